"""GPU tier: the C++ drop-in header (include/leco_codecs.hpp) driven by a
reference-style experiment loop (tests/cpp/dropin_driver.cpp), its block
images compared byte for byte with the oracle's."""
import os
import struct
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from gpu_helpers import mask_delta_last_fields

pytestmark = pytest.mark.gpu


def _keys():
    N = 200000
    k32 = np.zeros(N, np.uint32)
    k64 = np.zeros(N, np.uint64)
    state = 7
    M = (1 << 64) - 1
    for i in range(N):
        state = (state * 6364136223846793005 + 1442695040888963407) & M
        k32[i] = (1000 * i + ((state >> 40) & 255)) & 0xFFFFFFFF
        k64[i] = 5000000000 + 77 * i * i // 64 + ((state >> 20) & 4095)
    return k32, k64


def test_cpp_dropin_driver(tmp_path, orc, lc):
    exe = tmp_path / "dropin"
    lib_dir = os.path.dirname(lc.lib_path())
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "cpp", "dropin_driver.cpp"), "-L", lib_dir, "-lleco_b200",
                           f"-Wl,-rpath,{lib_dir}", "-o", str(exe)])
    out = tmp_path / "blocks.bin"
    fout = tmp_path / "filters.bin"
    r = subprocess.run([str(exe), str(out), str(fout)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    k32, k64 = _keys()
    data = out.read_bytes()
    pos = 0
    for codec, x, blocks in ((0, k32, 200), (0, k64, 49), (1, k64, 49), (2, k32, 200), (3, k64, 25)):
        nb = struct.unpack_from("<I", data, pos)[0]
        pos += 4
        sizes = np.frombuffer(data, np.uint32, nb, pos)
        pos += 4 * nb
        bs = len(x) // blocks
        for b in range(nb):
            img = data[pos:pos + int(sizes[b])]
            pos += int(sizes[b])
            ref = orc.encode_block(codec, x[b * bs:(b + 1) * bs])
            if codec == 2:
                s, m = x.dtype.itemsize, len(x[b * bs:(b + 1) * bs])
                off = np.array([0, len(img)], np.uint64)
                img = mask_delta_last_fields(np.frombuffer(img, np.uint8), off, s, m, m).tobytes()
                ref = mask_delta_last_fields(np.frombuffer(ref, np.uint8), np.array([0, len(ref)], np.uint64), s, m, m).tobytes()
            assert img == ref, (codec, b)
    # legacy u32 blocks (piecewise_fix_op_max::encodeArray8) == the oracle's legacy images
    nb = struct.unpack_from("<I", data, pos)[0]
    pos += 4
    sizes = np.frombuffer(data, np.uint32, nb, pos)
    pos += 4 * nb
    bs = len(k32) // 200
    for b in range(nb):
        img = data[pos:pos + int(sizes[b])]
        pos += int(sizes[b])
        assert img == orc.legacy_encode_block(k32[b * bs:(b + 1) * bs])[0], ("legacy", b)
    assert pos == len(data)

    # the filter experiments through the drop-in classes == the oracle's column loops
    fdata = fout.read_bytes()
    fpos = 0

    def take():
        nonlocal fpos
        c = struct.unpack_from("<i", fdata, fpos)[0]
        idx = np.frombuffer(fdata, np.uint32, c, fpos + 4)
        fpos += 4 + 4 * c
        return idx

    bs = len(k64) // 49
    med = int(k64[len(k64) // 2])
    for codec, f1, f2, base in ((0, med, med, 0), (0, 1 << 28, 1 << 29, 1 << 30), (1, 1000, 40000, 65536)):
        pay, off = orc.encode_column(codec, k64, bs)
        zmin = np.array([k64[i:i + bs].min() for i in range(0, len(k64), bs)], np.uint64)
        zmax = np.array([k64[i:i + bs].max() for i in range(0, len(k64), bs)], np.uint64)
        got = take()
        assert np.array_equal(got, orc.filter_column(codec, pay, off, len(k64), 8, bs, f1, zmax)), (codec, "range")
        got = take()
        if base:
            c, want = orc.filter_close_column(codec, pay, off, len(k64), 8, bs, f1, f2, base, zmin if codec == 0 else None)
            assert len(got) == c and np.array_equal(got, want[:c]), (codec, "close")
