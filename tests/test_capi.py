"""CPU tier: the C-ABI library loads without a GPU, exports every entry point
declared in include/leco.h, and its host-only logic (sizing, validation,
argument checks) agrees with the oracle."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, golden_cases


def declared_functions():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if h.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", h)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names += re.findall(r"\b(leco_[a-z0-9_]+)\s*\(", txt)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(lc):
    L = ctypes.CDLL(lc.lib_path())
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # and the Python binding declares a signature for each of them
    bound = {n for n, _, _ in lc.SIGNATURES}
    assert set(names) <= bound, sorted(set(names) - bound)


def test_version(lc):
    assert "sm_100a" in lc.version()


def test_block_bytes_match_reference_images(lc, golden):
    L = lc.lib()
    for key, codec, s, n, fam in golden_cases(golden):
        img = golden[key + "__image"]
        l = int(img[0])
        if l in (126, 127):
            continue
        assert L.leco_block_bytes(codec, s, l, n) == len(img), key


def test_max_payload_bound(lc, golden):
    L = lc.lib()
    for key, codec, s, n, fam in golden_cases(golden):
        img = golden[key + "__image"]
        assert L.leco_max_payload_bytes(codec, s, n, n) >= len(img) + lc.PAYLOAD_SLACK, key


def test_validate_accepts_reference_columns_and_rejects_corruption(lc, golden):
    L = lc.lib()
    P = ctypes.c_void_p
    for t, bs, s in (("u32", 1000, 4), ("u64", 4096, 8)):
        x = golden[f"column_leco_{t}__values"]
        pay = np.ascontiguousarray(golden[f"column_leco_{t}__payload"])
        off = np.ascontiguousarray(golden[f"column_leco_{t}__offsets"])
        bad = np.zeros(1, np.uint64)
        args = lambda p, o: (0, s, p.ctypes.data_as(P), len(p), o.ctypes.data_as(P), len(x), bs, bad.ctypes.data_as(P))
        assert L.leco_validate_host(*args(pay, off)) == 0
        # truncated payload
        assert L.leco_validate_host(*args(pay[:-5].copy(), off)) == -3
        # a header with an impossible width
        p2 = pay.copy()
        p2[int(off[3])] = 200
        assert L.leco_validate_host(*args(p2, off)) == -3 and int(bad[0]) == 3
        # non-monotone offsets
        o2 = off.copy()
        o2[2], o2[3] = o2[3], o2[2]
        assert L.leco_validate_host(*args(pay, o2)) == -3


def test_argument_errors_need_no_gpu(lc):
    L = lc.lib()
    P = ctypes.c_void_p
    dummy = P(16)
    # unsupported codec, zero block size, null pointers: rejected before any CUDA call
    assert L.leco_encode(9, 8, dummy, 10, 16, 0, dummy, 1024, dummy, None, dummy, 1024, None) == -6
    assert L.leco_encode(0, 8, dummy, 10, 0, 0, dummy, 1024, dummy, None, dummy, 1024, None) == -1
    assert L.leco_encode(0, 3, dummy, 10, 16, 0, dummy, 1024, dummy, None, dummy, 1024, None) == -1
    assert L.leco_encode(0, 8, None, 10, 16, 0, dummy, 1024, dummy, None, dummy, 1024, None) == -1
    assert L.leco_decode(0, 8, None, dummy, 10, 16, dummy, None) == -1
    assert L.leco_decode(0, 8, P(17), dummy, 10, 16, dummy, None) == -1  # misaligned payload
    assert b"block_size" in L.leco_last_error() or b"aligned" in L.leco_last_error()
    # outputs not aligned to the value size (the decoders store 16/32-byte vectors)
    assert L.leco_decode(0, 8, dummy, dummy, 10, 16, P(20), None) == -1
    assert b"misaligned" in L.leco_last_error()
    assert L.leco_varlen_decode(dummy, dummy, dummy, 1, 10, P(20), None) == -1
    assert b"aligned" in L.leco_last_error()
    assert L.leco_num_blocks(10, 4) == 3 and L.leco_num_blocks(0, 4) == 0


@pytest.mark.parametrize("codec", [0, 1, 2, 3])
@pytest.mark.parametrize("s", [4, 8])
def test_workspace_sizes(lc, codec, s):
    L = lc.lib()
    n, bs = 1_000_003, 4096
    ref_ws = L.leco_encode_workspace_bytes(codec, s, n, bs, 0)
    ex_ws = L.leco_encode_workspace_bytes(codec, s, n, bs, 1)
    nb = (n + bs - 1) // bs
    assert ex_ws >= nb * 8 + 8
    assert ref_ws >= ex_ws
