"""GPU tier: the legacy u32 format of the reference (piecewise_fix_op_max,
headers/piecewise_fix_op_minimize_maxerror.h) read by the library -- bulk
decode, range decode, random access, compressed-domain sum, zone map -- on
streams written by the reference's own encoder (tests/golden/reference_legacy.npz).
Bit-exact with the stored values, which is what the reference's random access
returns and what its drivers obtain after correcting its bulk decoder."""
import os

import numpy as np
import pytest

from conftest import ROOT
from gpu_helpers import to_np

pytestmark = pytest.mark.gpu

FIX = os.path.join(ROOT, "tests", "golden", "reference_legacy.npz")


@pytest.fixture(scope="module")
def fx():
    return np.load(FIX)


def test_blocks(lc, orc, dev, fx):
    m = lc.piecewise_fix_op_max()
    m.init(1, 10000)
    for k in fx.files:
        if not (k.startswith("legacy_") and k.endswith("__image")):
            continue
        key = k[: -len("__image")]
        x, img = fx[key + "__values"], fx[key + "__image"]
        n = len(x)
        col = lc.Column.from_host(lc.LINEAR_F32, 4, n, n, img, np.array([0, len(img)], np.uint64), device=dev)
        assert np.array_equal(to_np(col.decode(), 4), x), key
        assert np.array_equal(to_np(col.decode(), 4), orc.legacy_decode_block(img.tobytes(), n)), key
        import torch
        idx = torch.arange(n, device=dev)
        assert np.array_equal(to_np(col.gather(idx), 4), x), key
        assert col.sum() == int(x.astype(np.uint64).sum()), key
        assert np.array_equal(m.decodeArray8(img.tobytes(), n), x), key
        for kk, v in zip(fx[key + "__ra_k"], fx[key + "__ra_v"]):
            assert m.randomdecodeArray8(img.tobytes(), int(kk)) == int(v), (key, kk)


def test_column(lc, dev, fx):
    import torch

    x, pay, off = fx["column__values"], fx["column__payload"], fx["column__offsets"]
    bs = int(fx["column__block_size"][0])
    n = len(x)
    col = lc.Column.from_host(lc.LINEAR_F32, 4, n, bs, pay, off, device=dev)
    assert np.array_equal(to_np(col.decode(), 4), x)
    assert np.array_equal(to_np(col.decode_range(5000, 100_000), 4), x[5000:105_000])
    idx = torch.randint(0, n, (1 << 20,), device=dev)
    assert np.array_equal(to_np(col.gather(idx), 4), x[idx.cpu().numpy()])
    assert col.sum() == int(x.astype(np.uint64).sum())
    zmin, zmax = col.zonemap()
    assert np.array_equal(to_np(zmin, 8), [x[i:i + bs].min() for i in range(0, n, bs)])
    assert np.array_equal(to_np(zmax, 8), [x[i:i + bs].max() for i in range(0, n, bs)])
    lc.check()


def test_encode_is_refused(lc, dev):
    import torch

    with pytest.raises(lc.LecoError):
        lc.encode(torch.arange(1000, dtype=torch.int32, device=dev), lc.LINEAR_F32, 100)
    with pytest.raises(lc.LecoError):  # u64 columns do not exist in this format
        lc.Column.from_host(lc.LINEAR_F32, 8, 10, 10, np.zeros(13, np.uint8), np.array([0, 13], np.uint64), device=dev)
