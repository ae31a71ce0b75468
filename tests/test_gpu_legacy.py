"""GPU tier: the legacy u32 format of the reference (piecewise_fix_op_max,
headers/piecewise_fix_op_minimize_maxerror.h) read by the library -- bulk
decode, range decode, random access, compressed-domain sum, zone map -- on
streams written by the reference's own encoder (tests/golden/reference_legacy.npz);
and the library's encoder for the format, byte for byte against those streams and
the oracle.  Bit-exact with the stored values, which is what the reference's random
access returns and what its drivers obtain after correcting its bulk decoder."""
import os

import numpy as np
import pytest

from conftest import ROOT
from gpu_helpers import to_dev, to_np

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


def test_encode_blocks_match_reference(lc, dev, fx):
    """leco_encode(LINEAR_F32) and encodeArray8 write the reference's images."""
    m = lc.piecewise_fix_op_max()
    for k in fx.files:
        if not (k.startswith("legacy_") and k.endswith("__image")):
            continue
        key = k[: -len("__image")]
        x, img = fx[key + "__values"], fx[key + "__image"]
        n = len(x)
        col = lc.encode(to_dev(x, dev), lc.LINEAR_F32, n)
        pay, off = col.to_host()
        assert np.array_equal(pay, img), key
        assert np.array_equal(off, [0, len(img)]), key
        res = np.zeros(len(img) + 64, np.uint8)
        assert m.encodeArray8(x, n, res) == len(img), key
        assert np.array_equal(res[:len(img)], img), key
        assert np.array_equal(to_np(col.decode(), 4), x), key


def test_encode_column_matches_reference(lc, dev, fx):
    x, pay, off = fx["column__values"], fx["column__payload"], fx["column__offsets"]
    bs = int(fx["column__block_size"][0])
    for fit in (lc.FIT_REFERENCE, lc.FIT_EXACT):
        col = lc.encode(to_dev(x, dev), lc.LINEAR_F32, bs, fit_mode=fit)
        p, o = col.to_host()
        if fit == lc.FIT_REFERENCE:
            assert np.array_equal(o, off) and np.array_equal(p, pay)
        assert np.array_equal(to_np(col.decode(), 4), x)
        idx = np.random.default_rng(3).integers(0, len(x), 4096)
        import torch
        assert np.array_equal(to_np(col.gather(torch.from_numpy(idx).to(dev)), 4), x[idx])


def _legacy_families(n, rng):
    i = np.arange(n, dtype=np.float64)
    top = 2 ** 32 - 1
    yield np.clip(np.round(3e9 + 0.37 * i + rng.normal(0, 3, n)), 0, top)
    yield np.clip(np.round(1e8 + 7e3 * i + rng.normal(0, 2e4, n)), 0, top)
    yield np.clip(np.round(4e9 - 40 * i + rng.normal(0, 1e6, n)), 0, top)
    yield rng.integers(0, 2 ** 32, n).astype(np.float64)                      # raw blocks
    yield np.full(n, float(rng.integers(0, 2 ** 32)))                          # l == 0
    yield np.where((i // 2) % 2 == 0, 0.0, float(top))                         # wrapping residuals


@pytest.mark.parametrize("bs", [4096, 1000, 300, 64])
def test_encode_matches_oracle(lc, orc, dev, bs):
    """Seeded columns (block sizes on both the CTA and the warp-per-block path,
    ragged last blocks) against the oracle, block by block."""
    rng = np.random.default_rng(bs)
    for fam, xf in enumerate(_legacy_families(3 * bs + bs // 3 + 1, rng)):
        x = xf.astype(np.uint32)
        n = len(x)
        col = lc.encode(to_dev(x, dev), lc.LINEAR_F32, bs)
        pay, off = col.to_host()
        for b in range(len(off) - 1):
            img, _, _ = orc.legacy_encode_block(x[b * bs:(b + 1) * bs])
            assert pay[off[b]:off[b + 1]].tobytes() == img, (bs, fam, b)
        assert np.array_equal(to_np(col.decode(), 4), x), (bs, fam)


def test_encode_large_round_trip(lc, orc, dev):
    """20M values of mixed families: every block decodes to its values, and a
    sample of blocks equals the oracle's images."""
    import torch

    rng = np.random.default_rng(77)
    bs, per = 4096, 4096 * 800
    x = np.concatenate([f.astype(np.uint32) for f in _legacy_families(per, rng)])
    x = x[: 20_000_000] if len(x) > 20_000_000 else x
    col = lc.encode(to_dev(x, dev), lc.LINEAR_F32, bs)
    assert torch.equal(col.decode(), to_dev(x, dev))
    pay, off = col.to_host()
    for b in rng.integers(0, len(off) - 1, 200):
        img, _, _ = orc.legacy_encode_block(x[b * bs:(b + 1) * bs])
        assert pay[off[b]:off[b + 1]].tobytes() == img, b
    lc.check()


def test_encode_u64_is_refused(lc, dev):
    import torch

    with pytest.raises(lc.LecoError):  # the format stores u32 values only
        lc.encode(torch.arange(1000, dtype=torch.int64, device=dev), lc.LINEAR_F32, 100)
    with pytest.raises(lc.LecoError):
        lc.Column.from_host(lc.LINEAR_F32, 8, 10, 10, np.zeros(13, np.uint8), np.array([0, 13], np.uint64), device=dev)
