"""GPU tier: predicate pushdown (leco_filter_range, leco_filter_range_close,
leco_zonemap) through the C ABI against the oracle, which the CPU tier pins to
the reference's own filter results (tests/test_filter_oracle.py).  Index lists
are compared bit-exactly: same indices, same order, same count.

The oracle's close-range results are taken with windows appended (the layout
the library writes); the count is the reference's either way."""
import os

import numpy as np
import pytest

from conftest import ROOT
from gpu_helpers import to_dev, to_np

pytestmark = pytest.mark.gpu

FIX = os.path.join(ROOT, "tests", "golden", "reference_filters.npz")


def _fixture_columns():
    fx = np.load(FIX)
    i = 0
    while f"c{i}__meta" in fx.files:
        key = f"c{i}"
        s, codec, bs, n = (int(v) for v in fx[key + "__meta"])
        filters = []
        j = 0
        while f"{key}__f{j}__args" in fx.files:
            filters.append(tuple(int(v) for v in fx[f"{key}__f{j}__args"]))
            j += 1
        yield key, s, codec, bs, n, fx[key + "__values"], fx[key + "__payload"], fx[key + "__offsets"], filters
        i += 1


def _idx(t, c):
    return t[:c].cpu().numpy().view(np.uint32)


def test_zonemap_matches_values(lc, orc, dev):
    for key, s, codec, bs, n, x, pay, off, _ in _fixture_columns():
        col = lc.Column.from_host(codec, s, n, bs, pay, off, device=dev)
        zmin, zmax = col.zonemap()
        emin, emax = orc.zonemap(codec, pay, off, n, s, bs)
        assert np.array_equal(to_np(zmin, 8), emin), key
        assert np.array_equal(to_np(zmax, 8), emax), key
        assert lc.lib().leco_check(None) == 0


def test_filters_match_oracle_on_reference_columns(lc, orc, dev):
    """Every fixture column (reference-encoded, raw and l = 8s-1 blocks
    included) and filter, with and without the zone map."""
    import torch

    checked = 0
    for key, s, codec, bs, n, x, pay, off, filters in _fixture_columns():
        col = lc.Column.from_host(codec, s, n, bs, pay, off, device=dev)
        zmin_t, zmax_t = col.zonemap()
        zmin, zmax = orc.zonemap(codec, pay, off, n, s, bs)
        for kind, a, b, base in filters:
            if kind == 0:
                for zlo_t, zm_t, zm in ((None, None, None), (None, zmax_t, zmax), (zmin_t, zmax_t, zmax)):
                    want = orc.filter_column(codec, pay, off, n, s, bs, a, zm)
                    got, c = col.filter_range(a, zone_max=zm_t, zone_min=zlo_t)
                    assert c == len(want) and np.array_equal(_idx(got, c), want), (key, a, zm is None, zlo_t is None)
                    checked += 1
            else:
                zm_t, zm = (zmin_t, zmin) if codec == 0 else (None, None)
                if orc.filter_close_column(codec, pay, off, n, s, bs, a, b, base, zm, max_periods=4096)[0] < 0:
                    continue  # wide-residual blocks: more windows than the oracle is run for here
                want_c, want = orc.filter_close_column(codec, pay, off, n, s, bs, a, b, base, zm)
                got, c = col.filter_range_close(a, b, base, zone_min=zm_t)
                assert c == want_c and np.array_equal(_idx(got, c), want[:c]), (key, a, b, base)
                checked += 1
        torch.cuda.synchronize()
    assert lc.lib().leco_check(None) == 0
    assert checked > 300


@pytest.mark.parametrize("s", [4, 8])
def test_filters_on_gpu_encoded_columns(lc, orc, dev, s):
    """Columns encoded here (both fit modes), ragged tails, tiny and maximum
    block sizes, filters at the edges of the value range."""
    rng = np.random.default_rng(40 + s)
    dt = np.uint64 if s == 8 else np.uint32
    for n, bs in ((1, 16), (5, 64), (20011, 1000), (70001, 16384), (33333, 257)):
        i = np.arange(n, dtype=np.int64)
        for kind in range(3):
            if kind == 0:
                x = (np.cumsum(rng.integers(0, 2000, n)) + 7).astype(dt)
            elif kind == 1:
                x = ((i // 501) * 7000 + rng.integers(0, 60, n)).astype(dt)
            else:
                x = (3_000_000 - i * 11 + rng.integers(0, 9, n)).astype(dt)
            for codec in (0, 1):
                for fit in (lc.FIT_REFERENCE, lc.FIT_EXACT):
                    col = lc.encode(to_dev(x, dev), codec, bs, fit)
                    pay, off = col.to_host()
                    zmin_t, zmax_t = col.zonemap()
                    zmin, zmax = orc.zonemap(codec, pay, off, n, s, bs)
                    for f in (0, int(x.min()), int(np.median(x)), int(x.max()) - 1, int(x.max()), 2 ** (8 * s) - 1):
                        want = orc.filter_column(codec, pay, off, n, s, bs, f, zmax)
                        got, c = col.filter_range(f, zone_max=zmax_t, zone_min=zmin_t)
                        assert c == len(want) and np.array_equal(_idx(got, c), want), (n, bs, kind, codec, f)
                        got, c = col.filter_range(f)
                        assert c == len(want) and np.array_equal(_idx(got, c), want), (n, bs, kind, codec, f)
                    for base, f1, f2 in ((10000, 1000, 5000), (7919, 0, 3000), (1 << 20, 5, 1 << 19)):
                        zm_t, zm = (zmin_t, zmin) if codec == 0 else (None, None)
                        want_c, want = orc.filter_close_column(codec, pay, off, n, s, bs, f1, f2, base, zm)
                        got, c = col.filter_range_close(f1, f2, base, zone_min=zm_t)
                        assert c == want_c and np.array_equal(_idx(got, c), want[:c]), (n, bs, kind, codec, base)


def test_output_capacity_and_empty_column(lc, orc, dev):
    import torch

    x = np.arange(0, 50000, dtype=np.uint64) * 3
    col = lc.encode(to_dev(x, dev), 0, 1000, lc.FIT_REFERENCE)
    out = torch.full((100,), -1, dtype=torch.int32, device=dev)
    got, c = col.filter_range(10, out=out, out_cap=64)
    assert c == len(x) - 4  # values 12, 15, ... are above 10
    assert np.array_equal(_idx(got, 64), np.arange(4, 68, dtype=np.uint32))
    assert np.all(out[64:].cpu().numpy() == -1)  # nothing past out_cap
    # an output buffer that is not 16-byte aligned, and a cap inside a 4-index run
    out2 = torch.full((200,), -1, dtype=torch.int32, device=dev)
    got, c = col.filter_range(10, out=out2[1:], out_cap=63)
    assert c == len(x) - 4
    assert np.array_equal(_idx(got, 63), np.arange(4, 67, dtype=np.uint32))
    assert out2[0].item() == -1 and np.all(out2[64:].cpu().numpy() == -1)
    empty = lc.Column(0, 8, 0, 1000, col.payload, col.offsets)
    got, c = empty.filter_range(0)
    assert c == 0


def test_window_limit_reports_error(lc, orc, dev):
    """A LeCo block whose model allows every index for more than 65536 windows
    (40-bit residuals on a rising line, base 1): the close-range call reports
    LECO_ERR_UNSUPPORTED instead of running the reference's loop."""
    rng = np.random.default_rng(9)
    i = np.arange(64, dtype=np.uint64)
    x = (np.uint64(1 << 50) + i * np.uint64(1 << 34) + rng.integers(0, 2 ** 40, 64, dtype=np.uint64)).astype(np.uint64)
    col = lc.encode(to_dev(x, dev), 0, 64, lc.FIT_REFERENCE)
    pay, off = col.to_host()
    assert pay[0] < 64  # a packed block, not raw
    zmin, _ = orc.zonemap(0, pay, off, 64, 8, 64)
    assert orc.filter_close_column(0, pay, off, 64, 8, 64, 0, 1, 1, zmin, max_periods=65536)[0] == -1
    with pytest.raises(lc.LecoError) as e:
        col.filter_range_close(0, 1, 1, zone_min=col.zonemap()[0])
    assert e.value.code == -6
    assert lc.lib().leco_check(None) == 0  # the error word was cleared by the failing check


def test_bad_arguments_are_rejected(lc, dev):
    x = np.arange(1000, dtype=np.uint64)
    col = lc.encode(to_dev(x, dev), 2, 100, lc.FIT_REFERENCE)  # Delta: no filter in the reference
    with pytest.raises(lc.LecoError):
        col.filter_range(5)
    col = lc.encode(to_dev(x, dev), 1, 100, lc.FIT_REFERENCE)
    with pytest.raises(lc.LecoError):
        col.filter_range_close(1, 2, 0)
    with pytest.raises(lc.LecoError):
        col.filter_range_close(1, 2, 1 << 31)


def test_large_sorted_column_counts(lc, orc, dev):
    """20M sorted u64 keys in blocks of 4096 (the decode workload's shape, at a
    tenth of its size): indices equal the oracle's, and on this data they are
    also exactly the values above the filter."""
    rng = np.random.default_rng(3)
    n, bs = 20_000_000, 4096
    x = np.cumsum(rng.integers(1, 2000, n, dtype=np.uint64)).astype(np.uint64)
    col = lc.encode(to_dev(x, dev), 0, bs, lc.FIT_EXACT)
    pay, off = col.to_host()
    zmin_t, zmax_t = col.zonemap()
    for q in (0.5, 0.99):
        f = int(np.quantile(x, q))
        got, c = col.filter_range(f, zone_max=zmax_t, zone_min=zmin_t)
        want = orc.filter_column(0, pay, off, n, 8, bs, f)
        assert c == len(want) and np.array_equal(_idx(got, c), want)
        assert np.array_equal(want, np.nonzero(x > f)[0].astype(np.uint32))


def test_block_mirror_matches_reference_fixture(lc, orc):
    """Leco_int / FOR_int .filter_range / .filter_range_close one block at a
    time (the reference's call shape) against the reference's own per-block
    results stored in the fixtures (count always; indices where the
    reference's buffer is defined, i.e. not for l > 0 LeCo close range)."""
    fx = np.load(FIX)
    checked = 0
    for key, s, codec, bs, n, x, pay, off, filters in _fixture_columns():
        cls = lc.Leco_int if codec == 0 else lc.FOR_int
        c_ = cls(np.uint64 if s == 8 else np.uint32)
        c_.init(len(off) - 1, bs)
        for j, (kind, a, b, base) in enumerate(filters):
            counts, outs = fx[f"{key}__f{j}__counts"], fx[f"{key}__f{j}__out"]
            pos = 0
            for blk in range(len(off) - 1):
                img = pay[off[blk]:off[blk + 1]].tobytes()
                ln = min(bs, n - blk * bs)
                cr = int(counts[blk])
                ref = outs[pos:pos + max(cr, 0)]
                pos += max(cr, 0)
                if cr < 0 or (codec == 1 and img[0] == 8 * s - 1):
                    continue  # undefined in the reference (checked against the oracle elsewhere)
                buf = np.zeros(4 * ln + 8, np.uint32)
                if kind == 0:
                    c = c_.filter_range(img, ln, a, buf, blk)
                    assert c == cr and np.array_equal(buf[:c], ref), (key, j, blk)
                else:
                    f1, f2 = (int(fx[f"{key}__f{j}__w1"][blk]), int(fx[f"{key}__f{j}__w2"][blk])) if codec == 0 else (a, b)
                    c = c_.filter_range_close(img, ln, buf, blk, f1, f2, base)
                    assert c == cr, (key, j, blk)
                    if codec == 1 or img[0] == 0:
                        assert np.array_equal(buf[:c], ref), (key, j, blk)
                checked += 1
    assert checked > 1500
