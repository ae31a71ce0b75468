"""CPU tier: the product's host partitioner for variable-length segments
(leco_varlen_partition) reproduces the segmentation of the reference's
Leco_cost_merge_double_wo_round<uint64_t> (compiled reference headers)."""
import numpy as np
import pytest

from conftest import golden_cases  # noqa: F401


def _gen(rng, n, kind):
    i = np.arange(n, dtype=np.float64)
    if kind == 0:
        x = 1e9 + 37.5 * i + rng.normal(0, 256, n)
    elif kind == 1:
        x = 1e9 + 1e-3 * i * i + rng.normal(0, 256, n)
    elif kind == 2:
        x = np.cumsum(rng.integers(0, 3000, n)).astype(np.float64) + 1e12
    else:
        x = np.zeros(n)
        lvl, p = 1e9, 0
        while p < n:
            L = min(n - p, int(rng.geometric(1 / 5000)))
            k = int(rng.integers(3))
            j = np.arange(L, dtype=np.float64)
            seg = lvl + (rng.uniform(1, 2 ** 10) * j if k == 0 else (1e-3 * j * j if k == 1 else 0 * j))
            x[p:p + L] = seg
            lvl = seg[-1] + 1
            p += L
        x += np.round(rng.normal(0, 256, n))
    return np.round(np.clip(x, 0, None)).astype(np.uint64)


def test_partition_matches_reference(lc, ref):
    rng = np.random.default_rng(1)
    checked = 0
    for trial in range(24):
        n = int(rng.choice([1000, 5000, 20011, 100000]))
        x = _gen(rng, n, trial % 4)
        blocks = int(rng.choice([1, 3, 10, 50]))
        delta = int(rng.choice([0, 2, 12, 64]))
        bs = n // blocks
        if n % bs == 1:  # last coarse block of one value: see the next test
            continue
        st_ref, _, _, dec = ref.varlen_encode(x, blocks, delta)
        assert np.array_equal(dec, x)
        st = lc.varlen_partition(x, blocks, delta, threads=4)
        assert np.array_equal(st, st_ref.astype(np.uint64)), (trial, n, blocks, delta)
        checked += 1
    assert checked >= 15


def test_partition_single_value_tail_block(lc, ref):
    """When the last coarse block holds one value the reference reads one value
    past the column and starts a segment inside the previous block (its output
    still decodes correctly).  Here that value becomes its own segment."""
    rng = np.random.default_rng(3)
    x = _gen(rng, 20011, 0)
    st_ref, _, _, dec = ref.varlen_encode(x, 3, 12)
    st = lc.varlen_partition(x, 3, 12)
    assert np.array_equal(st[:-1], st_ref[:-1].astype(np.uint64))
    assert int(st_ref[-1]) == 20009 and int(st[-1]) == 20010


def test_partition_golden(lc, golden):
    x = golden["varlen__values"]
    assert np.array_equal(lc.varlen_partition(x, 10, 20), golden["varlen__starts"].astype(np.uint64))
