"""GPU tier: variable-length segments -- segment images byte-identical to the
reference's, bulk decode, random access and compressed-domain sum bit-exact."""
import numpy as np
import pytest

from test_varlen_partition import _gen

pytestmark = pytest.mark.gpu


def _dev(x, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x).view(np.int64)).to(dev)


def test_golden_segments_bytes(lc, golden, dev):
    x = golden["varlen__values"]
    col = lc.varlen_encode(_dev(x, dev), golden["varlen__starts"].astype(np.uint64), lc.FIT_REFERENCE)
    pay, off, st = col.to_host()
    assert np.array_equal(off, golden["varlen__offsets"])
    assert np.array_equal(pay, golden["varlen__payload"])
    assert np.array_equal(col.decode().cpu().numpy().view(np.uint64), x)


@pytest.mark.parametrize("kind", [0, 1, 2, 3])
def test_varlen_against_reference(lc, ref, orc, dev, kind):
    import torch

    rng = np.random.default_rng(40 + kind)
    n = 200_000
    x = _gen(rng, n, kind)
    st_ref, off_ref, pay_ref, _ = ref.varlen_encode(x, 100, 12)
    starts = lc.varlen_partition(x, 100, 12)
    assert np.array_equal(starts, st_ref.astype(np.uint64))
    xd = _dev(x, dev)
    col = lc.varlen_encode(xd, starts, lc.FIT_REFERENCE)
    pay, off, _ = col.to_host()
    assert np.array_equal(off, off_ref) and np.array_equal(pay, pay_ref), kind
    assert torch.equal(col.decode(), xd)
    idx = torch.randint(0, n, (100_000,), device=dev)
    assert torch.equal(col.gather(idx), xd[idx])
    edge = torch.tensor([0, n - 1] + [int(s) for s in starts[:50]], device=dev, dtype=torch.int64)
    assert torch.equal(col.gather(edge), xd[edge])
    assert col.sum() == int(x.sum(dtype=np.uint64))
    # the exact-fit stream decodes in the oracle's restatement of the reference decoder
    ce = lc.varlen_encode(xd, starts, lc.FIT_EXACT)
    pe, oe, se = ce.to_host()
    ends = list(se[1:]) + [n]
    for s in range(0, len(se), 7):
        seg = pe[oe[s]:oe[s + 1]].tobytes()
        assert np.array_equal(orc.varseg_decode(seg, int(ends[s] - se[s])), x[se[s]:ends[s]])
    assert torch.equal(ce.decode(), xd)
    lc.check()


def test_varlen_short_and_raw_segments(lc, orc, dev):
    """One- and two-value segments (sentinels 127/126) and raw segments."""
    import torch

    rng = np.random.default_rng(5)
    n = 5000
    x = np.cumsum(rng.integers(0, 100, n)).astype(np.uint64)
    x[3000:3100] = rng.integers(0, 2 ** 64 - 1, 100, dtype=np.uint64)  # forces a raw segment
    starts = np.array([0, 1, 3, 100, 101, 3000, 3100, 4998], np.uint64)
    xd = _dev(x, dev)
    col = lc.varlen_encode(xd, starts)
    pay, off, _ = col.to_host()
    ends = list(starts[1:]) + [n]
    for s in range(len(starts)):
        assert pay[off[s]:off[s + 1]].tobytes() == orc.varseg_encode(x, int(starts[s]), int(ends[s]) - 1), s
    assert torch.equal(col.decode(), xd)
    idx = torch.arange(n, device=dev)
    assert torch.equal(col.gather(idx), xd)
    lc.check()


def test_varlen_decode_paths_large(lc, orc, dev):
    """A column whose segment items take every decoder path: narrow segments
    decoded from the staged copy, runs of wide-residual segments whose eight-image
    items exceed the staging buffer (decoded from global memory), raw and
    one/two-value segments, and a segment count not a multiple of eight; decoded
    into an aligned and an 8-byte-offset output, summed and sampled at random."""
    import torch

    rng = np.random.default_rng(17)
    parts, starts, pos = [], [], 0
    for k in range(400):
        kind = k % 10
        if kind < 5:    # narrow: slope + small noise
            ln = int(rng.integers(500, 2000))
            seg = 10 ** 9 + 37 * pos + np.arange(ln) * 11 + rng.integers(0, 64, ln)
        elif kind < 8:  # wide residuals (about 40 bits): items of these exceed the buffer
            ln = int(rng.integers(1500, 2000))
            seg = 2 ** 50 + rng.integers(0, 2 ** 40, ln)
        elif kind == 8:  # raw
            ln = int(rng.integers(30, 300))
            seg = rng.integers(0, 2 ** 64 - 1, ln, dtype=np.uint64)
        else:            # one or two values
            ln = 1 + (k // 10) % 2
            seg = rng.integers(0, 2 ** 60, ln)
        starts.append(pos)
        parts.append(np.asarray(seg, dtype=np.uint64))
        pos += ln
    x = np.concatenate(parts)
    n = len(x)
    starts = np.array(starts, np.uint64)
    xd = _dev(x, dev)
    col = lc.varlen_encode(xd, starts, lc.FIT_REFERENCE)
    pay, off, _ = col.to_host()
    ends = list(starts[1:]) + [n]
    for s in range(0, len(starts), 13):
        assert pay[off[s]:off[s + 1]].tobytes() == orc.varseg_encode(x, int(starts[s]), int(ends[s]) - 1), s
    assert torch.equal(col.decode(), xd)
    buf = torch.zeros(n + 1, dtype=torch.int64, device=dev)
    col.decode(out=buf[1:])
    assert torch.equal(buf[1:], xd) and int(buf[0]) == 0
    assert col.sum() == int(x.sum(dtype=np.uint64))
    idx = torch.from_numpy(rng.integers(0, n, 1 << 16).astype(np.int64)).to(dev)
    assert torch.equal(col.gather(idx), xd[idx])
    lc.check()


def _starts(t):
    return t.cpu().numpy().view(np.uint64)


def test_device_partition_golden(lc, golden, dev):
    """The GPU partitioner on the reference fixture's column gives the
    reference's segment starts."""
    x = golden["varlen__values"]
    st = lc.varlen_partition_device(_dev(x, dev), 10, 20)
    assert np.array_equal(_starts(st), golden["varlen__starts"].astype(np.uint64))


def test_device_partition_matches_host(lc, dev):
    """GPU partitioner == host partitioner (which the CPU tier pins to the
    reference) over the value families, coarse block counts and merge
    penalties of the reference comparison, ragged and one-value tail blocks
    included."""
    rng = np.random.default_rng(5)
    checked = 0
    for trial in range(40):
        n = int(rng.choice([2, 3, 1000, 5000, 20011, 100000, 400_003]))
        x = _gen(rng, n, trial % 4)
        blocks = int(rng.choice([1, 3, 10, 50, 200]))
        blocks = max(1, min(blocks, n // 2))
        delta = int(rng.choice([0, 2, 12, 64]))
        want = lc.varlen_partition(x, blocks, delta, threads=8)
        got = _starts(lc.varlen_partition_device(_dev(x, dev), blocks, delta))
        assert np.array_equal(got, want), (trial, n, blocks, delta)
        checked += 1
    assert checked == 40


def test_device_partition_large(lc, dev):
    """20M keys of the regime-switching generator in coarse blocks of 2000
    values, merge penalty 12 bits (the variable-length benchmark's settings)."""
    from leco_b200 import workloads

    n = 20_000_000
    x = workloads.regime_switching_u64(n, seed=11, device=dev)
    xh = x.cpu().numpy().view(np.uint64)
    got = _starts(lc.varlen_partition_device(x, n // 2000, 12))
    want = lc.varlen_partition(xh, n // 2000, 12)
    assert np.array_equal(got, want)
