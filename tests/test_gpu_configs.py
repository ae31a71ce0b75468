"""GPU tier: parity at the benchmark configurations' own shapes.

* The CPU-runnable configuration exactly: 1,000,000 uint32 keys
  x_i = 1000*i + U[0,255], blocks of 1000 values.  The GPU block images equal
  the compiled reference's byte for byte; full decode and 1,000,000 uniform
  lookups are bit-exact; the reference's own decoder and random access read the
  GPU stream.  These are the reference driver's self-checks
  (experiments/leco_int_fix_template.cpp:158-173 decode, :194-206 random access).
* The batching configuration at its full column count: 4096 columns of mixed
  type, family and codec (lengths log-uniform 1K-4M, capped at 32768 values so
  the oracle finishes in seconds), each with the autotune table's block size,
  threads per block and unroll depth, through one persistent batch pass; every
  column's bytes are compared with the oracle's images, not only with the
  single-column path.
* The variable-length / degree-2 configuration at 5M keys: the host and GPU
  partitioners give the reference partitioner's segment starts
  (piecewise_cost_merge_integer_template_double_wo_round.h:283-572), the GPU
  segment images equal the reference's byte for byte
  (experiments/leco_double_int_template_wo_round.cpp:66-200 is the driver), and
  decode, random access and the sum are bit-exact; the degree-2 codec with
  8192-value blocks matches the compiled reference's images.
"""
import numpy as np
import pytest

from gpu_helpers import expected_gpu_column, mask_delta_last_fields, to_dev, to_np

pytestmark = pytest.mark.gpu


def test_cpu_runnable_config_exact(lc, ref, dev):
    import torch
    from leco_b200 import workloads

    n, bs = 1_000_000, 1000
    x = workloads.sorted_keys_u32(n, seed=1)
    pay_r, off_r = ref.encode_column(0, x, bs)
    col = lc.encode(to_dev(x, dev), lc.LINEAR, bs, lc.FIT_REFERENCE)
    pay, off = col.to_host()
    assert np.array_equal(off, off_r)
    assert np.array_equal(pay[: int(off[-1])], pay_r)
    assert col.nbytes == len(pay_r)  # same compression ratio as the reference
    assert np.array_equal(to_np(col.decode(), 4), x)
    rng = np.random.default_rng(2024)
    idx = rng.integers(0, n, n).astype(np.int64)
    got = to_np(col.gather(torch.from_numpy(idx).to(dev)), 4)
    assert np.array_equal(got, x[idx])
    # the GPU stream through the reference's own decoder and random access
    assert np.array_equal(ref.decode_column(0, pay[: int(off[-1])], off, n, 4, bs), x)
    assert np.array_equal(ref.random_column(0, pay[: int(off[-1])], off, 4, bs, idx.astype(np.uint64)), x[idx])
    assert col.sum() == int(x.astype(np.uint64).sum()) & (2 ** 64 - 1)
    lc.check()


def test_batch_config_4096_columns_against_oracle(lc, orc, dev):
    import torch
    from leco_b200 import autotune, workloads

    cols, host = [], []
    for x, codec, _ in workloads.batch_columns(4096, seed=3, max_len=32768):
        s = x.dtype.itemsize
        bs, g, u = autotune.pick(codec, s, len(x), autotune.classify(x))
        cols.append((to_dev(x, dev), codec, bs, g, u))
        host.append(x)
    b = lc.Batch(cols, fit_mode=lc.FIT_REFERENCE)
    b.encode()
    b.decode()
    torch.cuda.synchronize()
    lc.check()
    nbad = 0
    for x, (xd, codec, bs, _, _), c in zip(host, cols, b.cols):
        s, n = x.dtype.itemsize, len(x)
        opay, ooff = orc.encode_column(codec, x, bs)
        heads = opay[ooff[:-1].astype(np.int64)] if len(opay) else np.zeros(0, np.uint8)
        if codec != 2 and np.any(heads == 8 * s - 1):
            opay, ooff, _ = expected_gpu_column(orc, codec, x, bs)  # H1: such blocks are written raw
        gpay = c.payload[: int(ooff[-1])].cpu().numpy()
        goff = c.offsets.cpu().numpy().view(np.uint64)
        assert np.array_equal(goff, ooff), (codec, s, n, bs)
        if codec == 2:
            gpay = mask_delta_last_fields(gpay, goff, s, n, bs)
            opay = mask_delta_last_fields(opay, ooff, s, n, bs)
        nbad += not np.array_equal(gpay, opay)
        assert torch.equal(c.out, xd), (codec, s, n, bs)
    assert nbad == 0
    b.close()


def test_varlen_and_poly2_config_5m(lc, ref, dev):
    import torch
    from leco_b200 import workloads

    n = 5_000_000
    xd = workloads.regime_switching_u64(n, seed=5, device=dev)
    x = xd.cpu().numpy().view(np.uint64)
    coarse, delta = n // 2000, 12
    st_ref, off_ref, pay_ref, _ = ref.varlen_encode(x, coarse, delta)
    starts = lc.varlen_partition(x, coarse, delta)
    assert np.array_equal(starts, st_ref.astype(np.uint64))
    dstarts = lc.varlen_partition_device(xd, coarse, delta)
    assert np.array_equal(dstarts.cpu().numpy().view(np.uint64), starts)
    col = lc.varlen_encode(xd, starts, lc.FIT_REFERENCE)
    pay, off, _ = col.to_host()
    assert np.array_equal(off, off_ref) and np.array_equal(pay, pay_ref)
    assert torch.equal(col.decode(), xd)
    idx = torch.randint(0, n, (1 << 20,), device=dev)
    assert torch.equal(col.gather(idx), xd[idx])
    assert col.sum() == int(x.sum(dtype=np.uint64))
    # degree-2 polynomial, 8192-value blocks, against the compiled reference's images
    ppay_r, poff_r = ref.encode_column(3, x, 8192, threads=8)
    pc = lc.encode(xd, lc.POLY2, 8192, lc.FIT_REFERENCE)
    ppay, poff = pc.to_host()
    heads = ppay_r[poff_r[:-1].astype(np.int64)]
    assert not np.any(heads == 63)  # no H1 block in this column, so the images are the reference's
    assert np.array_equal(poff, poff_r) and np.array_equal(ppay[: int(poff[-1])], ppay_r)
    assert torch.equal(pc.decode(), xd)
    assert torch.equal(pc.gather(idx), xd[idx])
    assert pc.sum() == int(x.sum(dtype=np.uint64))
    lc.check()
