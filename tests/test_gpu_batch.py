"""GPU tier: the batch engine (one persistent launch per pass over many
columns of mixed codec, value type and length) produces exactly what the
single-column calls produce, and decodes every column bit-exactly."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _columns(dev, rng, ncols=64):
    import torch
    from leco_b200 import workloads

    cols = []
    fams = ["linear", "step", "walk", "uniform"]
    for i in range(ncols):
        n = int(rng.choice([1, 2, 3, 100, 1000, 4097, 20000, 123457]))
        s = 4 if i % 2 else 8
        x = workloads.families(n, fams[i % 4], s, rng)
        codec = [0, 1, 2, 3][(i // 2) % 4]
        bs = int(rng.choice([256, 1000, 2048, 4096, 8192]))
        t = torch.from_numpy(x.view(np.int64 if s == 8 else np.int32)).to(dev)
        cols.append((t, codec, bs))
    return cols


@pytest.mark.parametrize("fit", [0, 1])
def test_batch_matches_single_column_calls(lc, dev, fit):
    import torch

    rng = np.random.default_rng(12 + fit)
    cols = _columns(dev, rng)
    b = lc.Batch(cols, fit_mode=fit)
    assert b.total_blocks == sum((t.numel() + bs - 1) // bs for t, _, bs in cols)
    b.encode()
    b.decode()
    torch.cuda.synchronize()
    lc.check()
    for (x, codec, bs), col in zip(cols, b.cols):
        ref = lc.encode(x, codec, bs, fit)
        n = int(ref.offsets[-1].item())
        assert torch.equal(col.offsets, ref.offsets), (codec, bs, x.numel())
        assert torch.equal(col.payload[:n], ref.payload[:n]), (codec, bs, x.numel())
        assert torch.equal(col.dir, ref.dir)
        assert torch.equal(col.out, x), (codec, bs, x.numel())
    # graph replay (encode + decode) reproduces the same bytes and values
    for c in b.cols:
        c.out.zero_()
    b.run_graph(3)
    b.run_graph(3)
    torch.cuda.synchronize()
    lc.check()
    for (x, codec, bs), col in zip(cols, b.cols):
        assert torch.equal(col.out, x)
    # per-column baseline path gives the same result
    for c in b.cols:
        c.out.zero_()
    b.encode_per_column()
    b.decode_per_column()
    torch.cuda.synchronize()
    for (x, codec, bs), col in zip(cols, b.cols):
        assert torch.equal(col.out, x)
    b.close()


@pytest.mark.parametrize("fit", [0, 1])
def test_batch_threads_and_unroll_variants(lc, dev, fit):
    """Every (threads per block, unroll depth) the autotuner may pick -- groups of
    32, 64, 128 and 256 threads side by side in one CTA, unroll 1, 2 and 4 --
    gives the single-column path's bytes and decodes bit-exactly, for every
    codec and value type, including tail blocks and columns of one block."""
    import torch
    from leco_b200 import autotune, workloads

    rng = np.random.default_rng(40 + fit)
    fams = ["linear", "step", "walk", "uniform"]
    cols = []
    i = 0
    for g in autotune.GROUPS:
        for u in autotune.UNROLLS:
            for codec in (0, 1, 2, 3):
                s = 8 if (i // 2) % 2 else 4
                bs = int(rng.choice([b for b in (256, 512, 1000, 2048, 4096, 8192) if autotune.feasible(b, s, g)]))
                n = int(rng.choice([1, 3, bs - 1, bs * 3 + 17, bs * 9]))
                x = workloads.families(n, fams[i % 4], s, rng)
                cols.append((torch.from_numpy(x.view(np.int64 if s == 8 else np.int32)).to(dev), codec, bs, g, u))
                i += 1
    b = lc.Batch(cols, fit_mode=fit)
    b.encode()
    b.decode()
    torch.cuda.synchronize()
    lc.check()
    for (x, codec, bs, g, u), col in zip(cols, b.cols):
        ref = lc.encode(x, codec, bs, fit)
        n = int(ref.offsets[-1].item())
        assert torch.equal(col.offsets, ref.offsets), (codec, bs, g, u, x.numel())
        assert torch.equal(col.payload[:n], ref.payload[:n]), (codec, bs, g, u, x.numel())
        assert torch.equal(col.dir, ref.dir), (codec, bs, g, u)
        assert torch.equal(col.out, x), (codec, bs, g, u, x.numel())
    for c in b.cols:
        c.out.zero_()
    b.run_graph(3)
    torch.cuda.synchronize()
    lc.check()
    for (x, *_), col in zip(cols, b.cols):
        assert torch.equal(col.out, x)
    b.close()


def test_batch_rejects_bad_launch_parameters(lc, dev):
    import torch

    x = torch.arange(10000, dtype=torch.int64, device=dev)
    for spec in ((x, 0, 4096, 48, 2), (x, 0, 4096, 256, 3), (x, 0, 8192, 32, 2)):
        with pytest.raises(lc.LecoError):
            lc.Batch([spec])
