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
