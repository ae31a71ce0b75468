"""GPU tier: columns saved to and loaded from container files through device
memory (leco_container_save_device / leco_container_load_device), and a
checkpoint of the serving loop's resident columns resumed into a new server:
every result bit-exact with the column before the round trip."""
import numpy as np
import pytest

from gpu_helpers import to_dev, to_np
from test_gpu_serve import _expected, _requests, _setup

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("codec", [0, 1, 2, 3])
def test_column_save_load(lc, orc, dev, tmp_path, codec):
    import torch

    rng = np.random.default_rng(3 + codec)
    x = (np.cumsum(rng.integers(0, 7000, 300_001)) + 5).astype(np.uint64)
    col = lc.encode(to_dev(x, dev), codec, 4096, lc.FIT_REFERENCE)
    p = str(tmp_path / "c.leco")
    col.save(p)
    back = lc.Column.load(p, device=dev)
    assert (back.codec, back.dtype, back.n, back.block_size) == (codec, 8, len(x), 4096)
    pay, off = col.to_host()
    pay2, off2 = back.to_host()
    assert np.array_equal(pay, pay2) and np.array_equal(off, off2)
    assert np.array_equal(to_np(back.decode(), 8), x)
    idx = torch.randint(0, len(x), (100_000,), device=dev)
    assert torch.equal(back.gather(idx), col.gather(idx))
    assert back.sum() == col.sum()
    # the file is the reference's column: the oracle decodes it
    info, fpay, foff, _ = lc.container_read(p)
    assert np.array_equal(orc.decode_column(codec, fpay, foff, len(x), 8, 4096), x)


def test_varlen_save_load(lc, golden, dev, tmp_path):
    x = golden["varlen__values"]
    col = lc.varlen_encode(to_dev(x, dev), golden["varlen__starts"].astype(np.uint64), lc.FIT_REFERENCE)
    p = str(tmp_path / "v.leco")
    col.save(p)
    back = lc.VarlenColumn.load(p, device=dev)
    pay, off, st = back.to_host()
    assert np.array_equal(pay, golden["varlen__payload"]) and np.array_equal(off, golden["varlen__offsets"])
    assert np.array_equal(to_np(back.decode(), 8), x)
    with pytest.raises(lc.LecoError):
        lc.Column.load(p, device=dev)


def test_server_checkpoint_resume(lc, dev, tmp_path):
    import torch

    rng = np.random.default_rng(12)
    raw, cols = _setup(lc, dev)
    reqs = _requests(raw, rng, nreq=60)
    srv = lc.Server(cols, slots=2, max_requests_per_batch=16)

    def run(server):
        outs = [torch.empty(r[3], dtype=raw[r[0]].dtype).pin_memory() for r in reqs]
        ids = [server.submit(r[0], o, idx=r[1], first=r[2] or 0, count=r[3]) for r, o in zip(reqs, outs)]
        for i in ids:
            server.wait(i)
        return outs

    before = run(srv)
    srv.checkpoint(str(tmp_path / "ckpt"))
    srv.close()
    del cols
    torch.cuda.synchronize()
    srv2 = lc.Server.resume(str(tmp_path / "ckpt"), device=dev)
    assert srv2.options == {"slots": 2, "max_requests_per_batch": 16, "hbm_budget_bytes": 0, "max_items_per_batch": 0}
    after = run(srv2)
    srv2.close()
    lc.check()
    for r, a, b in zip(reqs, before, after):
        assert np.array_equal(b.numpy(), a.numpy())
        assert np.array_equal(a.numpy(), _expected(raw, r).numpy())
