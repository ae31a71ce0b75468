"""GPU tier: the serving loop.  Every request's result is the same when it is
served alone (one request per launch) and when it is served in the mix
(continuous batching, several batches in flight, requests from several
threads), and equals the stored values -- bit-exact.  Admission by device
memory: requests larger than the budget are refused, the rest wait for memory
and complete."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(lc, dev):
    import torch

    g = torch.Generator(device="cpu").manual_seed(4)
    a = torch.cumsum(torch.randint(0, 20000, (2_000_000,), generator=g), 0).to(torch.int64)
    b = (torch.arange(500_000, dtype=torch.int64) * 77 + torch.randint(0, 300, (500_000,), generator=g)).to(torch.int32)
    c = torch.cumsum(torch.randint(0, 9, (300_000,), generator=g), 0).to(torch.int64)
    raw = [a, b, c]
    cols = [lc.encode(a.to(dev), lc.LINEAR, 4096), lc.encode(b.to(dev), lc.FOR, 1000), lc.encode(c.to(dev), lc.DELTA, 256)]
    return raw, cols


def _requests(raw, rng, nreq=160):
    import torch

    reqs = []
    for i in range(nreq):
        ci = int(rng.integers(len(raw)))
        n = raw[ci].numel()
        if rng.random() < 0.8:
            m = int(np.exp(rng.uniform(0, np.log(20000))))
            idx = torch.from_numpy(rng.integers(0, n, m).astype(np.int64)).pin_memory()
            reqs.append((ci, idx, None, m))
        else:
            cnt = int(np.exp(rng.uniform(np.log(16), np.log(200000))))
            cnt = min(cnt, n)
            first = int(rng.integers(0, n - cnt + 1))
            reqs.append((ci, None, first, cnt))
    return reqs


def _expected(raw, req):
    ci, idx, first, cnt = req
    return raw[ci][idx] if idx is not None else raw[ci][first:first + cnt]


def _serve(lc, cols, raw, reqs, threads=1, **opt):
    import torch

    srv = lc.Server(cols, **opt)
    outs = [torch.empty(r[3], dtype=raw[r[0]].dtype).pin_memory() for r in reqs]
    ids = [None] * len(reqs)

    def client(lo, hi):
        for i in range(lo, hi):
            ci, idx, first, cnt = reqs[i]
            ids[i] = srv.submit(ci, outs[i], idx=idx, first=first or 0, count=cnt)

    step = (len(reqs) + threads - 1) // threads
    th = [threading.Thread(target=client, args=(k * step, min(len(reqs), (k + 1) * step))) for k in range(threads)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for i in ids:
        srv.wait(i)
    st = srv.stats()
    srv.close()
    return outs, st


def test_results_identical_alone_and_in_the_mix(lc, dev):
    rng = np.random.default_rng(8)
    raw, cols = _setup(lc, dev)
    reqs = _requests(raw, rng)
    alone, st1 = _serve(lc, cols, raw, reqs, threads=1, slots=1, max_requests_per_batch=1)
    mixed, st2 = _serve(lc, cols, raw, reqs, threads=4, slots=4, max_requests_per_batch=64)
    lc.check()
    assert st1["batches"] == len(reqs) and st1["max_requests_in_batch"] == 1
    assert st2["completed"] == len(reqs)
    for r, a, m in zip(reqs, alone, mixed):
        exp = _expected(raw, r)
        assert np.array_equal(a.numpy(), exp.numpy())
        assert np.array_equal(m.numpy(), a.numpy())


def test_admission_by_device_memory(lc, dev):
    import torch

    rng = np.random.default_rng(9)
    raw, cols = _setup(lc, dev)
    budget = 1 << 20  # 1 MiB of device memory for indices + results
    srv = lc.Server(cols, slots=4, max_requests_per_batch=64, hbm_budget_bytes=budget)
    big = torch.empty(200_000, dtype=torch.int64).pin_memory()  # 1.6 MB of results: never fits
    with pytest.raises(lc.LecoError):
        srv.submit(0, big, first=0, count=200_000)
    reqs = []
    for _ in range(60):  # each fits alone; together they need many times the budget
        m = int(rng.integers(1000, 20000))
        idx = torch.from_numpy(rng.integers(0, raw[0].numel(), m).astype(np.int64)).pin_memory()
        out = torch.empty(m, dtype=torch.int64).pin_memory()
        reqs.append((idx, out, srv.submit(0, out, idx=idx)))
    for idx, out, rid in reqs:
        srv.wait(rid)
        assert torch.equal(out, raw[0][idx])
    st = srv.stats()
    assert st["completed"] == 60 and st["arena_bytes"] == budget
    srv.close()
    lc.check()


def test_unaligned_budget(lc, dev):
    """The arena hands out 256-byte multiples, so a budget that is not one is
    rounded down: a request sized between the rounded and the given budget is
    refused at submit (it could never be admitted), and a request of exactly
    the rounded budget is admitted and completes."""
    import torch

    raw, cols = _setup(lc, dev)
    budget = (1 << 20) + 100
    srv = lc.Server(cols, slots=2, max_requests_per_batch=8, hbm_budget_bytes=budget)
    assert srv.stats()["arena_bytes"] == 1 << 20
    over = torch.empty((1 << 17) + 12, dtype=torch.int64).pin_memory()  # (1 << 20) + 96 bytes of results
    with pytest.raises(lc.LecoError):
        srv.submit(0, over, first=0, count=over.numel())
    whole = torch.empty(1 << 17, dtype=torch.int64).pin_memory()  # exactly the usable arena
    small = torch.empty(1000, dtype=torch.int64).pin_memory()
    r1 = srv.submit(0, whole, first=5, count=whole.numel())
    r2 = srv.submit(0, small, first=7, count=small.numel())  # queued behind it, admitted after it retires
    srv.wait(r1)
    srv.wait(r2)
    assert torch.equal(whole, raw[0][5:5 + (1 << 17)])
    assert torch.equal(small, raw[0][7:1007])
    srv.close()
    lc.check()
