"""GPU test of leco_encode_noalloc, the encode entry point for callers that
cannot allocate device memory (an engine whose buffer manager owns every byte
of device memory, or a thread that must not call cudaMalloc/cudaFree because
they can synchronize the device).  It must produce exactly what leco_encode
with a caller workspace produces, call after call, since the built-in scratch
array keeps the previous call's contents.

This file sorts last so that a run stopping at the first failure has already
run every other test; it also passes on its own in a fresh process."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

P = ctypes.c_void_p


def _encode_both(lc, x, codec, bs, fit_mode):
    import torch

    L = lc.lib()
    s = x.element_size()
    n = x.numel()
    nb = L.leco_num_blocks(n, bs)
    cap = L.leco_max_payload_bytes(codec, s, n, bs)
    stream = P(torch.cuda.current_stream().cuda_stream)
    ref = lc.encode(x, codec, bs, fit_mode)  # leco_encode with a workspace
    pay = torch.full((cap,), 0xA5, dtype=torch.uint8, device=x.device)
    off = torch.empty(nb + 1, dtype=torch.int64, device=x.device)
    d = torch.empty(nb * 32, dtype=torch.uint8, device=x.device)
    rc = L.leco_encode_noalloc(codec, s, P(x.data_ptr()), n, bs, fit_mode, P(pay.data_ptr()), cap, P(off.data_ptr()),
                               P(d.data_ptr()), stream)
    assert rc == 0, L.leco_last_error()
    torch.cuda.synchronize()
    lc.check()
    total = int(off[-1].item())
    assert torch.equal(off, ref.offsets)
    assert torch.equal(pay[:total], ref.payload[:total])
    assert torch.equal(d, ref.dir)
    col = lc.Column(codec, s, n, bs, pay, off, d)
    assert torch.equal(col.decode(), x)


def test_noalloc_encode_matches_workspace_encode_twice(lc):
    import torch

    dev = torch.device("cuda:0")
    g = torch.Generator(device="cpu").manual_seed(3)
    # two calls in a row with different columns: the second sees the first call's leftovers
    a = torch.cumsum(torch.randint(0, 5000, (3_000_001,), generator=g), 0).to(torch.int64).to(dev)
    b = (torch.arange(900_000, dtype=torch.int64) * 3 + torch.randint(0, 7, (900_000,), generator=g)).to(dev)
    for fit in (0, 1):
        _encode_both(lc, a, 0, 4096, fit)
        _encode_both(lc, b, 0, 1000, fit)
    _encode_both(lc, b.to(torch.int32), 1, 2048, 0)
    _encode_both(lc, a[:500_000], 3, 8192, 0)


def test_noalloc_encode_allocates_nothing(lc):
    """A call after the first on the device (which loads the library's kernels)
    changes neither the device's free memory nor torch's allocator counters."""
    import torch

    L = lc.lib()
    dev = torch.device("cuda:0")
    x = torch.cumsum(torch.randint(0, 999, (2_000_000,), device=dev), 0)
    n, bs = x.numel(), 4096
    cap = L.leco_max_payload_bytes(0, 8, n, bs)
    pay = torch.empty(cap, dtype=torch.uint8, device=dev)
    off = torch.empty(L.leco_num_blocks(n, bs) + 1, dtype=torch.int64, device=dev)
    stream = P(torch.cuda.current_stream().cuda_stream)
    args = (0, 8, P(x.data_ptr()), n, bs, 0, P(pay.data_ptr()), cap, P(off.data_ptr()), None, stream)
    assert L.leco_encode_noalloc(*args) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    stats0 = torch.cuda.memory_stats()
    for _ in range(3):
        assert L.leco_encode_noalloc(*args) == 0, L.leco_last_error()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    stats1 = torch.cuda.memory_stats()
    # any device allocation takes at least one 2 MiB page off the free count
    assert abs(free1 - free0) < (1 << 21), (free0, free1)
    for key in ("allocation.all.allocated", "segment.all.allocated", "reserved_bytes.all.current"):
        assert stats1.get(key) == stats0.get(key), key
    lc.check()


def test_noalloc_rejects_columns_beyond_its_scratch(lc):
    import torch

    L = lc.lib()
    maxb = L.leco_encode_noalloc_max_blocks()
    assert maxb == 32768
    n = (maxb + 1) * 16
    x = torch.zeros(n, dtype=torch.int64, device="cuda:0")
    cap = L.leco_max_payload_bytes(0, 8, n, 16)
    pay = torch.empty(cap, dtype=torch.uint8, device="cuda:0")
    off = torch.empty(maxb + 2, dtype=torch.int64, device="cuda:0")
    rc = L.leco_encode_noalloc(0, 8, P(x.data_ptr()), n, 16, 0, P(pay.data_ptr()), cap, P(off.data_ptr()), None,
                               P(torch.cuda.current_stream().cuda_stream))
    assert rc == -1
    assert b"at most 32768" in L.leco_last_error()
