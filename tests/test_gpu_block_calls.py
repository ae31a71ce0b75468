"""GPU tier: the per-block drop-in calls (leco_block_encode / _decode / _random)
keep one stream and grow-only buffers per calling thread.  Blocks of growing
size reuse and then enlarge them; several threads call at once, each on its
own resources; leco_thread_release frees a thread's resources and a later call
creates them again.  Every image equals the oracle's and every value the input."""
import ctypes
import threading

import numpy as np
import pytest

from gpu_helpers import expected_gpu_column

pytestmark = pytest.mark.gpu

P = ctypes.c_void_p


def _roundtrip(lc, orc, x, codec):
    L = lc.lib()
    s, n = x.dtype.itemsize, len(x)
    buf = np.zeros(n * s * 2 + 256, np.uint8)
    nb = L.leco_block_encode(codec, s, P(x.ctypes.data), n, lc.FIT_REFERENCE, P(buf.ctypes.data))
    assert nb > 0, L.leco_last_error()
    img = buf[:nb].copy()
    want, _, _ = expected_gpu_column(orc, codec, x, n)
    assert img.tobytes() == want.tobytes(), (codec, s, n)
    out = np.zeros(n, x.dtype)
    assert L.leco_block_decode(codec, s, P(img.ctypes.data), nb, n, P(out.ctypes.data)) == 0
    assert np.array_equal(out, x)
    v = np.zeros(1, x.dtype)
    for k in (0, n // 2, n - 1):
        assert L.leco_block_random(codec, s, P(img.ctypes.data), nb, n, k, P(v.ctypes.data)) == 0
        assert v[0] == x[k]


def _blocks(seed):
    rng = np.random.default_rng(seed)
    for n in (7, 300, 4096, 16384):  # the buffers grow past their first size
        for dt in (np.uint32, np.uint64):
            x = np.cumsum(rng.integers(0, 1 << 12, n)).astype(dt)
            yield x


def test_block_calls_grow_and_release(lc, orc, dev):
    for x in _blocks(1):
        for codec in (0, 1, 3):
            _roundtrip(lc, orc, x, codec)
    assert lc.lib().leco_thread_release() == 0
    assert lc.lib().leco_thread_release() == 0  # nothing left to free
    _roundtrip(lc, orc, next(_blocks(2)), 0)     # resources created again
    lc.check()


def test_block_calls_from_several_threads(lc, orc, dev):
    import torch

    errors = []

    def work(seed):
        try:
            torch.cuda.set_device(0)
            for x in _blocks(seed):
                _roundtrip(lc, orc, x, seed % 2)
            assert lc.lib().leco_thread_release() == 0
        except Exception as e:  # reported to the main thread
            errors.append(repr(e))

    th = [threading.Thread(target=work, args=(10 + i,)) for i in range(4)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errors, errors
    lc.check()
