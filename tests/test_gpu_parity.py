"""GPU tier: the CUDA library against the oracle / the reference on the same
seeded inputs.  Integer/byte work, so every comparison is bit-exact."""
import numpy as np
import pytest

from gpu_helpers import expected_gpu_column, mask_delta_last_fields, to_dev, to_np

pytestmark = pytest.mark.gpu

CODECS = [0, 1, 2, 3]


def columns(rng, s):
    dt = np.uint64 if s == 8 else np.uint32
    top = 2 ** (8 * s)
    n = 20011  # not a multiple of any block size: ragged tail
    yield "sorted_keys", (1000 * np.arange(n, dtype=np.uint64) + rng.integers(0, 256, n, dtype=np.uint64)).astype(dt)
    yield "linear_noise", np.clip(np.arange(n) * 37.25 + rng.normal(0, 2000, n) + 1e4, 0, top / 4).astype(np.float64).astype(np.uint64).astype(dt)
    yield "quadratic", np.clip(2e-3 * np.arange(n, dtype=np.float64) ** 2 + rng.normal(0, 64, n) + 1e5, 0, top / 4).astype(np.uint64).astype(dt)
    yield "walk", np.cumsum(rng.geometric(1 / 64, n)).astype(dt)
    yield "uniform_full", rng.integers(0, top, n, dtype=np.uint64).astype(dt)
    yield "uniform_half", rng.integers(0, top // 2, n, dtype=np.uint64).astype(dt)  # l = 8s-1 blocks
    yield "small", rng.integers(0, 4, n, dtype=np.uint64).astype(dt)
    yield "constant", np.full(n, 123456789, dt)
    yield "near_max", (np.uint64(top - 1) - rng.integers(0, 100000, n, dtype=np.uint64)).astype(dt)


@pytest.mark.parametrize("s", [4, 8])
@pytest.mark.parametrize("bs", [1000, 4096, 257])
def test_encode_bytes_match_reference(lc, orc, dev, s, bs):
    rng = np.random.default_rng(s * 1000 + bs)
    for name, x in columns(rng, s):
        for codec in CODECS:
            col = lc.encode(to_dev(x, dev), codec, bs, lc.FIT_REFERENCE)
            pay, off = col.to_host()
            epay, eoff, _ = expected_gpu_column(orc, codec, x, bs)
            if codec == 2:
                pay, epay = mask_delta_last_fields(pay, off, s, len(x), bs), mask_delta_last_fields(epay, eoff, s, len(x), bs)
            assert np.array_equal(off, eoff), (name, codec, s, bs)
            assert np.array_equal(pay, epay), (name, codec, s, bs)
            assert np.array_equal(to_np(col.decode(), s), x), (name, codec, s, bs)
    lc.check()


@pytest.mark.parametrize("s", [4, 8])
def test_decode_reference_streams(lc, orc, dev, s):
    """Reference-encoded columns (including l == 8s-1 blocks, which the
    reference's own bulk decoder gets wrong) decode bit-exactly on the GPU."""
    rng = np.random.default_rng(11 + s)
    bs = 1000
    for name, x in columns(rng, s):
        for codec in CODECS:
            pay, off = orc.encode_column(codec, x, bs)
            col = lc.Column.from_host(codec, s, len(x), bs, pay, off)
            assert np.array_equal(to_np(col.decode(), s), x), (name, codec)
            idx = rng.integers(0, len(x), 5000).astype(np.int64)
            import torch
            ti = torch.from_numpy(idx).to(dev)
            assert np.array_equal(to_np(col.gather(ti), s), x[idx]), (name, codec)
            assert np.array_equal(to_np(col.gather(ti, use_dir=False), s), x[idx]), (name, codec)
            assert col.sum() == int(x.astype(np.uint64).sum(dtype=np.uint64)), (name, codec)
    lc.check()


@pytest.mark.parametrize("s", [4, 8])
def test_exact_fit_streams_decode_in_reference(lc, orc, ref, dev, s):
    """LECO_FIT_EXACT streams are valid reference streams: the compiled
    reference's own decodeArray8 / randomdecodeArray8 reproduce the input."""
    rng = np.random.default_rng(21 + s)
    bs = 4096
    for name, x in columns(rng, s):
        if name in ("uniform_half",):
            continue
        for codec in (0, 3):
            col = lc.encode(to_dev(x, dev), codec, bs, lc.FIT_EXACT)
            pay, off = col.to_host()
            assert np.array_equal(ref.decode_column(codec, pay, off, len(x), s, bs), x), (name, codec)
            idx = rng.integers(0, len(x), 2000).astype(np.uint64)
            assert np.array_equal(ref.random_column(codec, pay, off, s, bs, idx), x[idx]), (name, codec)
            assert np.array_equal(to_np(col.decode(), s), x)
    lc.check()


@pytest.mark.parametrize("s", [4, 8])
def test_gpu_streams_decode_in_reference_decoder(lc, ref, dev, s):
    """GPU-encoded streams (reference fit) decode bit-exactly in the compiled
    reference's bulk decoder -- including columns whose blocks would have
    l == 8s-1, which this encoder writes raw."""
    rng = np.random.default_rng(31 + s)
    bs = 1000
    for name, x in columns(rng, s):
        for codec in (0, 1, 3):
            col = lc.encode(to_dev(x, dev), codec, bs, lc.FIT_REFERENCE)
            pay, off = col.to_host()
            assert np.array_equal(ref.decode_column(codec, pay, off, len(x), s, bs), x), (name, codec)


@pytest.mark.parametrize("s", [4, 8])
def test_range_decode(lc, dev, s):
    import torch
    rng = np.random.default_rng(41 + s)
    dt = np.uint64 if s == 8 else np.uint32
    x = np.cumsum(rng.integers(0, 5000, 50000)).astype(dt)
    for codec in CODECS:
        col = lc.encode(to_dev(x, dev), codec, 1000)
        for first, count in ((0, 1), (1, 3), (999, 2), (12345, 7777), (49990, 10), (0, 50000), (3, 49997)):
            assert np.array_equal(to_np(col.decode_range(first, count), s), x[first:first + count]), (codec, first, count)
    lc.check()


def test_edge_sizes(lc, orc, dev):
    for s in (4, 8):
        dt = np.uint64 if s == 8 else np.uint32
        for n in (1, 2, 3, 31, 32, 33, 4095, 4097):
            x = np.cumsum(np.arange(n) % 7).astype(dt) + dt(5)
            for codec in CODECS:
                for bs in (1, 2, 3, 64, 4096):
                    col = lc.encode(to_dev(x, dev), codec, bs)
                    pay, off = col.to_host()
                    epay, eoff, _ = expected_gpu_column(orc, codec, x, bs)
                    if codec == 2:
                        pay, epay = mask_delta_last_fields(pay, off, s, n, bs), mask_delta_last_fields(epay, eoff, s, n, bs)
                    assert np.array_equal(pay, epay) and np.array_equal(off, eoff), (s, n, codec, bs)
                    assert np.array_equal(to_np(col.decode(), s), x), (s, n, codec, bs)
    lc.check()


def test_every_width(lc, orc, dev):
    """Every bit width l in 0..8s: residual magnitudes 2^(l-2) force each l."""
    import torch
    for s in (4, 8):
        dt = np.uint64 if s == 8 else np.uint32
        for l in range(0, 8 * s + 1):
            n = 300
            x = np.full(n, 1 << (8 * s - 2), dtype=np.uint64)
            if l >= 2:
                amp = np.uint64(1) << np.uint64(l - 2)
                x = x + np.where(np.arange(n) % 2 == 0, amp, 0).astype(np.uint64)
            x = x.astype(dt)
            for codec in (1, 2):
                col = lc.encode(to_dev(x, dev), codec, 128)
                epay, eoff, _ = expected_gpu_column(orc, codec, x, 128)
                pay, off = col.to_host()
                if codec == 2:
                    pay, epay = mask_delta_last_fields(pay, off, s, n, 128), mask_delta_last_fields(epay, eoff, s, n, 128)
                assert np.array_equal(pay, epay), (s, l, codec)
                assert np.array_equal(to_np(col.decode(), s), x)
                idx = torch.arange(n, device=dev, dtype=torch.int64)
                assert np.array_equal(to_np(col.gather(idx), s), x)
    lc.check()


def test_block_mirrors_match_reference_methods(lc, ref):
    """The per-block Python mirrors return the reference methods' results."""
    rng = np.random.default_rng(5)
    for s, dt in ((4, np.uint32), (8, np.uint64)):
        x = np.cumsum(rng.integers(0, 1 << 12, 1000)).astype(dt)
        for cls, codec in ((lc.Leco_int, 0), (lc.FOR_int, 1), (lc.Delta_int, 2), (lc.Leco_int_poly, 3)):
            c = cls(dt)
            c.init(1, len(x))
            res = np.zeros(len(x) * s + 64, np.uint8)
            nbytes = c.encodeArray8_int(x, len(x), res, 0)
            img = res[:nbytes].tobytes()
            rimg = ref.encode_block(codec, x)
            if codec == 2:
                from gpu_helpers import mask_delta_last_fields as m
                off = np.array([0, nbytes], np.uint64)
                assert np.array_equal(m(np.frombuffer(img, np.uint8), off, s, len(x), len(x)),
                                      m(np.frombuffer(rimg, np.uint8), off, s, len(x), len(x)))
            else:
                assert img == rimg
            assert np.array_equal(c.decodeArray8(img, len(x)), x)
            for k in (0, 1, 500, 999):
                assert c.randomdecodeArray8(img, k, None, 0, length=len(x)) == int(x[k])


def test_corrupt_header_sets_error_word(lc, orc, dev):
    """A header width the codec cannot have is caught by the kernel's own
    check (no out-of-range access) and reported through leco_check."""
    x = np.arange(4000, dtype=np.uint64) * 3
    pay, off = orc.encode_column(0, x, 1000)
    pay = pay.copy()
    pay[int(off[2])] = 100  # l = 100 > 64
    col = lc.Column.from_host(0, 8, len(x), 1000, pay, off, validate=False)
    col.decode()
    with pytest.raises(lc.LecoError):
        lc.check()
    lc.check()  # cleared


@pytest.mark.parametrize("s,codec,bs,shift", [(8, 0, 4096, 0), (8, 3, 4096, 0), (4, 0, 4096, 0), (4, 5, 4096, 0),
                                              (8, 0, 4096, 1), (8, 0, 4099, 0), (4, 0, 2050, 0), (8, 3, 4096, 1),
                                              (4, 3, 2050, 0)])
def test_reference_fit_large_columns(lc, orc, dev, s, codec, bs, shift):
    """Columns of >= 4096 blocks under the reference fit (the sequential-fit
    kernel, then the encoder), with values 8 bytes off 16-byte alignment and block
    sizes whose rows are not a multiple of 16 bytes among them: aligned columns take
    the cp.async ring fit, the others the register-tiled fit (which also serves
    columns of more than one wave of the ring kernel), for linear and degree-2 fits.
    Every image equals the oracle's; large values make the reference's sequential
    FP64 sums round."""
    import torch
    rng = np.random.default_rng(7 * s + codec + bs + shift)
    dt = np.uint64 if s == 8 else np.uint32
    n = bs * 4100 + 777
    i = np.arange(n, dtype=np.float64)
    if s == 8:
        x = 2.0 ** 41 + np.cumsum(rng.exponential(2.0 ** 14, n)) + rng.normal(0, 2 ** 10, n)
    else:
        x = 1e8 + i * 0.9 + rng.normal(0, 40, n)
    if codec == 3:
        x = x + 1e-6 * (i % 8192) ** 2
    x = np.sort(x).astype(np.uint64).astype(dt)
    buf = torch.from_numpy(np.concatenate([np.zeros(shift, dt), x]).view(np.int64 if s == 8 else np.int32)).to(dev)
    col = lc.encode(buf[shift:], codec, bs, lc.FIT_REFERENCE)
    pay, off = col.to_host()
    if codec == 5:
        for b in list(range(0, 300)) + list(range(col.nblocks - 300, col.nblocks)):
            img, _, _ = orc.legacy_encode_block(x[b * bs:(b + 1) * bs])
            assert pay[off[b]:off[b + 1]].tobytes() == img, b
    else:
        epay, eoff, _ = expected_gpu_column(orc, codec, x, bs)
        assert np.array_equal(off, eoff)
        assert np.array_equal(pay, epay)
    assert np.array_equal(to_np(col.decode(), s), x)
    lc.check()


@pytest.mark.parametrize("s", [4, 8])
def test_staged_decode_large_mixed(lc, orc, dev, s):
    """Columns of >= 1024 blocks take the persistent TMA-staged decoder; mix
    narrow blocks (staged), blocks wider than 32 bits and raw blocks (decoded
    from global memory) in one column.  Delta blocks run the row scan on the
    staged copy (narrow) or on global memory (wide, raw)."""
    import torch
    rng = np.random.default_rng(99 + s)
    dt = np.uint64 if s == 8 else np.uint32
    top = 2 ** (8 * s)
    n = 2_100_003
    i = np.arange(n, dtype=np.float64)
    x = np.clip(1e6 + i * 3.5 + rng.normal(0, 300, n), 0, top / 4)
    seg = (np.arange(n) // 50_000) % 4
    wide = rng.integers(0, 2 ** (8 * s - 20), n, dtype=np.uint64).astype(np.float64)
    x = np.where(seg == 1, x + wide, x)                      # wide residuals (l > 32 for u64)
    x = x.astype(np.uint64)
    unif = rng.integers(0, top, n, dtype=np.uint64)
    x = np.where(seg == 2, unif, x).astype(dt)                # raw blocks
    for codec in (0, 1, 2, 3):
        for bs in (1000, 2048):
            col = lc.encode(to_dev(x, dev), codec, bs, lc.FIT_EXACT)
            assert col.nblocks >= 1024
            y = to_np(col.decode(), s)
            assert np.array_equal(y, x), (codec, bs)
            assert col.sum() == int(x.astype(np.uint64).sum(dtype=np.uint64)), (codec, bs)
        # and a reference-encoded copy of a slice decodes the same way
        pay, off = orc.encode_column(codec, x[:1_100_000], 1000)
        c2 = lc.Column.from_host(codec, s, 1_100_000, 1000, pay, off)
        assert np.array_equal(to_np(c2.decode(), s), x[:1_100_000]), codec
    lc.check()


def test_bounded_wait_times_out_without_faulting(lc):
    """Failure detection on the GPU: a look-back wait on a flag nothing sets gives
    up after its poll limit, the kernel reports LECO_ERR_TIMEOUT through the error
    word and the context keeps working."""
    import ctypes

    import torch

    res = ctypes.c_uint64()
    rc = lc.lib().leco_test_bounded_wait(2000, ctypes.byref(res))
    assert rc == -5 and res.value == 0xFFFFFFFFFFFFFFFF
    lc.check()  # the error word was read and cleared
    x = torch.arange(10000, dtype=torch.int64, device="cuda:0") * 3
    assert torch.equal(lc.encode(x, lc.LINEAR, 1000).decode(), x)
