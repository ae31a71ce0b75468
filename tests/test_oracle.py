"""CPU tier: the oracle restatement (oracle/leco_oracle.c) against the
reference's own outputs -- the committed golden fixtures (made by the compiled
reference headers) and, when oracle/_ref is present, the compiled reference
itself on fresh seeded inputs."""
import numpy as np
import pytest

from conftest import golden_cases

TB = {4: 32, 8: 64}


def _mask_delta_last_field(img: bytes, s: int, n: int) -> bytes:
    """The reference Delta encoder packs n fields from n-1 deltas
    (delta_integer_template.h:83): its last field is out-of-bounds memory.
    The oracle writes zeros there; comparisons clear that field."""
    l = img[0]
    if n < 2 or l in (0, 8 * s):
        return img
    b = bytearray(img)
    for bit in range((n - 1) * l, n * l):
        b[1 + s + bit // 8] &= ~(1 << (bit % 8)) & 0xFF
    return bytes(b)


def test_golden_images_match_oracle(golden, orc):
    bad = []
    for key, codec, s, n, fam in golden_cases(golden):
        x = golden[key + "__values"]
        ref_img = golden[key + "__image"].tobytes()
        img = orc.encode_block(codec, x)
        if codec == 2:
            img, ref_img = _mask_delta_last_field(img, s, n), _mask_delta_last_field(ref_img, s, n)
        if img != ref_img:
            bad.append(key)
    assert not bad, f"oracle encoder differs from the reference on {len(bad)} cases: {bad[:8]}"


def test_golden_decode_and_random_access(golden, orc):
    for key, codec, s, n, fam in golden_cases(golden):
        x = golden[key + "__values"]
        img = golden[key + "__image"].tobytes()
        # reference bulk decode (including its known bugs) == oracle strict_raw=0 path
        ref_dec = golden[key + "__decoded"] if key + "__decoded" in golden.files else x
        l = img[0]
        if not (codec == 2 and l == TB[s]):  # Delta raw: the reference reads garbage (no raw path)
            got = orc.decode_block(codec, img, n, s, strict_raw=0 if codec != 2 else 1)
            # an l == 8s-1 block is "raw" to the reference's bulk decoder, which then
            # copies n*s bytes starting inside the image and running past its end:
            # only the values that lie inside the image are defined
            m = min(n, (len(img) - 1) // s) if (l == TB[s] - 1 and codec != 2) else n
            assert np.array_equal(got[:m], ref_dec[:m]), key
        # the rule used by this library (raw iff l == 8s) always round-trips
        assert np.array_equal(orc.decode_block(codec, img, n, s, strict_raw=1), x), key
        for k, v in zip(golden[key + "__ra_k"], golden[key + "__ra_v"]):
            assert orc.random_block(codec, img, int(k), s) == int(v) == int(x[k]), (key, k)


def test_reference_bulk_decoder_hazards_are_pinned(golden):
    """The fixtures record where the reference's own bulk decoders are wrong:
    l == 8s-1 blocks (LeCo, FOR, poly) and raw Delta blocks."""
    wrong = [k[: -len("__decoded")] for k in golden.files if k.endswith("__decoded") and not k.startswith("varlen")]
    assert wrong, "expected the l == 8s-1 / Delta-raw hazards in the fixtures"
    for key in wrong:
        img = golden[key + "__image"]
        s = 4 if "_u32_" in key else 8
        assert img[0] in (8 * s - 1, 8 * s), key


def test_golden_columns(golden, orc):
    for t, bs in (("u32", 1000), ("u64", 4096)):
        x = golden[f"column_leco_{t}__values"]
        pay, off = orc.encode_column(0, x, bs)
        assert np.array_equal(pay, golden[f"column_leco_{t}__payload"])
        assert np.array_equal(off, golden[f"column_leco_{t}__offsets"])
        assert np.array_equal(orc.decode_column(0, pay, off, len(x), x.dtype.itemsize, bs), x)


def test_golden_varlen_segments(golden, orc):
    x = golden["varlen__values"]
    st, off, pay = golden["varlen__starts"], golden["varlen__offsets"], golden["varlen__payload"]
    ends = list(st[1:]) + [len(x)]
    for i in range(len(st)):
        seg = pay[off[i]:off[i + 1]].tobytes()
        assert orc.varseg_encode(x, int(st[i]), int(ends[i]) - 1) == seg
        assert np.array_equal(orc.varseg_decode(seg, int(ends[i] - st[i])), x[st[i]:ends[i]])
        for g in (int(st[i]), int(ends[i]) - 1):
            assert orc.varseg_random(seg, g) == int(x[g])
    assert np.array_equal(golden["varlen__decoded"], x)


@pytest.mark.parametrize("s", [4, 8])
def test_oracle_matches_compiled_reference_fresh(ref, orc, s):
    rng = np.random.default_rng(77 + s)
    dt = np.uint64 if s == 8 else np.uint32
    for trial in range(40):
        n = int(rng.choice([1, 2, 5, 31, 200, 1000, 2048, 3000]))
        kind = trial % 4
        if kind == 0:
            x = np.sort(rng.integers(0, 2 ** (8 * s - 2), n, dtype=np.uint64)).astype(dt)
        elif kind == 1:
            x = (np.arange(n) * float(rng.uniform(0, 2 ** 20)) + rng.normal(0, 2 ** rng.uniform(0, 14), n) + 2 ** 20).astype(dt)
        elif kind == 2:
            x = rng.integers(0, 2 ** int(rng.integers(1, 8 * s)), n, dtype=np.uint64).astype(dt)
        else:
            x = (2.0 ** (8 * s - 1) + np.cumsum(rng.integers(0, 1000, n))).astype(np.float64).astype(np.uint64).astype(dt)
        for codec in range(4):
            a, b = orc.encode_block(codec, x), ref.encode_block(codec, x)
            if codec == 2:
                a, b = _mask_delta_last_field(a, s, n), _mask_delta_last_field(b, s, n)
            assert a == b, (codec, s, n, kind)


def test_oracle_varlen_matches_reference_partitions(ref, orc):
    rng = np.random.default_rng(9)
    n = 20000
    x = np.cumsum(rng.integers(0, 3000, n)).astype(np.uint64) + np.uint64(10 ** 12)
    st, off, pay, dec = ref.varlen_encode(x, 4, 64)
    assert np.array_equal(dec, x)
    ends = list(st[1:]) + [n]
    for i in range(len(st)):
        assert orc.varseg_encode(x, int(st[i]), int(ends[i]) - 1) == pay[off[i]:off[i + 1]].tobytes()
