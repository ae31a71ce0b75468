"""CPU tier: the column container file (leco_container_*) and the import /
export of the reference drivers' per-block byte strings (leco_import_blocks,
leco_export_blocks).  Host-only entry points of the library: no GPU needed.

The reference has no file format (its drivers hold each block as a malloc'ed
byte string, experiments/leco_int_fix_template.cpp:108-127); what is checked
here is that a column survives the file byte for byte, that every kind of
damage is refused before a kernel could see it, and that the per-block strings
round-trip with the reference encoder's own output."""
import os

import numpy as np
import pytest

from gpu_helpers import mask_delta_last_fields

CORRUPT = -3


def _column(orc, codec, s, n=20011, bs=1000, seed=0):
    rng = np.random.default_rng(seed)
    dt = np.uint64 if s == 8 else np.uint32
    x = (np.cumsum(rng.integers(0, 5000, n)) + 12345).astype(dt)
    pay, off = orc.encode_column(codec, x, bs)
    return x, pay, off


@pytest.mark.parametrize("codec", [0, 1, 2, 3])
@pytest.mark.parametrize("s", [4, 8])
def test_round_trip(lc, orc, tmp_path, codec, s):
    x, pay, off = _column(orc, codec, s, seed=codec * 10 + s)
    p = str(tmp_path / "c.leco")
    lc.container_write(p, codec, s, 1000, len(x), pay, off)
    assert not os.path.exists(p + ".tmp")
    info, pay2, off2, st = lc.container_read(p)
    assert info == {"codec": codec, "dtype": s, "block_size": 1000, "n": len(x), "nunits": len(off) - 1,
                    "payload_bytes": len(pay), "has_starts": 0}
    assert st is None and np.array_equal(pay2, pay) and np.array_equal(off2, off)
    assert np.array_equal(orc.decode_column(codec, pay2, off2, len(x), s, 1000), x)


def test_variable_length_round_trip(lc, golden, tmp_path):
    pay, off = golden["varlen__payload"], golden["varlen__offsets"]
    st = golden["varlen__starts"].astype(np.uint64)
    n = len(golden["varlen__values"])
    p = str(tmp_path / "v.leco")
    lc.container_write(p, lc.VARLEN, 8, 0, n, pay, off, st)
    info, pay2, off2, st2 = lc.container_read(p)
    assert info["codec"] == lc.VARLEN and info["has_starts"] == 1 and info["nunits"] == len(st)
    assert np.array_equal(pay2, pay) and np.array_equal(off2, off) and np.array_equal(st2, st)


def _damaged(lc, p, q, mutate):
    data = bytearray(open(p, "rb").read())
    mutate(data)
    open(q, "wb").write(bytes(data))
    with pytest.raises(lc.LecoError) as e:
        lc.container_read(q)
    return e.value.code


def test_damage_is_refused(lc, orc, tmp_path):
    x, pay, off = _column(orc, 0, 8)
    p, q = str(tmp_path / "c.leco"), str(tmp_path / "d.leco")
    lc.container_write(p, 0, 8, 1000, len(x), pay, off)
    size = os.path.getsize(p)
    hdr = 64 + 8 * len(off)

    def flip(i):
        def m(d):
            d[i] ^= 0x10
        return m

    assert _damaged(lc, p, q, flip(hdr + len(pay) // 2)) == CORRUPT      # payload byte
    assert _damaged(lc, p, q, flip(64 + 8 * 5)) == CORRUPT               # an offset
    assert _damaged(lc, p, q, flip(24)) == CORRUPT                       # n in the header
    assert _damaged(lc, p, q, flip(0)) == CORRUPT                        # magic
    assert _damaged(lc, p, q, lambda d: d.__delitem__(slice(size - 100, size))) == CORRUPT  # truncated
    assert _damaged(lc, p, q, lambda d: d.__delitem__(slice(40, size))) == CORRUPT          # header only


def test_invalid_block_header_with_valid_checksum_is_refused(lc, orc, tmp_path):
    """A file written from a damaged column carries a valid checksum; the block
    headers are still checked on read."""
    x, pay, off = _column(orc, 0, 8)
    bad = pay.copy()
    bad[int(off[3])] = 200  # block 3's bit width
    p = str(tmp_path / "c.leco")
    lc.container_write(p, 0, 8, 1000, len(x), bad, off)
    with pytest.raises(lc.LecoError) as e:
        lc.container_read(p)
    assert e.value.code == CORRUPT


def test_bad_write_arguments(lc, orc, tmp_path):
    x, pay, off = _column(orc, 0, 8)
    with pytest.raises(lc.LecoError):
        lc.container_write(str(tmp_path / "a"), 0, 8, 500, len(x), pay, off)  # block count != offsets
    with pytest.raises(lc.LecoError):
        lc.container_write(str(tmp_path / "b"), lc.VARLEN, 8, 0, len(x), pay, off)  # varlen without starts


@pytest.mark.parametrize("codec", [0, 1, 2, 3])
def test_import_export_reference_blocks(lc, orc, ref, codec):
    """The reference encoder's per-block strings (as its drivers hold them)
    import to exactly the column the reference's column loop writes, and
    export back to the same strings."""
    rng = np.random.default_rng(7 + codec)
    x = (np.cumsum(rng.integers(0, 3000, 9001)) + 77).astype(np.uint64)
    bs = 512
    blocks = [ref.encode_block(codec, x[i:i + bs]) for i in range(0, len(x), bs)]
    pay, off = lc.import_blocks(blocks)
    rpay, roff = ref.encode_column(codec, x, bs)
    if codec == 2:  # the reference's Delta encoder packs its last field from out-of-bounds memory
        pay, rpay = mask_delta_last_fields(pay, off, 8, len(x), bs), mask_delta_last_fields(rpay, roff, 8, len(x), bs)
    assert np.array_equal(off, roff) and np.array_equal(pay, rpay)
    pay, off = lc.import_blocks(blocks)
    assert lc.export_blocks(pay, off) == blocks
