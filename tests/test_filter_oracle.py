"""CPU tier: the oracle's predicate-pushdown restatement (oracle/leco_oracle.c,
filters) against the reference's own filter results -- the committed fixtures
tests/golden/reference_filters.npz (made by the compiled reference,
tests/golden/gen_filter_golden.py) and, when oracle/_ref is present, the
compiled reference on fresh seeded columns.

Pinned per block: the count and the output buffer exactly as the reference
leaves it (for LeCo close-range that includes its overwriting of earlier
windows' indices, reproduced by the oracle's overwrite mode), and the per-block
window starts of the close-range experiment.  Where the reference has no
defined result the oracle's rule is checked instead against the values:
raw LeCo blocks (the reference reads their values as a model) and FOR blocks of
width 8*sizeof(T)-1 (the reference reads them as raw values)."""
import os

import numpy as np
import pytest

from conftest import ROOT

FIX = os.path.join(ROOT, "tests", "golden", "reference_filters.npz")


@pytest.fixture(scope="module")
def fx():
    return np.load(FIX)


def _columns(fx):
    i = 0
    while f"c{i}__meta" in fx.files:
        yield f"c{i}"
        i += 1


def _truth_close_any_window(v, f1, f2, base):
    """Raw LeCo block rule: a value counts once when it lies in some window
    (f1 + p*base, f2 + p*base), p >= 0."""
    v = v.astype(object)
    return [k for k, y in enumerate(v) if y > f1 and f2 > f1 and ((y - f1 - 1) % base) + 1 < f2 - f1]


def test_filter_fixtures_match_oracle(fx, orc):
    checked = {"ref": 0, "truth": 0}
    for key in _columns(fx):
        s, codec, bs, n = (int(v) for v in fx[key + "__meta"])
        x, pay, off = fx[key + "__values"], fx[key + "__payload"], fx[key + "__offsets"]
        nb = len(off) - 1
        j = 0
        while f"{key}__f{j}__args" in fx.files:
            fk = f"{key}__f{j}"
            kind, a, b, base = (int(v) for v in fx[fk + "__args"])
            counts, outs = fx[fk + "__counts"], fx[fk + "__out"]
            pos = 0
            for blk in range(nb):
                img = pay[off[blk]:off[blk + 1]].tobytes() + b"\0" * 64
                ln = min(bs, n - blk * bs)
                vals = x[blk * bs: blk * bs + ln]
                l = img[0]
                c_ref = int(counts[blk])
                ref_buf = outs[pos:pos + max(c_ref, 0)]
                pos += max(c_ref, 0)
                undefined = (codec == 0 and l == 8 * s) or (codec == 1 and l == 8 * s - 1)
                if kind == 0:
                    got = orc.block_filter(codec, img, ln, s, a, blk * bs)
                    if undefined:
                        assert np.array_equal(got, blk * bs + np.nonzero(vals > a)[0]), (fk, blk)
                        checked["truth"] += 1
                    else:
                        assert np.array_equal(got, ref_buf), (fk, blk)
                        checked["ref"] += 1
                    continue
                f1, f2 = a, b
                if codec == 0:
                    f1, f2 = orc.close_window_start(int(x[blk * bs: blk * bs + ln].min()), a, b, base, s)
                    assert (f1, f2) == (int(fx[fk + "__w1"][blk]), int(fx[fk + "__w2"][blk])) or c_ref == -1, (fk, blk)
                if c_ref == -2:  # too many windows for the reference's loop: the oracle agrees
                    assert orc.block_filter_close(codec, img, ln, s, f1, f2, base, max_periods=4096)[0] == -1
                    continue
                c, buf = orc.block_filter_close(codec, img, ln, s, f1, f2, base, blk * bs, overwrite=True)
                if undefined:
                    if codec == 0:
                        want = _truth_close_any_window(vals, f1, f2, base)
                    else:
                        r = vals.astype(np.uint64) % np.uint64(base)
                        want = list(np.nonzero((r > f1) & (r < f2))[0])
                    assert c == len(want) and list(buf[:c] - blk * bs) == want, (fk, blk)
                    checked["truth"] += 1
                else:
                    assert c == c_ref and np.array_equal(buf[:c], ref_buf), (fk, blk, c, c_ref)
                    checked["ref"] += 1
            j += 1
    assert checked["ref"] > 1000 and checked["truth"] > 10, checked


def test_overwrite_mode_only_changes_the_buffer(fx, orc):
    """Appending windows one after another (the layout the GPU writes) gives the
    same count, and every index the reference's overwritten buffer still shows
    is one of them."""
    for key in _columns(fx):
        s, codec, bs, n = (int(v) for v in fx[key + "__meta"])
        if codec != 0:
            continue
        pay, off = fx[key + "__payload"], fx[key + "__offsets"]
        for j in (6, 7, 8):
            fk = f"{key}__f{j}"
            kind, a, b, base = (int(v) for v in fx[fk + "__args"])
            for blk in range(len(off) - 1):
                img = pay[off[blk]:off[blk + 1]].tobytes()
                if img[0] == 8 * s or int(fx[fk + "__counts"][blk]) < 0:
                    continue
                ln = min(bs, n - blk * bs)
                f1, f2 = int(fx[fk + "__w1"][blk]), int(fx[fk + "__w2"][blk])
                c0, b0 = orc.block_filter_close(0, img, ln, s, f1, f2, base, blk * bs, overwrite=True)
                c1, b1 = orc.block_filter_close(0, img, ln, s, f1, f2, base, blk * bs, overwrite=False)
                assert c0 == c1
                written = set(b1[:c1].tolist())
                assert all(v in written or v == 0 for v in b0[:c0].tolist())


def test_column_drivers_match_reference_live(orc, ref):
    """The two experiment loops (zone-map skip, per-block window starts) over
    whole columns, against the compiled reference, on columns without raw LeCo
    blocks."""
    rng = np.random.default_rng(77)
    for s, dt in ((4, np.uint32), (8, np.uint64)):
        for trial in range(6):
            n = int(rng.integers(1, 30000))
            bs = int(rng.choice([64, 257, 1000, 4096]))
            x = (np.cumsum(rng.integers(0, int(rng.choice([10, 3000, 100000])), n)) + int(rng.integers(0, 10 ** 6))).astype(dt)
            for codec in (0, 1):
                pay, off = ref.encode_column(codec, x, bs)
                if codec == 0 and any(pay[o] == 8 * s for o in off[:-1]):
                    continue
                zmin, zmax = orc.zonemap(codec, pay, off, n, s, bs)
                assert np.array_equal(zmax, [x[i:i + bs].max() for i in range(0, n, bs)])
                for q in (0.0, 0.25, 0.999):
                    f = int(np.quantile(x, q))
                    assert np.array_equal(orc.filter_column(codec, pay, off, n, s, bs, f, zmax),
                                          ref.filter_column(codec, pay, off, n, s, bs, f, zmax))
                base = int(rng.choice([1000, 7919, 65536]))
                f1 = int(rng.integers(0, base // 2))
                f2 = f1 + int(rng.integers(1, base // 2))
                zm = zmin if codec == 0 else None
                if orc.filter_close_column(codec, pay, off, n, s, bs, f1, f2, base, zm, max_periods=4096)[0] < 0:
                    continue
                c0, b0 = orc.filter_close_column(codec, pay, off, n, s, bs, f1, f2, base, zm, overwrite=True)
                c1, b1 = ref.filter_close_column(codec, pay, off, n, s, bs, f1, f2, base, zm)
                assert c0 == c1 and np.array_equal(b0, b1)
