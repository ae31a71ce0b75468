"""CPU tier: the oracle's restatement of the reference's legacy u32 codec
piecewise_fix_op_max (headers/piecewise_fix_op_minimize_maxerror.h) against the
reference's own outputs (tests/golden/reference_legacy.npz, made by
tests/golden/gen_legacy_golden.py; and the compiled reference when present).

The reference's bulk decoder accumulates the prediction by addition while its
encoder and random access multiply; its drivers correct the difference with
lists the encoder keeps (experiments/fix_int.cpp:110-117).  The oracle
reproduces the reference's bulk output exactly (add_pred=1) and, with the
multiplied prediction, the stored values (what the library decodes)."""
import os

import numpy as np
import pytest

from conftest import ROOT

FIX = os.path.join(ROOT, "tests", "golden", "reference_legacy.npz")


@pytest.fixture(scope="module")
def fx():
    return np.load(FIX)


def _cases(fx):
    for k in fx.files:
        if k.startswith("legacy_") and k.endswith("__image"):
            yield k[: -len("__image")]


def test_fixtures_pin_the_oracle(fx, orc):
    seen_lists = 0
    for key in _cases(fx):
        x, img = fx[key + "__values"], fx[key + "__image"].tobytes()
        n = len(x)
        ours, dp, dm = orc.legacy_encode_block(x)
        assert ours == img, key
        assert np.array_equal(np.nonzero(dp)[0], fx[key + "__plus"]) and np.array_equal(np.nonzero(dm)[0], fx[key + "__minus"])
        assert np.array_equal(orc.legacy_decode_block(img, n, add_pred=True), fx[key + "__decoded"]), key
        assert np.array_equal(orc.legacy_decode_block(img, n), x), key
        patched = fx[key + "__decoded"].astype(np.int64)
        patched[fx[key + "__plus"]] += 1
        patched[fx[key + "__minus"]] -= 1
        assert np.array_equal(patched.astype(np.uint32), x), key  # the drivers' correction gives the values
        for k, v in zip(fx[key + "__ra_k"], fx[key + "__ra_v"]):
            assert orc.legacy_random(img, int(k)) == int(v) == int(x[k]), (key, k)
        seen_lists += len(fx[key + "__plus"]) + len(fx[key + "__minus"])
    assert seen_lists > 0  # the fixtures contain blocks where the two predictions differ


def test_live_reference(orc, ref):
    rng = np.random.default_rng(31)
    for trial in range(60):
        n = int(rng.choice([3, 500, 4096]))
        i = np.arange(n)
        x = np.clip(np.round(rng.uniform(0, 4e9) + rng.uniform(-3, 3) * i + rng.normal(0, rng.choice([0.5, 50, 5e5]), n)),
                    0, 2 ** 32 - 1).astype(np.uint32)
        a, ap, am = orc.legacy_encode_block(x)
        b, bp, bm = ref.legacy_encode_block(x)
        assert a == b and np.array_equal(ap, bp) and np.array_equal(am, bm)
        assert np.array_equal(orc.legacy_decode_block(b, n, add_pred=True), ref.legacy_decode_block(b, n))
        for k in rng.integers(0, n, 8):
            assert orc.legacy_random(b, int(k)) == ref.legacy_random(b, int(k))
