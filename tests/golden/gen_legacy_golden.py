"""Generates tests/golden/reference_legacy.npz from the UNMODIFIED reference's
legacy u32 codec piecewise_fix_op_max (headers/piecewise_fix_op_minimize_maxerror.h,
compiled by oracle/Makefile into oracle/_ref/libleco_ref.so).

Run where the reference sources exist:  python tests/golden/gen_legacy_golden.py

Per block case: the seeded values, the reference block image, the reference's own
bulk decode (decodeArray8, before its drivers' corrections), the encoder's
difference lists (mul_add_diff_set / _minus) and random-access samples.  Plus one
whole column (blocks of 4096) as its drivers lay it out.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
from oracle import Reference  # noqa: E402


def families(n, rng):
    i = np.arange(n, dtype=np.float64)
    yield "slow_slope", 2.5e9 + rng.uniform(1e-3, 1.0) * i + rng.normal(0, 2, n)
    yield "linear", 1e8 + rng.uniform(1, 5e4) * i + rng.normal(0, 300, n)
    yield "decreasing", 4e9 - rng.uniform(1, 1e5) * i + rng.normal(0, 50, n)
    yield "constant", np.full(n, float(rng.integers(0, 2 ** 32)))
    yield "uniform", rng.integers(0, 2 ** 32, n).astype(np.float64)
    yield "half", rng.integers(0, 2 ** 30, n).astype(np.float64)


def main():
    R = Reference()
    rng = np.random.default_rng(20241120)
    cases = {}
    for n in (1, 2, 17, 1000, 4096, 10000):
        for fam, x in families(n, rng):
            x = np.clip(np.round(x), 0, 2 ** 32 - 1).astype(np.uint32)
            img, dp, dm = R.legacy_encode_block(x)
            key = f"legacy_n{n}_{fam}"
            cases[key + "__values"] = x
            cases[key + "__image"] = np.frombuffer(img, np.uint8)
            cases[key + "__decoded"] = R.legacy_decode_block(img, n)
            cases[key + "__plus"] = np.nonzero(dp)[0].astype(np.int64)
            cases[key + "__minus"] = np.nonzero(dm)[0].astype(np.int64)
            ks = np.unique(np.array([0, n - 1, n // 2, n // 3], dtype=np.int64))
            cases[key + "__ra_k"] = ks
            cases[key + "__ra_v"] = np.array([R.legacy_random(img, int(k)) for k in ks], np.uint32)
    # palindromes of 0 and 2^32-1: slope 0, a residual of exactly -2^31 (the
    # reference's abs() leaves it negative, so it does not count toward the width)
    top = np.uint32(2 ** 32 - 1)
    for n in (4, 64, 1000):
        half = np.where(np.arange(n // 2) % 2 == 0, np.uint32(0), top).astype(np.uint32)
        x = np.concatenate([half, half[::-1]])
        img, dp, dm = R.legacy_encode_block(x)
        key = f"legacy_n{n}_wrap"
        cases[key + "__values"] = x
        cases[key + "__image"] = np.frombuffer(img, np.uint8)
        cases[key + "__decoded"] = R.legacy_decode_block(img, n)
        cases[key + "__plus"] = np.nonzero(dp)[0].astype(np.int64)
        cases[key + "__minus"] = np.nonzero(dm)[0].astype(np.int64)
        ks = np.unique(np.array([0, n - 1, n // 2, n // 3], dtype=np.int64))
        cases[key + "__ra_k"] = ks
        cases[key + "__ra_v"] = np.array([R.legacy_random(img, int(k)) for k in ks], np.uint32)
    # a column of blocks of 4096 values (sorted keys with a slow drift: difference lists occur)
    n, bs = 200_003, 4096
    i = np.arange(n, dtype=np.float64)
    x = np.clip(np.round(3e9 + 0.37 * i + 1e-7 * i * i + rng.normal(0, 3, n)), 0, 2 ** 32 - 1).astype(np.uint32)
    imgs = [R.legacy_encode_block(x[b:b + bs])[0] for b in range(0, n, bs)]
    off = np.zeros(len(imgs) + 1, np.uint64)
    off[1:] = np.cumsum([len(m) for m in imgs])
    cases["column__values"], cases["column__payload"] = x, np.frombuffer(b"".join(imgs), np.uint8)
    cases["column__offsets"], cases["column__block_size"] = off, np.array([bs])
    out = os.path.join(HERE, "reference_legacy.npz")
    np.savez_compressed(out, **cases)
    print(out, os.path.getsize(out), "bytes,", len(cases), "arrays")


if __name__ == "__main__":
    main()
