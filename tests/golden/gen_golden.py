"""Generates tests/golden/*.npz from the UNMODIFIED reference codec (the
headers compiled by oracle/Makefile into oracle/_ref/libleco_ref.so).

Run where the reference sources exist:  python tests/golden/gen_golden.py
Each case stores the seeded input values, the reference block image(s), the
reference's bulk-decoded values and random-access values.  The fixtures pin the
oracle restatement and the CUDA library without needing the reference at
test time.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
from oracle import Reference  # noqa: E402

CODECS = {0: "leco", 1: "for", 2: "delta", 3: "poly2"}


def families(n, s, rng):
    dt = np.uint64 if s == 8 else np.uint32
    top = 2 ** 64 if s == 8 else 2 ** 32
    yield "linear", np.clip(np.arange(n) * rng.uniform(1, 1e5) + rng.normal(0, 300, n) + 5000, 0, top / 4).astype(dt)
    yield "quad", np.clip(1e-3 * np.arange(n, dtype=np.float64) ** 2 + rng.normal(0, 50, n) + 1e6, 0, top / 4).astype(dt)
    yield "uniform", rng.integers(0, top, n, dtype=np.uint64).astype(dt)
    yield "const", np.full(n, rng.integers(0, top // 2), dt)
    yield "walk", np.cumsum(rng.geometric(1 / 64, n)).astype(dt)
    yield "near_max", (np.uint64(top - 1) - rng.integers(0, 5000, n, dtype=np.uint64)).astype(dt) if s == 4 else \
        (np.uint64(2 ** 64 - 1) - rng.integers(0, 5000, n, dtype=np.uint64))
    yield "halfwidth", rng.integers(0, top // 2, n, dtype=np.uint64).astype(dt)  # l = 8s-1 blocks
    yield "sorted_keys", (1000 * np.arange(n, dtype=np.uint64) + rng.integers(0, 256, n, dtype=np.uint64)).astype(dt)


def main():
    R = Reference()
    rng = np.random.default_rng(20240601)
    cases = {}
    for s in (4, 8):
        for n in (1, 2, 3, 17, 64, 1000, 4096):
            for fam, x in families(n, s, rng):
                if n == 4096 and fam not in ("linear", "sorted_keys", "halfwidth"):
                    continue
                for codec, cname in CODECS.items():
                    img = R.encode_block(codec, x)
                    dec = R.decode_block(codec, img, n, s)
                    ks = np.unique(np.array([0, n - 1, n // 2, n // 3], dtype=np.int64))
                    ra = np.array([R.random_block(codec, img, int(k), s) for k in ks], dtype=np.uint64)
                    key = f"{cname}_u{8*s}_n{n}_{fam}"
                    cases[key + "__values"] = x
                    cases[key + "__image"] = np.frombuffer(img, np.uint8)
                    if not np.array_equal(dec, x):  # stored only where the reference's bulk decoder is wrong
                        cases[key + "__decoded"] = dec
                    cases[key + "__ra_k"] = ks
                    cases[key + "__ra_v"] = ra
    # one whole column per dtype through the reference driver loop
    x32 = (1000 * np.arange(20000, dtype=np.uint64) + rng.integers(0, 256, 20000, dtype=np.uint64)).astype(np.uint32)
    pay, off = R.encode_column(0, x32, 1000)
    cases["column_leco_u32__values"], cases["column_leco_u32__payload"], cases["column_leco_u32__offsets"] = x32, pay, off
    x64 = np.cumsum(rng.integers(1, 1 << 20, 30000, dtype=np.uint64)).astype(np.uint64)
    pay, off = R.encode_column(0, x64, 4096)
    cases["column_leco_u64__values"], cases["column_leco_u64__payload"], cases["column_leco_u64__offsets"] = x64, pay, off
    # variable-length segments (Leco_cost_merge_double_wo_round<uint64_t>)
    n = 30000
    i = np.arange(n, dtype=np.float64)
    xv = np.where(i < 10000, 5e6 + 37.5 * i, np.where(i < 20000, 5e6 + 375000 + 2e-3 * (i - 10000) ** 2, 5e6 + 700000))
    xv = np.round(xv + rng.normal(0, 40, n)).astype(np.uint64)
    starts, boff, bpay, bdec = R.varlen_encode(xv, 10, 20)
    cases["varlen__values"], cases["varlen__starts"], cases["varlen__offsets"] = xv, starts, boff
    cases["varlen__payload"], cases["varlen__decoded"] = bpay, bdec
    out = os.path.join(HERE, "reference_blocks.npz")
    np.savez_compressed(out, **cases)
    print(out, os.path.getsize(out), "bytes,", len(cases), "arrays")


if __name__ == "__main__":
    main()
