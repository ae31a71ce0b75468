"""Generates tests/golden/reference_filters.npz from the UNMODIFIED reference
codec (headers compiled by oracle/Makefile into oracle/_ref/libleco_ref.so):
predicate-pushdown results of Leco_int<T>::filter_range / filter_range_close
and FOR_int<T>::filter_range / filter_range_close, one call per block as the
filter experiments make them (experiments/leco_int_fix_template.cpp:216-326,
experiments/FOR_int_fix_template.cpp:226-322).

Run where the reference sources exist:  python tests/golden/gen_filter_golden.py

Per column (key prefix c<i>): values, block size, codec, payload, offsets.
Per filter j of a column: the filter arguments, per-block counts and the
per-block output buffers exactly as the reference leaves them (concatenated;
block b's buffer holds counts[b] entries), and for LeCo close-range the
per-block window starts the experiment derives from the block minimum.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
from oracle import Oracle, Reference  # noqa: E402

MAX_WINDOWS = 4096


def kinds(n, s, rng):
    dt = np.uint64 if s == 8 else np.uint32
    i = np.arange(n, dtype=np.int64)
    yield "sorted", np.cumsum(rng.integers(0, 3000, n)).astype(dt)
    yield "noisy", (i * 1000 + rng.integers(0, 50000, n)).astype(dt)
    yield "step", ((i // 377) * 10000 + rng.integers(0, 100, n)).astype(dt)
    yield "dec", (10 ** 9 - np.cumsum(rng.integers(0, 3000, n))).astype(dt)
    yield "const", np.full(n, 123456, dt)
    yield "rand", rng.integers(0, 2 ** 30, n).astype(dt)
    yield "halfwidth", rng.integers(0, 2 ** (8 * s - 2), n, dtype=np.uint64).astype(dt) | dt(2 ** (8 * s - 2))
    yield "slow", (5_000_000 + i // 7 + rng.integers(0, 3, n)).astype(dt)


def main():
    R, O = Reference(), Oracle()
    rng = np.random.default_rng(20240917)
    cases = {}
    ci = 0
    for s in (4, 8):
        for kind, x in kinds(2003, s, rng):
            for codec in (0, 1):
                for bs in (1000, 257):
                    n = len(x)
                    pay, off = R.encode_column(codec, x, bs)
                    nb = len(off) - 1
                    key = f"c{ci}"
                    ci += 1
                    cases[key + "__values"], cases[key + "__payload"], cases[key + "__offsets"] = x, pay, off
                    cases[key + "__meta"] = np.array([s, codec, bs, n], np.int64)
                    zmin = np.array([x[b * bs:(b + 1) * bs].min() for b in range(nb)], np.uint64)
                    top = int(x.max())
                    filters = [("range", int(np.quantile(x, q)), 0, 0) for q in (0.0, 0.5, 0.9)]
                    filters += [("range", 0, 0, 0), ("range", top, 0, 0), ("range", 2 ** (8 * s) - 1, 0, 0)]
                    filters += [("close", 1000, 5000, 10000), ("close", 0, 3000, 7919), ("close", 10, 990, 1000)]
                    for j, (kindf, a, b, base) in enumerate(filters):
                        counts, bufs, w1, w2 = [], [], [], []
                        for blk in range(nb):
                            img = pay[off[blk]:off[blk + 1]].tobytes()
                            ln = min(bs, n - blk * bs)
                            if codec == 0 and img[0] == 8 * s:
                                # a raw LeCo block: the reference's filters read the raw
                                # values as a model (and its close-range loop need not end)
                                counts.append(-1)
                                w1.append(0)
                                w2.append(0)
                                continue
                            if kindf == "range":
                                c, out = R.block_filter(codec, img, ln, s, a, bs, blk)
                            else:
                                f1, f2 = a, b
                                if codec == 0:
                                    f1, f2 = R.close_window_start(int(zmin[blk]), a, b, base, s)
                                w1.append(f1)
                                w2.append(f2)
                                if codec == 0 and O.block_filter_close(codec, img, ln, s, f1, f2, base,
                                                                       max_periods=MAX_WINDOWS)[0] < 0:
                                    # more windows than MAX_WINDOWS: the reference's loop costs
                                    # windows x block length (wide residuals); not run
                                    counts.append(-2)
                                    continue
                                c, out = R.block_filter_close(codec, img, ln, s, f1, f2, base, bs, blk)
                            counts.append(c)
                            bufs.append(out[:c])
                        fk = f"{key}__f{j}"
                        cases[fk + "__args"] = np.array([0 if kindf == "range" else 1, a, b, base], np.uint64)
                        cases[fk + "__counts"] = np.array(counts, np.int64)
                        cases[fk + "__out"] = np.concatenate(bufs + [np.zeros(0, np.uint32)]).astype(np.uint32)
                        if kindf == "close" and codec == 0:
                            cases[fk + "__w1"] = np.array(w1, np.uint64)
                            cases[fk + "__w2"] = np.array(w2, np.uint64)
    out = os.path.join(HERE, "reference_filters.npz")
    np.savez_compressed(out, **cases)
    print(out, os.path.getsize(out), "bytes,", len(cases), "arrays,", ci, "columns")


if __name__ == "__main__":
    main()
