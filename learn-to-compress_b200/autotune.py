"""Block-size autotuner for the batch engine.

The tunable per column is the number of values per block (256 .. 16384).  The
table maps a column shape -- (codec, value type, data family, length bucket) --
to the block size that gives the smallest encoded column; among sizes within
0.5 % of that, the one with the shortest measured encode+decode time wins.
The table is produced on a B200 by ``python -m leco_b200.autotune`` (import
name of this package) and committed as ``autotune_table.json``; at run time
``pick_block_size`` looks it up, after ``classify`` has put the column in a
family from a sample of its values.  Threads per CTA are fixed at 256 by the
kernels and are not tuned.
"""
from __future__ import annotations

import json
import math
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = os.path.join(HERE, "autotune_table.json")
BLOCK_SIZES = (256, 512, 1024, 2048, 4096, 8192, 16384)
FAMILIES = ("linear", "step", "walk", "uniform")
LEN_BUCKETS = tuple(1 << k for k in range(10, 23, 2))  # 1K .. 4M


def max_block(dtype_bytes: int) -> int:
    """Largest block the batch engine stages in shared memory at 3+ CTAs/SM."""
    return 16384 if dtype_bytes == 4 else 8192


def length_bucket(n: int) -> int:
    k = max(10, min(22, int(round(math.log2(max(n, 1)) / 2) * 2)))
    return 1 << k


def classify(sample: np.ndarray) -> str:
    """Family of a column from (up to) its first 65536 values.

    step: most first differences are zero; walk: non-decreasing with small
    positive steps; uniform: neighbouring values are uncorrelated; otherwise
    linear (a trend plus noise)."""
    x = np.asarray(sample[:65536], dtype=np.float64)
    if len(x) < 3:
        return "linear"
    d = np.diff(x)
    if np.mean(d == 0) > 0.5:
        return "step"
    if np.all(d >= 0) and np.median(d) < 4096:
        return "walk"
    xc = x - x.mean()
    den = float(np.dot(xc, xc))
    r = float(np.dot(xc[1:], xc[:-1])) / den if den > 0 else 1.0
    if r < 0.5:
        return "uniform"
    return "linear"


_TABLE_CACHE = None


def load_table(path: str = TABLE) -> dict:
    global _TABLE_CACHE
    if _TABLE_CACHE is None:
        with open(path) as f:
            _TABLE_CACHE = json.load(f)
    return _TABLE_CACHE


def pick_block_size(codec: int, dtype_bytes: int, n: int, family: str, table: dict | None = None) -> int:
    t = table or load_table()
    key = f"{codec}|{dtype_bytes}|{family}|{length_bucket(n)}"
    bs = t["entries"].get(key, {}).get("block_size", 4096)
    return int(min(bs, max_block(dtype_bytes)))


def tune(device="cuda", seed: int = 11, reps: int = 3, out: str = TABLE) -> dict:
    """Measures every shape on the current GPU and writes the table."""
    import torch

    import leco_b200 as lc
    from leco_b200 import workloads

    rng = np.random.default_rng(seed)
    entries = {}
    stream = torch.cuda.current_stream()
    for codec in (lc.LINEAR, lc.FOR, lc.DELTA):
        for s in (4, 8):
            for fam in FAMILIES:
                for nb in LEN_BUCKETS:
                    x = workloads.families(nb, fam, s, rng)
                    t = torch.from_numpy(x.view(np.int64 if s == 8 else np.int32)).to(device)
                    res = []
                    for bs in BLOCK_SIZES:
                        if bs > max_block(s):
                            continue
                        col = lc.encode(t, codec, bs, lc.FIT_EXACT)
                        out_t = torch.empty_like(t)
                        col.decode(out=out_t)
                        torch.cuda.synchronize()
                        assert torch.equal(out_t, t)
                        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                        e0.record(stream)
                        for _ in range(reps):
                            col = lc.encode(t, codec, bs, lc.FIT_EXACT, payload=col.payload)
                            col.decode(out=out_t)
                        e1.record(stream)
                        torch.cuda.synchronize()
                        res.append((col.nbytes, e0.elapsed_time(e1) / reps, bs))
                    best = min(r[0] for r in res)
                    near = [r for r in res if r[0] <= best * 1.005]
                    nbytes, ms, bs = min(near, key=lambda r: r[1])
                    entries[f"{codec}|{s}|{fam}|{nb}"] = {
                        "block_size": bs, "ratio": round(nbytes / (nb * s), 5), "ms": round(ms, 4),
                        "candidates": {str(r[2]): [round(r[0] / (nb * s), 5), round(r[1], 4)] for r in res}}
    table = {"method": "smallest encoded size; ties within 0.5 % broken by encode+decode time (CUDA events)",
             "gpu": torch.cuda.get_device_name(), "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()),
             "key": "codec|dtype_bytes|family|length_bucket", "block_sizes": BLOCK_SIZES, "entries": entries}
    with open(out, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    return table


if __name__ == "__main__":
    import sys

    sys.path.insert(0, os.path.dirname(HERE))
    import leco_b200  # noqa: F401  (registers the package under its import name)

    tab = tune()
    print(len(tab["entries"]), "entries ->", TABLE)
