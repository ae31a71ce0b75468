"""Autotuner for the batch engine: block size, threads per block and unroll depth.

Three parameters are tuned per column shape -- (codec, value type, data family,
length bucket):

* values per block (256 .. 16384): the size that gives the smallest encoded
  column; among sizes within 0.5 % of that, the one with the shortest measured
  single-column encode+decode time;
* threads per block G (32, 64, 128, 256): the batch engine runs 256/G blocks
  of a work item side by side in one 256-thread CTA, one group of G threads per
  block (G = 32: one warp per block);
* unroll depth U (1, 2, 4): the decoder writes U 16-byte chunks per thread
  step; the u64 LeCo encoder keeps 2U 16-byte loads in flight per thread.

G and U are chosen by timing a batch pass (encode + decode, replayed as a CUDA
graph) over a batch of columns of that shape for every feasible (G, U) -- a
combination is feasible when the 256/G blocks of an item fit in the ~72 KB of
shared memory that keep three CTAs per SM (the batch encode kernel sizes every
CTA for the largest item) -- keeping the engine's default
(G = 32 for blocks of <= 512 values, else 256; U = 2) unless another is more
than 2 % faster.  The table is produced on a B200 by
``python -m leco_b200.autotune`` (import name of this package) and committed as
``autotune_table.json``; at run time ``pick`` looks a column up, after
``classify`` has put it in a family from a sample of its values.
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
GROUPS = (32, 64, 128, 256)
UNROLLS = (1, 2, 4)
FAMILIES = ("linear", "step", "walk", "uniform")
LEN_BUCKETS = tuple(1 << k for k in range(10, 23, 2))  # 1K .. 4M
BATCH_MAX_SMEM = 200 * 1024  # shared memory one work item may use (leco_batch.cu)
# The batch encode kernel takes the largest item's shared memory for every CTA, so
# the tuner keeps each choice within what the default launch already needs for the
# largest blocks (16384 u32 / 8192 u64 values, ~69 KB): three CTAs per SM.
TUNE_MAX_SMEM = 72 * 1024


def max_block(dtype_bytes: int) -> int:
    """Largest block the batch engine stages in shared memory at 3+ CTAs/SM."""
    return 16384 if dtype_bytes == 4 else 8192


def enc_smem_bytes(bs: int, s: int) -> int:
    """Encoder shared memory of one block (enc_smem_bytes in leco_encode.cuh),
    rounded to 16 bytes as the batch engine lays out its groups."""
    b = 1152 + ((bs // 32 + 9) * 4 + 15) // 16 * 16 + (bs + 31) // 32 * 32 * s + 16
    return (b + 15) // 16 * 16


def feasible(bs: int, s: int, group: int, limit: int = TUNE_MAX_SMEM) -> bool:
    return enc_smem_bytes(bs, s) * (256 // group) <= limit


def default_group(bs: int) -> int:
    return 32 if bs <= 512 else 256


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


def pick(codec: int, dtype_bytes: int, n: int, family: str, table: dict | None = None) -> tuple:
    """(block size, threads per block, unroll depth) for a column shape."""
    t = table or load_table()
    e = t["entries"].get(f"{codec}|{dtype_bytes}|{family}|{length_bucket(n)}", {})
    bs = int(min(e.get("block_size", 4096), max_block(dtype_bytes)))
    g = int(e.get("group_threads", default_group(bs)))
    u = int(e.get("unroll", 2))
    if not feasible(bs, dtype_bytes, g):
        g = default_group(bs)
    return bs, g, u


def pick_block_size(codec: int, dtype_bytes: int, n: int, family: str, table: dict | None = None) -> int:
    return pick(codec, dtype_bytes, n, family, table)[0]


def _time_pass(lc, torch, t, codec, bs, group, unroll, ncols, fit, reps):
    """ms of one batch pass (encode + decode, graph replay) over `ncols` columns
    that share the input tensor `t`; checks the decoded values."""
    b = lc.Batch([(t, codec, bs, group, unroll)] * ncols, fit_mode=fit)
    try:
        b.run_graph(3)
        torch.cuda.synchronize()
        lc.check()
        for c in b.cols:
            assert torch.equal(c.out, t)
        stream = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            b.run_graph(3)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps
    finally:
        b.close()


def tune(device="cuda", seed: int = 11, reps: int = 3, out: str = TABLE, fit: int | None = None) -> dict:
    """Measures every shape on the current GPU and writes the table."""
    import torch

    import leco_b200 as lc
    from leco_b200 import workloads

    fit = lc.FIT_REFERENCE if fit is None else fit
    rng = np.random.default_rng(seed)
    entries = {}
    stream = torch.cuda.current_stream()
    for codec in (lc.LINEAR, lc.FOR, lc.DELTA):
        for s in (4, 8):
            for fam in FAMILIES:
                for nb in LEN_BUCKETS:
                    x = workloads.families(nb, fam, s, rng)
                    t = torch.from_numpy(x.view(np.int64 if s == 8 else np.int32)).to(device)
                    # block size: smallest encoded column, ties by single-column time
                    res = []
                    for bs in BLOCK_SIZES:
                        if bs > max_block(s):
                            continue
                        col = lc.encode(t, codec, bs, fit)
                        out_t = torch.empty_like(t)
                        col.decode(out=out_t)
                        torch.cuda.synchronize()
                        assert torch.equal(out_t, t)
                        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                        e0.record(stream)
                        for _ in range(reps):
                            col = lc.encode(t, codec, bs, fit, payload=col.payload)
                            col.decode(out=out_t)
                        e1.record(stream)
                        torch.cuda.synchronize()
                        res.append((col.nbytes, e0.elapsed_time(e1) / reps, bs))
                    best = min(r[0] for r in res)
                    near = [r for r in res if r[0] <= best * 1.005]
                    nbytes, ms, bs = min(near, key=lambda r: r[1])
                    # threads per block and unroll depth: a batch of columns of this shape
                    ncols = max(1, min(256, (1 << 22) // nb))
                    variants = {}
                    for g in GROUPS:
                        if not feasible(bs, s, g):
                            continue
                        for u in UNROLLS:
                            variants[(g, u)] = _time_pass(lc, torch, t, codec, bs, g, u, ncols, fit, reps)
                    dflt = (default_group(bs), 2)
                    g, u = min(variants, key=variants.get)
                    if variants[(g, u)] > variants[dflt] / 1.02:
                        g, u = dflt
                    entries[f"{codec}|{s}|{fam}|{nb}"] = {
                        "block_size": bs, "group_threads": g, "unroll": u, "ratio": round(nbytes / (nb * s), 5),
                        "ms": round(ms, 4), "batch_columns": ncols, "batch_pass_ms": round(variants[(g, u)], 4),
                        "batch_pass_ms_default": round(variants[dflt], 4),
                        "candidates": {str(r[2]): [round(r[0] / (nb * s), 5), round(r[1], 4)] for r in res},
                        "variants": {f"{vg}x{vu}": round(v, 4) for (vg, vu), v in sorted(variants.items())}}
                    print(f"{codec}|{s}|{fam}|{nb}: bs {bs} G {g} U {u} "
                          f"({variants[(g, u)]:.3f} vs default {variants[dflt]:.3f} ms)", flush=True)
    table = {"method": "block size: smallest encoded size, ties within 0.5 % broken by encode+decode time; "
                       "threads per block and unroll depth: fastest batch pass (encode+decode, CUDA graph) over "
                       "a batch of columns of the shape, the default kept unless another is > 2 % faster "
                       "(CUDA events)",
             "gpu": torch.cuda.get_device_name(), "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()),
             "fit_mode": int(fit), "key": "codec|dtype_bytes|family|length_bucket", "block_sizes": BLOCK_SIZES,
             "groups": GROUPS, "unrolls": UNROLLS, "entries": entries}
    with open(out, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    return table


if __name__ == "__main__":
    import sys

    sys.path.insert(0, os.path.dirname(HERE))
    import leco_b200  # noqa: F401  (registers the package under its import name)

    tab = tune()
    print(len(tab["entries"]), "entries ->", TABLE)
