"""Multi-GPU sharding of LeCo columns: one process per GPU, no data-path
collective.

Blocks (and the columns made of them) are independent, so a column is split
into contiguous block ranges, one per rank; every rank encodes, decodes and
serves its own range.  The only exchanges are small:

* ``global_offsets``: the byte offset of each rank's part of a column-wide
  encoded stream -- an exclusive scan of the per-rank compressed sizes (one
  8-byte all-gather);
* ``max_over_ranks``: the time of a step is the slowest rank's;
* ``route_lookups``: a batch of global indices is split by owning rank
  (host-side), with the permutation that puts the answers back in order.

The reference has no multi-node or multi-device code; its drivers run one
column in one process (experiments/leco_int_fix_template.cpp:63-336).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class Shard:
    rank: int
    first_block: int
    nblocks: int
    first_value: int
    nvalues: int


def shard_blocks(n: int, block_size: int, world: int) -> list:
    """Contiguous block ranges, block counts differing by at most one."""
    nb = (n + block_size - 1) // block_size
    out = []
    b = 0
    for r in range(world):
        cnt = nb // world + (1 if r < nb % world else 0)
        v0 = min(n, b * block_size)
        v1 = min(n, (b + cnt) * block_size)
        out.append(Shard(r, b, cnt, v0, v1 - v0))
        b += cnt
    return out


def owner_of(idx: np.ndarray, shards: list, block_size: int) -> np.ndarray:
    """Rank that owns each global value index."""
    starts = np.array([s.first_block for s in shards], dtype=np.int64)
    blk = np.asarray(idx, dtype=np.int64) // block_size
    return np.searchsorted(starts, blk, side="right") - 1


def route_lookups(idx: np.ndarray, shards: list, block_size: int):
    """Splits global indices by owner.  Returns (per-rank local index arrays,
    per-rank positions in the original batch)."""
    idx = np.asarray(idx, dtype=np.int64)
    own = owner_of(idx, shards, block_size)
    local, where = [], []
    for s in shards:
        pos = np.nonzero(own == s.rank)[0]
        where.append(pos)
        local.append(idx[pos] - s.first_value)
    return local, where


def merge_answers(parts: list, where: list, m: int, dtype) -> np.ndarray:
    out = np.empty(m, dtype=dtype)
    for p, w in zip(parts, where):
        out[w] = p
    return out


def global_offsets(local_bytes: int, dist=None, device=None) -> tuple:
    """(exclusive byte offset of this rank's stream part, total bytes) over all
    ranks -- one all-gather of one 8-byte count per rank."""
    import torch

    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return 0, local_bytes
    world, rank = dist.get_world_size(), dist.get_rank()
    t = torch.tensor([local_bytes], dtype=torch.int64, device=device)
    allv = [torch.zeros(1, dtype=torch.int64, device=device) for _ in range(world)]
    dist.all_gather(allv, t)
    sizes = [int(v.item()) for v in allv]
    return sum(sizes[:rank]), sum(sizes)


def max_over_ranks(value: float, dist=None, device=None) -> float:
    import torch

    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return value
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shift_offsets(offsets: np.ndarray, byte_base: int) -> np.ndarray:
    """A rank's block offsets moved to their place in the column-wide stream."""
    return np.asarray(offsets, dtype=np.uint64) + np.uint64(byte_base)
