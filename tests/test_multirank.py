"""CPU tier, world_size 2 over gloo: the multi-GPU sharding logic.  Each rank
encodes its contiguous block range (the codec step here is the oracle -- this
test checks the host-side plumbing, not the kernels), the ranks exchange only
their compressed sizes to place their parts in one column-wide stream, and the
concatenation is byte-identical to encoding the whole column in one process.
Lookups are routed to owning ranks and merged back in order; timing is the
max over ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, outdir):
    import sys

    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import datetime

    import torch.distributed as dist

    from leco_b200 import shard
    from oracle import Oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    orc = Oracle()
    rng = np.random.default_rng(11)
    n, bs = 100_003, 1000
    x = np.cumsum(rng.integers(0, 5000, n)).astype(np.uint64)
    shards = shard.shard_blocks(n, bs, world)
    me = shards[rank]
    pay, off = orc.encode_column(0, x[me.first_value:me.first_value + me.nvalues], bs)
    base, total = shard.global_offsets(len(pay), dist)
    goff = shard.shift_offsets(off[:-1], base)
    np.save(os.path.join(outdir, f"pay{rank}.npy"), pay)
    np.save(os.path.join(outdir, f"off{rank}.npy"), goff)
    # routed lookups: every rank answers its part from its own shard
    idx = rng.integers(0, n, 5000)
    local, where = shard.route_lookups(idx, shards, bs)
    mine = orc.random_column(0, pay, off, 8, bs, local[rank].astype(np.uint64))
    np.save(os.path.join(outdir, f"ans{rank}.npy"), mine)
    np.save(os.path.join(outdir, f"where{rank}.npy"), where[rank])
    t = shard.max_over_ranks(float(rank + 1), dist)
    np.save(os.path.join(outdir, f"t{rank}.npy"), np.array([t, total]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sharded_encode_matches_single_process(tmp_path, orc):
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True, start_method="spawn")
    rng = np.random.default_rng(11)
    n, bs = 100_003, 1000
    x = np.cumsum(rng.integers(0, 5000, n)).astype(np.uint64)
    pay, off = orc.encode_column(0, x, bs)
    cat = np.concatenate([np.load(tmp_path / f"pay{r}.npy") for r in range(world)])
    goff = np.concatenate([np.load(tmp_path / f"off{r}.npy") for r in range(world)] + [np.array([len(cat)], np.uint64)])
    assert np.array_equal(cat, pay)
    assert np.array_equal(goff, off)
    idx = rng.integers(0, n, 5000)
    ans = np.empty(len(idx), np.uint64)
    for r in range(world):
        ans[np.load(tmp_path / f"where{r}.npy")] = np.load(tmp_path / f"ans{r}.npy")
    assert np.array_equal(ans, x[idx])
    for r in range(world):
        t, total = np.load(tmp_path / f"t{r}.npy")
        assert t == world and int(total) == len(pay)


def test_shard_plan_covers_column_exactly():
    from leco_b200 import shard

    for n, bs, world in ((10, 3, 4), (100_003, 1000, 8), (4096, 4096, 2), (1, 16, 3)):
        sh = shard.shard_blocks(n, bs, world)
        assert sum(s.nvalues for s in sh) == n
        assert sum(s.nblocks for s in sh) == (n + bs - 1) // bs
        v = 0
        for s in sh:
            assert s.first_value == v
            v += s.nvalues
        idx = np.arange(n)
        own = shard.owner_of(idx, sh, bs)
        for s in sh:
            assert np.all(own[s.first_value:s.first_value + s.nvalues] == s.rank)
