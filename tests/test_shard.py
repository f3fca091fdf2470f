"""Multi-rank sharding of independent instances (CPU, gloo, world size 2)."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from tamc_b200.shard import gather, partition, restart_seeds


def test_partition_balances_and_covers():
    rng = np.random.default_rng(0)
    costs = rng.integers(1, 100, 257).astype(float)
    for world in (1, 2, 3, 8):
        parts = partition(costs, world)
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(costs)))
        loads = [costs[p].sum() for p in parts]
        assert max(loads) - min(loads) <= costs.max()
    with pytest.raises(ValueError):
        partition(costs, 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, costs, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = partition(costs, world)[rank]
        seeds = restart_seeds(1000, rank, 4)
        res = gather({"rank": rank, "units": mine, "seeds": seeds}, world)
        if rank == 0:
            q.put(res)
    finally:
        dist.destroy_process_group()


def test_two_rank_shard_and_gather():
    costs = [float(c) for c in np.random.default_rng(1).integers(1, 50, 40)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    units = sorted(k for r in res for k in r["units"])
    assert units == list(range(40))
    seeds = [s for r in res for s in r["seeds"]]
    assert len(set(seeds)) == len(seeds)
