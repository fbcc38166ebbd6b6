"""Instance sharding and the multi-rank host path, as two gloo ranks on CPU."""
import os

import pytest
import torch.multiprocessing as mp

from pyheartsim_b200 import distributed


def test_shard_balances_and_covers():
    costs = [5.0, 1.0, 3.0, 3.0, 2.0, 8.0, 1.0, 4.0]
    parts = distributed.shard(costs, 3)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        costs = [float(c) for c in (7, 3, 5, 2, 9, 4, 6, 1)]
        mine = distributed.shard(costs, world)[rank]
        work = sum(costs[i] for i in mine)
        t = distributed.max_over_ranks(10.0 + rank)
        got = distributed.gather({"rank": rank, "instances": mine, "work": work})
        if rank == 0:
            q.put((t, got))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_shard_max_and_gather():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 2000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    t, got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert t == 11.0                                         # MAX over ranks
    assert sorted(i for g in got for i in g["instances"]) == list(range(8))
    assert abs(got[0]["work"] - got[1]["work"]) <= 9.0
