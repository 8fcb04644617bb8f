"""Host logic of the multi-GPU (replica) form, on CPU with gloo, world size 2."""

import os
import socket

import pytest
import torch.multiprocessing as mp

from cardiotrust_b200 import replicas


def test_shard_balances_and_covers():
    costs = [replicas.scenario_cost(v, t, b) for v, t, b in
             [(500, 1000, 1), (30000, 4000, 8), (8000, 2000, 1), (1200, 3000, 2), (20000, 1000, 4)]]
    shards = replicas.shard_scenarios(costs, 2)
    assert sorted(i for s in shards for i in s) == list(range(len(costs)))
    loads = [sum(costs[i] for i in s) for s in shards]
    assert max(loads) - min(loads) <= max(costs)
    assert replicas.shard_scenarios(costs, 2) == shards  # deterministic
    assert replicas.shard_scenarios(costs, 1) == [list(range(len(costs)))]
    assert replicas.shard_scenarios([], 3) == [[], [], []]
    with pytest.raises(ValueError):
        replicas.shard_scenarios(costs, 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        costs = [10, 7, 5, 3, 2, 1]
        mine = replicas.shard_scenarios(costs, world)[rank]
        # each rank "times" its share; the job time is the slowest rank
        t = float(sum(costs[i] for i in mine))
        tmax = replicas.max_over_ranks(t)
        total = replicas.sum_over_ranks(len(mine))
        got = replicas.gather_metrics({i: {"loss": float(i)} for i in mine})
        q.put((rank, mine, tmax, total, got))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_rank_gloo():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    shards = replicas.shard_scenarios([10, 7, 5, 3, 2, 1], world)
    for rank, mine, tmax, total, got in res:
        assert mine == shards[rank]
        assert tmax == max(sum([10, 7, 5, 3, 2, 1][i] for i in s) for s in shards)
        assert total == 6
        merged = {k for d in got for k in d}
        assert merged == set(range(6))
