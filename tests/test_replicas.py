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


def _specs():
    from cardiotrust_b200 import scenario as sc

    return [sc.ScenarioSpec(shape=shape, num_steps=steps, num_beats=beats, num_sensors=6, patho_size=2,
                            patho_origin=(1, 1, 1), pulse_onset=1, pulse_sigma_samples=3.0, noise_fraction=0.01,
                            seed=seed)
            for shape, steps, beats, seed in [((4, 4, 3), 40, 1, 1), ((5, 4, 4), 30, 2, 2), ((3, 3, 3), 50, 1, 3),
                                              ((4, 3, 3), 35, 2, 4), ((6, 4, 3), 25, 1, 5)]]


def _epoch_losses(spec):
    """One oracle epoch (f32, reference order, Adam) of the scenario a spec builds: its batch loss and
    the updated gains' checksum."""
    import numpy as np

    import oracle
    from cardiotrust_b200 import scenario as sc

    from conftest import oracle_forward

    oracle.set_threads(1)
    scn = sc.attach_measurements(sc.build(spec), oracle_forward(oracle))
    o = oracle.from_scenario(scn)
    o.run_epoch(oracle.algo(optimizer=1, learning_rate=1e-2, freeze_delays=0),
                beat_order=np.arange(scn.num_beats, dtype=np.int32))
    return {"loss_batch": float(o.loss_batch[0]), "gains_sum": float(np.sum(o.gains.astype(np.float64))),
            "cost": replicas.scenario_cost(scn.num_voxels, scn.num_steps, scn.num_beats)}


def _epoch_worker(rank, world, port, q):
    import datetime
    import sys

    import torch.distributed as dist

    sys.path.insert(0, os.path.dirname(__file__))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        from cardiotrust_b200 import scenario as sc

        specs = _specs()
        costs = [replicas.scenario_cost(sc.voxel_count(s), s.num_steps, s.num_beats) for s in specs]
        mine = replicas.shard_scenarios(costs, world)[rank]
        got = replicas.gather_metrics({i: _epoch_losses(specs[i]) for i in mine})
        q.put((rank, mine, got))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_rank_gloo_scenario_epochs_equal_one_rank():
    """Each of two gloo ranks runs the oracle epoch of its share of five scenarios (greedy balance of
    voxel-steps from the specs' masks); the gathered results equal the one-process run bit for bit."""
    import oracle

    oracle.build()
    want = {i: _epoch_losses(s) for i, s in enumerate(_specs())}
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_epoch_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    shards = {rank: mine for rank, mine, _ in res}
    assert sorted(i for s in shards.values() for i in s) == list(range(len(want)))
    assert all(len(s) > 0 for s in shards.values())
    for _, _, got in res:
        merged = {k: v for d in got for k, v in d.items()}
        assert merged == want
