"""Multi-GPU form of the epoch: independent scenarios spread over ranks.

One scenario's epoch does not shard: every step reads the delayed states of
all 26 neighbours, so a spatial split would need a halo exchange of depth
max-delay at every step (src/core/algorithm/estimation/prediction.rs:56-84).
Scenarios are independent (the reference scheduler runs one per thread,
src/scheduler.rs:68-114), so the multi-GPU form assigns whole scenarios to
ranks, one process per GPU, with no collective on the data path. The only
collectives are host-side bookkeeping: the max-over-ranks timing and an
optional gather of per-scenario metrics after the epoch.
"""

from __future__ import annotations

from typing import List, Sequence


def scenario_cost(num_voxels: int, num_steps: int, num_beats: int) -> int:
    """Work of one epoch, proportional to voxel-steps (V * T * B)."""
    return int(num_voxels) * int(num_steps) * int(num_beats)


def shard_scenarios(costs: Sequence[int], world_size: int) -> List[List[int]]:
    """Greedy longest-processing-time assignment of scenarios to ranks.

    Deterministic: ties break on scenario index, then rank. Returns, per rank,
    the sorted indices of its scenarios.
    """
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    load = [0] * world_size
    shards: List[List[int]] = [[] for _ in range(world_size)]
    for i in sorted(range(len(costs)), key=lambda j: (-int(costs[j]), j)):
        r = min(range(world_size), key=lambda k: (load[k], k))
        shards[r].append(i)
        load[r] += int(costs[i])
    return [sorted(s) for s in shards]


def max_over_ranks(value: float) -> float:
    """Max of a host float over all ranks (identity without an initialised process group)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float) -> float:
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gather_metrics(local: dict) -> list:
    """All ranks' {scenario index: metrics} dicts, gathered on every rank (a few KB)."""
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [local]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, local)
    return out
