"""Batched jobs over several GPUs, one process per GPU (torch.distributed).

Independent jobs (the CLI's `reps`, src/main.rs:82 and :152) shard with no
device collective: every process takes a share chosen by longest-processing-
time-first over the estimated work (n^3 for a rank, n^2 for a linear
complexity), runs it as one batched launch on its own GPU, and the results
(one integer per job) are gathered on the host.
"""
from __future__ import annotations

import heapq


def lpt_partition(costs, world: int) -> list[list[int]]:
    """Job indices per rank: jobs in decreasing cost, each to the least loaded
    rank (ties to the lowest rank), so every process ends at about the same
    time. Deterministic: every process computes the same partition."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(p) for p in parts]


def run_sharded(items, compute, cost, group=None) -> list[int]:
    """Results of compute(items) computed in shares over the process group
    (the default group when torch.distributed is initialised, else this
    process alone). `compute` maps a list of jobs to a list of results,
    `cost` estimates one job's work."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return list(compute(list(items)))
    world = dist.get_world_size(group)
    me = dist.get_rank(group)
    parts = lpt_partition([cost(it) for it in items], world)
    mine = parts[me]
    res = list(compute([items[i] for i in mine])) if mine else []
    gathered = [None] * world
    dist.all_gather_object(gathered, (mine, res), group=group)
    out = [None] * len(items)
    for idx, vals in gathered:
        for i, v in zip(idx, vals):
            out[i] = v
    return out


def _side(a) -> int:
    return int(round(len(a) ** 0.5))


def rank_batch_sharded(items, group=None) -> list[int]:
    """modlin.rank_batch over [(p, matrix), ...], sharded over the group."""
    from .fp import rank_batch
    return run_sharded(items, rank_batch, lambda it: _side(it[1]) ** 3, group)


def lc_batch_sharded(items, group=None) -> list[int]:
    """modlin.lc_batch over [(p, sequence), ...], sharded over the group."""
    from .fp import lc_batch
    return run_sharded(items, lc_batch, lambda it: len(it[1]) ** 2, group)
