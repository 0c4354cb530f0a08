"""Batched jobs sharded over processes (world size 2, gloo, CPU): the
partition covers every job once and balances the work; the gathered results
equal a single process's. The per-job compute here is the CPU oracle (the
GPU batch is covered by the -m gpu tests)."""
import os
import socket

import numpy as np
import pytest

from conftest import M61


def test_lpt_partition_covers_and_balances():
    from modlin.shard import lpt_partition
    rng = np.random.default_rng(3)
    costs = [int(x) ** 3 for x in rng.integers(64, 1025, 500)]
    for world in (1, 2, 3, 8):
        parts = lpt_partition(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)
    assert lpt_partition([], 2) == [[], []]
    assert lpt_partition([5, 5, 5], 2) == lpt_partition([5, 5, 5], 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    for p in (root, os.path.join(root, "modlin-rs_b200"), here):
        if p not in sys.path:
            sys.path.insert(0, p)
    import torch.distributed as dist
    from datetime import timedelta
    import oracle
    from modlin.shard import run_sharded
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        items = []
        for i in range(12):
            n = 20 + 7 * i
            items.append((M61 if i % 2 else 65521, oracle.gen_uniform(M61 if i % 2 else 65521, 100 + i, n * n)))
        seen = []

        def compute(jobs):
            seen.extend(int(round(len(a) ** 0.5)) for _, a in jobs)
            return [oracle.rank(p, a) for p, a in jobs]
        got = run_sharded(items, compute, lambda it: len(it[1]) ** 1.5)
        q.put((rank, got, seen))
    finally:
        dist.destroy_process_group()


def test_run_sharded_gloo_world2(O):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    out = {}
    while not q.empty():
        r, got, seen = q.get()
        out[r] = (got, seen)
    items_want = []
    for i in range(12):
        n = 20 + 7 * i
        p = M61 if i % 2 else 65521
        items_want.append(O.rank(p, O.gen_uniform(p, 100 + i, n * n)))
    assert out[0][0] == items_want and out[1][0] == items_want
    # Each rank computed a disjoint share, together every job.
    assert sorted(out[0][1] + out[1][1]) == sorted(20 + 7 * i for i in range(12))
    assert out[0][1] and out[1][1]
