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


# ---- the column-sharded single rank ------------------------------------------

SHARD_CASES = [("uniform", M61, 200, 0), ("planted", M61, 200, 100), ("uniform", 2, 150, 0),
               ("uniform", 65521, 130, 0), ("uniform", M61, 40, 0), ("planted", 97, 170, 120)]


def _case_matrix(O, kind, p, n, L):
    return O.gen_planted(p, L, 9, n * n) if kind == "planted" else O.gen_uniform(p, 9, n * n)


def test_sharded_rank_layout():
    from modlin.shard import local_columns
    for n in (40, 64, 130, 200, 1000):
        for world in (1, 2, 3, 5):
            cols = sorted(c for r in range(world) for c in local_columns(n, r, world))
            assert cols == list(range(n)), (n, world)


def test_sharded_rank_one_process(O):
    import torch
    from modlin.shard import rank_sharded, scatter_columns
    from shard_host_ops import HostOps

    class Counting(HostOps):
        blocks = general = 0

        def block_inverse(self, *a):
            r = super().block_inverse(*a)
            Counting.blocks += r is not None
            return r

        def panel_pivots(self, *a):
            Counting.general += 1
            return super().panel_pivots(*a)

    # Steps taken: block steps on every full panel of the uniform matrix over
    # 2^61-1 and general steps on its ragged last panel; the planted rank-100
    # matrix takes one block step and then general steps on the panels of its
    # rank-36 Schur complement (no gather of the remaining block).
    steps = {("uniform", M61, 200): (3, 1), ("planted", M61, 200): (1, 3), ("uniform", M61, 40): (0, 1)}
    for kind, p, n, L in SHARD_CASES:
        a = _case_matrix(O, kind, p, n, L)
        local = torch.from_numpy(scatter_columns(a, n, 0, 1).view(np.int64))
        Counting.blocks = Counting.general = 0
        assert rank_sharded(p, local, n, ops=Counting(p, O)) == O.rank(p, a, n), (kind, p, n)
        if (kind, p, n) in steps:
            assert (Counting.blocks, Counting.general) == steps[(kind, p, n)], (kind, p, n, Counting.blocks,
                                                                               Counting.general)


def _shard_worker(rank, world, port, q):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    for p in (root, os.path.join(root, "modlin-rs_b200"), here):
        if p not in sys.path:
            sys.path.insert(0, p)
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    import oracle
    from modlin.shard import rank_sharded, scatter_columns
    from shard_host_ops import HostOps
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=120))
    try:
        got = []
        for kind, p, n, L in SHARD_CASES:
            a = _case_matrix(oracle, kind, p, n, L)
            local = torch.from_numpy(scatter_columns(a, n, rank, world).view(np.int64))
            got.append(rank_sharded(p, local, n, ops=HostOps(p, oracle)))
        q.put((rank, got))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_rank_gloo(O, world):
    """Column panels dealt over `world` processes, the panel owner's pivots
    and multipliers broadcast per step (block steps, pivoted general steps,
    look-ahead on the next panel's owner): every process returns the
    oracle's rank."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
    assert all(p.exitcode == 0 for p in procs)
    out = {}
    while not q.empty():
        r, got = q.get()
        out[r] = got
    want = [O.rank(p, _case_matrix(O, kind, p, n, L), n) for kind, p, n, L in SHARD_CASES]
    assert sorted(out) == list(range(world))
    for r in range(world):
        assert out[r] == want, (r, out[r], want)
