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


# ---------------------------------------------------------------------------
# One large rank over several GPUs (src/fp.rs:125-255, sharded by columns).
#
# The 64-column panels are dealt block-cyclically: panel k lives on process
# k mod world, each process holding its panels side by side (n rows x its
# columns, row-major). Block step k, as on one GPU: the diagonal block
# P = A[64k .. 64k+64, panel k] is inverted by its owner, which forms the
# multipliers H = X * P^-1 of the rows below (X = those rows' panel entries)
# and broadcasts H (rows x 64 residues) and whether P was invertible; every
# process then updates its own panels right of k:
#     A[rows below, its columns] -= H * A[64k .. 64k+64, its columns].
# The rank grows by 64 per step. When a diagonal block is singular, or fewer
# than 64 rows and columns remain, the remaining block (the Schur complement,
# square) is gathered to process 0 and ranked there by the one-GPU engine,
# which takes the reference's pivoting path; rank(A) = 64k + its rank, the
# same invariant as the one-GPU block steps. One broadcast per step, one
# gather at the end; no device-side waits between processes.
# ---------------------------------------------------------------------------
PANEL = 64


def panel_owner(k: int, world: int) -> int:
    return k % world


def local_panels(n: int, me: int, world: int) -> list[int]:
    """Global panel indices held by process `me`, in local order."""
    npan = (n + PANEL - 1) // PANEL
    return list(range(me, npan, world))


def panel_width(n: int, k: int) -> int:
    return min(PANEL, n - PANEL * k)


def local_columns(n: int, me: int, world: int) -> list[int]:
    """Global column indices of process `me`'s local columns, in order."""
    cols = []
    for k in local_panels(n, me, world):
        cols.extend(range(PANEL * k, PANEL * k + panel_width(n, k)))
    return cols


class DeviceOps:
    """The per-process compute of the sharded rank on this process's GPU,
    through the C ABI (modlin_block_inverse_device, modlin_trailing_update_
    device, modlin_rank_device); local blocks are int64 CUDA tensors holding
    residues. Work is queued on the legacy default stream, so it is ordered
    with torch's default-stream copies and collectives."""

    def __init__(self, p: int):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("DeviceOps needs a CUDA device")
        self.p = p
        self.torch = torch

    def block_inverse(self, local, r0: int, c0: int):
        """-P^-1 of P = local[r0:r0+64, c0:c0+64], or None if P is singular."""
        from .fp import block_inverse_device
        t = self.torch
        V = t.empty(PANEL * PANEL, dtype=t.int64, device=local.device)
        ld = local.shape[1]
        ok = block_inverse_device(self.p, local.data_ptr() + 8 * (r0 * ld + c0), ld, V.data_ptr())
        return V if ok else None

    def multipliers(self, local, r0: int, c0: int, Vneg):
        """H = X * P^-1 = 0 - X * (-P^-1), X = local[r0+64:, c0:c0+64]."""
        from .fp import trailing_update_device
        t = self.torch
        X = local[r0 + PANEL:, c0:c0 + PANEL].contiguous()
        H = t.zeros_like(X)
        if X.shape[0]:
            trailing_update_device(self.p, H.data_ptr(), PANEL, X.shape[0], PANEL, X.data_ptr(), Vneg.data_ptr(),
                                   PANEL, PANEL, kernel="auto")
        return H

    def empty_h(self, rows: int, like):
        return self.torch.empty((rows, PANEL), dtype=self.torch.int64, device=like.device)

    def update(self, local, r0: int, cstart: int, H):
        """local[r0+64:, cstart:] -= H * local[r0:r0+64, cstart:]."""
        from .fp import trailing_update_device
        ld = local.shape[1]
        M, N = local.shape[0] - r0 - PANEL, ld - cstart
        if M > 0 and N > 0:
            trailing_update_device(self.p, local.data_ptr() + 8 * ((r0 + PANEL) * ld + cstart), ld, M, N,
                                   H.data_ptr(), local.data_ptr() + 8 * (r0 * ld + cstart), ld, PANEL, kernel="auto")

    def rank(self, block) -> int:
        """Rank of a square block (clobbered) on this GPU."""
        from .fp import rank_device
        n = block.shape[0]
        block = block.contiguous()
        return rank_device(self.p, block.data_ptr(), n) if n else 0


def rank_sharded(p: int, local, n: int, ops=None, group=None) -> int:
    """Rank of the n x n matrix whose columns are dealt to the processes of
    `group` as local_columns(n, rank, world) describes; `local` is this
    process's n x len(local_columns) block (clobbered). Every process returns
    the rank. `ops` is the per-process compute (DeviceOps(p) by default).
    Without an initialised process group this process holds every column."""
    import torch
    import torch.distributed as dist
    if ops is None:
        ops = DeviceOps(p)
    dist_on = dist.is_available() and dist.is_initialized()
    world = dist.get_world_size(group) if dist_on else 1
    me = dist.get_rank(group) if dist_on else 0
    mine = local_panels(n, me, world)
    npan = (n + PANEL - 1) // PANEL
    dev = local.device

    def bcast(t, src):
        if world > 1:
            dist.broadcast(t, src=dist.get_global_rank(group, src) if group is not None else src, group=group)
        return t

    rank, k = 0, 0
    while k < npan and panel_width(n, k) == PANEL and n - PANEL * k >= PANEL:
        r0 = PANEL * k
        owner = panel_owner(k, world)
        rows = n - r0 - PANEL
        H = None
        flag = torch.zeros(1, dtype=torch.int64, device=dev)
        if me == owner:
            c0 = PANEL * mine.index(k)
            V = ops.block_inverse(local, r0, c0)
            if V is not None:
                flag.fill_(1)
                H = ops.multipliers(local, r0, c0, V)
        bcast(flag, owner)
        if int(flag.item()) == 0:
            break
        if H is None:
            H = ops.empty_h(rows, local)
        if rows:
            bcast(H, owner)
        # This process's panels right of k start at local panel index j0.
        j0 = sum(1 for q in mine if q <= k)
        ops.update(local, r0, PANEL * j0, H)
        rank += PANEL
        k += 1
    # The rest: the square block rows r0.., columns of panels >= k.
    r0 = PANEL * k
    rest = n - r0
    if rest > 0:
        j0 = sum(1 for q in mine if q < k)
        part = local[r0:, PANEL * j0:].contiguous()
        if world > 1:
            widths = [len(local_columns(n, r, world)) - PANEL * sum(1 for q in local_panels(n, r, world) if q < k)
                      for r in range(world)]
            wmax = max(widths)
            pad = torch.zeros((rest, wmax), dtype=torch.int64, device=dev)
            pad[:, :part.shape[1]] = part
            parts = [torch.empty_like(pad) for _ in range(world)] if me == 0 else None
            dst = dist.get_global_rank(group, 0) if group is not None else 0
            dist.gather(pad, parts, dst=dst, group=group)
            if me == 0:
                cols = [parts[r][:, :widths[r]] for r in range(world)]
                # Reassemble global column order: panel q >= k is the next
                # PANEL columns of process q mod world.
                pos = [0] * world
                blocks = []
                for q in range(k, npan):
                    r = panel_owner(q, world)
                    w = panel_width(n, q)
                    blocks.append(cols[r][:, pos[r]:pos[r] + w])
                    pos[r] += w
                block = torch.cat(blocks, dim=1)
        else:
            block = part
        res = torch.zeros(1, dtype=torch.int64, device=dev)
        if me == 0:
            res.fill_(ops.rank(block))
        bcast(res, 0)
        rank += int(res.item())
    return rank


def scatter_columns(a, n: int, me: int, world: int):
    """This process's local block of the n x n row-major array `a`."""
    import numpy as np
    m = np.asarray(a).reshape(n, n)
    return np.ascontiguousarray(m[:, local_columns(n, me, world)])
