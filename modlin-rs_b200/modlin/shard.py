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
# columns, row-major). Step k eliminates panel k on the active rows r0 .. n:
#   * its owner finds the panel's pivots: when the 64 x 64 diagonal block P is
#     invertible its rows and columns are the pivots (a block step);
#     otherwise the reference's in-panel elimination (first nonzero row per
#     column, src/fp.rs:146-178) gives pb <= 64 pivot rows and columns, and
#     P is the pb x pb block they cross, which is invertible;
#   * every process moves the pivot rows to the top of the active rows (the
#     reference's row swaps, src/fp.rs:158-162; none for a block step);
#   * the owner forms the multipliers of the rows below, H = X P^-1 (X: those
#     rows' entries in the pivot columns), and broadcasts H (rows x 64);
#   * every process updates its columns right of panel k:
#       A[rows below, its columns] -= H * A[pivot rows, its columns],
#     the Schur complement, whose rank is the rank of what remains.
# The rank grows by pb per step. Look-ahead: the owner of panel k+1 updates
# that panel first, finds its pivots and multipliers and starts their
# broadcast before the rest of its step-k update, so the next step's chain
# overlaps this step's wide update. Per step the host reads one small header
# (pivot count, block or general, pivot rows); the buffers are allocated once.
# No device-side waits between processes, no TMA multicast.
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
    through the C ABI (modlin_block_inverse_device, modlin_panel_pivots_device,
    modlin_trailing_update_device); local blocks are int64 CUDA tensors
    holding residues. Work is queued on the legacy default stream, so it is
    ordered with torch's default-stream copies and collectives."""

    def __init__(self, p: int):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("DeviceOps needs a CUDA device")
        self.p = p
        self.torch = torch
        self.device = torch.device("cuda", torch.cuda.current_device())
        self._X = None
        self._P = None

    def zeros(self, *shape):
        return self.torch.zeros(shape, dtype=self.torch.int64, device=self.device)

    def _xbuf(self, rows):
        if self._X is None or self._X.shape[0] < rows:
            self._X = self.zeros(max(rows, 1), PANEL)
        return self._X[:rows]

    def block_inverse(self, local, r0: int, c0: int):
        """-P^-1 of P = local[r0:r0+64, c0:c0+64] (64 x 64), or None if singular."""
        from .fp import block_inverse_device
        if self._P is None:
            self._P = self.zeros(2, PANEL * PANEL)
        V = self._P[0]
        ld = local.shape[1]
        ok = block_inverse_device(self.p, local.data_ptr() + 8 * (r0 * ld + c0), ld, V.data_ptr())
        return V if ok else None

    def panel_pivots(self, local, r0: int, c0: int, W: int):
        """Pivot rows (relative to r0) and columns (within the panel) of
        local[r0:, c0:c0+W]."""
        from .fp import panel_pivots_device
        ld = local.shape[1]
        return panel_pivots_device(self.p, local.data_ptr() + 8 * (r0 * ld + c0), ld, local.shape[0] - r0, W)

    def sub_inverse(self, local, rows, cols):
        """-P^-1 embedded in 64 x 64 ([[P, 0], [0, I]]) for P = local[rows][:, cols]."""
        from .fp import block_inverse_device
        t = self.torch
        pb = len(rows)
        P = self.zeros(PANEL, PANEL)
        P[pb:, pb:] = t.eye(PANEL - pb, dtype=t.int64, device=self.device)
        ri = t.tensor(rows, device=self.device)
        ci = t.tensor(cols, device=self.device)
        P[:pb, :pb] = local.index_select(0, ri).index_select(1, ci)
        V = self._P[1] if self._P is not None else self.zeros(PANEL * PANEL)
        if not block_inverse_device(self.p, P.data_ptr(), PANEL, V.data_ptr()):
            raise RuntimeError("pivot block of a panel is singular")
        return V

    def multipliers(self, local, r0: int, rows_below, cols, V, out):
        """out[:m] = X P^-1 = 0 - X (-P^-1), X = local[rows_below][:, cols]
        padded to 64 columns; rows_below is a range (block step) or a list."""
        from .fp import trailing_update_device
        t = self.torch
        m = len(rows_below)
        X = self._xbuf(m)
        if isinstance(rows_below, range) and len(cols) == PANEL and cols[-1] - cols[0] == PANEL - 1:
            X.copy_(local[rows_below.start:rows_below.stop, cols[0]:cols[0] + PANEL])
        else:
            X.zero_()
            if m:
                ri = t.tensor(list(rows_below), device=self.device)
                ci = t.tensor(cols, device=self.device)
                X[:, :len(cols)] = local.index_select(0, ri).index_select(1, ci)
        H = out[:m]
        H.zero_()
        if m:
            trailing_update_device(self.p, H.data_ptr(), PANEL, m, PANEL, X.data_ptr(), V.data_ptr(), PANEL, PANEL,
                                   kernel="auto")
        return H

    def move_rows(self, local, r0: int, perm):
        """Rows r0.. of local take the order perm (absolute row indices)."""
        t = self.torch
        local[r0:] = local.index_select(0, t.tensor(perm, device=self.device))

    def update(self, local, r0: int, pb: int, c_from: int, c_to: int, H):
        """local[r0+pb:, c_from:c_to] -= H[:, :pb] * local[r0:r0+pb, c_from:c_to]."""
        from .fp import trailing_update_device
        ld = local.shape[1]
        M, N = local.shape[0] - r0 - pb, c_to - c_from
        if M > 0 and N > 0 and pb > 0:
            trailing_update_device(self.p, local.data_ptr() + 8 * ((r0 + pb) * ld + c_from), ld, M, N,
                                   H.data_ptr(), local.data_ptr() + 8 * (r0 * ld + c_from), ld, pb, kernel="auto")


def _factor(ops, local, n, r0, c0, W, out):
    """The owner's part of a step on panel columns c0 .. c0+W of its block:
    (pb, block_step, pivot rows in their new order, H = multipliers of the
    rows below, in the new row order)."""
    rows_active = n - r0
    if rows_active <= 0:
        return 0, True, [], out[:0]
    if W == PANEL and rows_active >= PANEL:
        V = ops.block_inverse(local, r0, c0)
        if V is not None:
            H = ops.multipliers(local, r0, range(r0 + PANEL, n), list(range(c0, c0 + PANEL)), V, out)
            return PANEL, True, list(range(r0, r0 + PANEL)), H
    prow, pcol = ops.panel_pivots(local, r0, c0, W)
    pb = len(prow)
    if pb == 0:
        return 0, False, [], out[:0]
    piv = [r0 + r for r in prow]
    below = [r for r in range(r0, n) if r not in set(piv)]
    V = ops.sub_inverse(local, piv, [c0 + c for c in pcol])
    H = ops.multipliers(local, r0, below, [c0 + c for c in pcol], V, out)
    return pb, False, piv, H


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
    pos = {q: i for i, q in enumerate(mine)}
    npan = (n + PANEL - 1) // PANEL
    width = local.shape[1]

    def src(r):
        return dist.get_global_rank(group, r) if group is not None else r

    def bcast(t, owner):
        if world == 1:
            return None
        return dist.broadcast(t, src=src(owner), group=group, async_op=True)

    # Header: [pb, block step, pivot rows (64)]; two multiplier buffers so
    # that a send can still be in flight while the next step's is formed.
    hdr = [ops.zeros(2 + PANEL) for _ in range(2)]
    Hbuf = [ops.zeros(max(n, 1), PANEL) for _ in range(2)]
    pending = [[], []]  # sends still in flight from each buffer pair

    def lead(k, r0):
        """Owner of panel k: factor it; everyone: exchange its header and
        multipliers. Returns (pb, block, pivot rows, H, H work)."""
        b = k & 1
        for w in pending[b]:
            w.wait()
        pending[b] = []
        owner = panel_owner(k, world)
        if me == owner:
            c0 = PANEL * pos[k]
            pb, block, piv, H = _factor(ops, local, n, r0, c0, panel_width(n, k), Hbuf[b])
            vals = [pb, int(block)] + piv + [0] * (PANEL - len(piv))
            hdr[b].copy_(torch.tensor(vals, dtype=torch.int64))
        w = bcast(hdr[b], owner)
        if w is not None:
            if me == owner:
                pending[b].append(w)
            else:
                w.wait()
        h = hdr[b].tolist()
        pb, block, piv = int(h[0]), bool(h[1]), [int(x) for x in h[2:2 + int(h[0])]]
        rows = n - r0 - pb
        H = Hbuf[b][:max(rows, 0)]
        wh = bcast(H, owner) if pb > 0 and rows > 0 else None
        if me == owner:
            if wh is not None:
                pending[b].append(wh)  # the buffer is reused two steps later
            wh = None
        return pb, block, piv, H, wh

    r0, k = 0, 0
    cur = lead(0, 0) if npan else None
    while k < npan and r0 < n:
        pb, block, piv, H, wh = cur
        if pb > 0 and not block:
            below = [r for r in range(r0, n) if r not in set(piv)]
            ops.move_rows(local, r0, piv + below)
        if wh is not None:
            wh.wait()
        # Local columns right of panel k.
        j0 = sum(1 for q in mine if q <= k)
        c_from = PANEL * j0
        nxt_owner = panel_owner(k + 1, world) if k + 1 < npan else -1
        r1 = r0 + pb
        if nxt_owner == me and pb > 0 and r1 < n:
            # Look-ahead: panel k+1 first, then its factorization and the
            # start of its broadcast, then the rest of this step's update.
            c1 = PANEL * pos[k + 1]
            ops.update(local, r0, pb, c1, c1 + panel_width(n, k + 1), H)
            nxt = lead(k + 1, r1)
            ops.update(local, r0, pb, c1 + panel_width(n, k + 1), width, H)
        else:
            if pb > 0:
                ops.update(local, r0, pb, c_from, width, H)
            nxt = lead(k + 1, r1) if k + 1 < npan and r1 < n else None
        r0, k = r1, k + 1
        cur = nxt
        if cur is None:
            break
    for ws in pending:
        for w in ws:
            w.wait()
    return r0


def scatter_columns(a, n: int, me: int, world: int):
    """This process's local block of the n x n row-major array `a`."""
    import numpy as np
    m = np.asarray(a).reshape(n, n)
    return np.ascontiguousarray(m[:, local_columns(n, me, world)])
