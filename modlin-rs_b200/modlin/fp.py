"""``modlin::fp`` over the C ABI: Field, rank, linear_complexity (src/fp.rs)."""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import (Job, LcOpts, PROGRESS, RankOpts, check, lib, szt, u64p)
from ._lib import Field as _CField

KERNELS = {"auto": 0, "plain": 1, "tc": 2}
LC_KERNELS = {"auto": 0, "block": 1, "grid": 2, "cluster": 3}
_NO_PROGRESS = ctypes.cast(None, PROGRESS)


class Field:
    """``Field`` (src/fp.rs:34-114): Barrett reduction modulo a prime p < 2^63."""

    def __init__(self, p: int):
        self._f = _CField()
        check(lib().modlin_field_new(p, ctypes.byref(self._f)), "Field::new")
        self.p = p

    @property
    def safe_batch(self) -> int:
        return int(self._f.safe_batch)

    @property
    def mu(self) -> int:
        return (int(self._f.mu_hi) << 64) | int(self._f.mu_lo)

    def reduce(self, x: int) -> int:
        """src/fp.rs:65-67."""
        return int(lib().modlin_field_reduce(ctypes.byref(self._f), x))

    def reduce_u128(self, t: int) -> int:
        """src/fp.rs:71-79."""
        return int(lib().modlin_field_reduce_u128(ctypes.byref(self._f), (t >> 64) & (2**64 - 1), t & (2**64 - 1)))

    def mul(self, a: int, b: int) -> int:
        """src/fp.rs:93-95 (canonical inputs)."""
        return int(lib().modlin_field_mul(ctypes.byref(self._f), a, b))


def _p(field) -> int:
    return field.p if isinstance(field, Field) else int(field)


def _as_u64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint64).reshape(-1))


def rank(field, m, n: int | None = None, *, kernel: str = "auto", pivot_cols: bool = False,
         check_input: bool = False, progress=None):
    """``fp::rank`` (src/fp.rs:125): rank of the n x n row-major matrix ``m``.

    ``m`` may be any array-like of residues; it is not modified. With
    ``pivot_cols`` the column profile (pivot columns, increasing) is returned
    too.
    """
    a = _as_u64(m)
    if n is None:
        n = int(round(a.size ** 0.5))
    if a.size != n * n:
        raise ValueError(f"matrix has {a.size} entries, expected {n}x{n}")
    opts = RankOpts(KERNELS[kernel], int(check_input))
    out = szt(0)
    pc = np.zeros(max(n, 1), dtype=np.uintp) if pivot_cols else None
    cb = PROGRESS(lambda ctx, done, total: progress(done, total)) if progress else _NO_PROGRESS
    rc = lib().modlin_rank_ex(_p(field), a.ctypes.data_as(u64p), n, ctypes.byref(opts), ctypes.byref(out),
                              pc.ctypes.data_as(ctypes.POINTER(szt)) if pivot_cols else None, cb, None)
    check(rc, "rank")
    r = int(out.value)
    if pivot_cols:
        return r, [int(x) for x in pc[:r]]
    return r


def rank_device(field, ptr: int, n: int, *, kernel: str = "auto", stream: int = 0, pivot_cols: bool = False):
    """Rank of a device-resident n x n matrix at ``ptr`` (clobbered)."""
    opts = RankOpts(KERNELS[kernel], 0)
    out = szt(0)
    pc = np.zeros(max(n, 1), dtype=np.uintp) if pivot_cols else None
    rc = lib().modlin_rank_device(_p(field), ptr, n, ctypes.byref(opts), ctypes.byref(out),
                                  pc.ctypes.data_as(ctypes.POINTER(szt)) if pivot_cols else None, stream or None)
    check(rc, "rank_device")
    r = int(out.value)
    return (r, [int(x) for x in pc[:r]]) if pivot_cols else r


def block_inverse_device(field, src_ptr: int, ld: int, out_ptr: int, stream: int = 0) -> bool:
    """-P^-1 of the 64 x 64 block at ``src_ptr`` (row stride ``ld``) into
    ``out_ptr``; False when P is singular."""
    sing = ctypes.c_int(0)
    check(lib().modlin_block_inverse_device(_p(field), src_ptr, ld, out_ptr, ctypes.byref(sing), stream or None),
          "block_inverse_device")
    return sing.value == 0


def rank_prng(field, gen, n: int, *, kernel: str = "auto", progress=None) -> int:
    """Rank of the next n x n outputs of ``gen`` (a ``prng.Prng``) reduced
    mod p, generated and ranked in device memory (src/main.rs:94-112)."""
    opts = RankOpts(KERNELS[kernel], 0)
    out = szt(0)
    cb = PROGRESS(lambda ctx, done, total: progress(done, total)) if progress else _NO_PROGRESS
    check(lib().modlin_rank_prng(_p(field), gen.handle, n, ctypes.byref(opts), ctypes.byref(out), cb, None),
          "rank_prng")
    return int(out.value)


def rank_prng_batch(field, gen, n: int, reps: int, *, kernel: str = "auto") -> list[int]:
    """Ranks of the next ``reps`` n x n matrices of ``gen``'s outputs reduced
    mod p (the CLI's -R reps loop, src/main.rs:82-125), in batched launches."""
    opts = RankOpts(KERNELS[kernel], 0)
    out = (szt * max(reps, 1))()
    check(lib().modlin_rank_prng_batch(_p(field), gen.handle, n, reps, ctypes.byref(opts), out, _NO_PROGRESS,
                                       None), "rank_prng_batch")
    return [int(out[i]) for i in range(reps)]


def linear_complexity(field, s, *, kernel: str = "auto", grid_ctas: int = 0, check_input: bool = False) -> int:
    """``fp::linear_complexity`` (src/fp.rs:260)."""
    a = _as_u64(s)
    out = szt(0)
    opts = LcOpts(LC_KERNELS[kernel], int(check_input), grid_ctas)
    rc = lib().modlin_linear_complexity_ex(_p(field), a.ctypes.data_as(u64p), a.size, ctypes.byref(opts),
                                           ctypes.byref(out))
    check(rc, "linear_complexity")
    return int(out.value)


def linear_complexity_device(field, ptr: int, n: int, *, kernel: str = "auto", grid_ctas: int = 0,
                             stream: int = 0) -> int:
    out = szt(0)
    opts = LcOpts(LC_KERNELS[kernel], 0, grid_ctas)
    rc = lib().modlin_linear_complexity_device(_p(field), ptr, n, ctypes.byref(opts), ctypes.byref(out),
                                               stream or None)
    check(rc, "linear_complexity_device")
    return int(out.value)


def _jobs(items):
    arrs = [(_p(p), _as_u64(x)) for p, x in items]
    jobs = (Job * max(len(arrs), 1))()
    for i, (p, a) in enumerate(arrs):
        jobs[i] = Job(p, a.ctypes.data_as(u64p), 0)
    return jobs, arrs


def rank_batch(items) -> list[int]:
    """Ranks of ``[(p, matrix), ...]`` (square matrices of any sides)."""
    jobs, arrs = _jobs(items)
    for i, (_, a) in enumerate(arrs):
        jobs[i].n = int(round(a.size ** 0.5))
    out = (szt * max(len(arrs), 1))()
    check(lib().modlin_rank_batch(jobs, len(arrs), out), "rank_batch")
    return [int(out[i]) for i in range(len(arrs))]


def rank_batch_device(ps, ptrs, ns, stream: int = 0, kernel: str = "auto") -> list[int]:
    """Device-resident batch: ``ptrs[i]`` points at an ``ns[i]`` x ``ns[i]``
    matrix mod ``ps[i]`` (clobbered). ``kernel``: "auto" (tuned split),
    "tc" (tensor-core batch kernel) or "plain"."""
    k = len(ptrs)
    P = (ctypes.c_uint64 * max(k, 1))(*ps)
    D = (ctypes.c_void_p * max(k, 1))(*ptrs)
    N = (szt * max(k, 1))(*ns)
    out = (szt * max(k, 1))()
    opts = RankOpts(KERNELS[kernel], 0)
    check(lib().modlin_rank_batch_device_ex(P, D, N, k, ctypes.byref(opts), out, stream or None),
          "rank_batch_device")
    return [int(out[i]) for i in range(k)]


def lc_batch(items) -> list[int]:
    """Linear complexities of ``[(p, sequence), ...]`` in one persistent launch."""
    jobs, arrs = _jobs(items)
    for i, (_, a) in enumerate(arrs):
        jobs[i].n = a.size
    out = (szt * max(len(arrs), 1))()
    check(lib().modlin_lc_batch(jobs, len(arrs), out), "lc_batch")
    return [int(out[i]) for i in range(len(arrs))]


def lc_batch_device(ps, ptrs, ns, stream: int = 0) -> list[int]:
    """Device-resident batch: ``ptrs[i]`` points at ``ns[i]`` residues mod ``ps[i]``."""
    k = len(ptrs)
    P = (ctypes.c_uint64 * k)(*ps)
    D = (ctypes.c_void_p * k)(*ptrs)
    N = (szt * k)(*ns)
    out = (szt * k)()
    check(lib().modlin_lc_batch_device(P, D, N, k, out, stream or None), "lc_batch_device")
    return [int(out[i]) for i in range(k)]


def trailing_update_device(field, c_ptr: int, ldc: int, M: int, N: int, l_ptr: int, u_ptr: int, ldu: int, K: int,
                           *, kernel: str = "tc", stream: int = 0) -> None:
    """C[M x N] -= L[M x K] * U[K x N] mod p on device buffers (L row stride 64)."""
    rc = lib().modlin_trailing_update_device(_p(field), c_ptr, ldc, M, N, l_ptr, u_ptr, ldu, K, KERNELS[kernel],
                                             stream or None)
    check(rc, "trailing_update_device")


class BatchPlan:
    """A device batch of ranks (kind "rank") or linear complexities ("lc"):
    built once, then launched asynchronously (capturable in a CUDA graph) any
    number of times; every launch writes job i's result to the device int64
    array at `out_ptr` (slot i)."""

    def __init__(self, kind: str, ps, ptrs, ns, out_ptr: int):
        self.kind, self.count = kind, len(ptrs)
        k = self.count
        P = (ctypes.c_uint64 * max(k, 1))(*ps)
        D = (ctypes.c_void_p * max(k, 1))(*ptrs)
        N = (szt * max(k, 1))(*ns)
        h = ctypes.c_void_p()
        rc = getattr(lib(), f"modlin_{kind}_batch_plan_new")(P, D, N, k, out_ptr, ctypes.byref(h))
        check(rc, f"{kind}_batch_plan_new")
        self._h = h

    def launch(self, stream: int = 0) -> None:
        check(getattr(lib(), f"modlin_{self.kind}_batch_plan_launch")(self._h, stream or None), "plan_launch")

    def free(self) -> None:
        if getattr(self, "_h", None):
            getattr(lib(), f"modlin_{self.kind}_batch_plan_free")(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def plain_mac_peak(field) -> float:
    """Modular multiply-adds per second of the plain trailing update's inner
    loop alone (shared-memory operands, no global traffic): the plain
    kernel's roofline on this GPU."""
    out = ctypes.c_double(0)
    check(lib().modlin_plain_mac_peak(_p(field), ctypes.byref(out)), "plain_mac_peak")
    return out.value


def panel_pivots_device(field, ptr: int, ld: int, rows: int, W: int, stream: int = 0):
    """Pivot rows and columns (within the panel) of the rows x W device panel
    at ``ptr`` (row stride ``ld``), as the reference's in-panel elimination
    finds them; the panel is not modified."""
    prow = (szt * 64)()
    pcol = (szt * 64)()
    pb = szt(0)
    check(lib().modlin_panel_pivots_device(_p(field), ptr, ld, rows, W, prow, pcol, ctypes.byref(pb),
                                           stream or None), "panel_pivots_device")
    return [int(prow[k]) for k in range(pb.value)], [int(pcol[k]) for k in range(pb.value)]
