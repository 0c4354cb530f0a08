"""Synthetic workloads: uniform residues and planted recurrences (SplitMix64)."""
from __future__ import annotations

import numpy as np

from ._lib import check, lib, u64p


def uniform(p: int, seed: int, count: int) -> np.ndarray:
    out = np.zeros(count, dtype=np.uint64)
    check(lib().modlin_gen_uniform(p, seed, out.ctypes.data_as(u64p), count), "gen_uniform")
    return out


def uniform_device(p: int, seed: int, ptr: int, count: int, stream: int = 0) -> None:
    check(lib().modlin_gen_uniform_device(p, seed, ptr, count, stream or None), "gen_uniform_device")


def planted(p: int, L: int, seed: int, count: int) -> np.ndarray:
    out = np.zeros(count, dtype=np.uint64)
    check(lib().modlin_gen_planted(p, L, seed, out.ctypes.data_as(u64p), count), "gen_planted")
    return out


def reduce_device(p: int, ptr: int, count: int, stream: int = 0) -> None:
    check(lib().modlin_reduce_device(p, ptr, count, stream or None), "reduce_device")


def planted_device(p: int, L: int, seed: int, ptr: int, count: int, stream: int = 0) -> None:
    """Planted order-L recurrence written to device memory (same stream as ``planted``)."""
    check(lib().modlin_gen_planted_device(p, L, seed, ptr, count, stream or None), "gen_planted_device")


def planted_batch_device(ps, Ls, seeds, ptrs, counts, stream: int = 0) -> None:
    """Many planted sequences on the device in one launch."""
    import ctypes
    k = len(ptrs)
    P = (ctypes.c_uint64 * k)(*ps)
    Lz = (ctypes.c_size_t * k)(*Ls)
    S = (ctypes.c_uint64 * k)(*seeds)
    D = (ctypes.c_void_p * k)(*ptrs)
    N = (ctypes.c_size_t * k)(*counts)
    check(lib().modlin_gen_planted_batch_device(P, Lz, S, D, N, k, stream or None), "gen_planted_batch_device")
