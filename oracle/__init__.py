"""CPU oracle (TEST INFRASTRUCTURE ONLY).

ctypes wrapper over ``oracle/liboracle.so``, the plain-C restatement of the
reference crate's ``src/fp.rs``, ``src/stats.rs`` and ``src/prng.rs``.  Only
``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package; the product library never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "liboracle.so")
_lib = None

u64p = ctypes.POINTER(ctypes.c_uint64)
szp = ctypes.POINTER(ctypes.c_size_t)


def build(force: bool = False) -> str:
    """Compile liboracle.so with the committed Makefile (gcc, OpenMP)."""
    if _SO != os.path.join(_HERE, "liboracle.so"):
        return _SO
    if force or not os.path.exists(_SO) or _stale():
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


def use_native(path: str) -> str:
    """Build the oracle with -march=native for the CPU this process runs on
    (the reference's release builds use target-cpu=native) into `path`, and
    load that library from now on. Must be called before the first use."""
    global _SO
    assert _lib is None, "use_native() must come before the oracle is loaded"
    subprocess.run(["make", "-s", "-C", _HERE, "native", f"NATIVE_OUT={path}"], check=True)
    _SO = path
    return path


def _stale() -> bool:
    t = os.path.getmtime(_SO)
    for f in os.listdir(_HERE):
        if f.endswith((".c", ".h")) or f == "Makefile":
            if os.path.getmtime(os.path.join(_HERE, f)) > t:
                return True
    return False


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_SO)
        L.oracle_rank.restype = ctypes.c_size_t
        L.oracle_rank.argtypes = [ctypes.c_uint64, u64p, ctypes.c_size_t, szp, ctypes.c_int]
        L.oracle_rank_naive.restype = ctypes.c_size_t
        L.oracle_rank_naive.argtypes = [ctypes.c_uint64, u64p, ctypes.c_size_t]
        L.oracle_linear_complexity.restype = ctypes.c_size_t
        L.oracle_linear_complexity.argtypes = [ctypes.c_uint64, u64p, ctypes.c_size_t, u64p, u64p]
        L.oracle_lc_naive.restype = ctypes.c_size_t
        L.oracle_lc_naive.argtypes = [ctypes.c_uint64, u64p, ctypes.c_size_t]
        for name in ("oracle_corank_prob", "oracle_corank_tail_pvalue", "oracle_lc_left_tail_pvalue"):
            fn = getattr(L, name)
            fn.restype = ctypes.c_double
            fn.argtypes = [ctypes.c_uint64, ctypes.c_size_t, ctypes.c_size_t]
        L.oracle_pretty_p_value.restype = ctypes.c_int
        L.oracle_pretty_p_value.argtypes = [ctypes.c_double, ctypes.c_char_p, ctypes.c_size_t]
        L.oracle_prng_fill.restype = ctypes.c_int
        L.oracle_prng_fill.argtypes = [ctypes.c_int, ctypes.c_uint64, u64p, ctypes.c_size_t]
        L.oracle_is_prime.restype = ctypes.c_int
        L.oracle_is_prime.argtypes = [ctypes.c_uint64]
        L.oracle_field_new.restype = ctypes.c_int
        L.oracle_reduce_u128_parts.restype = ctypes.c_uint64
        L.oracle_reduce_u128_parts.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64]
        L.oracle_mul.restype = ctypes.c_uint64
        L.oracle_mul.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64]
        for name in ("oracle_mix_rank", "oracle_mix_lc"):
            fn = getattr(L, name)
            fn.restype = ctypes.c_uint64
            fn.argtypes = [ctypes.c_uint64]
        L.oracle_test_rank_case.restype = None
        L.oracle_test_rank_case.argtypes = [ctypes.c_uint64, ctypes.c_size_t, ctypes.c_size_t, u64p, u64p]
        L.oracle_test_lc_random.restype = None
        L.oracle_test_lc_random.argtypes = [ctypes.c_uint64, ctypes.c_size_t, u64p, u64p]
        L.oracle_test_lc_lfsr.restype = None
        L.oracle_test_lc_lfsr.argtypes = [ctypes.c_uint64, ctypes.c_size_t, ctypes.c_size_t, u64p, u64p]
        L.oracle_gen_uniform.restype = None
        L.oracle_gen_uniform.argtypes = [ctypes.c_uint64, u64p, u64p, ctypes.c_size_t]
        L.oracle_gen_planted.restype = None
        L.oracle_gen_planted.argtypes = [ctypes.c_uint64, ctypes.c_size_t, u64p, u64p, ctypes.c_size_t]
        L.oracle_gen_dependent.restype = None
        L.oracle_gen_dependent.argtypes = [ctypes.c_uint64, ctypes.c_size_t, u64p, ctypes.c_size_t, ctypes.c_size_t,
                                           u64p, szp]
        _lib = L
    return _lib


def _u64(a):
    a = np.ascontiguousarray(a, dtype=np.uint64)
    return a, a.ctypes.data_as(u64p)


def rank(p: int, m, n: int | None = None, threads: int = 0, with_pcols: bool = False):
    """Blocked rank (src/fp.rs:125-255) of an n x n matrix; `m` is copied."""
    a = np.array(m, dtype=np.uint64, copy=True).reshape(-1)
    if n is None:
        n = int(round(len(a) ** 0.5))
    assert a.size == n * n
    ptr = a.ctypes.data_as(u64p)
    pc = np.zeros(max(n, 1), dtype=np.uint64) if with_pcols else None
    r = lib().oracle_rank(p, ptr, n, pc.ctypes.data_as(szp) if with_pcols else None, threads)
    if with_pcols:
        return int(r), [int(x) for x in pc[:r]]
    return int(r)


def rank_naive(p: int, m, n: int) -> int:
    """Naive elimination of tests/test_rank.rs:44-72; `m` is copied."""
    a = np.array(m, dtype=np.uint64, copy=True).reshape(-1)
    return int(lib().oracle_rank_naive(p, a.ctypes.data_as(u64p), n))


def linear_complexity(p: int, s, with_macs: bool = False):
    a, ptr = _u64(s)
    d = ctypes.c_uint64(0)
    x = ctypes.c_uint64(0)
    lc = int(lib().oracle_linear_complexity(p, ptr, a.size, ctypes.byref(d), ctypes.byref(x)))
    return (lc, int(d.value), int(x.value)) if with_macs else lc


def lc_naive(p: int, s) -> int:
    a, ptr = _u64(s)
    return int(lib().oracle_lc_naive(p, ptr, a.size))


def corank_prob(p: int, n: int, d: int) -> float:
    return lib().oracle_corank_prob(p, n, d)


def corank_tail_pvalue(p: int, n: int, c: int) -> float:
    return lib().oracle_corank_tail_pvalue(p, n, c)


def lc_left_tail_pvalue(p: int, n: int, ell: int) -> float:
    return lib().oracle_lc_left_tail_pvalue(p, n, ell)


def pretty_p_value(x: float) -> str:
    buf = ctypes.create_string_buffer(512)
    lib().oracle_pretty_p_value(x, buf, 512)
    return buf.value.decode()


PRNG_KINDS = {"xoroshiro128pp": 0, "mixmax17": 17, "mixmax": 240, "mixmax256": 256}


def prng(kind: str, seed: int, count: int) -> np.ndarray:
    out = np.zeros(count, dtype=np.uint64)
    rc = lib().oracle_prng_fill(PRNG_KINDS[kind], seed, out.ctypes.data_as(u64p), count)
    if rc != 0:
        raise ValueError(f"prng {kind} rejected seed {seed} (rc={rc})")
    return out


def is_prime(n: int) -> bool:
    return bool(lib().oracle_is_prime(n))


class _Field(ctypes.Structure):
    _fields_ = [("p", ctypes.c_uint64), ("pad", ctypes.c_uint64), ("mu_lo", ctypes.c_uint64),
                ("mu_hi", ctypes.c_uint64), ("safe_batch", ctypes.c_uint64), ("pad2", ctypes.c_uint64)]


class Field:
    """src/fp.rs:34-114 — Barrett field (reduce_u128 / reduce / mul)."""

    def __init__(self, p: int):
        # oracle_field is {u64 p; u128 mu; u64 safe_batch} with 16-byte alignment.
        self._buf = ctypes.create_string_buffer(64)
        self._ptr = ctypes.addressof(self._buf) + (-ctypes.addressof(self._buf)) % 16
        L = lib()
        L.oracle_field_new.argtypes = [ctypes.c_uint64, ctypes.c_void_p]
        if L.oracle_field_new(p, self._ptr) != 0:
            raise ValueError("modulus must satisfy 2 <= p < 2^63")
        self.p = p

    def reduce_u128(self, t: int) -> int:
        return int(lib().oracle_reduce_u128_parts(self._ptr, (t >> 64) & (2**64 - 1), t & (2**64 - 1)))

    def reduce(self, x: int) -> int:
        return self.reduce_u128(x)

    def mul(self, a: int, b: int) -> int:
        return int(lib().oracle_mul(self._ptr, a, b))

    @property
    def safe_batch(self) -> int:
        raw = ctypes.string_at(self._ptr, 48)
        return int.from_bytes(raw[32:40], "little")


class TestStream:
    """The reference tests' running counter (`seed`, pre-incremented) shared by
    every case of one test function."""

    def __init__(self):
        self._seed = ctypes.c_uint64(0)

    def rank_case(self, p: int, n: int, target: int) -> np.ndarray:
        """tests/test_rank.rs:104-138 — one blocked_matches_reference matrix."""
        a = np.zeros(max(n * n, 1), dtype=np.uint64)
        lib().oracle_test_rank_case(p, n, target, ctypes.byref(self._seed), a.ctypes.data_as(u64p))
        return a[: n * n].reshape(n, n)

    def lc_random(self, p: int, n: int) -> np.ndarray:
        """tests/test_linear_complexity.rs:110 — n random residues."""
        s = np.zeros(max(n, 1), dtype=np.uint64)
        lib().oracle_test_lc_random(p, n, ctypes.byref(self._seed), s.ctypes.data_as(u64p))
        return s[:n]

    def lc_lfsr(self, p: int, k: int, length: int = 150) -> np.ndarray:
        """tests/test_linear_complexity.rs:119-127 — order-k LFSR stream."""
        s = np.zeros(length, dtype=np.uint64)
        lib().oracle_test_lc_lfsr(p, k, length, ctypes.byref(self._seed), s.ctypes.data_as(u64p))
        return s


def gen_uniform(p: int, seed: int, count: int) -> np.ndarray:
    """Uniform residues: top bitlen(p-1) bits of SplitMix64(seed), rejection."""
    st = ctypes.c_uint64(seed)
    out = np.zeros(count, dtype=np.uint64)
    lib().oracle_gen_uniform(p, ctypes.byref(st), out.ctypes.data_as(u64p), count)
    return out


def gen_dependent(p: int, n: int, seed: int, ncols: int, nrows: int):
    """n x n uniform matrix (SplitMix64(seed)) with `ncols` planted dependent
    columns and its last `nrows` rows replaced by combinations of earlier
    rows; returns (matrix as a flat array, sorted planted columns)."""
    st = ctypes.c_uint64(seed)
    out = np.zeros(n * n, dtype=np.uint64)
    dep = np.zeros(max(ncols, 1), dtype=np.uint64)
    lib().oracle_gen_dependent(p, n, ctypes.byref(st), ncols, nrows, out.ctypes.data_as(u64p),
                               dep.ctypes.data_as(szp))
    return out, [int(x) for x in dep[:ncols]]


def gen_planted(p: int, L: int, seed: int, count: int) -> np.ndarray:
    """Planted order-L recurrence stream (coefficients, then initial state)."""
    st = ctypes.c_uint64(seed)
    out = np.zeros(count, dtype=np.uint64)
    lib().oracle_gen_planted(p, L, ctypes.byref(st), out.ctypes.data_as(u64p), count)
    return out
