"""``modlin::stats`` over the C ABI (src/stats.rs)."""
from __future__ import annotations

import ctypes

from ._lib import lib

P_FLOOR = 1e-307  # src/stats.rs:16


def corank_prob(p: int, n: int, d: int) -> float:
    return float(lib().modlin_corank_prob(p, n, d))


def corank_tail_pvalue(p: int, n: int, c: int) -> float:
    return float(lib().modlin_corank_tail_pvalue(p, n, c))


def lc_left_tail_pvalue(p: int, n: int, ell: int) -> float:
    return float(lib().modlin_lc_left_tail_pvalue(p, n, ell))


def pretty_p_value(x: float) -> str:
    buf = ctypes.create_string_buffer(128)
    lib().modlin_pretty_p_value(x, buf, 128)
    return buf.value.decode()
