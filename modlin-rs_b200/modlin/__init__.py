"""Python binding of libmodlin_gpu.so — the B200 modular rank / linear-complexity engine.

Mirrors the modlin crate's library surface (``src/lib.rs:9-14``):

* ``fp``    — ``Field`` (``src/fp.rs:34-114``), ``rank`` (``src/fp.rs:125``),
              ``linear_complexity`` (``src/fp.rs:260``), plus batched and
              device-resident forms;
* ``stats`` — ``corank_prob``, ``corank_tail_pvalue``, ``lc_left_tail_pvalue``,
              ``pretty_p_value`` (``src/stats.rs``);
* ``prng``  — the generators under test (``src/prng.rs``).

Every call goes through the C ABI declared in ``include/modlin.h``; there is no
CPU fallback: if the shared library is missing the import fails.
"""
from __future__ import annotations

import ctypes
import os

from . import _lib
from ._lib import ModlinError, lib, library_path  # noqa: F401
from . import fp, prng, stats, gen, shard  # noqa: F401
from .fp import Field, rank, linear_complexity, rank_batch, lc_batch  # noqa: F401
from .stats import corank_prob, corank_tail_pvalue, lc_left_tail_pvalue, pretty_p_value  # noqa: F401


def kernel_launches() -> int:
    """Kernels this library has launched since it was loaded."""
    return int(lib().modlin_kernel_launches())


def last_trailing_ms() -> float:
    """CUDA-event time of the last rank call's trailing-update kernels."""
    return float(lib().modlin_last_trailing_ms())


def last_trailing_macs() -> float:
    """Modular multiply-adds done by those timed trailing updates."""
    return float(lib().modlin_last_trailing_macs())


def autotune() -> dict:
    """Measure this device's AUTO choices (a few seconds); returns the choices
    and the timings they came from."""
    import json
    buf = ctypes.create_string_buffer(1 << 16)
    rc = lib().modlin_autotune(buf, len(buf))
    if rc != 0:
        raise ModlinError(rc, "autotune: " + buf.value.decode(errors="replace")[-400:])
    return json.loads(buf.value.decode())
