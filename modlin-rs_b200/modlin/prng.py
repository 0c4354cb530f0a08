"""``modlin::prng`` over the C ABI (src/prng.rs), kind chosen at run time."""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import check, lib, u64p

KINDS = {"xoroshiro128pp": 0, "mixmax17": 17, "mixmax": 240, "mixmax240": 240, "mixmax256": 256}


class Prng:
    """A generator under test: ``Prng::try_new(seed)`` / ``next_u64``."""

    def __init__(self, kind: str, seed: int):
        err = ctypes.c_int(0)
        self._k = KINDS[kind]
        self._g = lib().modlin_prng_new(self._k, seed, ctypes.byref(err))
        if not self._g:
            check(err.value, f"Prng::try_new({kind}, {seed})")

    @property
    def name(self) -> str:
        return lib().modlin_prng_name(self._k).decode()

    def fill(self, count: int) -> np.ndarray:
        out = np.zeros(count, dtype=np.uint64)
        lib().modlin_prng_fill(self._g, out.ctypes.data_as(u64p), count)
        return out

    def next_u64(self) -> int:
        return int(self.fill(1)[0])

    def fill_device(self, ptr: int, count: int, p: int = 0, stream: int = 0) -> None:
        """The next ``count`` outputs written to device memory at ``ptr``
        (reduced mod ``p`` unless 0); bit-identical to ``fill``."""
        check(lib().modlin_prng_fill_device(self._g, p, ptr, count, stream or None), "prng_fill_device")

    def get_state(self) -> np.ndarray:
        n = lib().modlin_prng_state_words(self._k)
        out = np.zeros(n, dtype=np.uint64)
        check(lib().modlin_prng_get_state(self._g, out.ctypes.data_as(u64p), n), "prng_get_state")
        return out

    def set_state(self, words) -> None:
        a = np.ascontiguousarray(np.asarray(words, dtype=np.uint64))
        check(lib().modlin_prng_set_state(self._g, a.ctypes.data_as(u64p), a.size), "prng_set_state")

    @property
    def handle(self):
        return self._g

    def __del__(self):
        g = getattr(self, "_g", None)
        if g:
            lib().modlin_prng_free(g)
            self._g = None
