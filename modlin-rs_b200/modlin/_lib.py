"""Loading and prototypes of libmodlin_gpu.so."""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
library_path = os.path.join(os.path.dirname(_HERE), "libmodlin_gpu.so")

u64 = ctypes.c_uint64
u64p = ctypes.POINTER(ctypes.c_uint64)
szt = ctypes.c_size_t
sztp = ctypes.POINTER(ctypes.c_size_t)
vp = ctypes.c_void_p
PROGRESS = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t)

MODLIN_OK = 0
ERRORS = {
    -1: "EINVAL_P", -2: "EINVAL_N", -3: "EINPUT", -4: "ECUDA",
    -5: "ENOMEM", -6: "ETIMEOUT", -7: "ENODEV", -8: "EINVAL_ARG",
}


class ModlinError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        msg = lib().modlin_strerror(code).decode()
        super().__init__(f"{what}: {ERRORS.get(code, code)} ({msg})" if what else f"{ERRORS.get(code, code)} ({msg})")


class Field(ctypes.Structure):
    _fields_ = [("p", u64), ("mu_lo", u64), ("mu_hi", u64), ("safe_batch", u64)]


class RankOpts(ctypes.Structure):
    _fields_ = [("kernel", ctypes.c_int), ("check_input", ctypes.c_int)]


class LcOpts(ctypes.Structure):
    _fields_ = [("kernel", ctypes.c_int), ("check_input", ctypes.c_int), ("grid_ctas", ctypes.c_int)]


class Job(ctypes.Structure):
    _fields_ = [("p", u64), ("data", u64p), ("n", szt)]


_lib = None


def _proto(L, name, res, args):
    fn = getattr(L, name)
    fn.restype = res
    fn.argtypes = args


def lib():
    """The loaded library; raises ImportError when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(library_path):
        raise ImportError(f"{library_path} is missing: build it with `make -C modlin-rs_b200` "
                          "(or __graft_entry__.build()); there is no CPU fallback")
    L = ctypes.CDLL(library_path)
    ci = ctypes.c_int
    _proto(L, "modlin_strerror", ctypes.c_char_p, [ci])
    _proto(L, "modlin_field_new", ci, [u64, ctypes.POINTER(Field)])
    _proto(L, "modlin_field_reduce", u64, [ctypes.POINTER(Field), u64])
    _proto(L, "modlin_field_reduce_u128", u64, [ctypes.POINTER(Field), u64, u64])
    _proto(L, "modlin_field_mul", u64, [ctypes.POINTER(Field), u64, u64])
    _proto(L, "modlin_rank", ci, [u64, u64p, szt, sztp, PROGRESS, vp])
    _proto(L, "modlin_rank_ex", ci, [u64, u64p, szt, ctypes.POINTER(RankOpts), sztp, sztp, PROGRESS, vp])
    _proto(L, "modlin_rank_device", ci, [u64, vp, szt, ctypes.POINTER(RankOpts), sztp, sztp, vp])
    _proto(L, "modlin_trailing_update_device", ci, [u64, vp, szt, szt, szt, vp, vp, szt, szt, ci, vp])
    _proto(L, "modlin_linear_complexity", ci, [u64, u64p, szt, sztp, PROGRESS, vp])
    _proto(L, "modlin_linear_complexity_ex", ci, [u64, u64p, szt, ctypes.POINTER(LcOpts), sztp])
    _proto(L, "modlin_linear_complexity_device", ci, [u64, vp, szt, ctypes.POINTER(LcOpts), sztp, vp])
    _proto(L, "modlin_linear_complexity_device_noalloc", ci, [u64, vp, szt, vp, vp])
    _proto(L, "modlin_rank_batch", ci, [ctypes.POINTER(Job), szt, sztp])
    _proto(L, "modlin_lc_batch", ci, [ctypes.POINTER(Job), szt, sztp])
    _proto(L, "modlin_rank_batch_device", ci, [u64p, ctypes.POINTER(vp), sztp, szt, sztp, vp])
    _proto(L, "modlin_rank_batch_device_ex", ci, [u64p, ctypes.POINTER(vp), sztp, szt, ctypes.POINTER(RankOpts),
                                                  sztp, vp])
    _proto(L, "modlin_lc_batch_device", ci, [u64p, ctypes.POINTER(vp), sztp, szt, sztp, vp])
    for name in ("modlin_corank_prob", "modlin_corank_tail_pvalue", "modlin_lc_left_tail_pvalue"):
        _proto(L, name, ctypes.c_double, [u64, szt, szt])
    _proto(L, "modlin_pretty_p_value", ci, [ctypes.c_double, ctypes.c_char_p, szt])
    _proto(L, "modlin_prng_new", vp, [ci, u64, ctypes.POINTER(ci)])
    _proto(L, "modlin_prng_name", ctypes.c_char_p, [ci])
    _proto(L, "modlin_prng_fill", None, [vp, u64p, szt])
    _proto(L, "modlin_prng_free", None, [vp])
    _proto(L, "modlin_prng_fill_device", ci, [vp, u64, vp, szt, vp])
    _proto(L, "modlin_prng_state_words", szt, [ci])
    _proto(L, "modlin_prng_get_state", ci, [vp, u64p, szt])
    _proto(L, "modlin_prng_set_state", ci, [vp, u64p, szt])
    _proto(L, "modlin_block_inverse_device", ci, [u64, vp, szt, vp, ctypes.POINTER(ci), vp])
    _proto(L, "modlin_rank_prng", ci, [u64, vp, szt, ctypes.POINTER(RankOpts), sztp, PROGRESS, vp])
    _proto(L, "modlin_gen_uniform", ci, [u64, u64, u64p, szt])
    _proto(L, "modlin_gen_uniform_device", ci, [u64, u64, vp, szt, vp])
    _proto(L, "modlin_gen_planted", ci, [u64, szt, u64, u64p, szt])
    _proto(L, "modlin_gen_planted_device", ci, [u64, szt, u64, vp, szt, vp])
    _proto(L, "modlin_gen_planted_batch_device", ci, [u64p, sztp, u64p, ctypes.POINTER(vp), sztp, szt, vp])
    _proto(L, "modlin_reduce_device", ci, [u64, vp, szt, vp])
    _proto(L, "modlin_kernel_launches", u64, [])
    _proto(L, "modlin_testing_grid_timeout_once", ci, [ctypes.c_longlong, ci])
    _proto(L, "modlin_plain_mac_peak", ci, [u64, ctypes.POINTER(ctypes.c_double)])
    _proto(L, "modlin_panel_pivots_device", ci, [u64, vp, szt, szt, szt, sztp, sztp, sztp, vp])
    _proto(L, "modlin_set_tc_pairs", ci, [ci])
    _proto(L, "modlin_rank_prng_batch", ci, [u64, vp, szt, szt, ctypes.POINTER(RankOpts), sztp, PROGRESS, vp])
    _proto(L, "modlin_last_trailing_ms", ctypes.c_double, [])
    _proto(L, "modlin_last_trailing_macs", ctypes.c_double, [])
    _proto(L, "modlin_autotune", ci, [ctypes.c_char_p, szt])
    for kind in ("rank", "lc"):
        _proto(L, f"modlin_{kind}_batch_plan_new", ci, [u64p, ctypes.POINTER(vp), sztp, szt, vp,
                                                        ctypes.POINTER(vp)])
        _proto(L, f"modlin_{kind}_batch_plan_launch", ci, [vp, vp])
        _proto(L, f"modlin_{kind}_batch_plan_free", None, [vp])
    _lib = L
    return L


def check(rc: int, what: str = "") -> None:
    if rc != MODLIN_OK:
        raise ModlinError(rc, what)


# Names every build of the library must export (include/modlin.h).
EXPORTED = [
    "modlin_strerror", "modlin_field_new", "modlin_field_reduce", "modlin_field_reduce_u128",
    "modlin_field_mul", "modlin_rank", "modlin_rank_ex", "modlin_rank_device", "modlin_trailing_update_device",
    "modlin_linear_complexity", "modlin_linear_complexity_ex", "modlin_linear_complexity_device",
    "modlin_linear_complexity_device_noalloc", "modlin_testing_grid_timeout_once", "modlin_plain_mac_peak",
    "modlin_panel_pivots_device", "modlin_rank_prng_batch", "modlin_set_tc_pairs",
    "modlin_rank_batch", "modlin_rank_batch_device", "modlin_rank_batch_device_ex", "modlin_lc_batch", "modlin_lc_batch_device", "modlin_corank_prob",
    "modlin_corank_tail_pvalue", "modlin_lc_left_tail_pvalue", "modlin_pretty_p_value",
    "modlin_prng_new", "modlin_prng_name", "modlin_prng_fill", "modlin_prng_free", "modlin_prng_fill_device",
    "modlin_prng_state_words", "modlin_prng_get_state", "modlin_prng_set_state", "modlin_rank_prng",
    "modlin_block_inverse_device",
    "modlin_gen_uniform", "modlin_gen_uniform_device", "modlin_gen_planted", "modlin_reduce_device",
    "modlin_gen_planted_device", "modlin_gen_planted_batch_device",
    "modlin_kernel_launches", "modlin_last_trailing_ms", "modlin_last_trailing_macs", "modlin_autotune",
    "modlin_rank_batch_plan_new", "modlin_rank_batch_plan_launch", "modlin_rank_batch_plan_free",
    "modlin_lc_batch_plan_new", "modlin_lc_batch_plan_launch", "modlin_lc_batch_plan_free",
]
