"""Loader for the in-tree CUDA library (libfvmhd3d_b200.so) and its C-ABI
(include/fvmhd3d_b200.h).  There is no fallback: if the library is missing or
fails to load, every entry point raises."""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
SO_PATH = os.path.join(HERE, "libfvmhd3d_b200.so")

c_int, c_double, c_void_p, c_ll, c_ull, c_float = (ctypes.c_int, ctypes.c_double, ctypes.c_void_p,
                                                   ctypes.c_longlong, ctypes.c_ulonglong, ctypes.c_float)


# int (*)(void *user, double *dt_min): the reduction of fvm_set_reduce
REDUCE_FN = ctypes.CFUNCTYPE(c_int, c_void_p, ctypes.POINTER(c_double))


class FvmParams(ctypes.Structure):
    """Mirror of `struct fvm_params`."""
    _fields_ = [
        ("gamma", c_double),
        ("courant", c_double),
        ("box", c_double * 3),
        ("dtmax", c_double),
        ("eos", c_int),
        ("iso_GM", c_double),
        ("iso_cfac", c_double),
        ("precision", c_int),
        ("static_mesh", c_int),
    ]


# name -> (restype, argtypes); every symbol declared in include/fvmhd3d_b200.h
SIGNATURES = {
    "fvm_create": (c_void_p, [ctypes.POINTER(FvmParams), c_int]),
    "fvm_destroy": (None, [c_void_p]),
    "fvm_last_error": (ctypes.c_char_p, [c_void_p]),
    "fvm_set_mesh": (c_int, [c_void_p, c_int, c_int] + [c_void_p] * 8),
    "fvm_init_problem": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int]),
    "fvm_get_state": (c_int, [c_void_p] + [c_void_p] * 8),
    "fvm_set_state": (c_int, [c_void_p] + [c_void_p] * 7 + [c_ull]),
    "fvm_get_motion": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "fvm_clock": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "fvm_dump_binary": (c_int, [c_void_p, ctypes.c_char_p, c_void_p, c_void_p]),
    "fvm_begin_step": (c_int, [c_void_p]),
    "fvm_slope_limiter": (c_int, [c_void_p]),
    "fvm_compute_update": (c_int, [c_void_p]),
    "fvm_compute_pvel": (c_int, [c_void_p]),
    "fvm_compute_timesteps": (c_int, [c_void_p, c_int, c_void_p]),
    "fvm_collect_results": (c_int, [c_void_p]),
    "fvm_compute_update0": (c_int, [c_void_p]),
    "fvm_compute_reconstruction": (c_int, [c_void_p]),
    "fvm_end_step": (c_int, [c_void_p, c_int]),
    "fvm_step": (c_int, [c_void_p, c_int]),
    "fvm_step_host": (c_int, [c_void_p, c_int, c_ull] + [c_void_p] * 7),
    "fvm_set_positions": (c_int, [c_void_p, c_void_p, c_void_p]),
    "fvm_run": (c_int, [c_void_p, c_int, c_int, c_void_p]),
    "fvm_time": (c_double, [c_void_p]),
    "fvm_tsys_ticks": (c_ull, [c_void_p]),
    "fvm_get_active_faces": (c_int, [c_void_p, c_void_p, c_void_p]),
    "fvm_get_limited_wrec": (c_int, [c_void_p, c_void_p]),
    "fvm_get_step_dU": (c_int, [c_void_p, c_void_p]),
    "fvm_get_dt_list": (c_int, [c_void_p, c_void_p]),
    "fvm_get_counters": (c_int, [c_void_p, c_void_p]),
    "fvm_mlp_set_weights": (c_int, [c_void_p, c_void_p]),
    "fvm_mlp_eval": (c_int, [c_void_p, c_int, c_void_p, c_void_p]),
    "fvm_mlp_eval_counted": (c_int, [c_void_p, c_int, c_int, c_void_p, c_void_p]),
    "fvm_set_flux_surrogate": (c_int, [c_void_p, c_int]),
    "fvm_mlp_get_weights": (c_int, [c_void_p, c_void_p]),
    "fvm_mlp_grad": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "fvm_mlp_train": (c_int, [c_void_p, c_ll, c_void_p, c_void_p, c_void_p, c_int, c_int, c_float, c_ull,
                              c_void_p]),
    "fvm_set_flux_mode": (c_int, [c_void_p, c_int, c_float, c_float, c_float, c_float, c_int, c_int, c_ll]),
    "fvm_mlp_set_norm": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "fvm_learn_stats": (c_int, [c_void_p, c_void_p]),
    "fvm_harvest_count": (c_ll, [c_void_p]),
    "fvm_get_harvest": (c_int, [c_void_p, c_ll, c_void_p, c_void_p]),
    "fvm_autotune": (c_int, [c_void_p, c_int, c_int, c_void_p]),
    "fvm_set_tuning": (c_int, [c_void_p, c_void_p]),
    "fvm_set_fused": (c_int, [c_void_p, c_int]),
    "fvm_fused_step_count": (c_ll, [c_void_p]),
    "fvm_set_list_building": (c_int, [c_void_p, c_int]),
    "fvm_incremental_step_count": (c_ll, [c_void_p]),
    "fvm_set_reduce": (c_int, [c_void_p, REDUCE_FN, c_void_p]),
    "fvm_set_halo": (c_int, [c_void_p, c_void_p]),
    "fvm_compute_flux": (c_int, [c_void_p, c_int] + [c_void_p] * 8),
    "fvm_compute_flux_static": (c_int, [c_void_p, c_int] + [c_void_p] * 8),
    "fvm_last_step_ms": (c_float, [c_void_p]),
    "fvm_stream": (c_void_p, [c_void_p]),
    "fvm_last_step_counts": (c_int, [c_void_p, c_void_p, c_void_p]),
    "fvm_last_adjust_stats": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "fvm_launch_count": (c_ll, [c_void_p]),
    "fvm_set_profiling": (c_int, [c_void_p, c_int]),
    "fvm_fp64_peak": (c_int, [c_void_p, c_void_p]),
    "fvm_kernel_times": (c_int, [c_void_p, c_int, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(c_double),
                                 ctypes.POINTER(c_ll)]),
}

_LIB = None


def lib() -> ctypes.CDLL:
    """The loaded CUDA library; raises if it is not built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(SO_PATH):
            raise RuntimeError(f"{SO_PATH} is missing: build it with __graft_entry__.build() "
                               "(there is no CPU fallback)")
        so = ctypes.CDLL(SO_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(so, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = so
    return _LIB
