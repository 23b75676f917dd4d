"""ctypes binding of the C ABI in include/pgm_b200.h (libpgm_b200.so, built in-tree for sm_100a).

There is no fallback: if the library is missing or cannot be loaded, every engine call raises.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libpgm_b200.so"

c_int, c_double, c_void_p, c_longlong, c_long, c_char_p = (ctypes.c_int, ctypes.c_double, ctypes.c_void_p,
                                                          ctypes.c_longlong, ctypes.c_long, ctypes.c_char_p)
P_D = ctypes.POINTER(ctypes.c_double)
P_F = ctypes.POINTER(ctypes.c_float)
P_I = ctypes.POINTER(ctypes.c_int)
P_LL = ctypes.POINTER(ctypes.c_longlong)


class PgmSettings(ctypes.Structure):
    _fields_ = [("cutoff", c_double), ("beta", c_double), ("grid", c_int * 3), ("order", c_int), ("tol", c_double),
                ("max_iter", c_int), ("peek", c_double), ("predictor", c_int), ("ke", c_double), ("device", c_int),
                ("skin", c_double), ("precision", c_int), ("zero_guess", c_int), ("polarizable", c_int),
                ("refine", c_int)]


class PgmTerms(ctypes.Structure):
    _fields_ = [("direct", c_double), ("reciprocal", c_double), ("self", c_double), ("background", c_double),
                ("polarization", c_double), ("gvdw", c_double)]


# name -> (restype, argtypes): every entry point declared in include/pgm_b200.h
SIGNATURES = {
    "pgm_settings_default": (None, [ctypes.POINTER(PgmSettings)]),
    "pgm_last_error": (c_char_p, []),
    "pgm_version": (c_char_p, []),
    "pgm_engine_create": (c_int, [ctypes.POINTER(PgmSettings), ctypes.POINTER(c_void_p)]),
    "pgm_engine_destroy": (None, [c_void_p]),
    "pgm_engine_set_atoms": (c_int, [c_void_p, c_int, P_D, P_D, P_D, P_I, c_int]),
    "pgm_engine_set_covalent": (c_int, [c_void_p, c_int, P_I, P_I, P_D]),
    "pgm_engine_set_candidates": (c_int, [c_void_p, c_int, P_I, P_I, P_I, P_I]),
    "pgm_engine_set_gvdw": (c_int, [c_void_p, c_int, c_double, P_D, P_D, P_D, c_int, P_I, P_I]),
    "pgm_engine_probe_barrier_timeout": (c_int, [c_void_p, P_I, P_D]),
    "pgm_gvdw_series": (c_int, [P_D, c_int]),
    "pgm_engine_compute": (c_int, [c_void_p, P_D, P_D, c_int, P_D, P_D, ctypes.POINTER(PgmTerms)]),
    "pgm_engine_compute_f": (c_int, [c_void_p, P_F, P_D, c_int, P_D, ctypes.POINTER(PgmTerms)]),
    "pgm_engine_forces": (P_D, [c_void_p]),
    "pgm_engine_release_positions": (c_int, [c_void_p]),
    "pgm_engine_launch_device": (c_int, [c_void_p, c_void_p, P_D, c_int, c_void_p, c_int, c_double, c_void_p]),
    "pgm_engine_finish_device": (c_int, [c_void_p, ctypes.POINTER(PgmTerms), P_I]),
    "pgm_engine_wait_device": (c_int, [c_void_p, c_void_p]),
    "pgm_engine_compute_device": (c_int, [c_void_p, c_void_p, P_D, c_int, c_void_p, c_int, c_double, c_void_p,
                                          ctypes.POINTER(PgmTerms)]),
    "pgm_engine_launch_resident": (c_int, [c_void_p, c_void_p, P_D, c_int, c_void_p, c_void_p]),
    "pgm_engine_iterations": (c_int, [c_void_p]),
    "pgm_engine_residual": (c_double, [c_void_p]),
    "pgm_engine_induced_dipoles": (c_int, [c_void_p, P_D]),
    "pgm_engine_permanent_dipoles": (c_int, [c_void_p, P_D]),
    "pgm_engine_reset_history": (c_int, [c_void_p]),
    "pgm_engine_list_builds": (c_long, [c_void_p]),
    "pgm_engine_late_list_checks": (c_long, [c_void_p]),
    "pgm_engine_num_candidates": (c_int, [c_void_p]),
    "pgm_engine_strain": (c_int, [c_void_p, P_D]),
    "pgm_engine_field": (c_int, [c_void_p, P_D, P_D, P_D, P_D, P_D]),
    "pgm_engine_pairs": (c_int, [c_void_p, P_I, P_I, c_longlong, P_LL]),
    "pgm_engine_history_size": (c_longlong, [c_void_p]),
    "pgm_engine_get_history": (c_int, [c_void_p, c_void_p]),
    "pgm_engine_set_history": (c_int, [c_void_p, c_void_p]),
    "pgm_engine_param_grad": (c_int, [c_void_p, P_D, P_D, P_D, P_D]),
    "pgm_engine_evaluate_fixed": (c_int, [c_void_p, P_D, P_D, P_D, c_int, P_D, P_D, ctypes.POINTER(PgmTerms)]),
    "pgm_engine_solve": (c_int, [c_void_p, P_D, P_D, c_double, P_I]),
    "pgm_engine_force_matching_grad": (c_int, [c_void_p, P_D, c_double, P_D, P_D, P_D, P_D, P_D, P_I]),
    "pgm_engine_kernel_launches": (c_int, [c_void_p]),
    "pgm_engine_active_systems": (c_int, [c_void_p, P_I, c_int]),
    "pgm_engine_kernel_times": (c_int, [c_void_p, c_int, P_D]),
    "pgm_engine_kernel_times_cold": (c_int, [c_void_p, c_int, c_void_p, ctypes.c_size_t, P_D]),
    "pgm_engine_time_evaluations": (c_int, [c_void_p, c_int, P_D]),
    "pgm_engine_set_pair_lanes": (c_int, [c_void_p, c_int]),
    "pgm_engine_set_pme_kernels": (c_int, [c_void_p, c_int]),
    "pgm_engine_pme_kernels": (c_int, [c_void_p]),
    "pgm_engine_pair_lanes": (c_int, [c_void_p]),
    "pgm_engine_set_transforms": (c_int, [c_void_p, c_int]),
    "pgm_engine_transforms": (c_int, [c_void_p]),
    "pgm_engine_set_systems": (c_int, [c_void_p, c_int, P_I, P_D, P_D, P_I, P_D, P_D, P_D, P_I, P_I, P_I, P_D]),
    "pgm_engine_compute_batch": (c_int, [c_void_p, P_D, P_D, P_D, P_D, P_D, P_I]),
    "pgm_pair_list_noalloc": (c_int, [c_int, c_void_p, P_D, c_double, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                      P_I]),
}

_lib = None


def load():
    """Loads libpgm_b200.so and declares every entry point; raises if it is missing."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"pgm_b200: {LIB_PATH} is missing; build it with __graft_entry__.build() "
                               "(there is no CPU fallback)")
        lib = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib
