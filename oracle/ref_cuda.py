"""ctypes access to the reference GPU engine ``pgmcuda::Engine`` (core/cuda/pgm_cuda.h:47-127), built unchanged
from the reference's own source core/cuda/pgm_cuda.cu into ``oracle/_ref/libpgmcuda_ref.so`` by
``make -C oracle cuda``.

TEST INFRASTRUCTURE ONLY: the reference engine timed beside pgm_b200 on the same GPU in the reference arm of
bench.py.  pgm_b200 never calls it.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "_ref" / "libpgmcuda_ref.so"
_lib = None

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_VP = ctypes.c_void_p


def available() -> bool:
    return LIB_PATH.exists()


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(f"{LIB_PATH} not built (make -C oracle cuda)")
        L = ctypes.CDLL(str(LIB_PATH))
        L.refcuda_last_error.restype = ctypes.c_char_p
        L.refcuda_create.restype = _VP
        L.refcuda_create.argtypes = [ctypes.c_double, ctypes.c_double, _I, ctypes.c_int, ctypes.c_double,
                                     ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                     ctypes.c_double]
        L.refcuda_destroy.argtypes = [_VP]
        L.refcuda_set_atoms.argtypes = [_VP, ctypes.c_int, _D, _D, _D]
        L.refcuda_set_covalent.argtypes = [_VP, ctypes.c_int, _I, _I, _D]
        L.refcuda_compute.argtypes = [_VP, _D, _D, ctypes.c_int, _D, _D, _D]
        L.refcuda_launch_device.argtypes = [_VP, _VP, _D, ctypes.c_int, _VP, ctypes.c_int, ctypes.c_double, _VP]
        L.refcuda_finish_device.argtypes = [_VP, _D]
        L.refcuda_wait_device.argtypes = [_VP, _VP]
        L.refcuda_iterations.restype = ctypes.c_int
        L.refcuda_iterations.argtypes = [_VP]
        L.refcuda_list_builds.restype = ctypes.c_long
        L.refcuda_list_builds.argtypes = [_VP]
        _lib = L
    return _lib


def _check(rc):
    if rc < 0:
        raise RuntimeError("reference pgm_cuda: " + lib().refcuda_last_error().decode())
    return rc


def _dp(a):
    return a.ctypes.data_as(_D)


class RefCudaEngine:
    """The reference GPU engine on one system (its own pair list with a skin, mixed precision, CUDA graph)."""

    def __init__(self, S, tol, predictor=0, peek=0.65, ke=138.935456, device=0, max_iter=200, skin=0.15):
        L = lib()
        grid = np.ascontiguousarray(S.grid, dtype=np.int32)
        self.h = L.refcuda_create(S.cutoff, S.beta, grid.ctypes.data_as(_I), S.order, tol, max_iter, peek,
                                  predictor, ke, device, skin)
        if not self.h:
            raise RuntimeError("reference pgm_cuda: " + L.refcuda_last_error().decode())
        self.n = S.n
        q, R, a = (np.ascontiguousarray(v, dtype=np.float64) for v in (S.q, S.radius, S.alpha))
        _check(L.refcuda_set_atoms(self.h, S.n, _dp(q), _dp(R), _dp(a)))
        ca = np.ascontiguousarray(S.cov_atom, dtype=np.int32)
        cp = np.ascontiguousarray(S.cov_partner, dtype=np.int32)
        cs = np.ascontiguousarray(S.cov_strength, dtype=np.float64)
        _check(L.refcuda_set_covalent(self.h, len(ca), ca.ctypes.data_as(_I), cp.ctypes.data_as(_I), _dp(cs)))
        self.terms = np.zeros(6)

    def compute(self, pos, box, new_step=True):
        """Host positions in; returns (total energy, forces)."""
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        box = np.ascontiguousarray(box, dtype=np.float64)
        f = np.zeros((self.n, 3))
        _check(lib().refcuda_compute(self.h, _dp(pos), _dp(box), int(new_step), _dp(f), None, _dp(self.terms)))
        return float(self.terms[5]), f

    def launch_device(self, posq4_ptr, box, new_step, force_fixed_ptr, stride, fixed_scale, stream_ptr):
        box = np.ascontiguousarray(box, dtype=np.float64)
        _check(lib().refcuda_launch_device(self.h, posq4_ptr, _dp(box), int(new_step), force_fixed_ptr, stride,
                                           fixed_scale, stream_ptr))

    def wait_device(self, stream_ptr):
        _check(lib().refcuda_wait_device(self.h, stream_ptr))

    def finish_device(self):
        """True when done; False when the list was out of date (launch again)."""
        return _check(lib().refcuda_finish_device(self.h, _dp(self.terms))) == 1

    def iterations(self):
        return lib().refcuda_iterations(self.h)

    def list_builds(self):
        return lib().refcuda_list_builds(self.h)

    def close(self):
        if self.h:
            lib().refcuda_destroy(self.h)
            self.h = None
