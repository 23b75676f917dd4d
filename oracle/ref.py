"""ctypes access to the reference FP64 engine ``pgmcore::Engine`` (core/pgm_core.h:47-115) built from
the reference's own sources into ``oracle/_ref/libpgmcore_ref.so`` by ``oracle/Makefile``.

TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline); the CUDA engine never calls it.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "_ref" / "libpgmcore_ref.so"
_lib = None

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def available() -> bool:
    return LIB_PATH.exists()


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(f"{LIB_PATH} not built (make -C oracle)")
        L = ctypes.CDLL(str(LIB_PATH))
        L.ref_create.restype = ctypes.c_void_p
        L.ref_create.argtypes = [ctypes.c_int, _D, _D, _D, ctypes.c_int, _I, _I, _D, ctypes.c_double, ctypes.c_double,
                                 _I, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                 ctypes.c_double, ctypes.c_int]
        L.ref_destroy.argtypes = [ctypes.c_void_p]
        L.ref_compute.restype = ctypes.c_double
        L.ref_compute.argtypes = [ctypes.c_void_p, _D, _D, _D]
        for name in ("ref_terms", "ref_strain", "ref_induced", "ref_permanent"):
            getattr(L, name).argtypes = [ctypes.c_void_p, _D]
        L.ref_iterations.restype = ctypes.c_int
        L.ref_iterations.argtypes = [ctypes.c_void_p]
        L.ref_residual.restype = ctypes.c_double
        L.ref_residual.argtypes = [ctypes.c_void_p]
        L.ref_set_history_key.argtypes = [ctypes.c_void_p, ctypes.c_longlong]
        L.ref_reset_history.argtypes = [ctypes.c_void_p]
        L.ref_field.argtypes = [ctypes.c_void_p, _D, _D, _D, _D, _D]
        L.ref_last_error.restype = ctypes.c_char_p
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(_D)


def _ip(a):
    return a.ctypes.data_as(_I)


class RefEngine:
    """pgmcore::Engine through ctypes.  Arrays are kept alive by the instance."""

    def __init__(self, top, s):
        L = lib()
        self.n = len(top.q)
        self._keep = [np.ascontiguousarray(top.q, np.float64), np.ascontiguousarray(top.radius, np.float64),
                      np.ascontiguousarray(top.alpha, np.float64), np.ascontiguousarray(top.cov_atom, np.int32),
                      np.ascontiguousarray(top.cov_partner, np.int32), np.ascontiguousarray(top.cov_strength, np.float64),
                      np.ascontiguousarray(s.grid, np.int32)]
        q, R, al, ca, cp, cs, g = self._keep
        self.h = L.ref_create(self.n, _dp(q), _dp(R), _dp(al), len(ca), _ip(ca), _ip(cp), _dp(cs), s.cutoff, s.beta,
                              _ip(g), s.order, s.tol, s.max_iter, s.peek, s.predictor, s.ke, int(s.polarizable))
        if not self.h:
            raise ValueError(L.ref_last_error().decode())

    def __del__(self):
        if getattr(self, "h", None):
            lib().ref_destroy(self.h)
            self.h = None

    def compute(self, pos, box, want_forces=True):
        pos = np.ascontiguousarray(pos, np.float64).reshape(-1)
        box = np.ascontiguousarray(box, np.float64).reshape(-1)
        self.forces = np.zeros((self.n, 3)) if want_forces else None
        e = lib().ref_compute(self.h, _dp(pos), _dp(box), _dp(self.forces) if want_forces else None)
        return e

    def terms(self):
        t = np.zeros(5)
        lib().ref_terms(self.h, _dp(t))
        return dict(zip(("direct", "reciprocal", "self", "background", "polarization"), t.tolist()))

    def strain(self):
        s = np.zeros(9)
        lib().ref_strain(self.h, _dp(s))
        return s

    def induced(self):
        m = np.zeros((self.n, 3))
        lib().ref_induced(self.h, _dp(m))
        return m

    def permanent(self):
        m = np.zeros((self.n, 3))
        lib().ref_permanent(self.h, _dp(m))
        return m

    def iterations(self):
        return lib().ref_iterations(self.h)

    def field(self, pos, box, q, d):
        pos = np.ascontiguousarray(pos, np.float64)
        box = np.ascontiguousarray(box, np.float64)
        q = np.ascontiguousarray(q, np.float64)
        d = np.ascontiguousarray(d, np.float64)
        E = np.zeros((self.n, 3))
        lib().ref_field(self.h, _dp(pos), _dp(box), _dp(q), _dp(d), _dp(E))
        return E


def threads_env():
    return int(os.environ.get("OMP_NUM_THREADS", "1"))
