"""pgm_b200: periodic pGM electrostatics (energies, forces, virial, induced dipoles) on one NVIDIA B200.

A new engine with the interface of the reference GPU engine pgmcuda::Engine (larryhuang98/pGM-MD,
core/cuda/pgm_cuda.h): hand-written sm_100a CUDA kernels behind the C ABI of include/pgm_b200.h,
reached from Python through ctypes.  The directory name is not a Python identifier; load the package
with ``load_package()`` of ``__graft_entry__`` (or importlib) under the name ``pgm_md_b200``.
"""

from .engine import FP64, MIXED, Engine, PgmArgumentError, PgmError, Result, Settings, Terms  # noqa: F401
from .engine import pair_list_noalloc  # noqa: F401
from . import systems  # noqa: F401

__all__ = ["Engine", "Settings", "Terms", "Result", "PgmError", "PgmArgumentError", "FP64", "MIXED", "systems"]
