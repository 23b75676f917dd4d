"""Builds the engine library in-tree: pgm-md_b200/libpgm_b200.so (sm_100a, nvcc, cuFFT).

    python pgm-md_b200/build.py            (or __graft_entry__.build())

The library exports the C ABI of include/pgm_b200.h.  It is built for sm_100a only.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libpgm_b200.so"
SOURCES = [CSRC / "engine.cu", CSRC / "capi.cpp"]
HEADERS = sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [ROOT / "include" / "pgm_b200.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def cuda_lib_dir() -> str:
    return str(Path(nvcc()).resolve().parent.parent / "lib64")


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(p.stat().st_mtime > t for p in SOURCES + HEADERS)


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not needs_build():
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "-shared",
           "-o", str(tmp), *map(str, SOURCES), "-lcufft", f"-L{cuda_lib_dir()}",
           f"-Xlinker", f"-rpath,{cuda_lib_dir()}"]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
    tmp.replace(LIB)
    return LIB


if __name__ == "__main__":
    p = build(force="--force" in sys.argv, verbose=True)
    print(p)
