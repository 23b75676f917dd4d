"""The C ABI library: it loads, exports every entry point include/pgm_b200.h declares, and rejects bad
arguments with a status and a message (no GPU work here)."""

import ctypes
import re
from pathlib import Path

import pytest

from conftest import PKG, ROOT

HEADER = ROOT / "include" / "pgm_b200.h"


def declared():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(pgm_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from pgm_md_b200 import _lib
    L = _lib.load()
    names = declared()
    assert len(names) >= 30
    for name in names:
        assert hasattr(L, name), name
    assert set(names) == set(_lib.SIGNATURES), set(names) ^ set(_lib.SIGNATURES)


def test_settings_defaults_match_reference():
    """pgm_settings_default gives pgmcuda::Settings' defaults (core/cuda/pgm_cuda.h:25-39)."""
    from pgm_md_b200 import _lib
    s = _lib.PgmSettings()
    _lib.load().pgm_settings_default(ctypes.byref(s))
    assert (s.cutoff, s.beta, tuple(s.grid), s.order, s.tol, s.max_iter, s.peek, s.predictor, s.ke, s.skin) == \
        (0.9, 3.5, (36, 36, 36), 6, 1e-5, 100, 0.65, 2, 138.935458, 0.15)


def test_invalid_order_rejected():
    with pytest.raises(PKG.PgmArgumentError, match="order"):
        PKG.Engine(PKG.Settings(order=2))
    with pytest.raises(PKG.PgmArgumentError, match="order"):
        PKG.Engine(PKG.Settings(order=13))


def test_null_engine_rejected():
    from pgm_md_b200 import _lib
    L = _lib.load()
    assert L.pgm_engine_set_atoms(None, 1, None, None, None, None, 1) == -1
    assert b"null" in L.pgm_last_error()


def test_header_is_plain_c_and_links(tmp_path):
    """include/pgm_b200.h compiles as strict C99 (a cgo / C caller's view), and a C program links the library and
    calls its host-only entry points with the header's struct layout (the Python binding's as well)."""
    import shutil
    import subprocess
    from pgm_md_b200 import _lib
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "caller.c"
    src.write_text(
        '#include "pgm_b200.h"\n#include <stdio.h>\n'
        "int main(void) {\n"
        "    pgm_settings s;\n    pgm_settings_default(&s);\n    double c[15];\n"
        "    const int rc = pgm_gvdw_series(c, 15);\n"
        '    printf("%zu %.17g %d %d %.17g\\n", sizeof(pgm_settings), s.cutoff, s.order, rc, c[1]);\n'
        "    return rc;\n}\n")
    lib_dir = _lib.LIB_PATH.parent
    exe = tmp_path / "caller"
    subprocess.run([gcc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", str(HEADER.parent),
                    str(src), "-L", str(lib_dir), "-lpgm_b200", f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    assert int(out[0]) == ctypes.sizeof(_lib.PgmSettings)
    assert float(out[1]) == 0.9 and int(out[2]) == 6 and int(out[3]) == 0 and float(out[4]) == -2.0


def build_core_engine_check(out_dir):
    """Compiles tests/cpp/core_engine_check.cpp (a pgmcore-style C++ caller of the engine through
    pgm-md_b200/csrc/pgm_core_b200.h) against the library; returns the executable."""
    import shutil
    import subprocess
    from pgm_md_b200 import _lib
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no C++ compiler")
    lib_dir = _lib.LIB_PATH.parent
    exe = Path(out_dir) / "core_engine_check"
    subprocess.run([gxx, "-std=c++17", "-O2", "-Wall", "-Werror", "-I", str(ROOT / "pgm-md_b200" / "csrc"),
                    str(ROOT / "tests" / "cpp" / "core_engine_check.cpp"), "-L", str(lib_dir), "-lpgm_b200",
                    f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], check=True)
    return exe


def test_core_shaped_cpp_surface_builds_and_links(tmp_path):
    """The pgmcore::Engine-shaped C++ class compiles as a caller sees it and links the library (it runs on
    the GPU in tests/test_gpu_core_api.py)."""
    assert build_core_engine_check(tmp_path).exists()


def test_openmm_kernel_recipe_needs_an_openmm_sdk():
    """The OpenMM CUDA-platform kernel (pgm-md_b200/openmm) builds only against an OpenMM SDK: without
    OPENMM_DIR its recipe stops with a message and status 2."""
    import os
    import subprocess
    env = {k: v for k, v in os.environ.items() if k != "OPENMM_DIR"}
    r = subprocess.run(["make", "-s", "-C", str(ROOT / "pgm-md_b200" / "openmm")], capture_output=True, text=True,
                       env=env)
    assert r.returncode == 2 and "OPENMM_DIR" in r.stdout
    src = (ROOT / "pgm-md_b200" / "openmm" / "PgmB200OpenMMKernel.cpp").read_text()
    for call in ("pgm_engine_launch_device", "pgm_engine_finish_device", "setForcesValid", "registerKernelFactories",
                 "getLongForceBuffer", "getAtomIndex"):
        assert call in src, call
