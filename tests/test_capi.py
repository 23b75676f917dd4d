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
