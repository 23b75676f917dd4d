"""The pgmcore::Engine-shaped C++ surface (pgm-md_b200/csrc/pgm_core_b200.h) driven by a C++ program the way
the reference's CPU tests drive pgmcore::Engine, on the 216-water golden (outputs of the reference pgm_core at
tol 1e-10): energy, terms, strain derivative, forces and induced dipoles of the FP64 path; the history key
(a second call with the same key reuses the stored solution); field() of the charges against the oracle's."""

import struct
import subprocess

import numpy as np
import pytest

from conftest import PKG, load_golden_system, oracle_settings, oracle_topology
from test_capi import build_core_engine_check

pytestmark = pytest.mark.gpu


def test_core_shaped_surface_against_reference(tmp_path):
    from oracle import pgm_oracle as O
    S, d = load_golden_system("water216")
    exe = build_core_engine_check(tmp_path)
    n, ncov = S.n, len(S.cov_atom)
    blob = struct.pack("<7i", n, ncov, *S.grid, S.order, 0) + struct.pack(
        "<4d", S.cutoff, S.beta, 1e-10, PKG.systems.KE_DEFAULT)
    blob += np.ascontiguousarray(S.box, "<f8").tobytes() + np.ascontiguousarray(S.pos, "<f8").tobytes()
    for a in (S.q, S.radius, S.alpha):
        blob += np.ascontiguousarray(a, "<f8").tobytes()
    blob += np.ascontiguousarray(S.cov_atom, "<i4").tobytes() + np.ascontiguousarray(S.cov_partner, "<i4").tobytes()
    blob += np.ascontiguousarray(S.cov_strength, "<f8").tobytes()
    inp, out = tmp_path / "in.bin", tmp_path / "out.bin"
    inp.write_bytes(blob)
    subprocess.run([str(exe), str(inp), str(out)], check=True, timeout=120)
    raw = out.read_bytes()
    k = 0

    def take(m):
        nonlocal k
        v = np.frombuffer(raw, "<f8", m, k)
        k += 8 * m
        return v

    e, terms, strain = take(1)[0], take(5), take(9)
    F, mu = take(3 * n).reshape(n, 3), take(3 * n).reshape(n, 3)
    e2, E = take(1)[0], take(3 * n).reshape(n, 3)
    it, it2 = struct.unpack_from("<2i", raw, k)
    e_ref = float(d["energy"])
    assert abs(e - e_ref) <= 1e-9 * abs(e_ref)
    assert np.abs(terms - d["terms"]).max() <= 1e-9 * abs(e_ref)
    assert np.linalg.norm(F - d["forces"]) <= 1e-7 * np.linalg.norm(d["forces"])
    assert np.linalg.norm(mu - d["mu"]) <= 1e-7 * np.linalg.norm(d["mu"])
    assert np.abs(strain - d["strain"]).max() <= 1e-7 * np.abs(d["strain"]).max()
    assert it == int(d["iterations"])
    assert abs(e2 - e) <= 1e-10 * abs(e) and it2 <= 1   # the same key: from the stored solution
    ora = O.Engine(oracle_topology(S), oracle_settings(S))
    ora.set_geometry(S.pos, S.box)
    E_ref = ora.field(S.q, np.zeros((n, 3)))
    assert np.linalg.norm(E - E_ref) <= 1e-9 * np.linalg.norm(E_ref)
