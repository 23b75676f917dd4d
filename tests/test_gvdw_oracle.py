"""The GVDW checker (oracle/gvdw.py, the reference's core/gvdw_kernel.h restated) pinned as the reference's own
test pins its kernel (core/tests/test_gvdw.cpp): the energy of its known-answer box (tests/data/gvdw_box.txt, in
tests/golden/gvdw_box.npz) against pmemd-pgm's VDWAALS for both repulsion forms, the series and closed forms
of G meeting at y = 0.6, dU/dr against central differences, and the forces and strain of the box sum against
finite differences of its energy."""

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import gvdw as GV

KCAL = 4.184


def box_params(d, model):
    arep, c6, B, slater, _ = model
    lj = d["lj"].astype(bool)
    sa = np.where(lj, np.sqrt(arep * KCAL), 0.0)
    sc = np.where(lj, np.sqrt(c6 * KCAL * 1e-6), 0.0)
    return sa, sc, np.full(len(lj), B), bool(slater)


@pytest.mark.parametrize("which", [0, 1])
def test_gvdw_box_matches_pmemd(which):
    d = np.load(GOLDEN / "gvdw_box.npz")
    model = d["models"][which]
    sa, sc, b, slater = box_params(d, model)
    E, _, _ = GV.gvdw_energy(d["pos"], d["box"], d["radius"], sa, sc, b, float(d["rvdw"]), slater,
                             d["excl"][:, 0], d["excl"][:, 1])
    assert abs(E / KCAL - model[4]) <= 1e-3   # the reference's own bar (core/tests/test_gvdw.cpp:92)


def test_gvdw_series_meets_closed_form():
    G1, H1 = GV.gvdw_g(np.array([GV.Y_SWITCH - 1e-12]))
    G2, H2 = GV.gvdw_g(np.array([GV.Y_SWITCH + 1e-12]))
    assert abs(G1[0] - G2[0]) <= 1e-9 * abs(G2[0]) and abs(H1[0] - H2[0]) <= 1e-7 * abs(H2[0])
    assert abs(GV.gvdw_g(np.array([0.0]))[0][0] - 8 / (9 * np.pi)) <= 1e-15


@pytest.mark.parametrize("slater", [False, True])
def test_gvdw_pair_finite_differences(slater):
    r = np.array([0.02, 0.05, 0.1, 0.2, 0.28, 0.35, 0.5, 0.9])
    bij, A, C6, B, h = 1.0 / np.sqrt(2.0 * (0.07 ** 2 + 0.07 ** 2)), 800.0, 0.0025, (4.52 if slater else 0.9453), 1e-6
    _, dEdR = GV.gvdw_pair(r, bij, A, C6, B, slater)
    up, _ = GV.gvdw_pair(r + h, bij, A, C6, B, slater)
    dn, _ = GV.gvdw_pair(r - h, bij, A, C6, B, slater)
    fd = -(up - dn) / (2 * h) / r
    assert np.all(np.abs(fd - dEdR) <= 1e-6 * np.maximum(np.abs(fd), 1e-12))


def test_gvdw_box_forces_and_strain_finite_differences():
    d = np.load(GOLDEN / "gvdw_box.npz")
    sa, sc, b, slater = box_params(d, d["models"][1])
    args = (d["radius"], sa, sc, b, float(d["rvdw"]), slater, d["excl"][:, 0], d["excl"][:, 1])
    pos, box = d["pos"], d["box"]
    E, F, S = GV.gvdw_energy(pos, box, *args)
    h = 1e-6
    for i in (0, 1, 2, 700):
        for a in range(3):
            p = pos.copy()
            p[i, a] += h
            ep = GV.gvdw_energy(p, box, *args)[0]
            p[i, a] -= 2 * h
            em = GV.gvdw_energy(p, box, *args)[0]
            assert abs(-(ep - em) / (2 * h) - F[i, a]) <= 1e-5 * np.abs(F).max()
    # S_ab = dE/d eps_ab under r -> (1 + eps) r, box rows -> rows (1 + eps)
    for a, bb in ((0, 0), (1, 2), (2, 2)):
        eps = np.zeros((3, 3))
        eps[a, bb] = h
        ep = GV.gvdw_energy(pos @ (np.eye(3) + eps).T, box @ (np.eye(3) + eps).T, *args)[0]
        em = GV.gvdw_energy(pos @ (np.eye(3) - eps).T, box @ (np.eye(3) - eps).T, *args)[0]
        assert abs((ep - em) / (2 * h) - S[3 * a + bb]) <= 1e-5 * np.abs(S).max()


def test_engine_series_matches_checker():
    """The engine's host derivation of the G(y) series (pgm_gvdw_series, double arithmetic) against the checker's
    exact rationals, and the reference's published table to its printed digits (core/gvdw_kernel.h:33-37 gives
    c_1 = -2, c_2 = 58/25, c_3 = -188/105)."""
    import ctypes
    from pgm_md_b200 import _lib
    c = np.zeros(GV.SERIES_TERMS)
    assert _lib.load().pgm_gvdw_series(c.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(c)) == 0
    ref = GV.series_coefficients()
    assert np.all(np.abs(c - ref) <= 1e-14 * np.abs(ref))
    assert c[0] == 1.0 and abs(c[1] + 2.0) < 1e-15 and abs(c[2] - 58 / 25) < 1e-15 and abs(c[3] + 188 / 105) < 1e-15
    bad = np.zeros(1)
    assert _lib.load().pgm_gvdw_series(bad.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 0) != 0
