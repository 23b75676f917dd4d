"""The combination-rule GVDW van der Waals (set_gvdw, pgmcuda::Engine::setGvdw, core/cuda/pgm_cuda.h:57-65) in
the engine's final pass:

- on the reference's GVDW known-answer box (tests/golden/gvdw_box.npz, no charges or polarizabilities) the
  engine's Terms.gvdw is pmemd-pgm's VDWAALS for both repulsion forms, FP64 within the reference's 1e-3 kcal/mol,
  mixed (float pair arithmetic, as the reference's GPU engine) within 1e-5 relative; its forces and strain are
  the oracle's (FP64 within 1e-10 relative RMS, mixed 1e-5);
- on a polarizable water box with GVDW beside the electrostatics (intramolecular pairs skipped) the totals,
  forces and strain derivative are the oracle's electrostatics plus its GVDW (FP64 1e-7 / 1e-6, mixed 1e-6 /
  1e-5);
- set_atoms drops it; a radius beyond the cutoff and parameter gradients while it is set are refused.
"""

import numpy as np
import pytest

from conftest import GOLDEN, PKG, oracle_settings, oracle_topology
from oracle import gvdw as GV
from oracle import pgm_oracle as O

pytestmark = pytest.mark.gpu
KCAL = 4.184


def rel_rms(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def box_case():
    d = np.load(GOLDEN / "gvdw_box.npz")
    n = len(d["radius"])
    S = PKG.systems.System(name="gvdw_box", pos=d["pos"], box=d["box"], q=np.zeros(n), radius=d["radius"],
                           alpha=np.zeros(n), cov_atom=np.zeros(0, np.int32), cov_partner=np.zeros(0, np.int32),
                           cov_strength=np.zeros(0), cutoff=float(d["rvdw"]), beta=3.5, grid=(28, 28, 28), order=6)
    return S, d


@pytest.mark.parametrize("precision", [PKG.FP64, PKG.MIXED])
@pytest.mark.parametrize("which", [0, 1])
def test_gvdw_box_matches_pmemd(which, precision):
    S, d = box_case()
    arep, c6, B, slater, pmemd = d["models"][which]
    lj = d["lj"].astype(bool)
    sa = np.where(lj, np.sqrt(arep * KCAL), 0.0)
    sc = np.where(lj, np.sqrt(c6 * KCAL * 1e-6), 0.0)
    b = np.full(S.n, B)
    eng = PKG.Engine(PKG.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=6, tol=1e-10, max_iter=100,
                                  peek=0.0, predictor=0, ke=PKG.systems.KE_DEFAULT, precision=precision,
                                  polarizable=False))
    eng.set_system(S)
    eng.set_gvdw(int(slater), S.cutoff, sa, sc, b, d["excl"][:, 0], d["excl"][:, 1])
    r = eng.compute(S.pos, S.box)
    if precision == PKG.FP64:   # the reference's own bar for its FP64 kernel (core/tests/test_gvdw.cpp:92)
        assert abs(r.terms.gvdw / KCAL - pmemd) <= 1e-3
    else:   # pair arithmetic in float, as the reference's GPU engine: the mixed path's relative bar
        assert abs(r.terms.gvdw / KCAL - pmemd) <= 1e-5 * pmemd
    E, F, Sg = GV.gvdw_energy(S.pos, S.box, S.radius, sa, sc, b, S.cutoff, bool(slater), d["excl"][:, 0],
                              d["excl"][:, 1])
    lim = 1e-10 if precision == PKG.FP64 else 1e-5
    assert abs(r.terms.gvdw - E) <= lim * abs(E)
    assert rel_rms(r.forces, F) <= lim
    assert np.abs(r.strain - Sg).max() <= lim * np.abs(Sg).max()


@pytest.mark.parametrize("precision", [PKG.FP64, PKG.MIXED])
def test_gvdw_beside_electrostatics(precision):
    S = PKG.systems.water216()
    rng = np.random.default_rng(17)
    sa = rng.uniform(20.0, 40.0, S.n) * (rng.uniform(size=S.n) < 0.8)   # a fifth of the atoms without the term
    sc = rng.uniform(0.02, 0.05, S.n)
    b = rng.uniform(0.8, 1.2, S.n)
    mol = np.arange(S.n) // 3
    ii, jj = np.triu_indices(S.n, 1)
    same = mol[ii] == mol[jj]
    skip_i, skip_j = ii[same], jj[same]
    rvdw = 0.8
    eng = PKG.Engine(PKG.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=S.order, tol=1e-10, max_iter=1000,
                                  peek=0.0, predictor=0, ke=PKG.systems.KE_DEFAULT, precision=precision))
    eng.set_system(S)
    eng.set_gvdw(0, rvdw, sa, sc, b, skip_i, skip_j)
    r = eng.compute(S.pos, S.box)
    ora = O.Engine(oracle_topology(S), oracle_settings(S))
    e = ora.compute(S.pos, S.box)
    Eg, Fg, Sg = GV.gvdw_energy(S.pos, S.box, S.radius, sa, sc, b, rvdw, False, skip_i, skip_j)
    lim_e, lim_f = (1e-7, 1e-6) if precision == PKG.FP64 else (1e-6, 1e-5)
    assert abs(r.terms.gvdw - Eg) <= lim_f * abs(Eg)
    assert abs(r.energy - (e + Eg)) <= lim_e * abs(e + Eg)
    assert rel_rms(r.forces, ora.forces + Fg) <= lim_f
    St = ora.strain + Sg
    assert np.abs(r.strain - St).max() <= 10 * lim_f * np.abs(St).max()
    with pytest.raises(RuntimeError):
        eng.param_grad()
    # set_atoms drops it
    eng.set_system(S)
    r2 = eng.compute(S.pos, S.box)
    assert r2.terms.gvdw == 0.0
    assert abs(r2.energy - e) <= lim_e * abs(e)


def test_gvdw_refused_beyond_cutoff():
    S = PKG.systems.water216()
    eng = PKG.Engine(PKG.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=S.order, precision=PKG.FP64))
    eng.set_system(S)
    ones = np.ones(S.n)
    with pytest.raises(RuntimeError):
        eng.set_gvdw(0, S.cutoff * 1.1, ones, ones, ones)
    with pytest.raises(RuntimeError):
        eng.set_gvdw(2, S.cutoff, ones, ones, ones)
