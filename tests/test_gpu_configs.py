"""The benchmark's other workloads held to the reference pgm_core at their own sizes (fixtures written by
tests/golden/make_golden.py from oracle/_ref at tol 1e-10):

  water98304   32768 waters, 104^3 grid: every energy term, the strain, the forces and the induced dipoles of
               both precisions (FP64 at tol 1e-10, mixed at the workload's tol 1e-5 and 1e-4);
  water_batch  the 1024 boxes of 8..512 waters in ONE batched launch, and a stratified sample of 32 of them
               (every 512-molecule box, every grid shape's smallest, median and largest box) in another: per
               system against pgm_core.

Bars (the reference GPU harness's, core/cuda/tests/test_cuda.cpp:177-191, and the metric's): FP64 energy
1e-9 relative, forces 1e-7 relative RMS; mixed energy 1e-6, forces 1e-5 (tol 1e-5).  Float32 storage of the
fixture's forces and dipoles contributes below 1e-7."""

import numpy as np
import pytest

from conftest import GOLDEN, PKG

pytestmark = pytest.mark.gpu

TERMS = ("direct", "reciprocal", "self", "background", "polarization")


def rel_rms(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def single_engine(S, precision, tol, pme=0):
    e = PKG.Engine(PKG.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=6, tol=tol, max_iter=500, peek=0.0,
                                predictor=0, ke=PKG.systems.KE_DEFAULT, precision=precision))
    e.set_system(S)
    e.set_pme_kernels(pme)
    return e


@pytest.fixture(scope="module")
def water98304():
    S = PKG.systems.water98304()
    d = np.load(GOLDEN / "ref_water98304.npz")
    assert np.allclose(d["pos_digest"], [S.pos.sum(), (S.pos ** 2).sum()], rtol=1e-13, atol=0)
    return S, d


@pytest.mark.parametrize("precision,tol,pme", [(PKG.FP64, 1e-10, 0), (PKG.MIXED, 1e-5, 0), (PKG.MIXED, 1e-4, 0),
                                               (PKG.MIXED, 1e-5, 1), (PKG.MIXED, 1e-5, 2),
                                               (PKG.MIXED, 1e-5, 3)])
def test_water98304_against_reference(water98304, precision, tol, pme):
    S, d = water98304
    eng = single_engine(S, precision, tol, pme)
    assert eng.pme_kernels() == pme
    r = eng.compute(S.pos, S.box)
    mu = eng.induced_dipoles()
    eng.close()
    e_ref = float(d["energy"])
    t = r.terms.as_dict()
    if precision == PKG.FP64:
        lim_e, lim_t, lim_f, lim_mu = 1e-9, 1e-8, 1e-7, 1e-7
        assert r.iterations == int(d["iterations"])
    else:   # the bar of the metric at tol 1e-5; tol 1e-4 stops the CG earlier
        lim_e, lim_t, lim_f, lim_mu = (1e-6, 1e-5, 1e-5, 1e-5) if tol == 1e-5 else (1e-5, 1e-4, 1e-4, 1e-4)
    assert abs(r.energy - e_ref) <= lim_e * abs(e_ref), (r.energy, e_ref)
    for k, name in enumerate(TERMS):
        ref = float(d["terms"][k])
        assert abs(t[name] - ref) <= lim_t * max(abs(ref), 1e-3 * abs(e_ref)), (name, t[name], ref)
    assert rel_rms(r.forces, d["forces"]) <= lim_f
    assert rel_rms(mu, d["mu"]) <= lim_mu
    assert np.abs(r.strain - d["strain"]).max() <= 10 * lim_f * np.abs(d["strain"]).max()


@pytest.fixture(scope="module")
def batch1024():
    boxes = PKG.systems.water_batch()
    d = np.load(GOLDEN / "ref_water_batch_sample.npz")
    return boxes, d


def batch_engine(boxes, precision, tol):
    s0 = boxes[0]
    eng = PKG.Engine(PKG.Settings(cutoff=s0.cutoff, beta=s0.beta, grid=s0.grid, order=6, tol=tol, max_iter=500,
                                  peek=0.0, predictor=0, ke=PKG.systems.KE_DEFAULT, precision=precision))
    eng.set_systems(boxes)
    return eng


def check_sample(boxes, d, out, mu, where, precision, tol):
    """Per-system checks of the sample boxes; where[k] = (index of the sample's box k in the launch, atom offset)."""
    foff = 0
    for k, b in enumerate(d["sample"]):
        S = boxes[int(b)]
        idx, aoff = where[k]
        n = S.n
        assert n == int(d["natoms"][k]) and S.grid[0] == int(d["grid"][k])
        e_ref = float(d["energy"][k])
        got = out["energies"][idx, :5].sum()
        F = out["forces"][aoff:aoff + n]
        Fr = d["forces"][foff:foff + n]
        mur = d["mu"][foff:foff + n]
        foff += n
        if precision == PKG.FP64:
            lim_e, lim_f = 1e-9, 1e-7
            assert int(out["iterations"][idx]) == int(d["iterations"][k]), (int(b), out["iterations"][idx])
        else:
            lim_e, lim_f = (1e-6, 1e-5) if tol <= 1e-5 else (1e-5, 1e-4)
        assert abs(got - e_ref) <= lim_e * abs(e_ref), (int(b), got, e_ref)
        for t in range(5):
            ref = float(d["terms"][k, t])
            assert abs(out["energies"][idx, t] - ref) <= 10 * lim_e * max(abs(ref), 1e-3 * abs(e_ref)), (int(b), t)
        assert rel_rms(F, Fr) <= lim_f, (int(b), rel_rms(F, Fr))
        assert rel_rms(mu[aoff:aoff + n], mur) <= 10 * lim_f, int(b)
        assert np.abs(out["strain"][idx] - d["strain"][k]).max() <= 10 * lim_f * np.abs(d["strain"][k]).max(), int(b)


@pytest.mark.parametrize("precision,tol", [(PKG.FP64, 1e-10), (PKG.MIXED, 1e-5)])
def test_batch1024_whole_launch_sample_against_reference(batch1024, precision, tol):
    """The timed workload itself: all 1024 boxes in one launch; the sample's systems against pgm_core."""
    boxes, d = batch1024
    eng = batch_engine(boxes, precision, tol)
    out = eng.compute_batch(np.concatenate([s.pos for s in boxes]), np.stack([s.box for s in boxes]))
    mu = eng.induced_dipoles()
    eng.close()
    offs = np.concatenate([[0], np.cumsum([s.n for s in boxes])])
    assert np.isfinite(out["energies"]).all()
    check_sample(boxes, d, out, mu, [(int(b), int(offs[b])) for b in d["sample"]], precision, tol)


@pytest.mark.parametrize("precision,tol", [(PKG.FP64, 1e-10), (PKG.MIXED, 1e-5)])
def test_batch_sample_launch_against_reference(batch1024, precision, tol):
    """The 32 sample boxes alone in one batched launch (ten grid shapes in one launch)."""
    boxes, d = batch1024
    sample = [boxes[int(b)] for b in d["sample"]]
    eng = batch_engine(sample, precision, tol)
    out = eng.compute_batch(np.concatenate([s.pos for s in sample]), np.stack([s.box for s in sample]))
    mu = eng.induced_dipoles()
    eng.close()
    offs = np.concatenate([[0], np.cumsum([s.n for s in sample])])
    check_sample(boxes, d, out, mu, [(k, int(offs[k])) for k in range(len(sample))], precision, tol)
