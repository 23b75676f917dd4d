"""Batched evaluation of many independent systems of uneven sizes in one launch, against the FP64 oracle per
system, and against the engine evaluating each system alone."""

import numpy as np
import pytest

from conftest import PKG, oracle_settings, oracle_topology
from oracle import pgm_oracle as O

pytestmark = pytest.mark.gpu


def batch_engine(systems, precision, tol=1e-10):
    s0 = systems[0]
    eng = PKG.Engine(PKG.Settings(cutoff=s0.cutoff, beta=s0.beta, grid=s0.grid, order=6, tol=tol, max_iter=1000,
                                  peek=0.0, predictor=0, ke=PKG.systems.KE_DEFAULT, precision=precision))
    eng.set_systems(systems)
    return eng


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_matches_oracle_per_system(precision):
    systems = PKG.systems.water_batch(nsys=12, seed=5, nmin=8, nmax=96, tol=1e-10)
    eng = batch_engine(systems, precision)
    pos = np.concatenate([s.pos for s in systems])
    boxes = np.stack([s.box for s in systems])
    out = eng.compute_batch(pos, boxes)
    off = 0
    for k, S in enumerate(systems):
        ora = O.Engine(oracle_topology(S), oracle_settings(S))
        e = ora.compute(S.pos, S.box)
        got = out["energies"][k, :5].sum()
        F = out["forces"][off:off + S.n]
        off += S.n
        tol_e, tol_f = (1e-9, 1e-7) if precision == 0 else (1e-6, 1e-5)
        assert abs(got - e) <= tol_e * abs(e), (k, got, e)
        assert np.linalg.norm(F - ora.forces) <= tol_f * np.linalg.norm(ora.forces), k
        assert np.abs(out["strain"][k] - ora.strain).max() <= 10 * tol_f * np.abs(ora.strain).max(), k
        if precision == 0:
            assert out["iterations"][k] == ora.iterations


def test_batch_equals_single_engines():
    """The batch gives each system what a single-system engine gives it (FP64)."""
    systems = PKG.systems.water_batch(nsys=6, seed=8, nmin=8, nmax=64, tol=1e-8)
    eng = batch_engine(systems, PKG.FP64, tol=1e-8)
    pos = np.concatenate([s.pos for s in systems])
    out = eng.compute_batch(pos, np.stack([s.box for s in systems]))
    off = 0
    for k, S in enumerate(systems):
        single = PKG.Engine(PKG.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=6, tol=1e-8, max_iter=1000,
                                         peek=0.0, predictor=0, ke=PKG.systems.KE_DEFAULT, precision=PKG.FP64))
        single.set_system(S)
        r = single.compute(S.pos, S.box)
        assert abs(out["energies"][k, :5].sum() - r.energy) <= 1e-11 * abs(r.energy)
        assert np.linalg.norm(out["forces"][off:off + S.n] - r.forces) <= 1e-10 * np.linalg.norm(r.forces)
        assert out["iterations"][k] == r.iterations
        off += S.n


def test_batch_tiny_boxes_half_box_cutoff():
    """Boxes of 8 molecules (6.2 A) with the cutoff at exactly half the box: pair sets and energies of the
    oracle."""
    systems = PKG.systems.water_batch(nsys=4, seed=2, nmin=8, nmax=8, tol=1e-10)
    eng = batch_engine(systems, PKG.FP64)
    out = eng.compute_batch(np.concatenate([s.pos for s in systems]), np.stack([s.box for s in systems]))
    for k, S in enumerate(systems):
        assert abs(S.cutoff - S.box[0, 0] / 2) < 1e-15
        ora = O.Engine(oracle_topology(S), oracle_settings(S))
        e = ora.compute(S.pos, S.box)
        assert abs(out["energies"][k, :5].sum() - e) <= 1e-9 * abs(e)


def test_batch_param_gradients():
    """Parameter gradients of every system of a batch (one launch) against the oracle's analytic gradient."""
    systems = PKG.systems.water_batch(nsys=5, seed=21, nmin=8, nmax=40, tol=1e-12)
    eng = batch_engine(systems, PKG.FP64, tol=1e-12)
    eng.compute_batch(np.concatenate([s.pos for s in systems]), np.stack([s.box for s in systems]))
    g = eng.param_grad()
    off, coff = 0, 0
    for S in systems:
        ora = O.Engine(oracle_topology(S), oracle_settings(S, tol=1e-12))
        ora.compute(S.pos, S.box)
        go = ora.param_gradients()
        sl = slice(off, off + S.n)
        cl = slice(coff, coff + len(S.cov_atom))
        for k, part in (("q", sl), ("radius", sl), ("alpha", sl), ("cov_strength", cl)):
            ref = go[k]
            assert np.linalg.norm(g[k][part] - ref) <= 1e-7 * np.linalg.norm(ref), (k, S.n)
        off += S.n
        coff += len(S.cov_atom)


def test_batch_retires_converged_systems():
    """The batched CG retires converged systems: the count of systems still iterating before each iteration
    (pgm_engine_active_systems) equals the number of systems whose own iteration count exceeds it, and falls to
    zero at the last iteration."""
    systems = PKG.systems.water_batch(nsys=10, seed=9, nmin=8, nmax=120, tol=1e-9)
    eng = batch_engine(systems, PKG.FP64, tol=1e-9)
    out = eng.compute_batch(np.concatenate([s.pos for s in systems]), np.stack([s.box for s in systems]))
    counts = eng.active_systems()
    its = np.asarray(out["iterations"])
    assert len(counts) == its.max() + 1
    assert counts == [int(np.sum(its > k)) for k in range(its.max() + 1)]
    assert counts[-1] == 0 and all(a >= b for a, b in zip(counts, counts[1:]))
    eng.close()
