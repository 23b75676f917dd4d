"""The dual first pass of a predicted step: with a guess from the history (mu3 / mu4 / the last solution), x0
does not depend on the permanent field, so the engine forms x0 first and takes E_perm and T x0 from one sweep
over the pair records and two PME passes (two grids), where an unpredicted step needs the permanent field before
x0 = alpha E_perm.  It runs with PGM_B200_DUAL=1 (the two passes apart are the default, and the faster).  Checked
over MD-like steps of the real 8550-atom liquid (mu4, Verlet list kept) against the same engine with the two
passes apart (PGM_B200_DUAL=0) and against a fresh unpredicted evaluation at tol 1e-10.

Bars: FP64 energies within 1e-10 relative and the same CG iterations as the separate passes (the same sums, in
another order only where atomics add), forces within 1e-9 relative RMS; mixed energies within 1e-6, forces 1e-5,
iterations within one; against the fresh evaluation FP64 within the reference bars (1e-9 / 1e-7) at tol 1e-8,
mixed within 2e-6 / 2e-5 at tol 1e-6."""

import os

import numpy as np
import pytest

from conftest import PKG, load_dmp_real

pytestmark = pytest.mark.gpu


def rel_rms(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def engine(S, precision, predictor=2, tol=1e-8, skin=0.15):
    e = PKG.Engine(PKG.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=6, tol=tol, max_iter=500, peek=0.0,
                                predictor=predictor, ke=PKG.systems.KE_DEFAULT, precision=precision, skin=skin))
    e.set_system(S)
    return e


def trajectory(S, steps, seed=3):
    rng = np.random.default_rng(seed)
    phase = rng.uniform(0, 2 * np.pi, S.pos.shape)
    for k in range(steps):   # smooth motion, amplitude 0.005 nm, period 60 steps
        yield S.pos + 0.005 * np.sin(2 * np.pi * k / 60 + phase)


@pytest.mark.parametrize("precision", [PKG.FP64, PKG.MIXED])
def test_dual_first_pass_matches_separate_passes(precision, monkeypatch):
    S, _ = load_dmp_real()
    fp64 = precision == PKG.FP64
    tol = 1e-8 if fp64 else 1e-6   # (the FP32 operator holds residuals to about 1e-7)
    dual = engine(S, precision, tol=tol)
    monkeypatch.setenv("PGM_B200_DUAL", "0")
    apart = engine(S, precision, tol=tol)
    lim_e, lim_f = (1e-10, 1e-9) if fp64 else (1e-6, 1e-5)
    for step, pos in enumerate(trajectory(S, 7)):
        monkeypatch.setenv("PGM_B200_DUAL", "1")
        a = dual.compute(pos, S.box)
        monkeypatch.setenv("PGM_B200_DUAL", "0")
        b = apart.compute(pos, S.box)
        assert abs(a.energy - b.energy) <= lim_e * abs(b.energy), (step, a.energy, b.energy)
        assert rel_rms(a.forces, b.forces) <= lim_f, step
        if fp64:
            assert a.iterations == b.iterations, (step, a.iterations, b.iterations)
        else:
            assert abs(a.iterations - b.iterations) <= 1, (step, a.iterations, b.iterations)
    monkeypatch.delenv("PGM_B200_DUAL")
    # the last step against a fresh unpredicted evaluation at tol 1e-10
    fresh = engine(S, precision, predictor=0, tol=1e-10, skin=0.0)
    f = fresh.compute(pos, S.box)
    lim_e, lim_f = (1e-9, 1e-7) if fp64 else (2e-6, 2e-5)
    assert abs(a.energy - f.energy) <= lim_e * abs(f.energy), (a.energy, f.energy)
    assert rel_rms(a.forces, f.forces) <= lim_f
    for e in (dual, apart, fresh):
        e.close()


def test_dual_first_pass_predicted_steps_save_iterations():
    """mu4 over the trajectory: later steps take fewer CG iterations than the first (unpredicted) one."""
    S, _ = load_dmp_real()
    e = engine(S, PKG.MIXED, tol=1e-5)
    os.environ["PGM_B200_DUAL"] = "1"
    try:
        its = [e.compute(pos, S.box).iterations for pos in trajectory(S, 6)]
    finally:
        os.environ.pop("PGM_B200_DUAL", None)
    e.close()
    assert its[-1] < its[0], its
