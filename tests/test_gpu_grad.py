"""Parameter gradients (the engine's adjoint of the stationary energy) against the FP64 oracle's analytic
gradient and central finite differences of the oracle energy (h = 1e-5 relative), per atom and per type
through the torch.autograd.Function.  Tolerance: 1e-5 relative (FP64 engine 1e-7 against the analytic
oracle gradient)."""

import numpy as np
import pytest

from conftest import PKG, oracle_settings, oracle_topology
from oracle import pgm_oracle as O

pytestmark = pytest.mark.gpu


def engine_for(S, precision, tol=1e-12):
    eng = PKG.Engine(PKG.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=S.order, tol=tol, max_iter=1000,
                                  peek=0.0, predictor=0, ke=PKG.systems.KE_DEFAULT, precision=precision))
    eng.set_system(S)
    return eng


@pytest.mark.parametrize("precision", [0, 1])
def test_param_grad_matches_oracle(precision):
    S = PKG.systems.tiny_triclinic(nmol=16, seed=23)
    eng = engine_for(S, precision)
    eng.compute(S.pos, S.box)
    g = eng.param_grad()
    ora = O.Engine(oracle_topology(S), oracle_settings(S, tol=1e-12))
    ora.compute(S.pos, S.box)
    go = ora.param_gradients()
    tol = 1e-7 if precision == 0 else 1e-5
    for k in ("q", "radius", "alpha", "cov_strength"):
        err = np.linalg.norm(g[k] - go[k]) / np.linalg.norm(go[k])
        assert err <= tol, (k, err)


@pytest.mark.parametrize("precision", [0, 1])
def test_autograd_per_type_vs_finite_differences(precision):
    import torch
    grad_mod = __import__("pgm_md_b200.autograd", fromlist=["autograd"])
    S = PKG.systems.waters(27, 9.6, seed=4, grid=(12, 12, 12), cutoff=4.7, tol=1e-12, lattice=3)
    eng = engine_for(S, precision)
    params = grad_mod.type_parameters(S)
    E = grad_mod.energy(eng, S, *params)
    E.backward()
    names = ("q", "cov_strength", "alpha", "radius")
    s = oracle_settings(S, tol=1e-12)
    for name, p in zip(names, params):
        for t in range(len(p)):
            fd = []
            for sgn in (1, -1):
                T = oracle_topology(S)
                vals = getattr(T, name).copy()
                idx = (S.cov_types if name == "cov_strength" else S.types) == t
                h = 1e-5 * abs(p[t].item())
                vals[idx] += sgn * h
                setattr(T, name, vals)
                fd.append(O.Engine(T, s).compute(S.pos, S.box, want_forces=False))
            d = (fd[0] - fd[1]) / (2 * h)
            got = float(p.grad[t])
            assert abs(got - d) <= 1e-5 * max(abs(d), 1e-2), (name, t, got, d)


def test_evaluate_fixed_and_solve():
    """Energy at the solved dipoles through evaluate_fixed equals compute's; the adjoint solve with the
    permanent field as right-hand side returns the induced dipoles (peek 0)."""
    S = PKG.systems.tiny_triclinic(nmol=12, seed=31)
    eng = engine_for(S, PKG.FP64)
    r = eng.compute(S.pos, S.box)
    mu = eng.induced_dipoles()
    rf = eng.evaluate_fixed(S.pos, S.box, mu, keep_list=True)
    assert abs(rf.energy - r.energy) <= 1e-12 * abs(r.energy)
    assert np.linalg.norm(rf.forces - r.forces) <= 1e-11 * np.linalg.norm(r.forces)
    # E_perm = field of charges and permanent dipoles; (alpha^-1 - T) mu = E_perm
    Eperm = eng.field(S.pos, S.box, S.q, eng.permanent_dipoles())
    eng.evaluate_fixed(S.pos, S.box, mu, keep_list=False)
    x, it = eng.solve(Eperm, tol=1e-12)
    assert np.abs(x - mu).max() <= 1e-8 * np.abs(mu).max()


@pytest.mark.parametrize("precision", [0, 1])
def test_force_matching_gradient_vs_finite_differences(precision):
    """dL/d(per-type parameter) of L = sum |F - F_target|^2 (F_target from parameters perturbed by
    N(0, 0.05)) by one adjoint solve, against central differences of L on the FP64 oracle (h = 1e-5 relative),
    to 1e-5 relative; and per atom against the oracle's analytic adjoint (FP64 1e-7, mixed 1e-5)."""
    import torch
    grad_mod = __import__("pgm_md_b200.autograd", fromlist=["autograd"])
    S = PKG.systems.waters(8, 6.3, seed=12, grid=(8, 8, 8), cutoff=3.1, tol=1e-12, lattice=2)
    Sp = PKG.systems.perturbed(S, rel=0.05, seed=3)
    ora_t = O.Engine(oracle_topology(Sp), oracle_settings(Sp, tol=1e-12))
    ora_t.compute(Sp.pos, Sp.box)
    Ft = ora_t.forces
    eng = engine_for(S, precision)
    params = grad_mod.type_parameters(S)
    L = grad_mod.force_matching_loss(eng, S, Ft, *params)
    ora = O.Engine(oracle_topology(S), oracle_settings(S, tol=1e-12))
    ora.compute(S.pos, S.box)
    Lo, go = ora.force_matching_gradients(Ft)
    eng.compute(S.pos, S.box)
    Lg, gg, _ = eng.force_matching_grad(Ft, tol=1e-12)
    lim = 1e-7 if precision == 0 else 1e-5
    assert abs(Lg - Lo) <= lim * Lo
    for k in ("q", "radius", "alpha", "cov_strength"):
        assert np.linalg.norm(gg[k] - go[k]) <= lim * np.linalg.norm(go[k]), k
    L.backward()
    s = oracle_settings(S, tol=1e-12)

    def loss(T):
        e = O.Engine(T, s)
        e.compute(S.pos, S.box)
        return float(np.sum((e.forces - Ft) ** 2))

    names = ("q", "cov_strength", "alpha", "radius")
    for name, p in zip(names, params):
        for t in range(len(p)):
            vals_fd = []
            h = 1e-5 * abs(p[t].item())
            for sgn in (1, -1):
                T = oracle_topology(S)
                vals = getattr(T, name).copy()
                idx = (S.cov_types if name == "cov_strength" else S.types) == t
                vals[idx] += sgn * h
                setattr(T, name, vals)
                vals_fd.append(loss(T))
            d = (vals_fd[0] - vals_fd[1]) / (2 * h)
            got = float(p.grad[t])
            assert abs(got - d) <= 1e-5 * max(abs(d), 1e-6 * abs(L.item())), (name, t, got, d)
