"""The Verlet pair list (radius cutoff + skin, kept while every atom stays within half the skin of its position at
the list's build and the box is unchanged; core/cuda/pgm_cuda.cu:1899-1940 keeps its list by the same rule):
over a moving trajectory the kept list gives the oracle's energies, forces and exact pair set at every step;
builds happen only when an atom moved beyond half the skin or the box changed; skin 0 builds at every
evaluation.

Tolerances as the parity tests: FP64 within 1e-7 relative in energy and 1e-6 relative RMS in forces against the
oracle at tol 1e-10, mixed within 1e-6 and 1e-5; the pair set bit-exact in both.
"""

import numpy as np
import pytest

from conftest import PKG, oracle_settings, oracle_topology
from oracle import pgm_oracle as O

pytestmark = pytest.mark.gpu


def water512():
    # 512 waters at 0.0334 molecules/A^3 (24.8 A box): the full 0.15 nm skin fits below half the box
    return PKG.systems.waters(512, (512 / 0.0334) ** (1 / 3), seed=5, grid=(25, 25, 25), tol=1e-10)


def make_engine(S, precision, **kw):
    eng = PKG.Engine(PKG.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=S.order, tol=1e-10,
                                  max_iter=1000, peek=0.0, predictor=0, ke=PKG.systems.KE_DEFAULT,
                                  precision=precision, **kw))
    eng.set_system(S)
    return eng


def rel_rms(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def check_step(engines, S, pos, box):
    ora = O.Engine(oracle_topology(S), oracle_settings(S))
    e = ora.compute(pos, box)
    oi, oj, _ = O.pair_set(pos, box, S.cutoff)
    for prec, eng in engines.items():
        r = eng.compute(pos, box)
        lim_e, lim_f = (1e-7, 1e-6) if prec == PKG.FP64 else (1e-6, 1e-5)
        assert abs(r.energy - e) <= lim_e * abs(e), (prec, r.energy, e)
        assert rel_rms(r.forces, ora.forces) <= lim_f, prec
        gi, gj = eng.pairs()
        assert np.array_equal(gi, oi) and np.array_equal(gj, oj), prec
        assert eng.num_candidates() == 2 * len(oi)


def test_verlet_list_kept_and_rebuilt():
    S = water512()
    engines = {p: make_engine(S, p) for p in (PKG.FP64, PKG.MIXED)}   # default skin 0.15 nm
    rng = np.random.default_rng(3)
    pos = S.pos.copy()
    for step in range(4):   # cumulative moves U(+-0.008 nm) per component: every atom stays within 0.075 nm
        if step:
            pos = pos + rng.uniform(-0.008, 0.008, pos.shape)
        check_step(engines, S, pos, S.box)
    drift = np.linalg.norm(pos - S.pos, axis=1).max()
    assert drift < 0.075
    for eng in engines.values():
        assert eng.list_builds() == 1
    # one atom beyond half the skin of its position at the build: the list is built anew
    pos = pos.copy()
    pos[7] += np.array([0.08, 0.0, 0.0])
    check_step(engines, S, pos, S.box)
    for eng in engines.values():
        assert eng.list_builds() == 2
    # another box (isotropic scaling): built anew
    box2 = S.box * 1.002
    pos2 = pos * 1.002
    check_step(engines, S, pos2, box2)
    for eng in engines.values():
        assert eng.list_builds() == 3


def test_skin_zero_builds_every_evaluation():
    S = water512()
    kept = make_engine(S, PKG.FP64)
    fresh = make_engine(S, PKG.FP64, skin=0.0)
    for _ in range(3):
        a = kept.compute(S.pos, S.box)
        b = fresh.compute(S.pos, S.box)
        assert abs(a.energy - b.energy) <= 1e-12 * abs(b.energy)
        assert rel_rms(a.forces, b.forces) <= 1e-12
    assert kept.list_builds() == 1
    assert fresh.list_builds() == 3
