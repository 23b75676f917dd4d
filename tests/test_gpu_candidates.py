"""The caller's pair candidates (set_candidates, pgmcuda::Engine::setCandidates, core/cuda/pgm_cuda.h:68-73) in
place of the engine's own pair search, as GROMACS hands its pair list over: segments of (i, box shift) with their
partners j, x = r_i + t.box - r_j, every pair once, the pairs beyond the cutoff left out at every evaluation.

Candidates are the oracle's pairs within cutoff + 0.15 nm (the reference's minimum image, i < j), grouped into
one segment per (i, shift).  With them the engine gives the energies, forces and pair set of its own list (FP64
within 1e-12 relative: only the order of the pair sums differs; mixed within 1e-6 and 1e-5) over a moving
trajectory, and the oracle's at tol 1e-10; the field entry point uses them too; a new set_atoms drops them; bad
input is refused.
"""

import numpy as np
import pytest

from conftest import PKG, oracle_settings, oracle_topology
from oracle import pgm_oracle as O

pytestmark = pytest.mark.gpu


def rel_rms(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def make_engine(S, precision, **kw):
    eng = PKG.Engine(PKG.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=S.order, tol=1e-10, max_iter=1000,
                                  peek=0.0, predictor=0, ke=PKG.systems.KE_DEFAULT, precision=precision, **kw))
    eng.set_system(S)
    return eng


def candidates(S, radius):
    """Segments (i, t) with their partners j from the oracle's pairs within radius (i < j)."""
    i, j, x = O.pair_set(S.pos, S.box, radius)
    d = S.pos[i] - S.pos[j]
    t = np.rint((x - d) @ np.linalg.inv(S.box)).astype(np.int64)   # x = r_i + t.box - r_j
    assert np.allclose(d + t @ S.box, x, atol=1e-9)
    key = np.lexsort((j, t[:, 2], t[:, 1], t[:, 0], i))
    i, j, t = i[key], j[key], t[key]
    new = np.ones(len(i), bool)
    new[1:] = (i[1:] != i[:-1]) | np.any(t[1:] != t[:-1], axis=1)
    starts = np.nonzero(new)[0]
    seg_begin = np.append(starts, len(i))
    return i[starts], t[starts], seg_begin, j


@pytest.mark.parametrize("precision", [PKG.FP64, PKG.MIXED])
def test_candidates_match_own_list(precision):
    S = PKG.systems.waters(512, (512 / 0.0334) ** (1 / 3), seed=5, grid=(25, 25, 25), tol=1e-10)
    own = make_engine(S, precision)
    ext = make_engine(S, precision)
    ext.set_candidates(*candidates(S, S.cutoff + 0.15))
    rng = np.random.default_rng(4)
    pos = S.pos.copy()
    lim_e, lim_f = (1e-12, 1e-11) if precision == PKG.FP64 else (1e-6, 1e-5)
    for step in range(3):   # moves within half of the 0.15 nm margin: the candidates still hold every pair
        if step:
            pos = pos + rng.uniform(-0.008, 0.008, pos.shape)
        a, b = own.compute(pos, S.box), ext.compute(pos, S.box)
        assert abs(a.energy - b.energy) <= lim_e * abs(a.energy)
        assert rel_rms(b.forces, a.forces) <= lim_f
        ga, gb = own.pairs(), ext.pairs()
        assert set(zip(*ga)) == set(zip(*gb))
        assert ext.num_candidates() == own.num_candidates()
    if precision == PKG.FP64:
        ora = O.Engine(oracle_topology(S), oracle_settings(S))
        e = ora.compute(pos, S.box)
        assert abs(b.energy - e) <= 1e-7 * abs(e)
        assert rel_rms(b.forces, ora.forces) <= 1e-6


def test_candidates_triclinic_and_reset():
    S = PKG.systems.tiny_triclinic(nmol=20, seed=9)
    own = make_engine(S, PKG.FP64)
    ext = make_engine(S, PKG.FP64)
    ext.set_candidates(*candidates(S, S.cutoff + 0.05))
    a, b = own.compute(S.pos, S.box), ext.compute(S.pos, S.box)
    assert abs(a.energy - b.energy) <= 1e-12 * abs(a.energy)
    assert rel_rms(b.forces, a.forces) <= 1e-11
    # the field entry point builds its list from the candidates too
    rng = np.random.default_rng(2)
    q, d = rng.normal(0, 0.5, S.n), rng.normal(0, 0.01, (S.n, 3))
    assert rel_rms(ext.field(S.pos, S.box, q, d), own.field(S.pos, S.box, q, d)) <= 1e-12
    # a new set_atoms drops the candidates: the own search again
    ext.set_system(S)
    c = ext.compute(S.pos, S.box)
    assert abs(c.energy - a.energy) <= 1e-12 * abs(a.energy)


def test_candidates_refused():
    S = PKG.systems.tiny_triclinic(nmol=20, seed=9)
    eng = make_engine(S, PKG.FP64)
    seg_i, seg_t, seg_begin, cand_j = candidates(S, S.cutoff)
    bad = cand_j.copy()
    bad[0] = S.n
    with pytest.raises(RuntimeError):
        eng.set_candidates(seg_i, seg_t, seg_begin, bad)
    far = seg_t.copy()
    far[0] = (200, 0, 0)
    with pytest.raises(RuntimeError):
        eng.set_candidates(seg_i, far, seg_begin, cand_j)
    # a shift the pair entries cannot hold (five boxes away) is refused at the evaluation
    far[0] = (5, 0, 0)
    eng.set_candidates(seg_i, far, seg_begin, cand_j)
    with pytest.raises(RuntimeError):
        eng.compute(S.pos, S.box)
