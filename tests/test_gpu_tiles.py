"""The cell-group tile spread and gather (PME kernels 3, mixed precision, one system): a block takes a group of
the pair search's cells, accumulates (spread) or reads (gather) the grid window of its atoms' stencils in shared
memory, and meets the grid once per window point.  Held to the reference pgm_core's outputs and, where no
fixture exists, to the FP64 path (itself held to the reference at 1e-7), with the warp-per-atom kernels
(PME kernels 0) beside them for the CG iteration count.

The small goldens (216 waters on 20^3, the 72-atom triclinic box on 48^3) have one group whose window is wider
than the grid: they run the tile kernels' direct path (global atomics / loads per point).  The 8550-atom liquid
(9 cells a side, groups of 2^3 cells) and the 98304-atom box (22 cells a side, groups of 4^3) run the tiles.

Bars as for every mixed path at tol 1e-10: energy 1e-6 relative, forces and induced dipoles 1e-5 relative RMS;
the warp-per-atom kernels' iteration count within one."""

import numpy as np
import pytest

from conftest import PKG, load_dmp_real, load_golden_system

pytestmark = pytest.mark.gpu


def rel_rms(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def engine(S, mode, pme, precision=None, tol=1e-10, lanes=16, skin=0.0, predictor=0, order=None):
    e = PKG.Engine(PKG.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=order or S.order, tol=tol,
                                max_iter=500, peek=0.0, predictor=predictor, ke=PKG.systems.KE_DEFAULT,
                                precision=PKG.MIXED if precision is None else precision, skin=skin))
    e.set_system(S)
    e.set_pair_lanes(lanes)
    e.set_transforms(mode)
    e.set_pme_kernels(pme)
    return e


def golden(name):
    if name == "dmp8550_real":
        return load_dmp_real()
    return load_golden_system(name)


@pytest.mark.parametrize("name", ["water216", "tiny_triclinic", "dmp8550_real"])
@pytest.mark.parametrize("mode", [0, 3])
def test_tile_spread_gather_against_reference(name, mode):
    """cuFFT (transforms 0) and the grid kernel (3, whose CG gather carries A p and alph) with the tile kernels."""
    S, d = golden(name)
    eng = engine(S, mode, 3)
    assert eng.pme_kernels() == 3
    r = eng.compute(S.pos, S.box)
    mu = eng.induced_dipoles()
    base = engine(S, mode, 0)
    g = base.compute(S.pos, S.box)
    e_ref = float(d["energy"])
    F = np.asarray(d["forces"], np.float64)
    assert abs(r.energy - e_ref) <= 1e-6 * abs(e_ref), (r.energy, e_ref)
    assert rel_rms(r.forces, F) <= 1e-5
    assert rel_rms(mu, d["mu"]) <= 1e-5
    assert abs(r.iterations - g.iterations) <= 1
    kt = eng.kernel_times(reps=3)
    assert kt["spread"] > 0 and kt["gather"] > 0
    eng.close()
    base.close()


@pytest.mark.parametrize("order", [4, 5, 8])
def test_tile_kernels_other_orders(order):
    """Orders 4, 5, 8 on the 8550-atom liquid (tiles), against the FP64 warp-per-atom path of the same order."""
    S, _ = golden("dmp8550_real")
    eng = engine(S, 0, 3, order=order)
    assert eng.pme_kernels() == 3
    r = eng.compute(S.pos, S.box)
    mu = eng.induced_dipoles()
    eng.close()
    ref = engine(S, 0, 0, precision=PKG.FP64, order=order)
    g = ref.compute(S.pos, S.box)
    mur = ref.induced_dipoles()
    ref.close()
    assert abs(r.energy - g.energy) <= 1e-6 * abs(g.energy), (order, r.energy, g.energy)
    assert rel_rms(r.forces, g.forces) <= 1e-5, order
    assert rel_rms(mu, mur) <= 1e-5, order


def test_tile_kernels_moving_atoms_kept_list():
    """MD-like steps with a 0.15 nm skin (the list kept while the atoms drift from the cells they were sorted
    into; windows grow by the drift) and the mu4 predictor: at every step the tile kernels against the
    warp-per-atom kernels of an engine fed the same positions."""
    S, _ = golden("dmp8550_real")
    rng = np.random.default_rng(5)
    tiles = engine(S, 3, 3, tol=1e-8, skin=0.15, predictor=4)
    warp = engine(S, 3, 0, tol=1e-8, skin=0.15, predictor=4)
    assert tiles.pme_kernels() == 3
    pos = S.pos.copy()
    vel = rng.normal(0.0, 0.004, pos.shape)   # nm per step
    for step in range(8):
        a = tiles.compute(pos, S.box)
        b = warp.compute(pos, S.box)
        assert abs(a.energy - b.energy) <= 2e-6 * abs(b.energy), (step, a.energy, b.energy)
        assert rel_rms(a.forces, b.forces) <= 2e-5, step
        pos = pos + vel
    tiles.close()
    warp.close()


def test_tile_kernels_not_applicable():
    """FP64 engines, batches and order 7 keep the warp-per-atom kernels; pme_kernels() tells."""
    S, _ = golden("water216")
    e = engine(S, 0, 3, precision=PKG.FP64, tol=1e-8)
    assert e.pme_kernels() == 0
    e.close()
    e = engine(S, 0, 3, order=7)
    assert e.pme_kernels() == 0
    e.close()
    boxes = PKG.systems.water_batch()[:4]
    s0 = boxes[0]
    b = PKG.Engine(PKG.Settings(cutoff=s0.cutoff, beta=s0.beta, grid=s0.grid, order=6, tol=1e-5, max_iter=500,
                                peek=0.0, predictor=0, ke=PKG.systems.KE_DEFAULT, precision=PKG.MIXED))
    b.set_systems(boxes)
    b.set_pme_kernels(3)
    assert b.pme_kernels() == 0
    b.close()
