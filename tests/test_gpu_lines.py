"""The float4 line spread and gather (PME kernels 2, mixed precision): a thread per (atom, x-plane of its
stencil) adds or loads each z line as aligned float4 words, with scalar atomics / loads where a line wraps
around z or the rows are not a whole number of words.  Held to the reference pgm_core's outputs and to the
oracle, with the warp-per-atom kernels (PME kernels 0) run beside them for the CG iteration count.

Bars as for every mixed path at tol 1e-10: energy 1e-6 relative, forces and induced dipoles 1e-5 relative RMS;
the iteration count of the warp-per-atom kernels within one (float sums in another order)."""

import numpy as np
import pytest

from conftest import GOLDEN, PKG, load_dmp_real, load_golden_system, oracle_settings, oracle_topology
from oracle import pgm_oracle as O

pytestmark = pytest.mark.gpu


def rel_rms(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def mixed_engine(S, mode, pme, tol=1e-10, lanes=16):
    e = PKG.Engine(PKG.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=S.order, tol=tol, max_iter=500,
                                peek=0.0, predictor=0, ke=PKG.systems.KE_DEFAULT, precision=PKG.MIXED, skin=0.0))
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
def test_line_spread_gather_against_reference(name, mode):
    """cuFFT (transforms 0) and the grid kernel (3, whose CG gather carries A p and alph) with the line kernels."""
    S, d = golden(name)
    eng = mixed_engine(S, mode, 2)
    assert eng.pme_kernels() == 2
    r = eng.compute(S.pos, S.box)
    mu = eng.induced_dipoles()
    base = mixed_engine(S, mode, 0)
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
def test_line_kernels_other_orders(order):
    """The orders the line kernels are built for besides 6, on a 48^3 triclinic box (rows of whole words) and a
    30^3 one (rows of 7.5 words: every line through the scalar path), against the oracle."""
    for grid in (48, 30):
        S = PKG.systems.tiny_triclinic(nmol=16, seed=21)
        S.order = order
        S.grid = (grid, grid, grid)
        eng = mixed_engine(S, 0, 2)
        assert eng.pme_kernels() == 2
        r = eng.compute(S.pos, S.box)
        eng.close()
        ora = O.Engine(oracle_topology(S), oracle_settings(S))
        e = ora.compute(S.pos, S.box)
        assert abs(r.energy - e) <= 1e-6 * abs(e), (order, grid, r.energy, e)
        assert rel_rms(r.forces, ora.forces) <= 1e-5, (order, grid)


def test_line_kernels_not_applicable():
    """FP64 engines and order 7 keep the warp-per-atom kernels; pme_kernels() tells."""
    S, _ = golden("water216")
    e = PKG.Engine(PKG.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=6, tol=1e-8, max_iter=500, peek=0.0,
                                predictor=0, ke=PKG.systems.KE_DEFAULT, precision=PKG.FP64))
    e.set_system(S)
    e.set_pme_kernels(2)
    assert e.pme_kernels() == 0
    e.close()
    S.order = 7
    e = mixed_engine(S, 0, 2)
    assert e.pme_kernels() == 0
    e.close()
    with pytest.raises(Exception):
        mixed_engine(S, 0, 4)


def test_line_kernels_batch_sample():
    """The 32 sample boxes of the 1024-box batch in one launch (grids 8..25: rows of whole words and not, system
    grid offsets aligned and not), per system against the reference pgm_core, the CG retiring systems as they
    converge (the gather maps its threads over the active systems' slots)."""
    boxes = PKG.systems.water_batch()
    d = np.load(GOLDEN / "ref_water_batch_sample.npz")
    sample = [boxes[int(b)] for b in d["sample"]]
    s0 = sample[0]
    eng = PKG.Engine(PKG.Settings(cutoff=s0.cutoff, beta=s0.beta, grid=s0.grid, order=6, tol=1e-5, max_iter=500,
                                  peek=0.0, predictor=0, ke=PKG.systems.KE_DEFAULT, precision=PKG.MIXED))
    eng.set_systems(sample)
    eng.set_pme_kernels(2)
    assert eng.pme_kernels() == 2
    out = eng.compute_batch(np.concatenate([s.pos for s in sample]), np.stack([s.box for s in sample]))
    mu = eng.induced_dipoles()
    eng.close()
    aoff = 0
    foff = 0
    for k, S in enumerate(sample):
        n = S.n
        e_ref = float(d["energy"][k])
        assert abs(out["energies"][k, :5].sum() - e_ref) <= 1e-6 * abs(e_ref), k
        assert rel_rms(out["forces"][aoff:aoff + n], d["forces"][foff:foff + n]) <= 1e-5, k
        assert rel_rms(mu[aoff:aoff + n], d["mu"][foff:foff + n]) <= 1e-4, k
        aoff += n
        foff += n
