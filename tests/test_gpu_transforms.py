"""The field passes' transforms by the cluster kernel (a thread-block cluster per system holding its half
spectrum in distributed shared memory) against the cuFFT plans + influence product path: the same energies and
forces (FP64 within 1e-12 relative, mixed within 1e-6 in energy and 1e-5 relative RMS in forces), for one
system (16 blocks per cluster) and a batch of many small systems (smaller clusters); grids with a prime factor
above 5 or beyond 64 points stay on cuFFT."""

import numpy as np
import pytest

from conftest import PKG

pytestmark = pytest.mark.gpu


def rel_rms(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def settings(S, precision):
    return PKG.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=S.order, tol=1e-10, max_iter=1000, peek=0.0,
                        predictor=0, ke=PKG.systems.KE_DEFAULT, precision=precision)


@pytest.mark.parametrize("precision", [0, 1])
def test_cluster_transforms_single_system(precision):
    S = PKG.systems.water216()   # 20^3 grid
    out = []
    for mode in (0, 1):
        eng = PKG.Engine(settings(S, precision))
        eng.set_system(S)
        eng.set_transforms(mode)
        assert eng.transforms() == mode
        out.append(eng.compute(S.pos, S.box))
        eng.close()
    a, b = out
    lim_e, lim_f = (1e-12, 1e-12) if precision == 0 else (1e-6, 1e-5)
    assert abs(a.energy - b.energy) <= lim_e * abs(a.energy)
    assert rel_rms(b.forces, a.forces) <= lim_f
    assert a.iterations == b.iterations or precision == 1


@pytest.mark.parametrize("precision", [0, 1])
def test_cluster_transforms_batch(precision):
    systems = []
    for k, (nm, K) in enumerate([(8, 8), (20, 9), (40, 12), (64, 15), (100, 16), (150, 18), (220, 20), (300, 24)]):
        L = (nm / 0.0334) ** (1 / 3)
        systems.append(PKG.systems.waters(nm, L, seed=50 + k, grid=(K, K, K), cutoff=min(9.0, L / 2.0), tol=1e-10))
    pos = np.concatenate([s.pos for s in systems])
    boxes = np.stack([s.box for s in systems])
    out = []
    for mode in (0, 1):
        eng = PKG.Engine(PKG.Settings(cutoff=0.9, beta=3.5, grid=(24, 24, 24), order=6, tol=1e-10, max_iter=1000,
                                      peek=0.0, predictor=0, ke=PKG.systems.KE_DEFAULT, precision=precision))
        eng.set_systems(systems)
        eng.set_transforms(mode)
        assert eng.transforms() == mode
        out.append(eng.compute_batch(pos, boxes))
        eng.close()
    a, b = out
    lim = 1e-12 if precision == 0 else 1e-6
    assert np.all(np.abs(a["energies"] - b["energies"]) <= lim * np.abs(a["energies"]))
    assert rel_rms(b["forces"], a["forces"]) <= (1e-12 if precision == 0 else 1e-5)


def test_cluster_transforms_need_small_235_grids():
    S = PKG.systems.waters(64, 12.4, seed=3, grid=(14, 14, 14), cutoff=6.0, tol=1e-6)   # 14 = 2 * 7
    eng = PKG.Engine(settings(S, PKG.FP64))
    eng.set_system(S)
    eng.set_transforms(1)
    assert eng.transforms() == 0
    assert np.isfinite(eng.compute(S.pos, S.box).energy)
