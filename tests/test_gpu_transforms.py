"""The field passes' transforms by the cluster kernel (a thread-block cluster per system holding its half
spectrum in distributed shared memory), by the split path (cuFFT 2D plans over the x-planes, one kernel for
the x-lines with the influence product) and by the grid kernel (one cooperative kernel, a block per x-plane,
planes and x-lines exchanged through L2 between two barriers) against the cuFFT 3D plans + influence product
path: the same energies and forces (FP64 within 1e-12 relative, mixed within 1e-6 in energy and 1e-5 relative
RMS in forces), for one system (16 blocks per cluster) and a batch of small systems (smaller clusters; grid
kernel blocks of several grid shapes in one launch); grids with a prime factor above 5 or beyond 64 points
stay on cuFFT."""

import numpy as np
import pytest

from conftest import PKG

pytestmark = pytest.mark.gpu


def rel_rms(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def settings(S, precision):
    return PKG.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=S.order, tol=1e-10, max_iter=1000, peek=0.0,
                        predictor=0, ke=PKG.systems.KE_DEFAULT, precision=precision)


@pytest.mark.parametrize("mode", [1, 2, 3])
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name", ["water216", "tiny_triclinic"])
def test_transforms_single_system(precision, mode, name):
    # 20^3 and 48^3 grids
    S = PKG.systems.water216() if name == "water216" else PKG.systems.tiny_triclinic(nmol=20, seed=9)
    out = []
    for m in (0, mode):
        eng = PKG.Engine(settings(S, precision))
        eng.set_system(S)
        eng.set_transforms(m)
        assert eng.transforms() == m
        out.append(eng.compute(S.pos, S.box))
        eng.close()
    a, b = out
    lim_e, lim_f = (1e-12, 1e-12) if precision == 0 else (1e-6, 1e-5)
    assert abs(a.energy - b.energy) <= lim_e * abs(a.energy)
    assert rel_rms(b.forces, a.forces) <= lim_f
    # the strain derivative too (the grid kernel's final pass sums the k-space strain itself)
    assert np.abs(b.strain - a.strain).max() <= lim_f * np.abs(a.strain).max()
    assert a.iterations == b.iterations or precision == 1


@pytest.mark.parametrize("K", [32, 40, 64])
@pytest.mark.parametrize("precision", [0, 1])
def test_grid_transforms_compiled_sizes(precision, K):
    # the grid kernel's compile-time sizes beside 48 (64^3 in FP64 takes 72 KB of shared memory per block)
    S = PKG.systems.waters(64, 12.4, seed=21, grid=(K, K, K), cutoff=6.0, tol=1e-10)
    out = []
    for m in (0, 3):
        eng = PKG.Engine(settings(S, precision))
        eng.set_system(S)
        eng.set_transforms(m)
        assert eng.transforms() == m
        out.append(eng.compute(S.pos, S.box))
        eng.close()
    a, b = out
    lim_e, lim_f = (1e-12, 1e-12) if precision == 0 else (1e-6, 1e-5)
    assert abs(a.energy - b.energy) <= lim_e * abs(a.energy)
    assert rel_rms(b.forces, a.forces) <= lim_f
    assert np.abs(b.strain - a.strain).max() <= lim_f * np.abs(a.strain).max()


@pytest.mark.parametrize("mode", [1, 2, 3])
@pytest.mark.parametrize("precision", [0, 1])
def test_transforms_batch(precision, mode):
    systems = []
    for k, (nm, K) in enumerate([(8, 8), (20, 9), (40, 12), (64, 15), (100, 16), (150, 18), (220, 20), (300, 24)]):
        L = (nm / 0.0334) ** (1 / 3)
        systems.append(PKG.systems.waters(nm, L, seed=50 + k, grid=(K, K, K), cutoff=min(9.0, L / 2.0), tol=1e-10))
    pos = np.concatenate([s.pos for s in systems])
    boxes = np.stack([s.box for s in systems])
    out = []
    for m in (0, mode):
        eng = PKG.Engine(PKG.Settings(cutoff=0.9, beta=3.5, grid=(24, 24, 24), order=6, tol=1e-10, max_iter=1000,
                                      peek=0.0, predictor=0, ke=PKG.systems.KE_DEFAULT, precision=precision))
        eng.set_systems(systems)
        eng.set_transforms(m)
        assert eng.transforms() == m
        out.append(eng.compute_batch(pos, boxes))
        eng.close()
    a, b = out
    lim = 1e-12 if precision == 0 else 1e-6
    assert np.all(np.abs(a["energies"] - b["energies"]) <= lim * np.abs(a["energies"]))
    assert rel_rms(b["forces"], a["forces"]) <= (1e-12 if precision == 0 else 1e-5)
    sa, sb = np.asarray(a["strain"]).reshape(len(systems), -1), np.asarray(b["strain"]).reshape(len(systems), -1)
    scale = np.abs(sa).max(axis=1, keepdims=True)
    assert np.all(np.abs(sb - sa) <= (1e-12 if precision == 0 else 1e-5) * scale)


def test_transforms_need_small_235_grids():
    S = PKG.systems.waters(64, 12.4, seed=3, grid=(14, 14, 14), cutoff=6.0, tol=1e-6)   # 14 = 2 * 7
    eng = PKG.Engine(settings(S, PKG.FP64))
    eng.set_system(S)
    for mode in (1, 2, 3):
        eng.set_transforms(mode)
        assert eng.transforms() == 0
    assert np.isfinite(eng.compute(S.pos, S.box).energy)
    S2 = PKG.systems.waters(64, 12.4, seed=3, grid=(12, 14, 14), cutoff=6.0, tol=1e-6)   # x extent 12: split only
    eng2 = PKG.Engine(settings(S2, PKG.FP64))
    eng2.set_system(S2)
    for mode in (1, 3):
        eng2.set_transforms(mode)
        assert eng2.transforms() == 0
    eng2.set_transforms(2)
    assert eng2.transforms() == 2
    ref = PKG.Engine(settings(S2, PKG.FP64))
    ref.set_system(S2)
    a, b = eng2.compute(S2.pos, S2.box), ref.compute(S2.pos, S2.box)
    assert abs(a.energy - b.energy) <= 1e-12 * abs(b.energy)
