"""The persistent CG kernel (transforms mode 4: the whole mixed-precision CG loop of one system as one
cooperative launch, PME planes spread, transformed and gathered in shared memory, the direct-space pass on the
other SMs) against the reference pgm_core's outputs and against the engine's own graph loop (mode 3), on the
committed goldens: the 216-water box (20^3 grid), the triclinic test box (48^3) and the real 8550-atom
dimethylphenol liquid (48^3).  Bars as for every mixed path: energy 1e-6, forces 1e-5 relative RMS at tol 1e-10
against the oracle; the CG iteration count of the graph loop within one."""

import numpy as np
import pytest

from conftest import PKG, load_dmp_real, load_golden_system

pytestmark = pytest.mark.gpu


def mixed_engine(S, mode, tol=1e-10, lanes=16, pme=0):
    e = PKG.Engine(PKG.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=6, tol=tol, max_iter=500, peek=0.0,
                                predictor=0, ke=PKG.systems.KE_DEFAULT, precision=PKG.MIXED, skin=0.0))
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
@pytest.mark.parametrize("lanes", [8, 32])
def test_persistent_cg_against_reference(name, lanes):
    S, d = golden(name)
    eng = mixed_engine(S, 4, lanes=lanes)
    assert eng.transforms() == 4
    r = eng.compute(S.pos, S.box)
    mu = eng.induced_dipoles()
    ref_graph = mixed_engine(S, 3, lanes=lanes)
    g = ref_graph.compute(S.pos, S.box)
    e_ref = float(d["energy"])
    assert abs(r.energy - e_ref) <= 1e-6 * abs(e_ref), (r.energy, e_ref)
    F = np.asarray(d["forces"], np.float64)
    assert np.linalg.norm(r.forces - F) <= 1e-5 * np.linalg.norm(F)
    assert np.linalg.norm(mu - d["mu"]) <= 1e-5 * np.linalg.norm(d["mu"])
    # the persistent kernel's spread sums in fixed point and its reductions in another fixed order: at tol 1e-10
    # the FP32 operator's rounding moves the last iteration by at most one
    assert abs(r.iterations - g.iterations) <= 1
    assert abs(r.energy - g.energy) <= 1e-6 * abs(e_ref)
    assert np.linalg.norm(r.forces - g.forces) <= 1e-5 * np.linalg.norm(F)
    # the launch count: the whole loop is one launch whatever the iterations
    assert eng.kernel_launches() < ref_graph.kernel_launches()
    eng.close()
    ref_graph.close()


def test_persistent_cg_repeated_calls_and_tolerance():
    """The benchmark's tolerance (1e-5) on the 8550-atom liquid, three calls in a row: the same iterations and
    energies within the mixed path's run-to-run spread (the field passes around the loop use float atomics)."""
    S, d = golden("dmp8550_real")
    eng = mixed_engine(S, 4, tol=1e-5)
    rs = [eng.compute(S.pos, S.box) for _ in range(3)]
    e_ref = float(d["energy"])
    F = np.asarray(d["forces"], np.float64)
    for r in rs:
        assert r.iterations == rs[0].iterations
        assert abs(r.energy - e_ref) <= 1e-6 * abs(e_ref)
        assert np.linalg.norm(r.forces - F) <= 1e-5 * np.linalg.norm(F)
    eng.close()


def test_persistent_cg_not_applicable_falls_back():
    """Batched engines and FP64 engines do not take mode 4; transforms() reports what runs."""
    S, _ = golden("water216")
    e = PKG.Engine(PKG.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=6, tol=1e-8, max_iter=500, peek=0.0,
                                predictor=0, ke=PKG.systems.KE_DEFAULT, precision=PKG.FP64))
    e.set_system(S)
    e.set_transforms(4)
    assert e.transforms() != 4
    e.close()


@pytest.mark.parametrize("name", ["water216", "tiny_triclinic", "dmp8550_real"])
@pytest.mark.parametrize("mode", [0, 3])
def test_plane_owner_spread_gather_against_reference(name, mode):
    """The plane-owner spread and gather (PME kernels 1: tiles of 16 rows of an x-plane in shared memory) with
    cuFFT (mode 0) and with the grid kernel (mode 3), against the reference's outputs and against the warp-per-atom
    kernels (the same CG iterations)."""
    S, d = golden(name)
    eng = mixed_engine(S, mode, pme=1)
    assert eng.pme_kernels() == 1
    r = eng.compute(S.pos, S.box)
    base = mixed_engine(S, mode, pme=0)
    g = base.compute(S.pos, S.box)
    e_ref = float(d["energy"])
    F = np.asarray(d["forces"], np.float64)
    assert abs(r.energy - e_ref) <= 1e-6 * abs(e_ref), (r.energy, e_ref)
    assert np.linalg.norm(r.forces - F) <= 1e-5 * np.linalg.norm(F)
    assert abs(r.iterations - g.iterations) <= 1
    kt = eng.kernel_times(reps=3)
    assert kt["spread"] > 0 and kt["gather"] > 0
    eng.close()
    base.close()


@pytest.mark.parametrize("name", ["tiny_triclinic", "dmp8550_real"])
def test_persistent_kernel_with_plane_owner_passes(name):
    """Mode 4 with the plane-owner spread and gather for the passes around its loop (the two share the plane
    bins), against the reference's outputs."""
    S, d = golden(name)
    eng = mixed_engine(S, 4, pme=1)
    assert eng.transforms() == 4 and eng.pme_kernels() == 1
    r = eng.compute(S.pos, S.box)
    e_ref = float(d["energy"])
    F = np.asarray(d["forces"], np.float64)
    assert abs(r.energy - e_ref) <= 1e-6 * abs(e_ref)
    assert np.linalg.norm(r.forces - F) <= 1e-5 * np.linalg.norm(F)
    eng.close()


@pytest.mark.parametrize("mode", [3, 4])
def test_kept_list_first_pass(mode):
    """With a kept Verlet list (skin 0.15 nm) the first pass compacts the list and forms the permanent field's pair
    part on the main stream beside its PME half on the side stream; the graph loop (3) and the persistent kernel
    (4), two calls at the same positions (the list built once), against the reference outputs on the real
    8550-atom liquid at tol 1e-10."""
    S, d = golden("dmp8550_real")
    e = PKG.Engine(PKG.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=6, tol=1e-10, max_iter=500,
                                peek=0.0, predictor=0, ke=PKG.systems.KE_DEFAULT, precision=PKG.MIXED, skin=0.15))
    e.set_system(S)
    e.set_pair_lanes(16)
    e.set_transforms(mode)
    assert e.transforms() == mode
    e_ref = float(d["energy"])
    F = np.asarray(d["forces"], np.float64)
    for _ in range(2):
        r = e.compute(S.pos, S.box)
        assert abs(r.energy - e_ref) <= 1e-6 * abs(e_ref), (r.energy, e_ref)
        assert np.linalg.norm(r.forces - F) <= 1e-5 * np.linalg.norm(F)
    assert e.list_builds() == 1
    e.close()
