"""The FP64 oracle against the reference: the committed outputs of the reference pgm_core itself, the
pGM-JAX goldens the reference ships, the reference's finite-difference known-answer test, and (when it is
built here) the reference library live."""

import numpy as np
import pytest

from conftest import GOLDEN, PKG, load_dmp_real, load_golden_system, oracle_settings, oracle_topology
from oracle import pgm_oracle as O
from oracle import ref as R

TERMS = ("direct", "reciprocal", "self", "background", "polarization")


@pytest.mark.parametrize("name", ["tiny_triclinic", "water216"])
def test_oracle_matches_reference_outputs(name):
    S, d = load_golden_system(name)
    eng = O.Engine(oracle_topology(S), oracle_settings(S))
    e = eng.compute(S.pos, S.box)
    assert abs(e - float(d["energy"])) <= 1e-12 * abs(float(d["energy"]))
    for k, t in enumerate(TERMS):
        assert abs(eng.terms[t] - d["terms"][k]) <= 1e-10 * max(1.0, abs(d["terms"][k]))
    assert np.linalg.norm(eng.forces - d["forces"]) <= 1e-12 * np.linalg.norm(d["forces"])
    assert np.abs(eng.strain - d["strain"]).max() <= 1e-10 * np.abs(d["strain"]).max()
    assert np.abs(eng.mu - d["mu"]).max() <= 1e-12 * np.abs(d["mu"]).max()
    assert np.abs(eng.perm - d["perm"]).max() <= 1e-14
    assert eng.iterations == int(d["iterations"])
    i, j, _ = O.pair_set(S.pos, S.box, S.cutoff)
    assert len(i) == int(d["npairs"])


@pytest.mark.parametrize("level", ["q", "qp", "qi", "qpi"])
def test_oracle_matches_pgmjax_goldens(level):
    g = np.load(GOLDEN / "w512_pgmjax.npz")
    cs = g["cov_strength"] if "p" in level else 0 * g["cov_strength"]
    top = O.Topology(g["q"], g["radius"], g["alpha"], g["cov_atom"], g["cov_partner"], cs)
    s = O.Settings(cutoff=float(g["cutoff"]), beta=float(g["beta"]), grid=tuple(g["grid"]), order=int(g["order"]),
                   tol=float(g["tol"]), max_iter=1000, peek=0.0, predictor=0, ke=float(g["ke"]),
                   polarizable="i" in level)
    eng = O.Engine(top, s)
    e = eng.compute(g["pos"], g["H"])
    eref = float(g[f"{level}_energy"])
    assert abs(e - eref) <= 1e-12 * abs(eref)
    F = g[f"{level}_forces"]
    assert np.linalg.norm(eng.forces - F) <= 1e-12 * np.linalg.norm(F)
    assert np.abs(eng.mu - g[f"{level}_mu"]).max() <= 1e-12
    assert eng.iterations == int(g[f"{level}_iterations"])


def test_oracle_matches_reference_on_real_dmp_liquid():
    """The numpy oracle on the reference's real 8550-atom dimethylphenol liquid (amber/test/dmp, the system the
    benchmark's synthetic stand-in imitates) against pgm_core's outputs at tol 1e-10: energy and iteration count;
    forces and induced dipoles to the float32 storage of the fixture."""
    S, d = load_dmp_real()
    eng = O.Engine(oracle_topology(S), oracle_settings(S))
    e = eng.compute(S.pos, S.box)
    assert abs(e - float(d["energy"])) <= 1e-12 * abs(float(d["energy"]))
    assert eng.iterations == int(d["iterations"])
    F = d["forces"].astype(np.float64)
    assert np.linalg.norm(eng.forces - F) <= 2e-7 * np.linalg.norm(F)
    assert np.abs(eng.mu - d["mu"]).max() <= 2e-7 * np.abs(d["mu"]).max()


def test_oracle_finite_differences():
    """core/tests/test_core.cpp: central differences of forces (h = 1e-5 nm) and of the strain derivative
    (h = 1e-6, upper triangle) agree to 1e-5 of the largest component."""
    S = PKG.systems.tiny_triclinic(nmol=12, seed=5)
    s = oracle_settings(S, tol=1e-13)
    top = oracle_topology(S)
    eng = O.Engine(top, s)
    eng.compute(S.pos, S.box)
    F, Sd = eng.forces.copy(), eng.strain.copy()
    h = 1e-5
    err, fmax = 0.0, np.abs(F).max()
    for i in (0, 1, 7):
        for k in range(3):
            p = S.pos.copy()
            p[i, k] += h
            ep = O.Engine(top, s).compute(p, S.box, want_forces=False)
            p[i, k] -= 2 * h
            em = O.Engine(top, s).compute(p, S.box, want_forces=False)
            err = max(err, abs(-(ep - em) / (2 * h) - F[i, k]))
    assert err <= 1e-5 * fmax
    hs = 1e-6
    errS = 0.0
    for a in range(3):
        for b in range(a, 3):
            ef = []
            for eps in (hs, -hs):
                p = S.pos.copy()
                p[:, a] += eps * p[:, b]
                bx = S.box.copy()
                bx[:, a] += eps * bx[:, b]
                ef.append(O.Engine(top, s).compute(p, bx, want_forces=False))
            errS = max(errS, abs((ef[0] - ef[1]) / (2 * hs) - Sd[3 * a + b]))
    assert errS <= 1e-5 * np.abs(Sd).max()


def test_param_gradients_finite_differences():
    """The oracle's analytic parameter gradients (the FP64 reference gradient) against central differences."""
    S = PKG.systems.tiny_triclinic(nmol=8, seed=11)
    s = oracle_settings(S, tol=1e-13)
    eng = O.Engine(oracle_topology(S), s)
    eng.compute(S.pos, S.box)
    g = eng.param_gradients()
    for field, idx in (("q", [0, 4]), ("radius", [1, 6]), ("alpha", [2, 3]), ("cov_strength", [0, 5])):
        for k in idx:
            vals = []
            for sgn in (1, -1):
                T = oracle_topology(S)
                arr = getattr(T, field).copy()
                h = 1e-5 * abs(arr[k])
                arr[k] += sgn * h
                setattr(T, field, arr)
                vals.append(O.Engine(T, s).compute(S.pos, S.box, want_forces=False))
            fd = (vals[0] - vals[1]) / (2 * h)
            assert abs(fd - g[field][k]) <= 1e-5 * max(abs(fd), 1e-3), (field, k, fd, g[field][k])


def test_pair_set_knife_edge():
    """Pairs exactly at the cutoff (r^2 == rc^2 in double) are out, one ulp inside are in."""
    rc = 0.9
    box = np.eye(3) * 2.0
    pos = np.array([[0.1, 0.1, 0.1], [0.1 + rc, 0.1, 0.1], [0.1, 0.1 + np.nextafter(rc, 0), 0.1],
                    [1.0, 1.0, 1.0], [1.0, 1.0, 1.0 + 1.0]])
    i, j, x = O.pair_set(pos, box, rc)
    got = set(zip(i.tolist(), j.tolist()))
    r2 = lambda a, b: (lambda v: v[0] * v[0] + v[1] * v[1] + v[2] * v[2])(O.min_image((pos[a] - pos[b])[None], box)[0])
    for a in range(5):
        for b in range(a + 1, 5):
            assert ((a, b) in got) == (r2(a, b) < rc * rc)
    assert (0, 1) not in got and (0, 2) in got


def test_round_half_away():
    v = np.array([0.5, -0.5, 1.5, -2.5, 0.49999999999999994, 2.4999999999999996, 0.0])
    np.testing.assert_array_equal(O.round_half_away(v), [1.0, -1.0, 2.0, -3.0, 0.0, 2.0, 0.0])


@pytest.mark.skipif(not R.available(), reason="oracle/_ref not built")
def test_oracle_matches_reference_live():
    S = PKG.systems.tiny_triclinic(nmol=16, seed=21)
    s = oracle_settings(S, tol=1e-10, predictor=2, peek=0.65)
    ref = R.RefEngine(oracle_topology(S), s)
    ora = O.Engine(oracle_topology(S), s)
    rng = np.random.default_rng(0)
    pos = S.pos.copy()
    for step in range(6):   # the mu3/mu4 predictor and the history over moved steps
        pos = pos + rng.uniform(-0.002, 0.002, pos.shape)
        e1 = ref.compute(pos, S.box)
        e2 = ora.compute(pos, S.box)
        assert abs(e1 - e2) <= 1e-11 * abs(e1)
        assert np.linalg.norm(ref.forces - ora.forces) <= 1e-10 * np.linalg.norm(ref.forces)
        assert ref.iterations() == ora.iterations


def test_pair_set_cells_equals_all_pairs():
    S = PKG.systems.water216()
    i, j, _ = O.pair_set(S.pos, S.box, 0.6)
    ci, cj = O.pair_set_cells(S.pos, S.box, 0.6)
    assert np.array_equal(i, ci) and np.array_equal(j, cj)


def test_oracle_force_matching_adjoint_against_reference_differences():
    """The oracle's analytic force-matching gradient (one adjoint solve, tangent pair and PME passes) against
    central differences of the reference pgm_core's loss: per type, on two of the 64-water boxes of the
    differentiation workload (tests/golden/grad_water64x16.npz), to 1e-6 relative."""
    import numpy as np
    from oracle import pgm_oracle as O
    d = np.load(GOLDEN / "grad_water64x16.npz")
    boxes = PKG.systems.water64_boxes(nsys=2)
    for k in (0, 1):
        S = boxes[k]
        e = O.Engine(oracle_topology(S), oracle_settings(S, tol=1e-12))
        e.compute(S.pos, S.box)
        L, g = e.force_matching_gradients(d[f"b{k}_Ft"])
        assert abs(L - float(d[f"b{k}_loss"])) <= 1e-8 * L
        for name in ("q", "cov_strength", "alpha", "radius"):
            ty = S.cov_types if name == "cov_strength" else S.types
            fd = d[f"b{k}_dL_{name}"]
            got = np.zeros(len(fd))
            np.add.at(got, ty, g[name])
            assert np.linalg.norm(got - fd) <= 1e-6 * np.linalg.norm(fd), (k, name, got, fd)
