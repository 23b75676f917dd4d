"""The differentiation workload at its own sizes: per-type parameter gradients of the total energy and of the
force-matching loss L = sum |F - F_target|^2 on (a) 16 of the 256 boxes of 64 waters, in one batched launch,
and (b) the 8550-atom dimethylphenol liquid, with the engine at the workload's tol 1e-8.

The goldens (tests/golden/grad_*.npz, from tests/golden/make_golden.py) are central differences of the
reference pgm_core itself (h = 1e-5 relative to each type's value, or to its kind's RMS value where that is
larger) with F_target from pgm_core at every
per-type parameter scaled by (1 + N(0, 0.05)); they are taken at tol 1e-12 so that the differences carry no CG
noise.  Bar: 1e-5 relative, per parameter kind as a vector norm and per element against the larger of the
element and 1e-3 of the kind's largest element (the energy differences of a 2.7e5 kJ/mol system resolve small
gradients only to about 1e-4 of their size)."""

import numpy as np
import pytest

from conftest import GOLDEN, PKG

pytestmark = pytest.mark.gpu

NAMES = ("q", "cov_strength", "alpha", "radius")


def per_type(values, index, ntypes):
    out = np.zeros(ntypes)
    np.add.at(out, index, values)
    return out


def check(got, fd, what, lim=1e-5, elem=(1e-5, 1e-3)):
    """The kind's vector within lim (norm-relative); each element within elem[0] of the larger of itself and
    elem[1] times the kind's largest element."""
    got = np.asarray(got, np.float64)
    fd = np.asarray(fd, np.float64)
    assert np.linalg.norm(got - fd) <= lim * np.linalg.norm(fd), (what, got, fd)
    floor = elem[1] * np.abs(fd).max()
    assert (np.abs(got - fd) <= elem[0] * np.maximum(np.abs(fd), floor) + 1e-300).all(), (what, got, fd)


# Mixed precision's force-matching gradient: the 1e-5 bar holds for each parameter kind as a vector; single
# elements may reach 1e-4 of the larger of themselves and 1 % of their kind's largest, because w = 2 (F - F_target)
# is a difference of forces about 20 times smaller than the forces (F_target from parameters perturbed by 5 %), so
# the mixed path's force error (3e-7 relative RMS) enters dL/dtheta about 20 times enlarged.  (Measured on a B200:
# the largest element error of the 64-water batch moves between 3e-5 and 5e-5 from run to run with the float
# atomics' order; the FP64 path holds every element to 1e-5.)
FM_ELEM = {PKG.FP64: (1e-5, 1e-3), PKG.MIXED: (1e-4, 1e-2)}
# and the kind's norm: FP64 1e-5; mixed 2e-5, because a kind with one type (the water's bond dipole) is a single
# element, measured on a B200 between 0.6e-5 and 1.2e-5 from run to run (the same amplification of the mixed
# forces' error through w)
FM_NORM = {PKG.FP64: 1e-5, PKG.MIXED: 2e-5}


def engine(S, precision, tol=1e-8):
    e = PKG.Engine(PKG.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=6, tol=tol, max_iter=1000, peek=0.0,
                                predictor=0, ke=PKG.systems.KE_DEFAULT, precision=precision))
    return e


@pytest.fixture(scope="module")
def water64():
    d = np.load(GOLDEN / "grad_water64x16.npz")
    boxes = PKG.systems.water64_boxes(nsys=int(d["boxes"].max()) + 1)
    return [boxes[int(k)] for k in d["boxes"]], d


@pytest.mark.parametrize("precision", [PKG.FP64, PKG.MIXED])
def test_water64_batch_energy_gradients(water64, precision):
    boxes, d = water64
    eng = engine(boxes[0], precision)
    eng.set_systems(boxes)
    out = eng.compute_batch(np.concatenate([s.pos for s in boxes]), np.stack([s.box for s in boxes]))
    g = eng.param_grad()
    eng.close()
    off, coff = 0, 0
    for k, S in zip(d["boxes"], boxes):
        assert abs(out["energies"][list(d["boxes"]).index(k), :5].sum() - float(d[f"b{k}_energy"])) <= \
            1e-6 * abs(float(d[f"b{k}_energy"]))
        for name in NAMES:
            if name == "cov_strength":
                part, ty = g[name][coff:coff + len(S.cov_atom)], S.cov_types
            else:
                part, ty = g[name][off:off + S.n], S.types
            fd = d[f"b{k}_dE_{name}"]
            check(per_type(part, ty, len(fd)), fd, (int(k), name))
        off += S.n
        coff += len(S.cov_atom)


@pytest.mark.parametrize("precision", [PKG.FP64, PKG.MIXED])
def test_water64_batch_force_matching_gradients(water64, precision):
    """The 16 boxes in ONE batched evaluation and ONE batched adjoint (every system's solve at once)."""
    grad_mod = __import__("pgm_md_b200.autograd", fromlist=["autograd"])
    boxes, d = water64
    eng = engine(boxes[0], precision)
    eng.set_systems(boxes)
    Ft = np.concatenate([d[f"b{k}_Ft"] for k in d["boxes"]])
    L, g, _ = grad_mod.force_matching_atom_grads(eng, boxes, Ft, tol=1e-8)
    eng.close()
    assert abs(L - sum(float(d[f"b{k}_loss"]) for k in d["boxes"])) <= 1e-5 * L
    off, coff = 0, 0
    for k, S in zip(d["boxes"], boxes):
        for name in NAMES:
            if name == "cov_strength":
                part, ty = g[name][coff:coff + len(S.cov_atom)], S.cov_types
            else:
                part, ty = g[name][off:off + S.n], S.types
            fd = d[f"b{k}_dL_{name}"]
            check(per_type(part, ty, len(fd)), fd, (int(k), name), lim=FM_NORM[precision], elem=FM_ELEM[precision])
        off += S.n
        coff += len(S.cov_atom)


@pytest.fixture(scope="module")
def dmp():
    d = np.load(GOLDEN / "grad_dimethylphenol8550.npz")
    return PKG.systems.dimethylphenol8550(tol=1e-8), d


@pytest.mark.parametrize("precision", [PKG.FP64, PKG.MIXED])
def test_dimethylphenol8550_energy_gradients(dmp, precision):
    S, d = dmp
    eng = engine(S, precision)
    eng.set_system(S)
    r = eng.compute(S.pos, S.box)
    g = eng.param_grad()
    eng.close()
    assert abs(r.energy - float(d["energy"])) <= 1e-6 * abs(float(d["energy"]))
    for name in NAMES:
        ty = S.cov_types if name == "cov_strength" else S.types
        check(per_type(g[name], ty, len(d["dE_" + name])), d["dE_" + name], name)


@pytest.mark.parametrize("precision", [PKG.FP64, PKG.MIXED])
def test_dimethylphenol8550_force_matching_gradients(dmp, precision):
    grad_mod = __import__("pgm_md_b200.autograd", fromlist=["autograd"])
    S, d = dmp
    eng = engine(S, precision)
    eng.set_system(S)
    L, g, _ = grad_mod.force_matching_atom_grads(eng, S, d["Ft"], tol=1e-8)
    eng.close()
    assert abs(L - float(d["loss"])) <= (1e-6 if precision == PKG.FP64 else 1e-5) * float(d["loss"])
    for name in NAMES:
        ty = S.cov_types if name == "cov_strength" else S.types
        check(per_type(g[name], ty, len(d["dL_" + name])), d["dL_" + name], name, lim=FM_NORM[precision],
              elem=FM_ELEM[precision])
