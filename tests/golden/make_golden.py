"""Generates the committed golden fixtures under tests/golden/ (run here, where the reference is mounted;
the fixtures travel, the reference does not):

  w512_pgmjax.npz   the reference's pGM-JAX FP64 goldens of 512 pGM3P-25 waters
                    (tests/data/ref_w512_{q,qp,qi,qpi}_novdw.npz of larryhuang98/pGM-MD: positions, box,
                    energies, forces, induced dipoles at tol 1e-10, no predictor, no peek) together with the
                    pGM parameters read from tests/data/water512/pgm3p25_512.prmtop (POL_GAUSS_* sections,
                    converted to nm as openmm/python/pgm_prmtop.py:96-116 does).
  ref_<name>.npz    outputs of the reference pgm_core itself (core/pgm_core.cpp, built from its sources
                    into oracle/_ref by oracle/Makefile) on the seeded synthetic systems: energy terms,
                    forces, strain derivative, induced and permanent dipoles, iterations, tol 1e-10,
                    predictor none, peek 0.
  gvdw_box.npz      the GVDW known-answer box of the reference (tests/data/gvdw_box.txt, written by
                    tests/gvdw_input.py: 512 waters, reduced triclinic box, radii, which atoms carry the van der
                    Waals term, the prmtop's excluded pairs) with pmemd-pgm's energies of it at 1 nm for the two
                    repulsion forms and their parameters (core/tests/test_gvdw.cpp:66-70).
  ref_water98304.npz           pgm_core on the 98304-atom water box (tol 1e-10; forces and dipoles float32)
  ref_water_batch_sample.npz   pgm_core on a stratified sample of 32 of the 1024 batch boxes (tol 1e-10)
  grad_water64x16.npz,
  grad_dimethylphenol8550.npz  central differences of pgm_core's energy and force-matching loss per parameter
                               type (GOLDEN_GRAD_TOL=1e-12 python tests/golden/make_golden.py grad)
  dmp8550_real.npz  the reference's real 8550-atom dimethylphenol liquid (amber/test/dmp: pGM parameters from
                    the POL_GAUSS_* sections of prmtop.gz, coordinates and box from the NetCDF restart restrt0)
                    with the benchmark's settings (cutoff 0.9 nm, beta 3.5 / nm, 48^3, order 6), and pgm_core's
                    outputs on it at tol 1e-10 (predictor none, peek 0).  The 450 molecules carry identical
                    parameters, so one molecule's 19 atoms and 38 covalent dipoles are stored (the system tiles
                    them); coordinates, forces and dipoles as float32 (the coordinates are the inputs of both
                    the reference run and the tests, so their rounding is part of the case).

    make -C oracle && PGM_REFERENCE=<reference tree> python tests/golden/make_golden.py [--ref <reference tree>]
"""

from __future__ import annotations

import importlib.util
import os
import re
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
def _reference_tree() -> Path:
    """The reference tree: --ref <path>, else $PGM_REFERENCE (no default: the fixtures are made where it lies)."""
    import os
    if "--ref" in sys.argv:
        return Path(sys.argv[sys.argv.index("--ref") + 1])
    if os.environ.get("PGM_REFERENCE"):
        return Path(os.environ["PGM_REFERENCE"])
    raise SystemExit("make_golden.py: give the reference tree with --ref <path> or PGM_REFERENCE")


REF = _reference_tree() if __name__ == "__main__" else None
OUT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))


def load_systems():
    spec = importlib.util.spec_from_file_location("pgm_md_b200_systems", ROOT / "pgm-md_b200" / "systems.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = mod
    spec.loader.exec_module(mod)
    return mod


def read_prmtop_sections(path, wanted):
    """Reads the named %FLAG sections of an Amber prmtop (fixed-width fields given by %FORMAT)."""
    out, name, fmt, lines = {}, None, None, []

    def flush():
        if name in wanted:
            m = re.match(r"\((\d+)([aAiIeEfF])(\d+)", fmt)
            width = int(m.group(3))
            kind = m.group(2).lower()
            toks = [ln[k:k + width].strip() for ln in lines for k in range(0, len(ln), width)]
            toks = [t for t in toks if t]
            out[name] = np.array([int(t) for t in toks]) if kind == "i" else np.array([float(t) for t in toks])

    for raw in open(path):
        line = raw.rstrip("\n")
        if line.startswith("%FLAG"):
            if name is not None:
                flush()
            name, fmt, lines = line.split()[1], None, []
        elif line.startswith("%FORMAT"):
            fmt = line[line.index("("):]
        elif line.startswith("%"):
            continue
        elif name is not None:
            lines.append(line)
    if name is not None:
        flush()
    return out


def w512():
    sec = read_prmtop_sections(REF / "tests/data/water512/pgm3p25_512.prmtop",
                               {"POL_GAUSS_MONOPOLES_LIST", "POL_GAUSS_RADII_LIST", "POL_GAUSS_POLARIZABILITY_LIST",
                                "POL_GAUSS_COVALENT_POINTERS_LIST", "POL_GAUSS_COVALENT_ATOMS_LIST",
                                "POL_GAUSS_COVALENT_DIPOLES_LIST"})
    nptr = sec["POL_GAUSS_COVALENT_POINTERS_LIST"].astype(np.int64)
    out = dict(q=sec["POL_GAUSS_MONOPOLES_LIST"], radius=sec["POL_GAUSS_RADII_LIST"] * 0.1,
               alpha=sec["POL_GAUSS_POLARIZABILITY_LIST"] * 1e-3,
               cov_atom=np.repeat(np.arange(len(nptr)), nptr).astype(np.int32),
               cov_partner=(sec["POL_GAUSS_COVALENT_ATOMS_LIST"] - 1).astype(np.int32),
               cov_strength=sec["POL_GAUSS_COVALENT_DIPOLES_LIST"] * 0.1)
    for lvl in ("q", "qp", "qi", "qpi"):
        d = np.load(REF / f"tests/data/ref_w512_{lvl}_novdw.npz")
        if lvl == "q":
            out["pos"] = d["pos"]
            out["H"] = d["H"]
        else:
            assert np.array_equal(out["pos"], d["pos"]) and np.array_equal(out["H"], d["H"])
        out[f"{lvl}_energy"] = d["term_elec"]
        out[f"{lvl}_forces"] = d["forces"]
        out[f"{lvl}_mu"] = d["mu"]
        out[f"{lvl}_iterations"] = d["iterations"]
    # settings of the goldens: tests/openmm_tests.sh:18-21, tests/ref_pgmjax.py:22-40
    out.update(ke=138.935458, beta=3.5, cutoff=0.9, grid=np.array([36, 36, 36]), order=6, tol=1e-10)
    np.savez_compressed(OUT / "w512_pgmjax.npz", **out)
    print("w512_pgmjax.npz", {k: np.shape(v) for k, v in out.items()})


def gvdw_box():
    lines = open(REF / "tests/data/gvdw_box.txt").read().split("\n")
    n = int(lines[0])
    box = np.array([[float(v) for v in lines[1 + a].split()] for a in range(3)])
    atoms = np.array([[float(v) for v in lines[4 + i].split()] for i in range(n)])
    excl = np.array([[int(v) for v in ln.split()] for ln in lines[4 + n:] if ln.strip()], dtype=np.int32)
    # pmemd-pgm VDWAALS of this box at 10 A (kcal/mol) with the global parameters of the two repulsion forms:
    # A_rep [kcal/mol], C6 [kcal/mol A^6], B, 1 = Slater (core/tests/test_gvdw.cpp:66-70)
    models = np.array([[87500.0, 594.825035, 4.52, 1, 784.7282], [422.0, 594.825035, 0.9453, 0, 868.3699]])
    np.savez_compressed(OUT / "gvdw_box.npz", box=box, pos=atoms[:, :3], radius=atoms[:, 3],
                        lj=atoms[:, 4].astype(np.uint8), excl=excl, rvdw=1.0, models=models)
    print("gvdw_box.npz", n, "atoms", len(excl), "exclusions")


def dmp8550_real():
    import gzip
    import tempfile
    from scipy.io import netcdf_file
    from oracle import pgm_oracle as O
    from oracle import ref as R
    systems = load_systems()
    with tempfile.NamedTemporaryFile("w", suffix=".prmtop") as t:
        t.write(gzip.open(REF / "amber/test/dmp/prmtop.gz", "rt").read())
        t.flush()
        sec = read_prmtop_sections(t.name, {"POL_GAUSS_MONOPOLES_LIST", "POL_GAUSS_RADII_LIST",
                                            "POL_GAUSS_POLARIZABILITY_LIST", "POL_GAUSS_COVALENT_POINTERS_LIST",
                                            "POL_GAUSS_COVALENT_ATOMS_LIST", "POL_GAUSS_COVALENT_DIPOLES_LIST"})
    nat, nmol = 19, 450
    q, rad, alp = (sec[k] for k in ("POL_GAUSS_MONOPOLES_LIST", "POL_GAUSS_RADII_LIST",
                                    "POL_GAUSS_POLARIZABILITY_LIST"))
    ptr = sec["POL_GAUSS_COVALENT_POINTERS_LIST"].astype(np.int64)
    catom = np.repeat(np.arange(len(ptr)), ptr)
    cpart = sec["POL_GAUSS_COVALENT_ATOMS_LIST"].astype(np.int64) - 1
    cstr = sec["POL_GAUSS_COVALENT_DIPOLES_LIST"]
    ncov = int(ptr[:nat].sum())
    mol = dict(q=q[:nat], radius=rad[:nat] * 0.1, alpha=alp[:nat] * 1e-3, cov_atom=catom[:ncov].astype(np.int32),
               cov_partner=cpart[:ncov].astype(np.int32), cov_strength=cstr[:ncov] * 0.1)
    for m in range(nmol):   # the tiling is exact
        a = slice(nat * m, nat * m + nat)
        c = slice(ncov * m, ncov * m + ncov)
        assert np.array_equal(q[a], q[:nat]) and np.array_equal(rad[a], rad[:nat]) and np.array_equal(alp[a], alp[:nat])
        assert np.array_equal(catom[c] - nat * m, catom[:ncov]) and np.array_equal(cpart[c] - nat * m, cpart[:ncov])
        assert np.array_equal(cstr[c], cstr[:ncov])
    nc = netcdf_file(str(REF / "amber/test/dmp/restrt0"), "r", mmap=False)
    assert np.allclose(nc.variables["cell_angles"][:], 90.0)
    pos = (np.array(nc.variables["coordinates"][:], dtype=np.float64) * 0.1).astype(np.float32)
    box = np.diag(np.array(nc.variables["cell_lengths"][:], dtype=np.float64) * 0.1)
    S = dmp_system(mol, pos, box, systems)
    top = O.Topology(S.q, S.radius, S.alpha, S.cov_atom, S.cov_partner, S.cov_strength)
    st = O.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=S.order, tol=1e-10, max_iter=500, peek=0.0,
                    predictor=0, ke=systems.KE_DEFAULT)
    eng = R.RefEngine(top, st)
    e = eng.compute(S.pos, S.box)
    t = eng.terms()
    np.savez_compressed(
        OUT / "dmp8550_real.npz", nmol=nmol, pos=pos, box=box, cutoff=S.cutoff, beta=S.beta, grid=np.array(S.grid),
        order=S.order, ke=systems.KE_DEFAULT, tol=1e-10, energy=e,
        terms=np.array([t[k] for k in ("direct", "reciprocal", "self", "background", "polarization")]),
        forces=eng.forces.astype(np.float32), strain=eng.strain(), mu=eng.induced().astype(np.float32),
        iterations=eng.iterations(), **{"mol_" + k: v for k, v in mol.items()})
    print("dmp8550_real.npz", S.n, "atoms", e, eng.iterations(), "iterations")


def dmp_system(mol, pos, box, systems):
    """The DMP liquid as a System: the molecule's parameters and covalent dipoles tiled over the molecules
    (the same construction as tests/conftest.py's loader)."""
    nat, ncov, nmol = len(mol["q"]), len(mol["cov_atom"]), len(pos) // len(mol["q"])
    off = np.repeat(np.arange(nmol) * nat, ncov)
    return systems.System(name="dmp8550_real", pos=np.asarray(pos, dtype=np.float64), box=box,
                          q=np.tile(mol["q"], nmol), radius=np.tile(mol["radius"], nmol),
                          alpha=np.tile(mol["alpha"], nmol),
                          cov_atom=(np.tile(mol["cov_atom"], nmol) + off).astype(np.int32),
                          cov_partner=(np.tile(mol["cov_partner"], nmol) + off).astype(np.int32),
                          cov_strength=np.tile(mol["cov_strength"], nmol), cutoff=0.9, beta=3.5, grid=(48, 48, 48),
                          order=6)


def ref_outputs():
    from oracle import pgm_oracle as O
    from oracle import ref as R
    systems = load_systems()
    cases = {"tiny_triclinic": systems.tiny_triclinic(), "water216": systems.water216()}
    for name, S in cases.items():
        top = O.Topology(S.q, S.radius, S.alpha, S.cov_atom, S.cov_partner, S.cov_strength)
        st = O.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=S.order, tol=1e-10, max_iter=500, peek=0.0,
                        predictor=0, ke=systems.KE_DEFAULT)
        eng = R.RefEngine(top, st)
        e = eng.compute(S.pos, S.box)
        t = eng.terms()
        i, j, _ = O.pair_set(S.pos, S.box, S.cutoff)
        np.savez_compressed(
            OUT / f"ref_{name}.npz", pos=S.pos, box=S.box, q=S.q, radius=S.radius, alpha=S.alpha,
            cov_atom=S.cov_atom, cov_partner=S.cov_partner, cov_strength=S.cov_strength, cutoff=S.cutoff,
            beta=S.beta, grid=np.array(S.grid), order=S.order, ke=systems.KE_DEFAULT, tol=1e-10, energy=e,
            terms=np.array([t[k] for k in ("direct", "reciprocal", "self", "background", "polarization")]),
            forces=eng.forces, strain=eng.strain(), mu=eng.induced(), perm=eng.permanent(),
            iterations=eng.iterations(), npairs=len(i))
        print(f"ref_{name}.npz", S.n, "atoms", e, eng.iterations(), "iterations", len(i), "pairs")


TERM_NAMES = ("direct", "reciprocal", "self", "background", "polarization")


def _ref_eval(S, tol, want=("forces", "mu")):
    """One pgm_core evaluation (the reference itself, oracle/_ref) at tol, predictor none, peek 0."""
    from oracle import pgm_oracle as O
    from oracle import ref as R
    systems = load_systems()
    top = O.Topology(S.q, S.radius, S.alpha, S.cov_atom, S.cov_partner, S.cov_strength)
    st = O.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=S.order, tol=tol, max_iter=1000, peek=0.0,
                    predictor=0, ke=systems.KE_DEFAULT)
    eng = R.RefEngine(top, st)
    e = eng.compute(S.pos, S.box)
    t = eng.terms()
    out = dict(energy=e, terms=np.array([t[k] for k in TERM_NAMES]), strain=eng.strain(),
               iterations=eng.iterations())
    if "forces" in want:
        out["forces"] = eng.forces.copy()
    if "mu" in want:
        out["mu"] = eng.induced()
    return out


def water98304_ref():
    """The 98304-atom water box (32768 waters, 104^3) through pgm_core at tol 1e-10: terms, strain, iterations,
    forces and induced dipoles (float32), and a digest of the generator's positions."""
    systems = load_systems()
    S = systems.water98304()
    r = _ref_eval(S, 1e-10)
    np.savez_compressed(OUT / "ref_water98304.npz", pos_digest=np.array([S.pos.sum(), (S.pos ** 2).sum()]),
                        energy=r["energy"], terms=r["terms"], strain=r["strain"], iterations=r["iterations"],
                        forces=r["forces"].astype(np.float32), mu=r["mu"].astype(np.float32), tol=1e-10)
    print("ref_water98304.npz", S.n, "atoms", r["energy"], r["iterations"], "iterations")


def batch_sample_indices(systems_list, per_grid=3):
    """A stratified sample of the 1024-box batch: every box of the largest molecule count, and per distinct grid
    shape its smallest, its largest and its median box (at least one of each shape)."""
    counts = np.array([len(S.q) for S in systems_list])
    grids = np.array([S.grid[0] for S in systems_list])
    pick = set(np.flatnonzero(counts == counts.max()).tolist())
    for K in sorted(set(grids.tolist())):
        idx = np.flatnonzero(grids == K)
        order = idx[np.argsort(counts[idx], kind="stable")]
        for k in {0, len(order) // 2, len(order) - 1} if per_grid >= 3 else {0}:
            pick.add(int(order[k]))
    return np.array(sorted(pick))


def batch_sample_ref():
    """pgm_core at tol 1e-10 on a stratified sample of the 1024 water boxes (water_batch(), seed 1024):
    per-system terms, strain, iterations, forces (float32) and induced dipoles (float32), concatenated in the
    sample's order."""
    systems = load_systems()
    boxes = systems.water_batch()
    sample = batch_sample_indices(boxes)
    rows = [_ref_eval(boxes[k], 1e-10) for k in sample]
    np.savez_compressed(OUT / "ref_water_batch_sample.npz", sample=sample,
                        natoms=np.array([len(boxes[k].q) for k in sample]),
                        grid=np.array([boxes[k].grid[0] for k in sample]),
                        energy=np.array([r["energy"] for r in rows]), terms=np.stack([r["terms"] for r in rows]),
                        strain=np.stack([r["strain"] for r in rows]),
                        iterations=np.array([r["iterations"] for r in rows]),
                        forces=np.concatenate([r["forces"] for r in rows]).astype(np.float32),
                        mu=np.concatenate([r["mu"] for r in rows]).astype(np.float32), tol=1e-10)
    print("ref_water_batch_sample.npz", len(sample), "boxes, grids", sorted(set(boxes[k].grid[0] for k in sample)))


def _with_params(S, name, values):
    from dataclasses import replace
    return replace(S, **{name: values})


def _as_fields(S):
    return {k: getattr(S, k) for k in S.__dataclass_fields__}


def _fd_job(args):
    """(+h, -h) energies and forces of pgm_core with one per-type parameter moved (a worker of the FD pool; the
    system travels as its fields)."""
    fields, name, t, h, tol = args
    S = load_systems().System(**fields)
    out = []
    for sgn in (1.0, -1.0):
        vals = getattr(S, name).copy()
        idx = (S.cov_types if name == "cov_strength" else S.types) == t
        vals[idx] += sgn * h
        r = _ref_eval(_with_params(S, name, vals), tol, want=("forces",))
        out.append((r["energy"], r["forces"]))
    return out


PARAM_NAMES = ("q", "cov_strength", "alpha", "radius")


def type_values(S, name):
    ty = S.cov_types if name == "cov_strength" else S.types
    v = np.zeros(int(ty.max()) + 1)
    v[ty] = getattr(S, name)
    return v


def gradient_fixture(S, F_target, tol, pool):
    """Central differences of pgm_core's energy and of the force-matching loss L = sum |F - F_target|^2 per
    parameter type, plus the energy and L at the unperturbed parameters.  The step is 1e-5 relative to the
    type's value, or to the RMS of its kind's values where that is larger: a value near zero (a bond dipole of
    1e-6 e nm) would otherwise give a step whose energy change drowns in the rounding of the energy."""
    jobs, keys = [], []
    for name in PARAM_NAMES:
        vals = type_values(S, name)
        scale = float(np.sqrt(np.mean(vals ** 2)))
        for t in range(len(vals)):
            h = 1e-5 * max(abs(vals[t]), scale)
            jobs.append((_as_fields(S), name, t, h, tol))
            keys.append((name, t, h))
    res = pool.map(_fd_job, jobs)
    out = {}
    for (name, t, h), ((ep, fp), (em, fm)) in zip(keys, res):
        lp = float(np.sum((fp - F_target) ** 2))
        lm = float(np.sum((fm - F_target) ** 2))
        out.setdefault("dE_" + name, []).append((ep - em) / (2 * h))
        out.setdefault("dL_" + name, []).append((lp - lm) / (2 * h))
    r0 = _ref_eval(S, tol, want=("forces",))
    out = {k: np.array(v) for k, v in out.items()}
    out["energy"] = r0["energy"]
    out["loss"] = float(np.sum((r0["forces"] - F_target) ** 2))
    return out


def gradients_ref():
    """Gradient goldens of the differentiation workload (FP64 pgm_core, central differences with h = 1e-5
    relative, at tol $GOLDEN_GRAD_TOL; the committed files use 1e-12, where the differences carry no CG noise,
    while the tests run the engine at the workload's 1e-8): (a) 16 of the 256 boxes of 64 waters, (b) the
    8550-atom dimethylphenol liquid.  The
    force-matching target F_target is pgm_core's forces with every per-type parameter scaled by
    (1 + N(0, 0.05)) (systems.perturbed, seed 1 + box index), stored with the fixture."""
    import multiprocessing as mp
    systems = load_systems()
    tol = float(os.environ.get("GOLDEN_GRAD_TOL", "1e-8"))
    ctx = mp.get_context("spawn")
    with ctx.Pool(int(os.environ.get("GOLDEN_PROCS", "8"))) as pool:
        boxes = systems.water64_boxes()
        sel = np.arange(16)
        fx = {}
        for k in sel:
            S = boxes[k]
            St = systems.perturbed(S, rel=0.05, seed=1 + int(k))
            Ft = _ref_eval(St, tol, want=("forces",))["forces"]
            g = gradient_fixture(S, Ft, tol, pool)
            fx[f"b{k}_Ft"] = Ft
            for key, v in g.items():
                fx[f"b{k}_{key}"] = v
            print("water64 box", k, "E", g["energy"], "L", g["loss"])
        np.savez_compressed(OUT / "grad_water64x16.npz", boxes=sel, tol=tol, **fx)
        S = systems.dimethylphenol8550(tol=tol)
        St = systems.perturbed(S, rel=0.05, seed=8550)
        Ft = _ref_eval(St, tol, want=("forces",))["forces"]
        g = gradient_fixture(S, Ft, tol, pool)
        np.savez_compressed(OUT / "grad_dimethylphenol8550.npz", tol=tol, Ft=Ft,
                            **{k: v for k, v in g.items()})
        print("dimethylphenol8550 E", g["energy"], "L", g["loss"])


if __name__ == "__main__":
    which = sys.argv[1:] or ["w512", "ref", "dmp", "gvdw"]
    which = [w for w in which if not w.startswith("--") and w != (sys.argv[sys.argv.index("--ref") + 1]
                                                                  if "--ref" in sys.argv else None)]
    if "water98304" in which:
        water98304_ref()
    if "batch" in which:
        batch_sample_ref()
    if "grad" in which:
        gradients_ref()
    if "w512" in which:
        w512()
    if "ref" in which:
        ref_outputs()
    if "dmp" in which:
        dmp8550_real()
    if "gvdw" in which:
        gvdw_box()
