"""Seeded synthetic pGM systems: the benchmark and parity workloads.

The reference measures on real liquids (pGM3P water boxes, the 8550-atom DMP liquid of
``amber/test/dmp``); these seeded systems stand in for them with the same sizes, densities and
parameter magnitudes.  Every builder takes a seed; inputs are in Angstrom / e / e A / A^3 as the
workload descriptions are written and are converted to the engine's units (nm, e, e nm, nm^3) here:
A -> 0.1 nm, A^3 -> 1e-3 nm^3, e A -> 0.1 e nm, 1/A -> 10/nm.

Workloads
  water216      216 rigid 3-site waters, 18.64 A cubic box, beta 0.35/A, rc 9 A, 20^3, order 6, tol 1e-6
  dimethylphenol8550
                450 rigid 19-atom C8H10O molecules (8550 atoms), 44.5 A box, 48^3, order 6, tol 1e-5
  water98304    32768 waters, 99.4 A box, 104^3, order 6
  water_batch   independent water boxes of 8..512 molecules at 0.0334 molecules/A^3, grids <= 1 A (2-3-5 sizes)
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

KE_DEFAULT = 138.935456   # Coulomb constant [kJ mol^-1 nm e^-2], used for every engine and the oracle


@dataclass
class System:
    """One periodic pGM system in engine units (nm, e, e nm, nm^3)."""
    name: str
    pos: np.ndarray          # (n, 3)
    box: np.ndarray          # (3, 3) rows a, b, c (reduced triclinic)
    q: np.ndarray
    radius: np.ndarray
    alpha: np.ndarray
    cov_atom: np.ndarray
    cov_partner: np.ndarray
    cov_strength: np.ndarray
    cutoff: float
    beta: float
    grid: tuple
    order: int = 6
    tol: float = 1e-5
    types: np.ndarray = None         # per-atom parameter type (for per-type gradients)
    cov_types: np.ndarray = None     # per-dipole parameter type
    meta: dict = field(default_factory=dict)

    @property
    def n(self):
        return len(self.q)


def random_rotations(rng, n):
    """Uniform random rotation matrices (Shoemake's uniform quaternions)."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    q0 = np.sqrt(1 - u1) * np.sin(2 * np.pi * u2)
    q1 = np.sqrt(1 - u1) * np.cos(2 * np.pi * u2)
    q2 = np.sqrt(u1) * np.sin(2 * np.pi * u3)
    q3 = np.sqrt(u1) * np.cos(2 * np.pi * u3)
    w, x, y, z = q3, q0, q1, q2
    R = np.empty((n, 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z)
    R[:, 0, 1] = 2 * (x * y - z * w)
    R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w)
    R[:, 1, 1] = 1 - 2 * (x * x + z * z)
    R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w)
    R[:, 2, 1] = 2 * (y * z + x * w)
    R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


def _lattice_sites(m, L, count, rng, jitter):
    g = (np.arange(m) + 0.5) * (L / m)
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    sites = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)[:count]
    return sites + rng.uniform(-jitter, jitter, size=sites.shape)


def _place(template, sites, rng):
    R = random_rotations(rng, len(sites))
    return (np.einsum("mij,aj->mai", R, template) + sites[:, None, :]).reshape(-1, 3)


def water_template():
    """Rigid 3-site water (r_OH 0.9572 A, HOH 104.52 deg), O at the origin [A]."""
    r, th = 0.9572, math.radians(104.52)
    return np.array([[0.0, 0.0, 0.0],
                     [r * math.sin(th / 2), 0.0, r * math.cos(th / 2)],
                     [-r * math.sin(th / 2), 0.0, r * math.cos(th / 2)]])


def waters(nmol, L, *, seed, grid, cutoff=9.0, beta=0.35, tol=1e-6, lattice=None, name="water"):
    """``nmol`` waters, O on a jittered cubic lattice (U(+-0.2 A)), uniform random orientations, cubic box
    of L [A].  q O -0.80 / H +0.40 e; R 0.90 / 0.70 A; alpha 1.00 / 0.40 A^3; a covalent dipole of
    0.10 e A along each O->H (atom O, partner H)."""
    rng = np.random.default_rng(seed)
    m = lattice or int(math.ceil(round(nmol ** (1 / 3), 9)))
    sites = _lattice_sites(m, L, nmol, rng, 0.2)
    pos = _place(water_template(), sites, rng)
    n = 3 * nmol
    q = np.tile([-0.80, 0.40, 0.40], nmol)
    R = np.tile([0.90, 0.70, 0.70], nmol)
    al = np.tile([1.00, 0.40, 0.40], nmol)
    types = np.tile([0, 1, 1], nmol)
    base = 3 * np.arange(nmol)
    ca = np.repeat(base, 2)
    cp = np.stack([base + 1, base + 2], axis=1).ravel()
    cs = np.full(2 * nmol, 0.10)
    return System(name=name, pos=pos * 0.1, box=np.eye(3) * L * 0.1, q=q, radius=R * 0.1, alpha=al * 1e-3,
                  cov_atom=ca.astype(np.int64), cov_partner=cp.astype(np.int64), cov_strength=cs * 0.1,
                  cutoff=cutoff * 0.1, beta=beta * 10.0, grid=tuple(grid), order=6, tol=tol, types=types,
                  cov_types=np.zeros(2 * nmol, np.int64), meta=dict(seed=seed, nmol=nmol, L_A=L))


def water216(seed=216):
    """216 waters on a 6^3 lattice, 18.64 A box, 20^3 grid, tol 1e-6 (zero initial guess)."""
    s = waters(216, 18.64, seed=seed, grid=(20, 20, 20), tol=1e-6, lattice=6, name="water216")
    return s


def water98304(seed=98304, tol=1e-5):
    """32768 waters on a 32^3 lattice, 99.4 A box, 104^3 grid."""
    return waters(32768, 99.4, seed=seed, grid=(104, 104, 104), tol=tol, lattice=32, name="water98304")


def dimethylphenol_template():
    """19-atom C8H10O template [A]: planar hexagonal ring (C-C 1.39), hydroxyl on C1 (C-O 1.36, O-H 0.96),
    ortho methyls on C2 and C6 (C-C 1.50, C-H 1.09), ring H on C3, C4, C5 (C-H 1.08).
    Returns (coordinates, element symbols, bonds (a, b) with a the atom nearer the ring)."""
    xyz, el, bonds = [], [], []
    ring = []
    for k in range(6):
        ang = math.radians(60 * k)
        ring.append([1.39 * math.cos(ang), 1.39 * math.sin(ang), 0.0])
    for k in range(6):
        xyz.append(ring[k])
        el.append("C")
    for k in range(6):
        bonds.append((k, (k + 1) % 6))

    def out(k, dist):
        ang = math.radians(60 * k)
        return [(1.39 + dist) * math.cos(ang), (1.39 + dist) * math.sin(ang), 0.0], [math.cos(ang), math.sin(ang), 0.0]

    # hydroxyl on ring atom 0
    o, u = out(0, 1.36)
    xyz.append(o)
    el.append("O")
    bonds.append((0, 6))
    # O-H at 109.5 deg in the ring plane
    perp = [-u[1], u[0], 0.0]
    th = math.radians(180 - 109.5)
    xyz.append([o[0] + 0.96 * (math.cos(th) * u[0] + math.sin(th) * perp[0]),
                o[1] + 0.96 * (math.cos(th) * u[1] + math.sin(th) * perp[1]), 0.0])
    el.append("H")
    bonds.append((6, 7))
    # methyls on ring atoms 1 and 5
    for k in (1, 5):
        c, u = out(k, 1.50)
        ci = len(xyz)
        xyz.append(c)
        el.append("C")
        bonds.append((k, ci))
        perp = np.array([-u[1], u[0], 0.0])
        zax = np.array([0.0, 0.0, 1.0])
        uu = np.array(u)
        cth, sth = math.cos(math.radians(180 - 109.47)), math.sin(math.radians(180 - 109.47))
        for phi in (0.0, 120.0, 240.0):
            ph = math.radians(phi)
            dvec = cth * uu + sth * (math.cos(ph) * zax + math.sin(ph) * perp)
            xyz.append(list(np.array(c) + 1.09 * dvec))
            el.append("H")
            bonds.append((ci, len(xyz) - 1))
    # ring H on 2, 3, 4
    for k in (2, 3, 4):
        h, _ = out(k, 1.08)
        xyz.append(h)
        el.append("H")
        bonds.append((k, len(xyz) - 1))
    xyz = np.array(xyz)
    xyz -= xyz.mean(axis=0)
    return xyz, el, bonds


def dimethylphenol8550(seed=8550, tol=1e-5):
    """450 rigid C8H10O molecules (8550 atoms) on the first 450 sites of a jittered 8^3 lattice in a
    44.5 A cubic box, random orientations.  Per-template-atom charges N(0, 0.3 e) shifted to neutrality,
    radii U(0.7, 1.1) A, polarizabilities C 1.3 / H 0.4 / O 0.8 A^3, one bond dipole U(-0.1, 0.1) e A per
    bond (atom: the bond's first atom, partner: its second).  beta 0.35/A, rc 9 A, 48^3, order 6."""
    rng = np.random.default_rng(seed)
    tmpl, el, bonds = dimethylphenol_template()
    na = len(tmpl)
    q_t = rng.normal(0.0, 0.3, na)
    q_t -= q_t.mean()
    R_t = rng.uniform(0.7, 1.1, na)
    al_t = np.array([{"C": 1.3, "H": 0.4, "O": 0.8}[e] for e in el])
    c_t = rng.uniform(-0.1, 0.1, len(bonds))
    nmol, L = 450, 44.5
    sites = _lattice_sites(8, L, nmol, rng, 0.2)
    pos = _place(tmpl, sites, rng)
    base = na * np.arange(nmol)
    b = np.array(bonds)
    ca = (base[:, None] + b[None, :, 0]).ravel()
    cp = (base[:, None] + b[None, :, 1]).ravel()
    return System(name="dimethylphenol8550", pos=pos * 0.1, box=np.eye(3) * L * 0.1, q=np.tile(q_t, nmol),
                  radius=np.tile(R_t, nmol) * 0.1, alpha=np.tile(al_t, nmol) * 1e-3, cov_atom=ca.astype(np.int64),
                  cov_partner=cp.astype(np.int64), cov_strength=np.tile(c_t, nmol) * 0.1, cutoff=0.9, beta=3.5,
                  grid=(48, 48, 48), order=6, tol=tol, types=np.tile(np.arange(na), nmol),
                  cov_types=np.tile(np.arange(len(bonds)), nmol), meta=dict(seed=seed, nmol=nmol, L_A=L))


def fft_size(x):
    """The smallest integer >= x with no prime factor above 5 (a PME grid size the transforms handle best)."""
    n = max(1, int(math.ceil(x)))
    while True:
        m = n
        for p in (2, 3, 5):
            while m % p == 0:
                m //= p
        if m == 1:
            return n
        n += 1


def water_batch(nsys=1024, seed=1024, nmin=8, nmax=512, density=0.0334, tol=1e-5):
    """``nsys`` independent water boxes, molecule counts U{nmin..nmax}, L = (n/density)^(1/3) A, grid the
    smallest size >= L / 1 A without a prime factor above 5 (at least the order; spacing <= 1 A), cutoff
    min(9 A, L/2), beta 0.35/A."""
    rng = np.random.default_rng(seed)
    counts = rng.integers(nmin, nmax + 1, size=nsys)
    out = []
    for k, nm in enumerate(counts):
        L = (nm / density) ** (1.0 / 3.0)
        K = max(6, fft_size(L / 1.0))
        rc = min(9.0, L / 2.0)
        out.append(waters(int(nm), L, seed=seed * 100003 + k, grid=(K, K, K), cutoff=rc, tol=tol,
                          name=f"water_batch[{k}]"))
    return out


def water64_boxes(nsys=256, seed=5000, density=0.0334, tol=1e-8):
    """The differentiation workload's boxes: ``nsys`` boxes of 64 waters built as water216 is (4^3 jittered
    lattice, random orientations, the same parameters) at 0.0334 molecules/A^3 (L = 12.4 A), grid the smallest
    2-3-5 size >= L / 1 A (15^3), cutoff L/2, beta 0.35/A; box k has seed ``seed + k``."""
    L = (64 / density) ** (1.0 / 3.0)
    K = fft_size(L / 1.0)
    return [waters(64, L, seed=seed + k, grid=(K, K, K), cutoff=min(9.0, L / 2.0), tol=tol, lattice=4,
                   name=f"water64[{k}]") for k in range(nsys)]


def perturbed(sys_: System, rel=0.05, seed=0):
    """The same system with every parameter scaled by (1 + N(0, rel)) per atom type / dipole type."""
    rng = np.random.default_rng(seed)
    nt = int(sys_.types.max()) + 1
    nc = int(sys_.cov_types.max()) + 1 if len(sys_.cov_types) else 0
    fq, fR, fa = (1 + rng.normal(0, rel, nt)), (1 + rng.normal(0, rel, nt)), (1 + rng.normal(0, rel, nt))
    fc = 1 + rng.normal(0, rel, nc)
    s = System(**{k: getattr(sys_, k) for k in sys_.__dataclass_fields__})
    s.q = sys_.q * fq[sys_.types]
    s.radius = sys_.radius * fR[sys_.types]
    s.alpha = sys_.alpha * fa[sys_.types]
    s.cov_strength = sys_.cov_strength * fc[sys_.cov_types] if nc else sys_.cov_strength
    return s


def tiny_triclinic(nmol=24, seed=7):
    """Water-like molecules at random positions in the reference unit test's triclinic box
    (2.0/1.9/1.8 nm, core/tests/test_core.cpp:12-46), beta 5/nm, rc 0.85 nm, 48^3, order 6."""
    rng = np.random.default_rng(seed)
    box = np.array([[2.0, 0, 0], [-0.5, 1.9, 0], [-0.4, -0.7, 1.8]])
    pos, q, R, al, ca, cp, cs = [], [], [], [], [], [], []
    for m in range(nmol):
        f = rng.random(3)
        o = f @ box
        b = len(pos)
        pos.append(o)
        for h in range(2):
            th, ph = 2 * np.pi * rng.random(), math.acos(2 * rng.random() - 1)
            pos.append(o + 0.096 * np.array([math.sin(ph) * math.cos(th), math.sin(ph) * math.sin(th), math.cos(ph)]))
        q += [-0.8, 0.4, 0.4]
        R += [0.0605, 0.0536, 0.0536]
        al += [1.1e-3, 0.33e-3, 0.33e-3]
        for h in (1, 2):
            ca += [b, b + h]
            cp += [b + h, b]
            cs += [-0.019, 0.0086]
    n = len(pos)
    return System(name="tiny_triclinic", pos=np.array(pos), box=box, q=np.array(q), radius=np.array(R),
                  alpha=np.array(al), cov_atom=np.array(ca), cov_partner=np.array(cp), cov_strength=np.array(cs),
                  cutoff=0.85, beta=5.0, grid=(48, 48, 48), order=6, tol=1e-10,
                  types=np.tile([0, 1, 1], nmol), cov_types=np.tile([0, 1, 0, 1], nmol), meta=dict(seed=seed))
