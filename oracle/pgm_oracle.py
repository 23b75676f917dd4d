"""FP64 CPU oracle of the periodic pGM energy + force + virial evaluation.

TEST INFRASTRUCTURE ONLY.  This module is the checker for the CUDA engine: only the tests, the smoke
check in ``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of ``bench.py`` may import it.  The
engine never calls it and has no CPU fallback.

It restates, in vectorised numpy, the reference engine ``core/pgm_core.cpp`` of larryhuang98/pGM-MD
(and the numerics header ``core/pgm_math.h`` it uses).  Every function names the reference lines it
follows.  Units: nm, e, e nm, nm^3, kJ/mol (the Coulomb constant ``ke`` is a setting).

Parity of this restatement is pinned in ``tests/test_oracle.py``:
  * against the reference ``pgm_core`` itself, compiled from its own sources into ``oracle/_ref``
    (fixtures committed under ``tests/golden/`` by ``tests/golden/make_golden.py``);
  * against the pGM-JAX FP64 goldens of 512 pGM3P-25 waters that the reference ships
    (``tests/data/ref_w512_{q,qp,qi,qpi}_novdw.npz``, converted by the same script);
  * by the reference's own known-answer test (central finite differences of forces and of the
    strain derivative, ``core/tests/test_core.cpp``).

The pair set is reproduced bit for bit: the minimum image is the reference's c -> b -> a rounding
with round-half-away-from-zero (``core/pgm_math.h:153-160``) and the cutoff test is the same double
expression ``x0*x0 + x1*x1 + x2*x2 < rc*rc`` (``core/pgm_core.cpp:64-87``), evaluated without fused
multiply-adds.

The FFT is numpy's (pocketfft, the same library the reference vendors as
``core/pocketfft_hdronly.h``): ``rfftn`` is its unnormalised forward r2c and ``irfftn * K1 K2 K3`` its
unnormalised backward c2r (``core/pgm_core.cpp:208-213, 237``).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field as dc_field

import numpy as np
from scipy.special import erf, erfc

SQRT_PI = 1.7724538509055160273   # core/pgm_math.h:154
PI = 3.14159265358979323846       # core/pgm_math.h:155
MIN_POLARIZABILITY = 1e-9         # core/pgm_constants.h:9


# ----------------------------------------------------------------------------------------- settings

@dataclass
class Settings:
    """core/pgm_core.h:22-34 (pgmcore::Settings)."""
    periodic: bool = True
    cutoff: float = 0.9
    beta: float = 0.0
    grid: tuple = (0, 0, 0)
    order: int = 6
    polarizable: bool = True
    tol: float = 1e-5
    max_iter: int = 100
    peek: float = 0.65
    predictor: int = 2
    ke: float = 138.935456


@dataclass
class Topology:
    """core/pgm_core.h:36-40 (pgmcore::Topology): per-atom q [e], radius [nm], alpha [nm^3];
    covalent dipoles p_atom += strength * unit(r_partner - r_atom) [e nm]."""
    q: np.ndarray
    radius: np.ndarray
    alpha: np.ndarray
    cov_atom: np.ndarray = dc_field(default_factory=lambda: np.zeros(0, np.int64))
    cov_partner: np.ndarray = dc_field(default_factory=lambda: np.zeros(0, np.int64))
    cov_strength: np.ndarray = dc_field(default_factory=lambda: np.zeros(0))


# ----------------------------------------------------------------------------------------- numerics

def round_half_away(v):
    """std::round: nearest integer, halves away from zero (exact for every double)."""
    v = np.asarray(v, dtype=np.float64)
    t = np.trunc(v)
    frac = v - t                     # exact
    return t + np.where(np.abs(frac) >= 0.5, np.sign(v), 0.0)


def min_image(v, box):
    """core/pgm_math.h:153-160: minimum image in a reduced triclinic box, c first, then b, then a.
    v: (..., 3) array (copied); box: rows a, b, c."""
    v = np.array(v, dtype=np.float64, copy=True)
    for c in (2, 1, 0):
        k = round_half_away(v[..., c] / box[c][c])
        for j in range(3):
            v[..., j] = v[..., j] - k * box[c][j]
    return v


def erf_kernels(a, r, nmax):
    """core/pgm_math.h:31-61 (erfKernels): B_0..B_{nmax-1} of erf(a r)/r, 15-term series for
    (a r)^2 < 1, upward recursion elsewhere.  a, r: arrays of equal shape.  Returns (nmax, ...)."""
    a = np.asarray(a, np.float64)
    r = np.asarray(r, np.float64)
    x = a * r
    s = x * x
    c0 = 2.0 * a / SQRT_PI
    a2 = 2.0 * a * a
    out = np.empty((nmax,) + x.shape)
    ser = s < 1.0
    # series branch
    t = [np.ones_like(s)]
    for m in range(1, 15):
        t.append(t[-1] * (-s) / m)
    pw = np.ones_like(s)
    for k in range(nmax):
        acc = np.zeros_like(s)
        for m in range(14, -1, -1):
            acc = acc + t[m] / (2 * m + 2 * k + 1)
        out[k] = np.where(ser, c0 * pw * acc, 0.0)
        pw = pw * a2
    # recursion branch
    with np.errstate(divide="ignore", invalid="ignore"):
        c = c0 * np.exp(-s)
        ir2 = 1.0 / (r * r)
        B = erf(x) / r
        rec = [B]
        pw = np.ones_like(s)
        for k in range(1, nmax):
            B = ((2 * k - 1) * B - pw * c) * ir2
            rec.append(B)
            pw = pw * a2
    for k in range(nmax):
        out[k] = np.where(ser, out[k], rec[k])
    return out


def erfc_kernels(a, r, nmax):
    """core/pgm_math.h:63-75 (erfcKernels): B_n of erfc(a r)/r by the all-positive recursion."""
    a = np.asarray(a, np.float64)
    r = np.asarray(r, np.float64)
    x = a * r
    c = (2.0 / SQRT_PI) * a * np.exp(-x * x)
    ir2 = 1.0 / (r * r)
    a2 = 2.0 * a * a
    out = np.empty((nmax,) + x.shape)
    out[0] = erfc(x) / r
    pw = np.ones_like(x)
    for k in range(1, nmax):
        out[k] = ((2 * k - 1) * out[k - 1] + pw * c) * ir2
        pw = pw * a2
    return out


def ewald_pair_kernels(a, beta, r, nmax=4):
    """core/pgm_math.h:77-93 (ewaldPairKernels): G_n = B_n[erf(a r)/r] - B_n[erf(beta r)/r], the
    series form for a r < 1, the erfc form Bc(beta) - Bc(a) elsewhere.  Returns (nmax, npairs)."""
    a = np.asarray(a, np.float64)
    r = np.asarray(r, np.float64)
    b = np.full_like(a, beta)
    near = a * r < 1.0
    G = np.empty((nmax,) + a.shape)
    if near.any():
        G[:, near] = erf_kernels(a[near], r[near], nmax) - erf_kernels(b[near], r[near], nmax)
    far = ~near
    if far.any():
        G[:, far] = erfc_kernels(b[far], r[far], nmax) - erfc_kernels(a[far], r[far], nmax)
    return G


def bspline_moduli(K, p):
    """core/pgm_math.h:98-126 (bsplineModuli): |sum_k M_p(k+1) exp(2 pi i m k/K)|^2, zeros replaced
    by the mean of their neighbours."""
    M = [0.0] * (p + 1)
    M[0] = 1.0
    for k in range(2, p + 1):
        tmp = [0.0] * (p + 1)
        for j in range(k):
            cur = M[j] if j < k - 1 else 0.0
            prev = M[j - 1] if j > 0 else 0.0
            tmp[j] = (j * cur + (k - j) * prev) / (k - 1)
        for j in range(k):
            M[j] = tmp[j]
    data = np.zeros(K)
    for k in range(min(p - 1, K)):
        data[k] = M[k + 1]
    kk = np.arange(K)
    mod = np.empty(K)
    for m in range(K):
        arg = 2 * PI * m * kk / K
        sc = float(np.sum(data * np.cos(arg)))
        ss = float(np.sum(data * np.sin(arg)))
        mod[m] = sc * sc + ss * ss
    out = mod.copy()
    for m in range(K):
        if mod[m] < 1e-7:
            out[m] = 0.5 * (mod[(m - 1 + K) % K] + mod[(m + 1) % K])
    return out


def box_inverse(box):
    """core/pgm_core.cpp:94-111: recip = H^-1 (H: box vectors as rows) by cofactors, and |det H|."""
    H = np.asarray(box, np.float64)
    det = (H[0][0] * (H[1][1] * H[2][2] - H[1][2] * H[2][1]) - H[0][1] * (H[1][0] * H[2][2] - H[1][2] * H[2][0])
           + H[0][2] * (H[1][0] * H[2][1] - H[1][1] * H[2][0]))
    inv = np.empty((3, 3))
    inv[0][0] = (H[1][1] * H[2][2] - H[1][2] * H[2][1]) / det
    inv[0][1] = (H[0][2] * H[2][1] - H[0][1] * H[2][2]) / det
    inv[0][2] = (H[0][1] * H[1][2] - H[0][2] * H[1][1]) / det
    inv[1][0] = (H[1][2] * H[2][0] - H[1][0] * H[2][2]) / det
    inv[1][1] = (H[0][0] * H[2][2] - H[0][2] * H[2][0]) / det
    inv[1][2] = (H[0][2] * H[1][0] - H[0][0] * H[1][2]) / det
    inv[2][0] = (H[1][0] * H[2][1] - H[1][1] * H[2][0]) / det
    inv[2][1] = (H[0][1] * H[2][0] - H[0][0] * H[2][1]) / det
    inv[2][2] = (H[0][0] * H[1][1] - H[0][1] * H[1][0]) / det
    return inv, abs(det)


def pair_set(pos, box, cutoff, chunk=2048):
    """core/pgm_core.cpp:64-87 (build_pairs), periodic branch: all i < j with the minimum-image
    x = r_i - r_j, r^2 < rc^2.  Returns (i, j, x) in the reference's order (i major, j ascending)."""
    pos = np.asarray(pos, np.float64)
    n = len(pos)
    rc2 = cutoff * cutoff
    I, J, X = [], [], []
    for i0 in range(0, n, chunk):
        i1 = min(n, i0 + chunk)
        for i in range(i0, i1):
            if i + 1 >= n:
                continue
            x = pos[i][None, :] - pos[i + 1:]
            x = min_image(x, box)
            r2 = x[:, 0] * x[:, 0] + x[:, 1] * x[:, 1] + x[:, 2] * x[:, 2]
            sel = np.nonzero(r2 < rc2)[0]
            if len(sel):
                I.append(np.full(len(sel), i, np.int64))
                J.append(sel + i + 1)
                X.append(x[sel])
    if not I:
        return np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros((0, 3))
    return np.concatenate(I), np.concatenate(J), np.concatenate(X)


def pair_set_cells(pos, box, cutoff):
    """The set of pair_set (core/pgm_core.cpp:64-87, the same exact test on every candidate) for large systems:
    candidates come from a grid of cells at least rc wide in every fractional direction (27 neighbour cells), so
    only nearby pairs are tested.  Needs at least 3 cells per dimension.  Returns (i, j) sorted, i < j."""
    pos = np.asarray(pos, np.float64)
    box = np.asarray(box, np.float64)
    recip, _ = box_inverse(box)
    n = len(pos)
    rc2 = cutoff * cutoff
    frac = pos @ recip
    frac -= np.floor(frac)
    nc = []
    for a in range(3):
        rho = cutoff * np.linalg.norm(recip[:, a])
        nc.append(int(np.floor(1.0 / rho)))
    if min(nc) < 3:
        raise ValueError("pair_set_cells needs at least 3 cells per dimension")
    cidx = np.minimum((frac * nc).astype(np.int64), np.array(nc) - 1)
    lin = (cidx[:, 0] * nc[1] + cidx[:, 1]) * nc[2] + cidx[:, 2]
    order = np.argsort(lin, kind="stable")
    starts = np.searchsorted(lin[order], np.arange(nc[0] * nc[1] * nc[2] + 1))
    I, J = [], []
    for c0 in range(nc[0]):
        for c1 in range(nc[1]):
            for c2 in range(nc[2]):
                ca = (c0 * nc[1] + c1) * nc[2] + c2
                A = order[starts[ca]:starts[ca + 1]]
                if len(A) == 0:
                    continue
                nb = set()
                for d0 in (-1, 0, 1):
                    for d1 in (-1, 0, 1):
                        for d2 in (-1, 0, 1):
                            nb.add((((c0 + d0) % nc[0]) * nc[1] + (c1 + d1) % nc[1]) * nc[2] + (c2 + d2) % nc[2])
                B = np.concatenate([order[starts[cb]:starts[cb + 1]] for cb in sorted(nb)])
                ii = np.repeat(A, len(B))
                jj = np.tile(B, len(A))
                keep = ii < jj
                ii, jj = ii[keep], jj[keep]
                x = min_image(pos[ii] - pos[jj], box)
                r2 = x[:, 0] * x[:, 0] + x[:, 1] * x[:, 1] + x[:, 2] * x[:, 2]
                sel = r2 < rc2
                I.append(ii[sel])
                J.append(jj[sel])
    I = np.concatenate(I)
    J = np.concatenate(J)
    o = np.lexsort((J, I))
    return I[o], J[o]


# ----------------------------------------------------------------------------------------- engine

class Engine:
    """core/pgm_core.h:47-115 (pgmcore::Engine), periodic (PME) case only."""

    def __init__(self, top: Topology, s: Settings):
        if not s.periodic:
            raise ValueError("oracle: only the periodic (PME) path is restated")
        self.s = s
        self.set_topology(top)
        self.history = []
        self.last_pos = None
        self.have_pos = False
        self.history_key = -1
        self.last_key = -1
        self.iterations = 0
        self.residual = 0.0
        if min(s.grid) <= 0 or s.order < 3 or s.beta <= 0:
            raise ValueError("oracle: PME grid, order >= 3 and beta must be set")   # pgm_core.cpp:30-38

    def set_topology(self, top: Topology):
        """core/pgm_core.cpp:17-21, 41-47: alpha <= 1e-9 nm^3 -> 0 (not polarizable)."""
        self.top = Topology(np.asarray(top.q, np.float64).copy(), np.asarray(top.radius, np.float64).copy(),
                            np.asarray(top.alpha, np.float64).copy(), np.asarray(top.cov_atom, np.int64).copy(),
                            np.asarray(top.cov_partner, np.int64).copy(), np.asarray(top.cov_strength, np.float64).copy())
        self.top.alpha[self.top.alpha <= MIN_POLARIZABILITY] = 0.0
        self.n = len(self.top.q)
        if len(self.top.radius) != self.n or len(self.top.alpha) != self.n:
            raise ValueError("oracle: per-atom arrays of different lengths")
        self.have_pos = False

    def reset_history(self):
        self.history = []
        self.have_pos = False

    # ---------------------------------------------------------------- geometry
    def set_geometry(self, pos, box):
        """core/pgm_core.cpp:89-119."""
        self.pos = np.asarray(pos, np.float64).copy()
        self.box = np.asarray(box, np.float64).copy()
        self.recip, self.volume = box_inverse(self.box)
        self.perm = self._perm_dipoles()
        self._build_pairs()
        self._setup_pme()
        self._compute_influence()

    def _cov_vectors(self):
        t = self.top
        v = self.pos[t.cov_partner] - self.pos[t.cov_atom]
        v = min_image(v, self.box)
        L = np.sqrt(v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1] + v[:, 2] * v[:, 2])
        return v, L

    def _perm_dipoles(self):
        """core/pgm_core.cpp:51-62: p_i = sum c unit(r_j - r_i) (minimum image)."""
        p = np.zeros((self.n, 3))
        if len(self.top.cov_atom):
            v, L = self._cov_vectors()
            contrib = self.top.cov_strength[:, None] * v / L[:, None]
            for k in range(3):
                p[:, k] = np.bincount(self.top.cov_atom, weights=contrib[:, k], minlength=self.n)
        return p

    def _build_pairs(self):
        """core/pgm_core.cpp:64-87: pairs i < j within the cutoff with G_0..G_3."""
        i, j, x = pair_set(self.pos, self.box, self.s.cutoff)
        R = self.top.radius
        r = np.sqrt(x[:, 0] * x[:, 0] + x[:, 1] * x[:, 1] + x[:, 2] * x[:, 2])
        a = 1.0 / np.sqrt(2.0 * (R[i] * R[i] + R[j] * R[j]))
        self.pi, self.pj, self.px, self.pr, self.pa = i, j, x, r, a
        self.pG = ewald_pair_kernels(a, self.s.beta, r, 4) if len(i) else np.zeros((4, 0))

    def _setup_pme(self):
        """core/pgm_core.cpp:123-153: base = floor(w), M_p(fr + j) on points base - j, and the first and
        second derivatives."""
        p = self.s.order
        n = self.n
        self.base = np.zeros((3, n), np.int64)
        self.theta = np.zeros((3, n, p))
        self.dtheta = np.zeros((3, n, p))
        self.d2theta = np.zeros((3, n, p))
        for a in range(3):
            t = self.pos[:, 0] * self.recip[0][a] + self.pos[:, 1] * self.recip[1][a] + self.pos[:, 2] * self.recip[2][a]
            t = t - np.floor(t)
            w = self.s.grid[a] * t
            base = np.floor(w)
            fr = w - base
            M = np.zeros((p + 1, p + 2, n))
            M[1][0] = 1.0

            def get(k, j):
                return M[k][j] if 0 <= j < k else 0.0

            for k in range(2, p + 1):
                for j in range(k):
                    M[k][j] = ((fr + j) * get(k - 1, j) + (k - fr - j) * get(k - 1, j - 1)) / (k - 1)
            for j in range(p):
                self.theta[a, :, j] = M[p][j]
                self.dtheta[a, :, j] = get(p - 1, j) - get(p - 1, j - 1)
                self.d2theta[a, :, j] = get(p - 2, j) - 2 * get(p - 2, j - 1) + get(p - 2, j - 2)
            self.base[a] = base.astype(np.int64)

    def _mvec(self):
        K1, K2, K3 = self.s.grid
        m1 = np.arange(K1)
        m2 = np.arange(K2)
        m3 = np.arange(K3 // 2 + 1)
        mm1 = np.where(m1 <= K1 // 2, m1, m1 - K1).astype(np.float64)
        mm2 = np.where(m2 <= K2 // 2, m2, m2 - K2).astype(np.float64)
        mm3 = m3.astype(np.float64)
        A, B, C = np.meshgrid(mm1, mm2, mm3, indexing="ij")
        ms = np.empty((3,) + A.shape)
        for k in range(3):
            ms[k] = A * self.recip[k][0] + B * self.recip[k][1] + C * self.recip[k][2]
        return A, B, C, ms

    def _compute_influence(self):
        """core/pgm_core.cpp:155-177: G(m) = exp(-pi^2 m^2/beta^2)/(pi V m^2)/(b1 b2 b3), G(0) = 0."""
        K1, K2, K3 = self.s.grid
        b1 = bspline_moduli(K1, self.s.order)
        b2 = bspline_moduli(K2, self.s.order)
        b3 = bspline_moduli(K3, self.s.order)
        A, B, C, ms = self._mvec()
        m2s = ms[0] * ms[0] + ms[1] * ms[1] + ms[2] * ms[2]
        fac = math.pi * math.pi / (self.s.beta * self.s.beta)
        bb = b1[:, None, None] * b2[None, :, None] * b3[None, None, : K3 // 2 + 1]
        with np.errstate(divide="ignore", invalid="ignore"):
            g = np.exp(-fac * m2s) / (math.pi * self.volume * m2s) / bb
        g[0, 0, 0] = 0.0
        self.influence = g
        self.ms = ms
        self.m2s = m2s

    def frac_dipoles(self, d):
        """core/pgm_core.cpp:179-185: e_a = K_a d . recip[:, a]."""
        e = np.empty((self.n, 3))
        for a in range(3):
            e[:, a] = self.s.grid[a] * (d[:, 0] * self.recip[0][a] + d[:, 1] * self.recip[1][a] + d[:, 2] * self.recip[2][a])
        return e

    def _grid_index(self, a, j):
        K = self.s.grid[a]
        return ((self.base[a] - j) % K + K) % K

    def pme_potential(self, q, d, strain=None):
        """core/pgm_core.cpp:187-239: spread q theta + e . grad theta, r2c, energy and (optionally) the
        k-space strain, multiply by the influence function, c2r.  Returns (energy [e^2/nm], phi)."""
        K1, K2, K3 = self.s.grid
        p = self.s.order
        e = self.frac_dipoles(d)
        qi = np.zeros(self.n) if q is None else q
        Q = np.zeros(K1 * K2 * K3)
        for j1 in range(p):
            g1 = self._grid_index(0, j1)
            t1, u1 = self.theta[0, :, j1], self.dtheta[0, :, j1]
            for j2 in range(p):
                g2 = self._grid_index(1, j2)
                t2, u2 = self.theta[1, :, j2], self.dtheta[1, :, j2]
                for j3 in range(p):
                    g3 = self._grid_index(2, j3)
                    t3, u3 = self.theta[2, :, j3], self.dtheta[2, :, j3]
                    w = qi * t1 * t2 * t3 + e[:, 0] * u1 * t2 * t3 + e[:, 1] * t1 * u2 * t3 + e[:, 2] * t1 * t2 * u3
                    Q += np.bincount((g1 * K2 + g2) * K3 + g3, weights=w, minlength=K1 * K2 * K3)
        F = np.fft.rfftn(Q.reshape(K1, K2, K3))
        g = self.influence
        w = np.full(g.shape, 2.0)
        w[:, :, 0] = 1.0
        if K3 % 2 == 0:
            w[:, :, K3 // 2] = 1.0
        nrm = F.real * F.real + F.imag * F.imag
        ew = 0.5 * w * g * nrm
        energy = float(np.sum(ew))
        if strain is not None:
            with np.errstate(divide="ignore", invalid="ignore"):
                c2 = 2.0 * (math.pi * math.pi / (self.s.beta * self.s.beta) + 1.0 / self.m2s)
            c2[0, 0, 0] = 0.0
            ms = self.ms
            for a in range(3):
                for b in range(3):
                    strain[3 * a + b] += float(np.sum(ew * ((-1.0 if a == b else 0.0) + c2 * ms[a] * ms[b])))
        phi = np.fft.irfftn(F * g, s=(K1, K2, K3), axes=(0, 1, 2)) * (K1 * K2 * K3)
        return energy, phi.reshape(-1)

    def _interp(self, phi, want_second=False, want_pot=False):
        """core/pgm_core.cpp:241-264 (field sums f) and :452-481 (second derivatives f2)."""
        K1, K2, K3 = self.s.grid
        p = self.s.order
        n = self.n
        f = np.zeros((n, 3))
        f2 = np.zeros((n, 6)) if want_second else None   # 00 11 22 01 02 12
        pot = np.zeros(n) if want_pot else None
        for j1 in range(p):
            g1 = self._grid_index(0, j1)
            t1, u1, v1 = self.theta[0, :, j1], self.dtheta[0, :, j1], self.d2theta[0, :, j1]
            for j2 in range(p):
                g2 = self._grid_index(1, j2)
                t2, u2, v2 = self.theta[1, :, j2], self.dtheta[1, :, j2], self.d2theta[1, :, j2]
                for j3 in range(p):
                    g3 = self._grid_index(2, j3)
                    t3, u3, v3 = self.theta[2, :, j3], self.dtheta[2, :, j3], self.d2theta[2, :, j3]
                    ph = phi[(g1 * K2 + g2) * K3 + g3]
                    f[:, 0] += u1 * t2 * t3 * ph
                    f[:, 1] += t1 * u2 * t3 * ph
                    f[:, 2] += t1 * t2 * u3 * ph
                    if want_second:
                        f2[:, 0] += v1 * t2 * t3 * ph
                        f2[:, 1] += t1 * v2 * t3 * ph
                        f2[:, 2] += t1 * t2 * v3 * ph
                        f2[:, 3] += u1 * u2 * t3 * ph
                        f2[:, 4] += u1 * t2 * u3 * ph
                        f2[:, 5] += t1 * u2 * u3 * ph
                    if want_pot:
                        pot += t1 * t2 * t3 * ph
        return f, f2, pot

    def pme_field(self, phi):
        """core/pgm_core.cpp:241-264: -grad phi at every atom."""
        f, _, _ = self._interp(phi)
        E = np.zeros((self.n, 3))
        for k in range(3):
            E[:, k] -= (self.s.grid[0] * self.recip[k][0] * f[:, 0] + self.s.grid[1] * self.recip[k][1] * f[:, 1]
                        + self.s.grid[2] * self.recip[k][2] * f[:, 2])
        return E

    def _pair_field(self, q, d):
        """core/pgm_core.cpp:274-284: direct field of charges q and dipoles d over the pair list."""
        E = np.zeros((self.n, 3))
        if len(self.pi) == 0:
            return E
        i, j, x, G = self.pi, self.pj, self.px, self.pG
        qi, qj = q[i], q[j]
        di, dj = d[i], d[j]
        djx = dj[:, 0] * x[:, 0] + dj[:, 1] * x[:, 1] + dj[:, 2] * x[:, 2]
        dix = di[:, 0] * x[:, 0] + di[:, 1] * x[:, 1] + di[:, 2] * x[:, 2]
        for k in range(3):
            ei = qj * x[:, k] * G[1] - dj[:, k] * G[1] + djx * x[:, k] * G[2]
            ej = -qi * x[:, k] * G[1] - di[:, k] * G[1] + dix * x[:, k] * G[2]
            E[:, k] += np.bincount(i, weights=ei, minlength=self.n) + np.bincount(j, weights=ej, minlength=self.n)
        return E

    def field(self, q, d):
        """core/pgm_core.cpp:268-295: field [e/nm^2] of charges q and dipoles d (direct + PME + self)."""
        q = np.asarray(q, np.float64)
        d = np.asarray(d, np.float64)
        E = self._pair_field(q, d)
        useq = bool(np.any(q != 0))
        _, phi = self.pme_potential(q if useq else None, d)
        E += self.pme_field(phi)
        cs = 4.0 * self.s.beta ** 3 / (3.0 * SQRT_PI)
        E += cs * d
        return E

    # ---------------------------------------------------------------- solver
    def solve(self):
        """core/pgm_core.cpp:297-401: Jacobi PCG on (alpha^-1 - T) mu = E_perm with the mu3/mu4
        predictor, convergence max|alpha r| / mean|alpha E_perm| <= tol, then the peek step."""
        n = self.n
        zero = np.zeros(n)
        b = self.field(self.top.q, self.perm)
        al = self.top.alpha
        norm = float(np.sum(np.abs(al[:, None] * b))) / (3.0 * n) + 1e-300
        same = self.have_pos and (self.last_key == self.history_key if self.history_key >= 0
                                  else np.array_equal(self.last_pos, self.pos))
        h = len(self.history)
        s = self.s
        if same and h > 0:
            x = self.history[0].copy()
        elif s.predictor == 2 and h >= 4:
            x = 4 * self.history[0] - 6 * self.history[1] + 4 * self.history[2] - self.history[3]
        elif s.predictor >= 1 and h >= 3:
            x = 3 * self.history[0] - 3 * self.history[1] + self.history[2]
        elif s.predictor >= 1 and h >= 1:
            x = self.history[0].copy()
        else:
            x = al[:, None] * b
        pol = (al > 0)[:, None]
        safe = np.where(al > 0, al, 1.0)[:, None]

        def applyA(v):
            Tv = self.field(zero, v)
            return np.where(pol, v / safe - Tv, 0.0)

        def err_of(r):
            return float(np.max(np.abs(al[:, None] * r))) / norm

        Ax = applyA(x)
        r = np.where(pol, b - Ax, 0.0)
        z = al[:, None] * r
        pdir = z.copy()
        rz = float(np.sum(r * z))
        err = err_of(r)
        it = 0
        while err > s.tol and it < s.max_iter:
            Ap = applyA(pdir)
            alph = rz / max(float(np.sum(pdir * Ap)), 1e-300)
            x = x + alph * pdir
            rnew = r - alph * Ap
            znew = al[:, None] * rnew
            beta = float(np.sum(znew * (rnew - r))) / max(rz, 1e-300)
            pdir = znew + beta * pdir
            r, z = rnew, znew
            rz = float(np.sum(r * z))
            err = err_of(r)
            it += 1
        if s.peek != 0:
            x = x + s.peek * al[:, None] * r
        self.mu = x
        self.iterations = it
        self.residual = err
        if not same:
            self.history.insert(0, x.copy())
            del self.history[4:]
        self.last_pos = self.pos.copy()
        self.last_key = self.history_key
        self.have_pos = True

    # ---------------------------------------------------------------- energy and forces
    def compute(self, pos, box, want_forces=True):
        """core/pgm_core.cpp:405-537.  Returns the total energy [kJ/mol]; sets ``terms`` (direct,
        reciprocal, self, background, polarization), ``forces`` (n, 3) [kJ/mol/nm], ``strain`` (9,
        dE/d eps_ab, row-major) and the total field ``E_total`` [e/nm^2]."""
        s = self.s
        self.set_geometry(pos, box)
        if s.polarizable:
            self.solve()
        else:
            self.mu = np.zeros((self.n, 3))
            self.iterations = 0
        d = self.perm + self.mu
        q = self.top.q
        n = self.n
        E = np.zeros((n, 3))
        F = np.zeros((n, 3))
        S = np.zeros(9)
        direct = 0.0
        if len(self.pi):
            i, j, x, G = self.pi, self.pj, self.px, self.pG
            qi, qj, di, dj = q[i], q[j], d[i], d[j]
            dix = di[:, 0] * x[:, 0] + di[:, 1] * x[:, 1] + di[:, 2] * x[:, 2]
            djx = dj[:, 0] * x[:, 0] + dj[:, 1] * x[:, 1] + dj[:, 2] * x[:, 2]
            didj = di[:, 0] * dj[:, 0] + di[:, 1] * dj[:, 1] + di[:, 2] * dj[:, 2]
            direct = float(np.sum(qi * qj * G[0] + (qi * djx - qj * dix) * G[1] + didj * G[1] - dix * djx * G[2]))
            sc = -qi * qj * G[1] - (qi * djx - qj * dix) * G[2] - didj * G[2] + dix * djx * G[3]
            for k in range(3):
                dedx = sc * x[:, k] + (qi * dj[:, k] - qj * di[:, k]) * G[1] - (djx * di[:, k] + dix * dj[:, k]) * G[2]
                for b_ in range(3):
                    S[3 * k + b_] += float(np.sum(dedx * x[:, b_]))
                F[:, k] += -np.bincount(i, weights=dedx, minlength=n) + np.bincount(j, weights=dedx, minlength=n)
                E[:, k] += (np.bincount(i, weights=qj * x[:, k] * G[1] - dj[:, k] * G[1] + djx * x[:, k] * G[2], minlength=n)
                            + np.bincount(j, weights=-qi * x[:, k] * G[1] - di[:, k] * G[1] + dix * x[:, k] * G[2], minlength=n))
        recip_e, phi = self.pme_potential(q, d, S)
        Erec = self.pme_field(phi)
        E += Erec
        for a in range(3):
            for b_ in range(3):
                S[3 * a + b_] += float(np.sum(Erec[:, a] * d[:, b_]))
        # reciprocal forces: core/pgm_core.cpp:452-487
        e = self.frac_dipoles(d)
        f1, f2v, pot = self._interp(phi, want_second=True, want_pot=True)
        f2 = np.empty((n, 3, 3))
        f2[:, 0, 0], f2[:, 1, 1], f2[:, 2, 2] = f2v[:, 0], f2v[:, 1], f2v[:, 2]
        f2[:, 0, 1] = f2[:, 1, 0] = f2v[:, 3]
        f2[:, 0, 2] = f2[:, 2, 0] = f2v[:, 4]
        f2[:, 1, 2] = f2[:, 2, 1] = f2v[:, 5]
        for a in range(3):
            c = q * f1[:, a] + e[:, 0] * f2[:, a, 0] + e[:, 1] * f2[:, a, 1] + e[:, 2] * f2[:, a, 2]
            for k in range(3):
                F[:, k] -= s.grid[a] * self.recip[k][a] * c
        cs = 4.0 * s.beta ** 3 / (3.0 * SQRT_PI)
        q2 = float(np.sum(q * q))
        d2 = float(np.sum(d * d))
        Q = float(np.sum(q))
        E += cs * d
        self_e = -(s.beta / SQRT_PI) * q2 - 0.5 * cs * d2
        bg = -PI * Q * Q / (2.0 * self.volume * s.beta * s.beta)
        for a in range(3):
            S[4 * a] -= bg
        al = self.top.alpha
        polz = float(np.sum(np.where(al > 0, np.sum(self.mu * self.mu, axis=1) / (2.0 * np.where(al > 0, al, 1.0)), 0.0)))
        self.terms = dict(direct=s.ke * direct, reciprocal=s.ke * recip_e, self=s.ke * self_e,
                          background=s.ke * bg, polarization=s.ke * polz)
        self.E_total = E
        self.phi_rec_atoms = pot
        self.d = d
        self.E_rec = Erec
        self.f2_rec = f2v
        # covalent chain rule: core/pgm_core.cpp:511-529
        if len(self.top.cov_atom):
            v, L = self._cov_vectors()
            u = v / L[:, None]
            ia, ja, c = self.top.cov_atom, self.top.cov_partner, self.top.cov_strength
            g = -E[ia]
            gu = np.sum(g * u, axis=1)
            t = c[:, None] * (g - gu[:, None] * u) / L[:, None]
            for k in range(3):
                F[:, k] += -np.bincount(ja, weights=t[:, k], minlength=n) + np.bincount(ia, weights=t[:, k], minlength=n)
                for b_ in range(3):
                    S[3 * k + b_] += float(np.sum(t[:, k] * v[:, b_]))
        self.strain = s.ke * S
        self.forces = s.ke * F
        return sum(self.terms.values())

    # ---------------------------------------------------------------- parameter gradients (extension)
    def param_gradients(self):
        """Analytic dE/d(parameter) at the solved dipoles of the last ``compute`` (no reference
        counterpart: the reference lists parameter derivatives as not implemented).  E is stationary in
        the induced dipoles (peek = 0), so these are partial derivatives at fixed mu:
          dE/dq_i     = ke [sum_j (q_j G0 + d_j.x_ij G1) + phi_rec(r_i) - 2 beta q_i/sqrt(pi) - pi Q/(V beta^2)]
          dE/dc_m     = -ke E_total(atom m) . u_m
          dE/dalpha_i = -ke |mu_i|^2 / (2 alpha_i^2)
          dE/dR_i     = ke sum_j U_pair(dG_n/da) da_ij/dR_i,  dG_n/da = (2/sqrt(pi)) (2a^2)^n exp(-a^2 r^2),
                        da_ij/dR_i = -2 R_i a_ij^3.
        Returns a dict of per-atom / per-dipole arrays."""
        s = self.s
        n = self.n
        q = self.top.q
        d = self.d
        R = self.top.radius
        dq = np.zeros(n)
        dR = np.zeros(n)
        if len(self.pi):
            i, j, x, G, r, a = self.pi, self.pj, self.px, self.pG, self.pr, self.pa
            qi, qj, di, dj = q[i], q[j], d[i], d[j]
            dix = np.sum(di * x, axis=1)
            djx = np.sum(dj * x, axis=1)
            didj = np.sum(di * dj, axis=1)
            dq += np.bincount(i, weights=qj * G[0] + djx * G[1], minlength=n)
            dq += np.bincount(j, weights=qi * G[0] - dix * G[1], minlength=n)
            ex = (2.0 / SQRT_PI) * np.exp(-(a * r) ** 2)
            H0 = ex
            H1 = ex * 2 * a * a
            H2 = H1 * 2 * a * a
            u = qi * qj * H0 + (qi * djx - qj * dix) * H1 + didj * H1 - dix * djx * H2
            dR += np.bincount(i, weights=u * (-2.0 * R[i] * a ** 3), minlength=n)
            dR += np.bincount(j, weights=u * (-2.0 * R[j] * a ** 3), minlength=n)
        dq += self.phi_rec_atoms
        dq += -2.0 * s.beta / SQRT_PI * q
        dq += -PI * float(np.sum(q)) / (self.volume * s.beta * s.beta)
        al = self.top.alpha
        dal = np.where(al > 0, -np.sum(self.mu * self.mu, axis=1) / (2.0 * np.where(al > 0, al, 1.0) ** 2), 0.0)
        dc = np.zeros(len(self.top.cov_atom))
        if len(dc):
            v, L = self._cov_vectors()
            u = v / L[:, None]
            dc = -np.sum(self.E_total[self.top.cov_atom] * u, axis=1)
        return dict(q=s.ke * dq, radius=s.ke * dR, alpha=s.ke * dal, cov_strength=s.ke * dc)


    # ---------------------------------------------------------------- force-matching adjoint (extension)
    def _pme_tangent(self, dip, quad_d=None, quad_w=None):
        """PME potential and field at every atom of the sources: dipoles dip and, when given, the quadrupoles
        quad_d (x) quad_w (the derivative of a dipole d moved along w: sum_ab ed_a ew_b d2 theta / dw_a dw_b).
        Returns (potential, field)."""
        K1, K2, K3 = self.s.grid
        p = self.s.order
        e = self.frac_dipoles(dip)
        ed = self.frac_dipoles(quad_d) if quad_d is not None else None
        ew = self.frac_dipoles(quad_w) if quad_w is not None else None
        Q = np.zeros(K1 * K2 * K3)
        th, dth, d2 = self.theta, self.dtheta, self.d2theta
        for j1 in range(p):
            g1 = self._grid_index(0, j1)
            for j2 in range(p):
                g2 = self._grid_index(1, j2)
                for j3 in range(p):
                    g3 = self._grid_index(2, j3)
                    t = (th[0, :, j1], th[1, :, j2], th[2, :, j3])
                    u = (dth[0, :, j1], dth[1, :, j2], dth[2, :, j3])
                    v = (d2[0, :, j1], d2[1, :, j2], d2[2, :, j3])
                    w = e[:, 0] * u[0] * t[1] * t[2] + e[:, 1] * t[0] * u[1] * t[2] + e[:, 2] * t[0] * t[1] * u[2]
                    if ed is not None:
                        for a in range(3):
                            for b in range(3):
                                fac = []
                                for c in range(3):
                                    if c == a and c == b:
                                        fac.append(v[c])
                                    elif c == a or c == b:
                                        fac.append(u[c])
                                    else:
                                        fac.append(t[c])
                                w = w + ed[:, a] * ew[:, b] * fac[0] * fac[1] * fac[2]
                    Q += np.bincount((g1 * K2 + g2) * K3 + g3, weights=w, minlength=K1 * K2 * K3)
        F = np.fft.rfftn(Q.reshape(K1, K2, K3))
        phi = (np.fft.irfftn(F * self.influence, s=(K1, K2, K3), axes=(0, 1, 2)) * (K1 * K2 * K3)).reshape(-1)
        f, _, pot = self._interp(phi, want_pot=True)
        E = np.zeros((self.n, 3))
        for k in range(3):
            E[:, k] -= (self.s.grid[0] * self.recip[k][0] * f[:, 0] + self.s.grid[1] * self.recip[k][1] * f[:, 1]
                        + self.s.grid[2] * self.recip[k][2] * f[:, 2])
        return pot, E

    def _pair_tangent(self, dr, dd):
        """Directional derivatives of the direct-space potential, field and radius gradient at every atom along
        the displacement dr of the positions and the change dd of the dipoles (charges fixed):
          D phi_i = sum_j -q_j G1 (x.dx) + dd_j.x G1 + d_j.dx G1 - (d_j.x) G2 (x.dx)
          D E_i   = sum_j q_j dx G1 - q_j x G2 (x.dx) - dd_j G1 + d_j G2 (x.dx) + (dd_j.x + d_j.dx) x G2
                          + (d_j.x) dx G2 - (d_j.x) x G3 (x.dx)
          D gR_i  = sum_j D U_a (-2 R_i a^3), U_a the pair energy with dG_n/da = H_n, D H_n = -2 a^2 (x.dx) H_n,
        with x = r_i - r_j, dx = dr_i - dr_j (dG_n = -G_{n+1} x.dx from dG_n/dr = -r G_{n+1})."""
        n = self.n
        q, d, R = self.top.q, self.d, self.top.radius
        Dphi = np.zeros(n)
        DE = np.zeros((n, 3))
        DgR = np.zeros(n)
        if len(self.pi) == 0:
            return Dphi, DE, DgR
        i, j, x, G, r, a = self.pi, self.pj, self.px, self.pG, self.pr, self.pa
        dx = dr[i] - dr[j]
        xd = np.sum(x * dx, axis=1)
        qi, qj, di, dj, ddi, ddj = q[i], q[j], d[i], d[j], dd[i], dd[j]
        djx, dix = np.sum(dj * x, axis=1), np.sum(di * x, axis=1)
        ddjx, ddix = np.sum(ddj * x, axis=1), np.sum(ddi * x, axis=1)
        djdx, didx = np.sum(dj * dx, axis=1), np.sum(di * dx, axis=1)
        Dphi += np.bincount(i, weights=-qj * G[1] * xd + ddjx * G[1] + djdx * G[1] - djx * G[2] * xd, minlength=n)
        Dphi += np.bincount(j, weights=-qi * G[1] * xd - ddix * G[1] - didx * G[1] + dix * G[2] * xd, minlength=n)
        for k in range(3):
            ei = (qj * dx[:, k] * G[1] - qj * x[:, k] * G[2] * xd - ddj[:, k] * G[1] + dj[:, k] * G[2] * xd
                  + (ddjx + djdx) * x[:, k] * G[2] + djx * dx[:, k] * G[2] - djx * x[:, k] * G[3] * xd)
            ej = (-qi * dx[:, k] * G[1] + qi * x[:, k] * G[2] * xd - ddi[:, k] * G[1] + di[:, k] * G[2] * xd
                  + (ddix + didx) * x[:, k] * G[2] + dix * dx[:, k] * G[2] - dix * x[:, k] * G[3] * xd)
            DE[:, k] += np.bincount(i, weights=ei, minlength=n) + np.bincount(j, weights=ej, minlength=n)
        H0 = (2.0 / SQRT_PI) * np.exp(-(a * r) ** 2)
        H1 = H0 * 2 * a * a
        H2 = H1 * 2 * a * a
        c = -2.0 * a * a * xd
        Ddjx, Ddix = ddjx + djdx, ddix + didx
        Ddidj = np.sum(ddi * dj + di * ddj, axis=1)
        didj = np.sum(di * dj, axis=1)
        DU = (qi * qj * c * H0 + (qi * Ddjx - qj * Ddix) * H1 + (qi * djx - qj * dix) * c * H1 + Ddidj * H1
              + didj * c * H1 - (Ddix * djx + dix * Ddjx) * H2 - dix * djx * c * H2)
        DgR += np.bincount(i, weights=DU * (-2.0 * R[i] * a ** 3), minlength=n)
        DgR += np.bincount(j, weights=DU * (-2.0 * R[j] * a ** 3), minlength=n)
        return Dphi, DE, DgR

    def _solve_rhs(self, rhs):
        """(alpha^-1 - T) x = rhs by Jacobi PCG from x = alpha rhs to tol 1e-14 (rows with alpha = 0: 0)."""
        al = self.top.alpha
        zero = np.zeros(self.n)
        pol = (al > 0)[:, None]
        safe = np.where(al > 0, al, 1.0)[:, None]

        def applyA(v):
            return np.where(pol, v / safe - self.field(zero, v), 0.0)

        b = np.where(pol, rhs, 0.0)
        x = al[:, None] * b
        r = b - applyA(x)
        z = al[:, None] * r
        pdir = z.copy()
        rz = float(np.sum(r * z))
        nb = float(np.sum(np.abs(al[:, None] * b))) + 1e-300
        for _ in range(1000):
            if float(np.sum(np.abs(al[:, None] * r))) <= 1e-14 * nb:
                break
            Ap = applyA(pdir)
            alph = rz / max(float(np.sum(pdir * Ap)), 1e-300)
            x = x + alph * pdir
            rn = r - alph * Ap
            zn = al[:, None] * rn
            beta = float(np.sum(zn * (rn - r))) / max(rz, 1e-300)
            pdir = zn + beta * pdir
            r, z = rn, zn
            rz = float(np.sum(r * z))
        return x

    def force_matching_gradients(self, F_target):
        """dL/d(parameter) of L = sum |F - F_target|^2 at the solved dipoles of the last ``compute`` (peek 0), by
        one adjoint solve (no reference counterpart).  With w = 2 (F - F_target), g = dE/dtheta at fixed mu and
        E_tot the total field at fixed mu,
            dL/dtheta = -D_w g + D_u g,   (alpha^-1 - T) u = -D_w E_tot,
        D_w the derivative along the displacement w of the positions (mu fixed; the covalent dipoles follow
        their bonds), D_u the derivative along u of the induced dipoles; every derivative analytic:
          D_w phi_i   = [direct part] + phi_tangent(r_i) - E_rec(r_i) . w_i
          D_w E_tot_i = [direct part] + E_tangent(r_i) - Hess phi_rec(r_i) w_i + cs D_w p_i
        where the tangent sources are the dipoles q_j w_j + D_w p_j and the quadrupoles d_j (x) w_j.
        Returns (L, dict of per-atom / per-dipole gradients)."""
        s = self.s
        n = self.n
        q, d, al = self.top.q, self.d, self.top.alpha
        F = self.forces
        w = 2.0 * (F - np.asarray(F_target, np.float64))
        L = float(np.sum((F - F_target) ** 2))
        cs = 4.0 * s.beta ** 3 / (3.0 * SQRT_PI)
        ncov = len(self.top.cov_atom)
        Dp = np.zeros((n, 3))
        if ncov:
            v, Lc = self._cov_vectors()
            u_c = v / Lc[:, None]
            ia, ja, c = self.top.cov_atom, self.top.cov_partner, self.top.cov_strength
            dv = w[ja] - w[ia]
            Du_c = (dv - np.sum(u_c * dv, axis=1)[:, None] * u_c) / Lc[:, None]
            for k in range(3):
                Dp[:, k] = np.bincount(ia, weights=c * Du_c[:, k], minlength=n)
        # along w (positions moved, mu fixed)
        Dphi, DE, DgR = self._pair_tangent(w, Dp)
        pot_t, E_t = self._pme_tangent(q[:, None] * w + Dp, d, w)
        H = np.zeros((n, 3, 3))
        f2 = self.f2_rec
        f2m = np.empty((n, 3, 3))
        f2m[:, 0, 0], f2m[:, 1, 1], f2m[:, 2, 2] = f2[:, 0], f2[:, 1], f2[:, 2]
        f2m[:, 0, 1] = f2m[:, 1, 0] = f2[:, 3]
        f2m[:, 0, 2] = f2m[:, 2, 0] = f2[:, 4]
        f2m[:, 1, 2] = f2m[:, 2, 1] = f2[:, 5]
        Kr = np.array([[s.grid[a] * self.recip[k][a] for a in range(3)] for k in range(3)])   # [k][a]
        H = np.einsum("ka,nab,lb->nkl", Kr, f2m, Kr)
        Dw_phi = Dphi + pot_t - np.sum(self.E_rec * w, axis=1)
        Dw_E = DE + E_t - np.einsum("nkl,nl->nk", H, w) + cs * Dp
        gw = dict(q=s.ke * Dw_phi, radius=s.ke * DgR, alpha=np.zeros(n), cov_strength=np.zeros(ncov))
        if ncov:
            gw["cov_strength"] = -s.ke * (np.sum(Dw_E[ia] * u_c, axis=1) + np.sum(self.E_total[ia] * Du_c, axis=1))
        # the adjoint solve, then along u (dipoles changed, positions fixed)
        u = self._solve_rhs(-Dw_E)
        zero3 = np.zeros((n, 3))
        Dphi_u, DE_u, DgR_u = self._pair_tangent(zero3, u)
        pot_u, E_u = self._pme_tangent(u)
        gu = dict(q=s.ke * (Dphi_u + pot_u), radius=s.ke * DgR_u,
                  alpha=np.where(al > 0, -s.ke * np.sum(self.mu * u, axis=1) / np.where(al > 0, al, 1.0) ** 2, 0.0),
                  cov_strength=np.zeros(ncov))
        if ncov:
            gu["cov_strength"] = -s.ke * np.sum((DE_u + E_u + cs * u)[ia] * u_c, axis=1)
        return L, {k: -gw[k] + gu[k] for k in gw}


def evaluate(pos, box, top: Topology, s: Settings):
    """One fresh evaluation (no history): returns the Engine after compute()."""
    eng = Engine(top, s)
    eng.compute(pos, box)
    return eng
