"""Numpy restatement of the combination-rule GVDW van der Waals of the reference (core/gvdw_kernel.h), the
pair term its GPU engine adds in the final pair pass (core/cuda/pgm_cuda.cu:398-413, setGvdw
core/cuda/pgm_cuda.cu:2634-2667).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the engine's GVDW pass; never by the engine.

With the pGM pair exponent b_ij = 1/sqrt(2 (R_i^2 + R_j^2)) and y = b_ij r:
    U_ij = A_ij exp(-B_ij y^2) (Gaussian) or A_ij exp(-B_ij y) (Slater) - C6_ij b_ij^6 G(y),
    G(y) = F(y) / y^6, F = A(y)^2 + g(y)^2 / 2, A(y) = erf y - (2y/sqrt(pi))(1 + 2y^2/3) e^{-y^2},
    g(y) = (4 y^3 / (3 sqrt(pi))) e^{-y^2}                                   (core/gvdw_kernel.h:4-20)
with A_ij = a_i a_j, C6_ij = c_i c_j, B_ij = (b_i + b_j)/2 from per-atom a = sqrt(A), c = sqrt(C6), b.
G is taken from its Taylor series in y^2 below y = 0.6 and in closed form above (core/gvdw_kernel.h:31-58).
The series coefficients are derived here from the series of erf and exp (exact rationals), not tabulated.
"""

from __future__ import annotations

from fractions import Fraction
from math import factorial

import numpy as np

from .pgm_oracle import min_image, pair_set

SERIES_TERMS = 15
Y_SWITCH = 0.6


def series_coefficients(k_terms=SERIES_TERMS):
    """c_k with G(y) = G(0) sum_k c_k y^(2k), G(0) = 8 / (9 pi): from erf y = (2/sqrt(pi)) sum (-1)^n
    y^(2n+1) / (n! (2n+1)) and e^{-y^2} = sum (-1)^n y^(2n) / n!, A(y) = (2/sqrt(pi)) sum_n a_n y^(2n+1) (a_0 = a_1
    = 0), so that G (pi/4) = y^4 (sum_{n>=2} a_n y^(2n-4))^2 + (2/9) e^{-2 y^2}."""
    a = []
    for n in range(k_terms + 3):
        t = Fraction((-1) ** n, factorial(n) * (2 * n + 1)) - Fraction((-1) ** n, factorial(n))
        if n >= 1:
            t -= Fraction(2, 3) * Fraction((-1) ** (n - 1), factorial(n - 1))
        a.append(t)
    b = a[2:]
    coef = [Fraction(2, 9) * Fraction((-2) ** k, factorial(k)) for k in range(k_terms)]
    for m1 in range(k_terms):
        for m2 in range(k_terms - 2 - m1):
            coef[m1 + m2 + 2] += b[m1] * b[m2]
    return np.array([float(x / coef[0]) for x in coef])


_C = series_coefficients()
_C0 = 8.0 / (9.0 * np.pi)


def gvdw_g(y):
    """G(y) = F(y)/y^6 and H(y) = G'(y)/y (core/gvdw_kernel.h:30-58), elementwise."""
    from scipy.special import erf
    y = np.asarray(y, np.float64)
    G = np.empty_like(y)
    H = np.empty_like(y)
    small = y < Y_SWITCH
    ys = y[small]
    y2 = ys * ys
    g = np.zeros_like(ys)
    h = np.zeros_like(ys)
    for k in range(SERIES_TERMS - 1, -1, -1):
        g = g * y2 + _C[k]
    for k in range(SERIES_TERMS - 1, 0, -1):
        h = h * y2 + 2.0 * k * _C[k]
    G[small] = _C0 * g
    H[small] = _C0 * h
    yl = y[~small]
    isp = 1.0 / np.sqrt(np.pi)
    y2 = yl * yl
    e = np.exp(-y2)
    A = erf(yl) - 2.0 * isp * yl * (1.0 + 2.0 * y2 / 3.0) * e
    gg = (4.0 / 3.0) * isp * y2 * yl * e
    F = A * A + 0.5 * gg * gg
    Ap = (8.0 / 3.0) * isp * y2 * y2 * e
    gp = 4.0 * isp * y2 * (1.0 - 2.0 * y2 / 3.0) * e
    Fp = 2.0 * A * Ap + gg * gp
    y6 = y2 * y2 * y2
    G[~small] = F / y6
    H[~small] = (Fp / y6 - 6.0 * F / (y6 * yl)) / yl
    return G, H


def gvdw_pair(r, bij, A, C6, B, slater):
    """Pair energy and dEdR = -(1/r) dU/dr (force on i = dEdR (r_i - r_j)), core/gvdw_kernel.h:64-78."""
    r = np.asarray(r, np.float64)
    y = bij * r
    b2 = bij * bij
    b6 = b2 * b2 * b2
    if slater:
        erep = A * np.exp(-B * y)
        drep = np.where(r > 0, -B * bij * erep / np.where(r > 0, r, 1.0), 0.0)
    else:
        erep = A * np.exp(-B * y * y)
        drep = -2.0 * B * b2 * erep
    G, H = gvdw_g(y)
    return erep - C6 * b6 * G, -(drep - C6 * b6 * b2 * H)


def gvdw_energy(pos, box, radius, sqrt_a, sqrt_c6, b, rvdw, slater, skip_i=(), skip_j=()):
    """The combination-rule sum over the pairs within rvdw (the reference's minimum image) except the skipped
    ones: energy [kJ/mol], forces (n, 3) and the strain derivative S_ab = sum (dU/dx_a) x_b (9)."""
    pos = np.asarray(pos, np.float64)
    i, j, x = pair_set(pos, box, rvdw)
    skip = {(min(a, c), max(a, c)) for a, c in zip(np.asarray(skip_i).tolist(), np.asarray(skip_j).tolist())}
    keep = np.array([(a, c) not in skip for a, c in zip(i.tolist(), j.tolist())], bool) if len(i) else np.zeros(0, bool)
    A = sqrt_a[i] * sqrt_a[j]
    C6 = sqrt_c6[i] * sqrt_c6[j]
    keep &= (A != 0) | (C6 != 0)
    i, j, x, A, C6 = i[keep], j[keep], x[keep], A[keep], C6[keep]
    r = np.sqrt(np.sum(x * x, axis=1))
    bij = 1.0 / np.sqrt(2.0 * (radius[i] ** 2 + radius[j] ** 2))
    U, dEdR = gvdw_pair(r, bij, A, C6, 0.5 * (b[i] + b[j]), slater)
    f = dEdR[:, None] * x
    F = np.zeros_like(pos)
    np.add.at(F, i, f)
    np.add.at(F, j, -f)
    S = -(dEdR[:, None, None] * x[:, :, None] * x[:, None, :]).sum(axis=0).reshape(9)
    return float(U.sum()), F, S


__all__ = ["series_coefficients", "gvdw_g", "gvdw_pair", "gvdw_energy", "min_image"]
