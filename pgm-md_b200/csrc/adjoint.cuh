// Kernels of the force-matching adjoint: the gradient of L = sum |F - F_target|^2 with respect to the per-atom
// charges, radii and polarizabilities and the per-dipole strengths, by one adjoint solve.  With w = 2 (F - F_t),
// g = dE/dtheta at fixed induced dipoles mu and E_tot the total field at fixed mu,
//     dL/dtheta = -D_w g + D_u g,    (alpha^-1 - T) u = -D_w E_tot,
// D_w the derivative along the displacement w of the positions (mu fixed, the covalent dipoles following their
// bonds), D_u the derivative along u of the induced dipoles.  Every derivative is analytic:
//   direct space  dG_n = -G_{n+1} (x . dx), the radial kernels recomputed per pair in double (G_0..G_3 and the
//                 radius derivatives H_n = dG_n/da = (2/sqrt(pi)) (2a^2)^n exp(-a^2 r^2), D H_n = -2a^2 (x.dx) H_n);
//   PME           the tangent sources (dipoles q_j w_j + D_w p_j, quadrupoles d_j (x) w_j, second derivatives of
//                 the splines) spread, transformed and gathered, plus the probe's own displacement through the
//                 final pass's field and potential Hessian at every atom.
// No reference counterpart (the reference lists parameter derivatives as not implemented).
#pragma once

#include "kernels.cuh"

namespace pgmb200 {

// Buffers of the adjoint (device, caller order unless stated).
struct FmBufs {
    double* w;        // 3n displacement w
    double* dp;       // 3n D_w p (covalent dipoles along w)
    double* pphi;     // n  direct-space D phi
    double* pE;       // 3n direct-space D E
    double* pR;       // n  direct-space D (dE/dR)
    double* tphi;     // n  PME tangent potential
    double* tE;       // 3n PME tangent field
    double* gq;       // n  assembled dq part
    double* gR;       // n  assembled dR part
    double* ga;       // n  assembled dalpha part
    double* gc;       // ncov assembled dc part
    double* Ed;       // 3n the pass's total-field derivative (D_w E_tot, or the field of u)
};

// D_w p_i = sum_m c_m D u_m over the covalent dipoles of atom i, D u = (dv - u (u . dv)) / L, dv = w_partner - w_atom
// (the bond vector's change), u and L of the minimum image (core/pgm_core.cpp:51-62 differentiated).
__global__ void k_fm_dp(Dev dv, const double* w, double* dp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= dv.nAtoms)
        return;
    const SysDev& S = dv.sys[dv.atomSys[i]];
    double acc[3] = {0, 0, 0};
    for (int k = dv.covByAtomOff[i]; k < dv.covByAtomOff[i + 1]; k++) {
        const int m = dv.covByAtom[k];
        const int j = dv.covPartner[m];
        double v[3] = {dv.posIn[3 * j] - dv.posIn[3 * i], dv.posIn[3 * j + 1] - dv.posIn[3 * i + 1],
                       dv.posIn[3 * j + 2] - dv.posIn[3 * i + 2]};
        int kk[3];
        minImageExact(v, S.H, kk);
        const double L = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        const double u[3] = {v[0] / L, v[1] / L, v[2] / L};
        const double dvv[3] = {w[3 * j] - w[3 * i], w[3 * j + 1] - w[3 * i + 1], w[3 * j + 2] - w[3 * i + 2]};
        const double ud = u[0] * dvv[0] + u[1] * dvv[1] + u[2] * dvv[2];
        for (int a = 0; a < 3; a++)
            acc[a] += dv.covStrength[m] * (dvv[a] - ud * u[a]) / L;
    }
    for (int a = 0; a < 3; a++)
        dp[3 * i + a] = acc[a];
}

// Direct-space derivatives at slot's atom i along the displacement dr (null: none) and the dipole change dd,
// over the evaluation's pairs within the cutoff (both directions listed, so each atom sums its own row):
//   D phi_i = sum_j -q_j G1 (x.dx) + dd_j.x G1 + d_j.dx G1 - (d_j.x) G2 (x.dx)
//   D E_i   = sum_j q_j dx G1 - q_j x G2 (x.dx) - dd_j G1 + d_j G2 (x.dx) + (dd_j.x + d_j.dx) x G2 + (d_j.x) dx G2
//                   - (d_j.x) x G3 (x.dx)
//   D gR_i  = sum_j D U_a (-2 R_i a^3),  D U_a the pair energy with G_n -> H_n differentiated,
// x = r_i - r_j, dx = dr_i - dr_j, d the final total dipoles.  Double precision, GS lanes per atom.
template <int GS>
__global__ void __launch_bounds__(256) k_pair_tangent(Dev dv, const double* dr, const double* dd, double* Dphi,
                                                      double* DE, double* DgR) {
    const int slot = (blockIdx.x * blockDim.x + threadIdx.x) / GS, lane = threadIdx.x % GS;
    if (slot >= dv.nAtoms)
        return;
    const int i = dv.slotAtom[slot];
    const SysDev& S = dv.sys[dv.atomSys[i]];
    const double4 pwi = dv.posS[slot];
    const double Ri = dv.radS[slot];
    const uint32_t* row = dv.list + (size_t) slot * dv.cap;
    const int cnt = dv.listCount[slot];
    const double qi = dv.q[i];
    const double di[3] = {dv.dtot[3 * i], dv.dtot[3 * i + 1], dv.dtot[3 * i + 2]};
    const double ddi[3] = {dd[3 * i], dd[3 * i + 1], dd[3 * i + 2]};
    const double dri[3] = {dr ? dr[3 * i] : 0.0, dr ? dr[3 * i + 1] : 0.0, dr ? dr[3 * i + 2] : 0.0};
    double aphi = 0.0, aE[3] = {0.0, 0.0, 0.0}, aR = 0.0;
    for (int t = lane; t < cnt; t += GS) {
        const uint32_t e = row[t];
        const int js = entrySlot(e);
        const int j = dv.slotAtom[js];
        double sh[3];
        entryShift(e, S.H, sh);
        const double4 pwj = dv.posS[js];
        const double x[3] = {pwi.x - pwj.x - sh[0], pwi.y - pwj.y - sh[1], pwi.z - pwj.z - sh[2]};
        const double r = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
        const double Rj = dv.radS[js];
        const double a = 1.0 / sqrt(2.0 * (Ri * Ri + Rj * Rj));
        double G[4];
        pairKernels<double, 4>(a, S.beta, r, G);
        const double qj = pwj.w;
        const double dj[3] = {dv.dtot[3 * j], dv.dtot[3 * j + 1], dv.dtot[3 * j + 2]};
        const double ddj[3] = {dd[3 * j], dd[3 * j + 1], dd[3 * j + 2]};
        double dx[3] = {dri[0], dri[1], dri[2]};
        if (dr)
            for (int k = 0; k < 3; k++)
                dx[k] -= dr[3 * j + k];
        const double xd = x[0] * dx[0] + x[1] * dx[1] + x[2] * dx[2];
        const double djx = dj[0] * x[0] + dj[1] * x[1] + dj[2] * x[2];
        const double dix = di[0] * x[0] + di[1] * x[1] + di[2] * x[2];
        const double ddjx = ddj[0] * x[0] + ddj[1] * x[1] + ddj[2] * x[2];
        const double ddix = ddi[0] * x[0] + ddi[1] * x[1] + ddi[2] * x[2];
        const double djdx = dj[0] * dx[0] + dj[1] * dx[1] + dj[2] * dx[2];
        const double didx = di[0] * dx[0] + di[1] * dx[1] + di[2] * dx[2];
        aphi += -qj * G[1] * xd + ddjx * G[1] + djdx * G[1] - djx * G[2] * xd;
        for (int k = 0; k < 3; k++)
            aE[k] += qj * dx[k] * G[1] - qj * x[k] * G[2] * xd - ddj[k] * G[1] + dj[k] * G[2] * xd +
                     (ddjx + djdx) * x[k] * G[2] + djx * dx[k] * G[2] - djx * x[k] * G[3] * xd;
        const double H0 = (2.0 / SQRT_PI) * exp(-(a * r) * (a * r)), H1 = H0 * 2.0 * a * a, H2 = H1 * 2.0 * a * a;
        const double c = -2.0 * a * a * xd;
        const double Ddjx = ddjx + djdx, Ddix = ddix + didx;
        const double Ddidj = ddi[0] * dj[0] + ddi[1] * dj[1] + ddi[2] * dj[2] + di[0] * ddj[0] + di[1] * ddj[1] +
                             di[2] * ddj[2];
        const double didj = di[0] * dj[0] + di[1] * dj[1] + di[2] * dj[2];
        const double DU = qi * qj * c * H0 + (qi * Ddjx - qj * Ddix) * H1 + (qi * djx - qj * dix) * c * H1 +
                          Ddidj * H1 + didj * c * H1 - (Ddix * djx + dix * Ddjx) * H2 - dix * djx * c * H2;
        aR += DU * (-2.0 * Ri * a * a * a);
    }
    const unsigned gm = groupMask<GS>();
#pragma unroll
    for (int o = GS / 2; o > 0; o >>= 1) {
        aphi += __shfl_xor_sync(gm, aphi, o, GS);
        aR += __shfl_xor_sync(gm, aR, o, GS);
#pragma unroll
        for (int k = 0; k < 3; k++)
            aE[k] += __shfl_xor_sync(gm, aE[k], o, GS);
    }
    if (lane == 0) {
        Dphi[i] = aphi;
        DgR[i] = aR;
        for (int k = 0; k < 3; k++)
            DE[3 * i + k] = aE[k];
    }
}

// Fractional-scaled vector e_a = K_a v . recip[:, a] (core/pgm_core.cpp:179-185).
__device__ __forceinline__ void fracScaled(const SysDev& S, const double* v, double* e) {
#pragma unroll
    for (int a = 0; a < 3; a++)
        e[a] = S.K[a] * (v[0] * S.recip[a] + v[1] * S.recip[3 + a] + v[2] * S.recip[6 + a]);
}

// Spread of the tangent sources onto the grid: dipoles dip_i (+ q_i qw_i when withQ) and, when qd is given, the
// quadrupoles qd_i (x) qw_i: per point sum_a e_a u_a (others t) + sum_ab Q_ab (d2 / dw_a dw_b of t1 t2 t3),
// Q = sym(frac(qd) (x) frac(qw)).  A warp per slot, the lanes over the p^3 points.
template <typename R>
__global__ void __launch_bounds__(256) k_spread_tangent(Dev dv, const double* dip, const double* qd, const double* qw,
                                                        int withQ) {
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int slot = blockIdx.x * 8 + wib;
    if (slot >= dv.nAtoms)
        return;
    const int i = dv.slotAtom[slot];
    const SysDev& S = dv.sys[dv.atomSys[i]];
    const int p = dv.order;
    double v[3] = {dip[3 * i], dip[3 * i + 1], dip[3 * i + 2]};
    if (withQ)
        for (int k = 0; k < 3; k++)
            v[k] += dv.q[i] * qw[3 * i + k];
    double e[3], Q[6] = {0, 0, 0, 0, 0, 0};   // 00 11 22 01 02 12
    fracScaled(S, v, e);
    if (qd) {
        const double a[3] = {qd[3 * i], qd[3 * i + 1], qd[3 * i + 2]};
        const double b[3] = {qw[3 * i], qw[3 * i + 1], qw[3 * i + 2]};
        double ea[3], eb[3];
        fracScaled(S, a, ea);
        fracScaled(S, b, eb);
        Q[0] = ea[0] * eb[0];
        Q[1] = ea[1] * eb[1];
        Q[2] = ea[2] * eb[2];
        Q[3] = ea[0] * eb[1] + ea[1] * eb[0];   // (twice the symmetric part: both orders of the mixed derivative)
        Q[4] = ea[0] * eb[2] + ea[2] * eb[0];
        Q[5] = ea[1] * eb[2] + ea[2] * eb[1];
    }
    const R* sp = (const R*) dv.spl + (size_t) slot * 9 * MAXP;
    const int4 b = dv.baseS[slot];
    R* grid = (R*) dv.grid + S.gridOff;
    const int K0 = S.K[0], K1 = S.K[1], K2 = S.K[2], pp = p * p;
    for (int t = lane; t < pp * p; t += 32) {
        const int j1 = t / pp, j2 = (t / p) % p, j3 = t % p;
        const double t1 = sp[0 * MAXP + j1], t2 = sp[1 * MAXP + j2], t3 = sp[2 * MAXP + j3];
        const double u1 = sp[3 * MAXP + j1], u2 = sp[4 * MAXP + j2], u3 = sp[5 * MAXP + j3];
        const double v1 = sp[6 * MAXP + j1], v2 = sp[7 * MAXP + j2], v3 = sp[8 * MAXP + j3];
        const double wpt = e[0] * u1 * t2 * t3 + e[1] * t1 * u2 * t3 + e[2] * t1 * t2 * u3 + Q[0] * v1 * t2 * t3 +
                           Q[1] * t1 * v2 * t3 + Q[2] * t1 * t2 * v3 + Q[3] * u1 * u2 * t3 + Q[4] * u1 * t2 * u3 +
                           Q[5] * t1 * u2 * u3;
        const int g1 = wrapIndex(b.x - j1, K0), g2 = wrapIndex(b.y - j2, K1), g3 = wrapIndex(b.z - j3, K2);
        atomicAdd(&grid[((size_t) g1 * K1 + g2) * K2 + g3], (R) wpt);
    }
}

// Potential and field of the convolved grid at every atom: pot_i = sum t1 t2 t3 phi, E_i = -sum_a K_a recip[:, a]
// f_a with f_a the derivative sums (core/pgm_core.cpp:241-264).  A warp per slot.
template <typename R>
__global__ void __launch_bounds__(256) k_gather_tangent(Dev dv, double* pot, double* E) {
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int slot = blockIdx.x * 8 + wib;
    if (slot >= dv.nAtoms)
        return;
    const int i = dv.slotAtom[slot];
    const SysDev& S = dv.sys[dv.atomSys[i]];
    const int p = dv.order, pp = p * p;
    const R* sp = (const R*) dv.spl + (size_t) slot * 9 * MAXP;
    const int4 b = dv.baseS[slot];
    const R* grid = (const R*) dv.grid + S.gridOff;
    const int K0 = S.K[0], K1 = S.K[1], K2 = S.K[2];
    double f[4] = {0, 0, 0, 0};
    for (int t = lane; t < pp * p; t += 32) {
        const int j1 = t / pp, j2 = (t / p) % p, j3 = t % p;
        const double t1 = sp[0 * MAXP + j1], t2 = sp[1 * MAXP + j2], t3 = sp[2 * MAXP + j3];
        const double u1 = sp[3 * MAXP + j1], u2 = sp[4 * MAXP + j2], u3 = sp[5 * MAXP + j3];
        const int g1 = wrapIndex(b.x - j1, K0), g2 = wrapIndex(b.y - j2, K1), g3 = wrapIndex(b.z - j3, K2);
        const double ph = (double) grid[((size_t) g1 * K1 + g2) * K2 + g3];
        f[0] += u1 * t2 * t3 * ph;
        f[1] += t1 * u2 * t3 * ph;
        f[2] += t1 * t2 * u3 * ph;
        f[3] += t1 * t2 * t3 * ph;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int k = 0; k < 4; k++)
            f[k] += __shfl_xor_sync(0xffffffffu, f[k], o);
    if (lane < 3) {
        const int k = lane;
        E[3 * i + k] = -(S.K[0] * S.recip[3 * k] * f[0] + S.K[1] * S.recip[3 * k + 1] * f[1] +
                         S.K[2] * S.recip[3 * k + 2] * f[2]);
    }
    if (lane == 0)
        pot[i] = f[3];
}

// The pass along w, per atom: D_w phi_i = pphi + tphi - E_rec . w_i; D_w E_tot = pE + tE - Hess phi_rec w_i +
// cs D_w p_i (the final pass's E_rec and Hessian sums), then dq and dR parts (times ke).
__global__ void k_fm_assemble_w(Dev dv, FmBufs B) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= dv.nAtoms)
        return;
    const SysDev& S = dv.sys[dv.atomSys[i]];
    const double cs = 4.0 * S.beta * S.beta * S.beta / (3.0 * SQRT_PI);
    const double* w = B.w + 3 * i;
    const double* h = dv.hrec + 6 * (size_t) i;
    const double f2[3][3] = {{h[0], h[3], h[4]}, {h[3], h[1], h[5]}, {h[4], h[5], h[2]}};
    double Kr[3][3];   // K_a recip[k][a]
    for (int k = 0; k < 3; k++)
        for (int a = 0; a < 3; a++)
            Kr[k][a] = S.K[a] * S.recip[3 * k + a];
    double Ew = 0.0;
    for (int k = 0; k < 3; k++)
        Ew += dv.Erec[3 * i + k] * w[k];
    for (int k = 0; k < 3; k++) {
        double Hw = 0.0;
        for (int l = 0; l < 3; l++) {
            double Hkl = 0.0;
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++)
                    Hkl += Kr[k][a] * f2[a][b] * Kr[l][b];
            Hw += Hkl * w[l];
        }
        B.Ed[3 * i + k] = B.pE[3 * i + k] + B.tE[3 * i + k] - Hw + cs * B.dp[3 * i + k];
    }
    B.gq[i] = dv.ke * (B.pphi[i] + B.tphi[i] - Ew);
    B.gR[i] = dv.ke * B.pR[i];
    B.ga[i] = 0.0;
}

// The pass along u (positions fixed, dipoles changed by u): dq, dR, dalpha parts and the total field of u.
__global__ void k_fm_assemble_u(Dev dv, FmBufs B, const double* u) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= dv.nAtoms)
        return;
    const SysDev& S = dv.sys[dv.atomSys[i]];
    const double cs = 4.0 * S.beta * S.beta * S.beta / (3.0 * SQRT_PI);
    double mu_u = 0.0;
    for (int k = 0; k < 3; k++) {
        B.Ed[3 * i + k] = B.pE[3 * i + k] + B.tE[3 * i + k] + cs * u[3 * i + k];
        mu_u += dv.mu[3 * i + k] * u[3 * i + k];
    }
    const double al = dv.alpha[i];
    B.gq[i] = dv.ke * (B.pphi[i] + B.tphi[i]);
    B.gR[i] = dv.ke * B.pR[i];
    B.ga[i] = al > 0 ? -dv.ke * mu_u / (al * al) : 0.0;
}

// Per covalent dipole m (atom i, partner j, unit u, length L): along w, dc = -ke (D_w E_tot(i) . u + E_tot(i) . D u);
// along u (alongW = 0), dc = -ke E_u(i) . u.
__global__ void k_fm_cov(Dev dv, FmBufs B, int alongW) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= dv.ncov)
        return;
    const int i = dv.covAtom[m], j = dv.covPartner[m];
    const SysDev& S = dv.sys[dv.atomSys[i]];
    double v[3] = {dv.posIn[3 * j] - dv.posIn[3 * i], dv.posIn[3 * j + 1] - dv.posIn[3 * i + 1],
                   dv.posIn[3 * j + 2] - dv.posIn[3 * i + 2]};
    int kk[3];
    minImageExact(v, S.H, kk);
    const double L = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    const double u[3] = {v[0] / L, v[1] / L, v[2] / L};
    double g = 0.0;
    for (int k = 0; k < 3; k++)
        g += B.Ed[3 * i + k] * u[k];
    if (alongW) {
        const double dvv[3] = {B.w[3 * j] - B.w[3 * i], B.w[3 * j + 1] - B.w[3 * i + 1], B.w[3 * j + 2] - B.w[3 * i + 2]};
        const double ud = u[0] * dvv[0] + u[1] * dvv[1] + u[2] * dvv[2];
        for (int k = 0; k < 3; k++)
            g += dv.Etot[3 * i + k] * (dvv[k] - ud * u[k]) / L;
    }
    B.gc[m] = -dv.ke * g;
}

// b = -D_w E_tot (the adjoint's right-hand side).
__global__ void k_fm_rhs(Dev dv, const double* Ed) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < 3 * dv.nAtoms)
        dv.b[t] = -Ed[t];
}

}  // namespace pgmb200
