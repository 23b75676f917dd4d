// Line PME spread and gather of the mixed-precision field passes (any number of systems; orders 4, 5, 6, 8).
//
// An atom's stencil is p^2 lines of p consecutive points along z (the grid's fastest dimension).  A thread owns
// one (atom, j1) x-plane of the stencil, its p lines, and moves each line as 2 or 3 aligned float4 words:
//   spread  float4 atomic adds (red.global.add.v4.f32) of the line's p weights, zero-padded to the aligned
//           16-byte words that hold them: about p^2 * 2.25 vector reductions per atom in place of p^3 scalar
//           ones, and no per-point index arithmetic;
//   gather  float4 loads of the same words, and the line's two sums (theta_z and dtheta_z weighted) in registers.
// The zero padding never leaves the row: a row is a multiple of 4 floats long, the words are aligned, and each
// word issued holds at least one of the line's points.  Lines that wrap around z (the atom's z base below p - 1)
// and systems whose rows are not a whole number of words take scalar atomics / loads per point.
// A warp holds 32 / p atoms (lanes beyond them idle), so all of an atom's threads share a warp.
#pragma once

#include "kernels.cuh"

namespace pgmb200 {

// The p coefficients of z at row positions a0 + k (k = 0 .. 11) of the aligned words, where the line starts at
// a0 + o: L[k] = src[p - 1 - (k - o)] for 0 <= k - o < p (the points run z = base - j3), else 0.  Two select
// stages (shift by o & 1, then by o & 2), the index pattern compile-time.
template <int P>
__device__ __forceinline__ void shiftLine(const float* src, int o, float* L) {
    float a[12];
#pragma unroll
    for (int k = 0; k < 12; k++)
        a[k] = k < P ? src[P - 1 - k] : 0.0f;
    const bool s1 = o & 1, s2 = o & 2;
#pragma unroll
    for (int k = 11; k >= 0; k--)
        a[k] = s1 ? (k >= 1 ? a[k - 1] : 0.0f) : a[k];
#pragma unroll
    for (int k = 11; k >= 0; k--)
        L[k] = s2 ? (k >= 2 ? a[k - 2] : 0.0f) : a[k];
}

// The y and z coefficients of a slot (theta and dtheta): float4 loads of the slot's spline record.
template <int P>
__device__ __forceinline__ void lineCoefficients(const float* sp, float* ty, float* uy, float* tz, float* uz) {
    constexpr int NV = (P + 3) / 4;
    const float4* s4 = (const float4*) sp;
#pragma unroll
    for (int v = 0; v < NV; v++) {
        const float4 a = s4[(1 * MAXP) / 4 + v], b = s4[(4 * MAXP) / 4 + v];
        const float4 c = s4[(2 * MAXP) / 4 + v], d = s4[(5 * MAXP) / 4 + v];
        const float av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w};
        const float cv[4] = {c.x, c.y, c.z, c.w}, dvv[4] = {d.x, d.y, d.z, d.w};
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (4 * v + k < P) {
                ty[4 * v + k] = av[k];
                uy[4 * v + k] = bv[k];
                tz[4 * v + k] = cv[k];
                uz[4 * v + k] = dvv[k];
            }
    }
}

static_assert(MAXP % 4 == 0, "line kernels load spline records as float4 words");

// Spread of charges and dipoles (the k_spread contract: mode 0 q and vec, 1 vec only, 2 the CG direction
// p = z + beta p first, vec = p; writes dS = (d, q)), Q[g] += q t1 t2 t3 + e0 u1 t2 t3 + e1 t1 u2 t3 + e2 t1 t2 u3
// (core/pgm_core.cpp:187-207).  The grid is cleared before.
template <int P>
__global__ void __launch_bounds__(256) k_spread_lines(Dev dv, int mode, double* vec) {
    constexpr int APW = 32 / P;
    const int lane = threadIdx.x & 31, a = lane / P, j1 = lane - a * P;
    const int warpG = (int) ((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    int slot = warpG * APW + a;
    bool on = a < APW;
    if (on && mode == 2 && dv.useActive)   // the CG direction of a batch: the active systems' slots only
        slot = activeSlot(dv, slot);
    on = on && slot >= 0 && slot < dv.nAtoms;
    int i = 0, s = 0;
    if (on) {
        i = dv.slotAtom[slot];
        s = dv.atomSys[i];
        on = !(mode == 2 && dv.scal[s * NSCAL + SC_DONE] != 0.0);
    }
    double d[3] = {0.0, 0.0, 0.0};
    if (on) {
        const double bt = mode == 2 ? dv.scal[s * NSCAL + SC_BETA] : 0.0;
#pragma unroll
        for (int k = 0; k < 3; k++)
            d[k] = mode == 2 ? dv.z[3 * i + k] + bt * vec[3 * i + k] : vec[3 * i + k];
    }
    __syncwarp();   // (every thread of the atom has read vec before its first thread writes p back)
    if (!on)
        return;
    const double qv = mode == 0 ? dv.q[i] : 0.0;
    if (j1 == 0) {
        if (mode == 2)
            for (int k = 0; k < 3; k++)
                vec[3 * i + k] = d[k];
        ((float4*) dv.dS)[slot] = make_float4((float) d[0], (float) d[1], (float) d[2], (float) qv);
    }
    const SysDev& S = dv.sys[s];
    float e[3];
#pragma unroll
    for (int k = 0; k < 3; k++)
        e[k] = (float) (S.K[k] * (d[0] * S.recip[k] + d[1] * S.recip[3 + k] + d[2] * S.recip[6 + k]));
    const float* sp = (const float*) dv.spl + (size_t) slot * 9 * MAXP;
    const float t1 = sp[j1], u1 = sp[3 * MAXP + j1];
    float ty[P], uy[P], tz[P], uz[P];
    lineCoefficients<P>(sp, ty, uy, tz, uz);
    const int K0 = S.K[0], K1 = S.K[1], K2 = S.K[2];
    const int4 b = dv.baseS[slot];
    const int bz = wrapIndex(b.z, K2), z0 = bz - (P - 1);
    float* plane = (float*) dv.grid + S.gridOff + (size_t) wrapIndex(b.x - j1, K0) * K1 * K2;
    // point (j2, j3) = t3 (t2 c1 + u2 c2) + u3 t2 c3
    const float c1 = (float) qv * t1 + e[0] * u1, c2 = e[1] * t1, c3 = e[2] * t1;
    if (z0 >= 0 && (K2 & 3) == 0 && (S.gridOff & 3) == 0) {
        const int o = z0 & 3;
        float T[12], U[12];
        shiftLine<P>(tz, o, T);
        shiftLine<P>(uz, o, U);
        constexpr int NQ = (P + 3 + 3) / 4;
#pragma unroll
        for (int j2 = 0; j2 < P; j2++) {
            const float A = ty[j2] * c1 + uy[j2] * c2, B = ty[j2] * c3;
            float4* row = (float4*) (plane + (size_t) wrapIndex(b.y - j2, K1) * K2 + (z0 - o));
#pragma unroll
            for (int w = 0; w < NQ; w++)
                if (4 * w < o + P)
                    atomicAdd(row + w, make_float4(A * T[4 * w] + B * U[4 * w], A * T[4 * w + 1] + B * U[4 * w + 1],
                                                   A * T[4 * w + 2] + B * U[4 * w + 2],
                                                   A * T[4 * w + 3] + B * U[4 * w + 3]));
        }
    } else {
#pragma unroll
        for (int j2 = 0; j2 < P; j2++) {
            const float A = ty[j2] * c1 + uy[j2] * c2, B = ty[j2] * c3;
            float* row = plane + (size_t) wrapIndex(b.y - j2, K1) * K2;
#pragma unroll
            for (int j3 = 0; j3 < P; j3++)
                atomicAdd(row + wrapIndex(bz - j3, K2), A * tz[j3] + B * uz[j3]);
        }
    }
}

// Gather of the reciprocal field of a field pass (the k_gather contract, FINAL false): per slot
// E_rec = -K recip . (sum_g Q[g] (u1 t2 t3, t1 u2 t3, t1 t2 u3)) (core/pgm_core.cpp:241-260).  A thread sums
// its x-plane's p^2 points per component (two line sums per line: t3 and u3 weighted); the atom's p partial sums
// are added in double in j1 order.  CGA as k_gather's: A p and the block partials of p . A p, the last block
// forming alph in block order.
template <int P, bool CGA>
__global__ void __launch_bounds__(256) k_gather_lines(Dev dv, int gateDone) {
    constexpr int APW = 32 / P;
    const int lane = threadIdx.x & 31, a = lane / P, j1 = lane - a * P, wib = threadIdx.x >> 5;
    const int warpG = (int) ((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (CGA && dv.scal[SC_DONE] != 0.0)
        return;   // every block alike (system 0)
    int slot = warpG * APW + a;
    bool on = a < APW;
    if (!CGA && on && gateDone && dv.useActive)   // a batch's CG iteration: the active systems' slots only
        slot = activeSlot(dv, slot);
    on = on && slot >= 0 && slot < dv.nAtoms;
    int i = 0, s = 0;
    if (on) {
        i = dv.slotAtom[slot];
        s = dv.atomSys[i];
        if (!CGA && gateDone && dv.scal[s * NSCAL + SC_DONE] != 0.0)
            on = false;
    }
    __shared__ float part[8][32][3];
    float f0 = 0.0f, f1 = 0.0f, f2 = 0.0f;
    const SysDev& S = dv.sys[s];
    if (on) {
        const float* sp = (const float*) dv.spl + (size_t) slot * 9 * MAXP;
        const float t1 = sp[j1], u1 = sp[3 * MAXP + j1];
        float ty[P], uy[P], tz[P], uz[P];
        lineCoefficients<P>(sp, ty, uy, tz, uz);
        const int K0 = S.K[0], K1 = S.K[1], K2 = S.K[2];
        const int4 b = dv.baseS[slot];
        const int bz = wrapIndex(b.z, K2), z0 = bz - (P - 1);
        const float* plane = (const float*) dv.grid + S.gridOff + (size_t) wrapIndex(b.x - j1, K0) * K1 * K2;
        float st[P], su[P];   // per line j2: sum_j3 t3 Q, sum_j3 u3 Q
        if (z0 >= 0 && (K2 & 3) == 0 && (S.gridOff & 3) == 0) {
            const int o = z0 & 3;
            float T[12], U[12];
            shiftLine<P>(tz, o, T);
            shiftLine<P>(uz, o, U);
            constexpr int NQ = (P + 3 + 3) / 4;
#pragma unroll
            for (int j2 = 0; j2 < P; j2++) {
                const float4* row = (const float4*) (plane + (size_t) wrapIndex(b.y - j2, K1) * K2 + (z0 - o));
                float x = 0.0f, y = 0.0f;
#pragma unroll
                for (int w = 0; w < NQ; w++)
                    if (4 * w < o + P) {
                        const float4 g = __ldcg(row + w);
                        x += T[4 * w] * g.x + T[4 * w + 1] * g.y + T[4 * w + 2] * g.z + T[4 * w + 3] * g.w;
                        y += U[4 * w] * g.x + U[4 * w + 1] * g.y + U[4 * w + 2] * g.z + U[4 * w + 3] * g.w;
                    }
                st[j2] = x;
                su[j2] = y;
            }
        } else {
#pragma unroll
            for (int j2 = 0; j2 < P; j2++) {
                const float* row = plane + (size_t) wrapIndex(b.y - j2, K1) * K2;
                float x = 0.0f, y = 0.0f;
#pragma unroll
                for (int j3 = 0; j3 < P; j3++) {
                    const float g = __ldcg(row + wrapIndex(bz - j3, K2));
                    x += tz[j3] * g;
                    y += uz[j3] * g;
                }
                st[j2] = x;
                su[j2] = y;
            }
        }
#pragma unroll
        for (int j2 = 0; j2 < P; j2++) {
            f0 += u1 * ty[j2] * st[j2];
            f1 += t1 * uy[j2] * st[j2];
            f2 += t1 * ty[j2] * su[j2];
        }
    }
    part[wib][lane][0] = f0;
    part[wib][lane][1] = f1;
    part[wib][lane][2] = f2;
    __syncwarp();
    double v = 0.0;   // CGA: the atom's p . A p (its first thread)
    if (on && j1 == 0) {
        double F[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int j = 0; j < P; j++)
#pragma unroll
            for (int k = 0; k < 3; k++)
                F[k] += (double) part[wib][lane + j][k];
        const double cs = 4.0 * S.beta * S.beta * S.beta / (3.0 * SQRT_PI);
        const double al = CGA ? dv.alpha[i] : 0.0;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const double E = -(S.K[0] * S.recip[3 * k] * F[0] + S.K[1] * S.recip[3 * k + 1] * F[1] +
                               S.K[2] * S.recip[3 * k + 2] * F[2]);
            dv.Erec[3 * i + k] = E;
            if (CGA) {   // A p = p / alpha - (E_pair + E_rec + cs p) (core/pgm_core.cpp:363)
                const double pk = dv.p[3 * i + k];
                const double apk = (al > 0) ? pk / al - (dv.Epair[3 * i + k] + E + cs * pk) : 0.0;
                dv.Ap[3 * i + k] = apk;
                v += pk * apk;
            }
        }
    }
    if constexpr (CGA) {
        __shared__ double asum[8 * APW];
        __shared__ int isLast;
        if (j1 == 0 && a < APW)
            asum[wib * APW + a] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int k = 0; k < 8 * APW; k++)   // the block's atoms in slot order
                t += asum[k];
            dv.gpartial[blockIdx.x] = t;
            __threadfence();
            isLast = atomicAdd(&dv.flags[10], 1) == (int) gridDim.x - 1;
        }
        __syncthreads();
        if (!isLast)
            return;
        __threadfence();
        double acc[1] = {0.0};   // thread t: blocks t, t + 256, ... in order; then the fixed block tree
        for (int k = threadIdx.x; k < (int) gridDim.x; k += blockDim.x)
            acc[0] += __ldcg(&dv.gpartial[k]);
        blockReduce<1>(acc, 0u);
        if (threadIdx.x == 0) {
            dv.scal[SC_ALPH] = dv.scal[SC_RZ] / fmax(acc[0], 1e-300);
            dv.flags[10] = 0;
        }
    }
}

// Blocks of 256 threads (8 warps of 32 / p atoms) covering n slots.
template <int P> inline int lineBlocks(int n) {
    constexpr int APW = 32 / P;
    const int warps = (n + APW - 1) / APW;
    return (warps + 7) / 8;
}

}   // namespace pgmb200
