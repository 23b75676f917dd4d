// The CG solve of one system in mixed precision as ONE persistent cooperative kernel (one block per SM), for
// grids whose dimensions have at most FFT_MAXK points and the prime factors 2, 3, 5.
//
// Every CG iteration of core/pgm_core.cpp:351-385 (A v = v/alpha - T v; T v = pair + reciprocal + self field)
// runs inside the kernel, with grid barriers between its phases instead of kernel boundaries and graph nodes:
//
//   S  (every block, 8 lanes per slot of its chunk)  p = z + beta p; the pair pass's float copy of p; the PME
//      weights (q, e_a = K_a p . recip[:, a]) and the spread of the atom into the 64-bit fixed-point grid
//      (global atomics, the same points and arithmetic as k_spread; integer sums do not depend on their order,
//      so the solve repeats bit for bit);                                                         grid barrier
//   F  blocks 0 .. K0-1 own the x-planes of the PME grid: the plane is read from the fixed-point grid (and
//      cleared for the next spread), transformed along z and y, the x-lines exchanged through L2 (two barriers
//      of the plane blocks), the influence product, transformed back and stored to the potential grid.
//      Blocks K0 .. end run the direct-space field pass of the iteration's direction over the pair records.
//                                                                                                  grid barrier
//   G  (every block, 8 lanes per slot of its chunk) E_rec at the atom from the potential grid, the atom's row of
//      A p and the block's share of p . A p;                                                        grid barrier
//   U  (every block) alph from the shares (fixed order), x, r, z of its slots, shares of z'.(r' - r), r'.z',
//      max |z'|;                                                                                    grid barrier
//   C  (every block, identically) beta, rz, err, the iteration count and the convergence test.
//
// Every reduction sums in a fixed order.  Data other blocks wrote in this launch is read past L1 (__ldcg).
// Barrier waits are bounded (about a second); a block that gives up sets flags[11] and returns, and the host
// reports the evaluation as failed.
#pragma once

#include "kernels.cuh"

namespace pgmb200 {

constexpr int PCG_THREADS = 512;
constexpr int PCG_MIN_PAIR_BLOCKS = 16;      // blocks left for the pair pass beside the plane blocks
constexpr int PCG_SLOT_LANES = 8;            // lanes per slot in the spread and gather phases
constexpr int PCG_BLOCKS_PER_SM = 1;         // resident blocks per SM (two, at 64 registers, measured slower)

// The spline record of one atom of the plane-owner kernels' bins (order P): its slot, b1, b2 and b0 mod K0, and
// theta and dtheta of the three dimensions, c[dim 2P + kind P + j].
template <int P> struct PmeRec {
    int4 idx;
    float c[6 * P];
};

// The spread of slot s (its atom's weights w = (q, e0, e1, e2)) into the 64-bit fixed-point grid by a group of L
// lanes (lane hl, mask `mask`, shared rows `row` for the evaluation's spline coefficients): a stencil column
// (j2, j3) per lane and round, a loop over j1; the groups of a warp keep several atoms' loads and atomics in
// flight.  The points and per-point arithmetic of k_spread, so both add the same integers.
// The group's share of slot s's spline coefficients (k = hl, hl + L, ...) and base index (lanes hl < 3), loaded
// ahead of the direction update that the spread waits for.
template <int P, int L> struct SpreadPre {
    float c[(6 * P + L - 1) / L];
    int bl;
    __device__ __forceinline__ void load(const Dev& dv, int s, int i, int hl) {
        const float* sp = (const float*) dv.spl + (size_t) s * 9 * MAXP;
#pragma unroll
        for (int m = 0; m < (6 * P + L - 1) / L; m++) {
            const int k = hl + m * L;
            if (k < 6 * P) {
                const int kind = k / (3 * P), dim = (k / P) % 3, j = k % P;
                c[m] = sp[(kind * 3 + dim) * MAXP + j];
            }
        }
        bl = hl < 3 ? dv.pmeBase[3 * i + hl] : 0;
    }
};

template <int P, int L>
__device__ __forceinline__ void pcgSpreadHalf(const Dev& dv, const SysDev& S, long long* gfix, float4 w,
                                             const SpreadPre<P, L>& pre, float (*sth)[3][P], float (*sdth)[3][P],
                                             int row, int hl, unsigned mask) {
#pragma unroll
    for (int m = 0; m < (6 * P + L - 1) / L; m++) {
        const int k = hl + m * L;
        if (k < 6 * P) {
            const int kind = k / (3 * P), dim = (k / P) % 3, j = k % P;
            if (kind == 0)
                sth[row][dim][j] = pre.c[m];
            else
                sdth[row][dim][j] = pre.c[m];
        }
    }
    const int bl = pre.bl;
    const int b0 = __shfl_sync(mask, bl, 0, L), b1 = __shfl_sync(mask, bl, 1, L), b2 = __shfl_sync(mask, bl, 2, L);
    __syncwarp(mask);
    const float qr = w.x, e0 = w.y, e1 = w.z, e2 = w.w;
    const int K0 = S.K[0], K1 = S.K[1], K2 = S.K[2];
    const size_t plane = (size_t) K1 * K2;
    for (int c = hl; c < P * P; c += L) {
        const int j2 = c / P, j3 = c % P;
        const float t2 = sth[row][1][j2], u2 = sdth[row][1][j2];
        const float t3 = sth[row][2][j3], u3 = sdth[row][2][j3];
        const float c23 = t2 * t3;
        const float a = qr * c23 + e1 * u2 * t3 + e2 * t2 * u3;
        const float b = e0 * c23;
        const size_t col = (size_t) wrapIndex(b1 - j2, K1) * K2 + wrapIndex(b2 - j3, K2);
#pragma unroll
        for (int j1 = 0; j1 < P; j1++)
            gridFixAdd(gfix + col + (size_t) wrapIndex(b0 - j1, K0) * plane,
                       (float) (a * sth[row][0][j1] + b * sdth[row][0][j1]));
    }
    __syncwarp(mask);   // (the next slot of this group overwrites the shared rows)
}

// E_rec at the atom of slot s from the potential grid gpot (written by other blocks in this launch: read past
// L1) by a group of L lanes (as pcgSpreadHalf): f_a = sum (d theta_a) theta theta phi over the stencil, E_rec =
// -sum_a K_a recip[:, a] f_a (core/pgm_core.cpp:241-264), the lanes' sums in double; or (CGA, the CG iterations)
// instead the atom's row of A p = p / alpha - (E_pair + E_rec + cs p) (core/pgm_core.cpp:363) and the returned
// share p_k (A p)_k of lanes hl = k < 3 (0 elsewhere).
template <int P, bool CGA, int L>
__device__ __forceinline__ double pcgGatherHalf(const Dev& dv, const SysDev& S, const float* gpot, int s,
                                               float (*sth)[3][P], float (*sdth)[3][P], int row, int hl,
                                               unsigned mask, double cs) {
    const int i = dv.slotAtom[s];
    double alI = 0.0, pI = 0.0, eI = 0.0;   // (CGA) the inputs of the atom's A p row, loaded first
    if (CGA && hl < 3) {
        alI = dv.alpha[i];
        pI = dv.p[3 * i + hl];
        eI = __ldcg(dv.Epair + 3 * i + hl);
    }
    const float* sp = (const float*) dv.spl + (size_t) s * 9 * MAXP;
    for (int k = hl; k < 6 * P; k += L) {
        const int kind = k / (3 * P), dim = (k / P) % 3, j = k % P;
        const float v = sp[(kind * 3 + dim) * MAXP + j];
        if (kind == 0)
            sth[row][dim][j] = v;
        else
            sdth[row][dim][j] = v;
    }
    const int bl = hl < 3 ? dv.pmeBase[3 * i + hl] : 0;
    const int b0 = __shfl_sync(mask, bl, 0, L), b1 = __shfl_sync(mask, bl, 1, L), b2 = __shfl_sync(mask, bl, 2, L);
    __syncwarp(mask);
    const int K0 = S.K[0], K1 = S.K[1], K2 = S.K[2];
    const size_t plane = (size_t) K1 * K2;
    float f0 = 0.f, f1 = 0.f, f2 = 0.f;
    for (int c = hl; c < P * P; c += L) {
        const int j2 = c / P, j3 = c % P;
        const float* col = gpot + (size_t) wrapIndex(b1 - j2, K1) * K2 + wrapIndex(b2 - j3, K2);
        float St = 0.f, Su = 0.f;
#pragma unroll
        for (int j1 = 0; j1 < P; j1++) {
            const float ph = __ldcg(col + (size_t) wrapIndex(b0 - j1, K0) * plane);
            St += sth[row][0][j1] * ph;
            Su += sdth[row][0][j1] * ph;
        }
        const float t2 = sth[row][1][j2], u2 = sdth[row][1][j2];
        const float t3 = sth[row][2][j3], u3 = sdth[row][2][j3];
        f0 += Su * t2 * t3;
        f1 += St * u2 * t3;
        f2 += St * t2 * u3;
    }
    double F[3] = {(double) f0, (double) f1, (double) f2};
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1)
#pragma unroll
        for (int k = 0; k < 3; k++)
            F[k] += __shfl_xor_sync(mask, F[k], o, L);
    double share = 0.0;
    if (hl < 3) {
        const int k = hl;
        const double E = -(S.K[0] * S.recip[3 * k] * F[0] + S.K[1] * S.recip[3 * k + 1] * F[1] +
                           S.K[2] * S.recip[3 * k + 2] * F[2]);
        if (CGA) {
            const double Tp = eI + E + cs * pI;
            const double apk = (alI > 0) ? pI / alI - Tp : 0.0;
            dv.Ap[3 * i + k] = apk;
            share = pI * apk;
        } else {
            dv.Erec[3 * i + k] = E;
        }
    }
    __syncwarp(mask);
    return share;
}

// Direct-space field of the direction p (mixed pair records) at slots g0, g0 + gstride, ...: GS lanes per slot,
// E_i = sum_j -p_j G1 + (p_j . x) x G2 (core/pgm_core.cpp:274-284), products in float, sums across lanes in
// double, written to Epair (caller order).
template <int GS, bool WITHQ>
__device__ __forceinline__ void pcgPairField(const Dev& dv, int g0, int gstride) {
    const int lane = threadIdx.x % GS;
    const unsigned gm = groupMask<GS>();
    const float4* dS = (const float4*) dv.dS;
    for (int slot = g0; slot < dv.nAtoms; slot += gstride) {
        const float4* arow = (const float4*) dv.pairA + (size_t) slot * dv.cap;
        const float2* brow = (const float2*) dv.pairB + (size_t) slot * dv.cap;
        const int cnt = dv.listCount[slot];
        float a0 = 0.f, a1 = 0.f, a2 = 0.f;
#pragma unroll 4
        for (int t = lane; t < cnt; t += GS) {
            const float4 xg = arow[t];
            const float2 gb = brow[t];
            const float4 dj = __ldcg(dS + realAsSlot(gb.y));   // (written by other blocks in this launch)
            float c = (dj.x * xg.x + dj.y * xg.y + dj.z * xg.z) * gb.x;
            if (WITHQ)
                c += dj.w * xg.w;
            a0 += c * xg.x - dj.x * xg.w;
            a1 += c * xg.y - dj.y * xg.w;
            a2 += c * xg.z - dj.z * xg.w;
        }
        double E0 = a0, E1 = a1, E2 = a2;
#pragma unroll
        for (int o = GS / 2; o > 0; o >>= 1) {
            E0 += __shfl_xor_sync(gm, E0, o, GS);
            E1 += __shfl_xor_sync(gm, E1, o, GS);
            E2 += __shfl_xor_sync(gm, E2, o, GS);
        }
        if (lane == 0) {
            const int i = dv.slotAtom[slot];
            dv.Epair[3 * i] = E0;
            dv.Epair[3 * i + 1] = E1;
            dv.Epair[3 * i + 2] = E2;
        }
    }
}

// Block-wide fixed-order sum (or max where the bit of maxMask is set) of NV values per block over the nb
// blocks' shares part[b * 4 + k]; every block obtains the same totals.
template <int NV>
__device__ __forceinline__ void pcgTotals(const double* part, int nb, unsigned maxMask, double* tot) {
    double v[NV];
#pragma unroll
    for (int k = 0; k < NV; k++)
        v[k] = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < NV; k++) {
            const double x = __ldcg(part + (size_t) b * 4 + k);
            v[k] = ((maxMask >> k) & 1u) ? fmax(v[k], x) : v[k] + x;
        }
    blockReduce<NV>(v, maxMask);
    __shared__ double out[NV];
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < NV; k++)
            out[k] = v[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; k++)
        tot[k] = out[k];
    __syncthreads();
}

// KC > 0: the grid is KC^3 (compile-time line transforms); 0: any grid the plane blocks handle.
// PASS 0: the CG loop.  PASS 1 / 2: ONE field pass of the same machinery -- the field at every atom of the dipoles
// vec (2: and the charges), E_pair and E_rec written per atom -- for the passes around the loop.
template <int P, int GS, int KC, int PASS>
__global__ void __launch_bounds__(PCG_THREADS, PCG_BLOCKS_PER_SM) k_cg_persistent(Dev dv, int nyc, const double* vec) {
    typedef cufftComplex C;
    const SysDev& S = dv.sys[0];
    double* sc = dv.scal;
    if (PASS == 0 && sc[SC_DONE] != 0.0)
        return;   // converged at the initial guess (every block alike)
    const int n = dv.nAtoms, nb = gridDim.x, tid = threadIdx.x, nT = blockDim.x;
    const int K0 = KC > 0 ? KC : S.K[0], K1 = KC > 0 ? KC : S.K[1], K2 = KC > 0 ? KC : S.K[2];
    const int K2h = K2 / 2 + 1, NP = (K1 + 1) / 2, ly = K1 + 1, lx = K0 + 1;
    const int x = blockIdx.x;
    const bool planeBlock = x < K0;
    const int nline = K1 * K2h, lpb = (nline + K0 - 1) / K0, l0 = x * lpb;
    const int nl = planeBlock ? max(0, min(nline, l0 + lpb) - l0) : 0;
    const float iK2 = __frcp_rn((float) K2), iK2h = __frcp_rn((float) K2h), iLpb = __frcp_rn((float) lpb);
    auto qd = [](int e, int d, float inv) { return KC > 0 ? e / d : fdiv(e, inv); };
    unsigned* const gbar = dv.pcgBar;        // every block
    unsigned* const pbar = dv.pcgBar + 1;    // the plane blocks
    extern __shared__ __align__(16) unsigned char smraw[];
    C* W0 = (C*) smraw;
    C* W1 = W0 + FFT_MAXK;
    C* W2 = W1 + FFT_MAXK;
    C* const b0 = W2 + FFT_MAXK;
    C* const b1 = b0 + dv.fftgBuf;
    const C* tw = (const C*) dv.twiddle;
    if (planeBlock) {
        for (int m = tid; m < K0; m += nT)
            W0[m] = tw[S.twOff[0] + m];
        for (int m = tid; m < K1; m += nT)
            W1[m] = tw[S.twOff[1] + m];
        for (int m = tid; m < K2; m += nT)
            W2[m] = tw[S.twOff[2] + m];
    }
    C* const spec = (C*) dv.spec + S.specOff;
    C* const myPlane = spec + (size_t) x * nline;
    double* const part = dv.pcgPartial;
    // the slot-group phases (spread, gather): the groups' shared spline rows, the fixed-point charge grid and the
    // float potential grid
    constexpr int SL = PCG_SLOT_LANES;
    __shared__ float psth[PCG_THREADS / SL][3][P], psdth[PCG_THREADS / SL][3][P];
    // the slot-group phases: SL lanes per slot
    const int hrow = tid / SL, hl = tid % SL, nhalves = nT / SL;
    const unsigned hmask = ((1u << SL) - 1u) << (tid & 31 & ~(SL - 1));
    long long* const gfix = dv.gridFix + S.gridOff;
    float* const gpot = (float*) dv.grid + S.gridOff;
    (void) nyc;
    const double cs = 4.0 * S.beta * S.beta * S.beta / (3.0 * SQRT_PI);
    // the block's chunk of slots for the per-atom phases
    const int per = (n + nb - 1) / nb, s0 = x * per, s1 = min(n, s0 + per);
    double rz = sc[SC_RZ], beta = sc[SC_BETA], it = sc[SC_IT];
    const double norm = sc[SC_NORM];
    for (;;) {
        // ---- S: SL lanes per slot: direction p = z + beta p (or the pass's sources), the float copy for the
        // pair pass, the PME weights (q, e_a = K_a p . recip[:, a]) and the spread
        for (int s = s0 + hrow; s < s1; s += nhalves) {
            const int i = dv.slotAtom[s];
            SpreadPre<P, SL> pre;
            pre.load(dv, s, i, hl);
            double dl = 0.0;
            if (hl < 3) {
                if (PASS == 0) {
                    dl = dv.z[3 * i + hl] + beta * dv.p[3 * i + hl];
                    dv.p[3 * i + hl] = dl;
                } else {
                    dl = vec[3 * i + hl];
                }
            }
            const double d0 = __shfl_sync(hmask, dl, 0, SL), d1 = __shfl_sync(hmask, dl, 1, SL),
                         d2 = __shfl_sync(hmask, dl, 2, SL);
            const float qf = PASS == 2 ? (float) dv.q[i] : 0.f;
            if (hl == 0)
                ((float4*) dv.dS)[s] = make_float4((float) d0, (float) d1, (float) d2, qf);
            const float4 w = make_float4(qf, (float) (S.K[0] * (d0 * S.recip[0] + d1 * S.recip[3] + d2 * S.recip[6])),
                                         (float) (S.K[1] * (d0 * S.recip[1] + d1 * S.recip[4] + d2 * S.recip[7])),
                                         (float) (S.K[2] * (d0 * S.recip[2] + d1 * S.recip[5] + d2 * S.recip[8])));
            pcgSpreadHalf<P, SL>(dv, S, gfix, w, pre, psth, psdth, hrow, hl, hmask);
        }
        if (!fftgBarrier(gbar, (unsigned) nb, dv.flags))
            return;
        // ---- F: the plane blocks' reciprocal part, the other blocks' direct part
        if (planeBlock) {
            // plane x from the fixed-point grid (cleared for the next spread): rows 2p, 2p + 1 as one complex row
            // [pair][z]; z; separation into y-lines [kz][y]; y
            long long* const fxx = gfix + (size_t) x * K1 * K2;
            auto take = [](long long* g) {
                const long long v = __ldcg(g);
                __stcg(g, 0ll);
                return (float) ((double) v * (1.0 / 4294967296.0));
            };
            for (int e = tid; e < NP * K2; e += nT) {
                const int pr = qd(e, K2, iK2), z = e - pr * K2;
                C v;
                v.x = take(fxx + 2 * pr * K2 + z);
                v.y = (2 * pr + 1 < K1) ? take(fxx + (2 * pr + 1) * K2 + z) : 0.f;
                b0[e] = v;
            }
            __syncthreads();
            C* Z = fftLinesK<float, -1, KC>(b0, b1, NP, K2, K2, W2);
            C* O = (Z == b0) ? b1 : b0;
            for (int e = tid; e < NP * K2h; e += nT) {
                const int pr = qd(e, K2h, iK2h), kz = e - pr * K2h;
                const C* zr = Z + pr * K2;
                const C zk = zr[kz], zm = zr[kz == 0 ? 0 : K2 - kz];
                C X, Y;
                X.x = 0.5f * (zk.x + zm.x);
                X.y = 0.5f * (zk.y - zm.y);
                Y.x = 0.5f * (zk.y + zm.y);
                Y.y = 0.5f * (zm.x - zk.x);
                C* o = O + kz * ly + 2 * pr;
                o[0] = X;
                if (2 * pr + 1 < K1)
                    o[1] = Y;
            }
            __syncthreads();
            const C* F = fftLinesK<float, -1, KC>(O, Z, K2h, K1, ly, W1);
            for (int e = tid; e < nline; e += nT) {
                const int ky = qd(e, K2h, iK2h), kz = e - ky * K2h;
                myPlane[e] = F[kz * ly + ky];
            }
            if (!fftgBarrier(pbar, (unsigned) K0, dv.flags))
                return;
            // my x-lines: forward along x, influence product, back
            for (int e = tid; e < lpb * K0; e += nT) {
                const int xx = qd(e, lpb, iLpb), li = e - xx * lpb;
                if (li < nl)
                    b0[li * lx + xx] = __ldcg(spec + (size_t) xx * nline + l0 + li);
            }
            __syncthreads();
            C* Fx = fftLinesK<float, -1, KC>(b0, b1, nl, K0, lx, W0);
            const float* infl = (const float*) dv.infl + S.specOff;
            for (int e = tid; e < lpb * K0; e += nT) {
                const int xx = qd(e, lpb, iLpb), li = e - xx * lpb;
                if (li < nl) {
                    const float gk = infl[(size_t) xx * nline + l0 + li];
                    C& v = Fx[li * lx + xx];
                    v.x *= gk;
                    v.y *= gk;
                }
            }
            __syncthreads();
            const C* Gx = fftLinesK<float, 1, KC>(Fx, Fx == b0 ? b1 : b0, nl, K0, lx, W0);
            for (int e = tid; e < lpb * K0; e += nT) {
                const int xx = qd(e, lpb, iLpb), li = e - xx * lpb;
                if (li < nl)
                    spec[(size_t) xx * nline + l0 + li] = Gx[li * lx + xx];
            }
            if (!fftgBarrier(pbar, (unsigned) K0, dv.flags))
                return;
            // plane x back: y-lines; y; two real rows from one complex row; z
            for (int e = tid; e < nline; e += nT) {
                const int ky = qd(e, K2h, iK2h), kz = e - ky * K2h;
                b0[kz * ly + ky] = __ldcg(myPlane + e);
            }
            __syncthreads();
            C* Gy = fftLinesK<float, 1, KC>(b0, b1, K2h, K1, ly, W1);
            C* O2 = (Gy == b0) ? b1 : b0;
            for (int e = tid; e < NP * K2; e += nT) {
                const int pr = qd(e, K2, iK2), k = e - pr * K2;
                const bool upper = k >= K2h;
                const int kk = upper ? K2 - k : k;
                const bool realOnly = (k == 0) || ((K2 & 1) == 0 && k == K2 / 2);
                const C* gy = Gy + kk * ly + 2 * pr;
                C X = gy[0], Y;
                Y.x = 0.f;
                Y.y = 0.f;
                if (2 * pr + 1 < K1)
                    Y = gy[1];
                if (upper) {
                    X.y = -X.y;
                    Y.y = -Y.y;
                }
                if (realOnly) {
                    X.y = 0.f;
                    Y.y = 0.f;
                }
                C Zv;
                Zv.x = X.x - Y.y;
                Zv.y = X.y + Y.x;
                O2[e] = Zv;
            }
            __syncthreads();
            const C* Zt = fftLinesK<float, 1, KC>(O2, Gy, NP, K2, K2, W2);
            float* const gx = gpot + (size_t) x * K1 * K2;   // plane x of the potential
            for (int e = tid; e < NP * K2; e += nT) {
                const int pr = qd(e, K2, iK2), z = e - pr * K2;
                gx[2 * pr * K2 + z] = Zt[e].x;
                if (2 * pr + 1 < K1)
                    gx[(2 * pr + 1) * K2 + z] = Zt[e].y;
            }
        } else {
            const int groups = nT / GS;
            pcgPairField<GS, PASS == 2>(dv, (x - K0) * groups + tid / GS, (nb - K0) * groups);
        }
        if (!fftgBarrier(gbar, (unsigned) nb, dv.flags))
            return;
        // ---- G: E_rec at the chunk's atoms (a field pass), or the rows of A p and the block's share of p . A p
        if (PASS != 0) {   // one field pass: E_pair and E_rec written
            for (int s = s0 + hrow; s < s1; s += nhalves)
                pcgGatherHalf<P, false, SL>(dv, S, gpot, s, psth, psdth, hrow, hl, hmask, cs);
            return;
        }
        {
            double v[1] = {0.0};
            for (int s = s0 + hrow; s < s1; s += nhalves)
                v[0] += pcgGatherHalf<P, true, SL>(dv, S, gpot, s, psth, psdth, hrow, hl, hmask, cs);
            blockReduce<1>(v, 0u);
            if (tid == 0)
                part[(size_t) x * 4] = v[0];
        }
        if (!fftgBarrier(gbar, (unsigned) nb, dv.flags))
            return;
        // ---- U: alph, x, r, z; shares of z'.(r' - r), r'.z', max|z'|
        {
            // the first slot's p, x, r, A p and alpha are loaded before the total of p . A p is formed
            const int sF = s0 + tid;
            const bool hasF = sF < s1;
            const int iF = hasF ? dv.slotAtom[sF] : 0;
            double pF[3] = {0, 0, 0}, xF[3] = {0, 0, 0}, rF[3] = {0, 0, 0}, aF[3] = {0, 0, 0}, alF = 0.0;
            if (hasF) {
                alF = dv.alpha[iF];
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    pF[k] = dv.p[3 * iF + k];
                    xF[k] = dv.x[3 * iF + k];
                    rF[k] = dv.r[3 * iF + k];
                    aF[k] = dv.Ap[3 * iF + k];
                }
            }
            double pap[1];
            pcgTotals<1>(part, nb, 0u, pap);
            const double alph = rz / fmax(pap[0], 1e-300);
            double v[3] = {0.0, 0.0, 0.0};
            auto update = [&](int i, double al, const double* pk, const double* xk, const double* rk, const double* ak) {
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    dv.x[3 * i + k] = xk[k] + alph * pk[k];
                    const double rold = rk[k];
                    const double rn = rold - alph * ak[k];
                    const double zn = al * rn;
                    dv.r[3 * i + k] = rn;
                    dv.z[3 * i + k] = zn;
                    v[0] += zn * (rn - rold);
                    v[1] += rn * zn;
                    v[2] = fmax(v[2], fabs(zn));
                }
            };
            if (hasF)
                update(iF, alF, pF, xF, rF, aF);
            for (int s = sF + nT; s < s1; s += nT) {
                const int i = dv.slotAtom[s];
                double pk[3], xk[3], rk[3], ak[3];
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    pk[k] = dv.p[3 * i + k];
                    xk[k] = dv.x[3 * i + k];
                    rk[k] = dv.r[3 * i + k];
                    ak[k] = dv.Ap[3 * i + k];
                }
                update(i, dv.alpha[i], pk, xk, rk, ak);
            }
            blockReduce<3>(v, 4u);
            if (tid == 0) {
                if (x == 0)
                    sc[SC_ALPH] = alph;
                part[(size_t) nb * 4 + (size_t) x * 4] = v[0];
                part[(size_t) nb * 4 + (size_t) x * 4 + 1] = v[1];
                part[(size_t) nb * 4 + (size_t) x * 4 + 2] = v[2];
            }
        }
        if (!fftgBarrier(gbar, (unsigned) nb, dv.flags))
            return;
        // ---- C: the same decision in every block
        double tot[3];
        pcgTotals<3>(part + (size_t) nb * 4, nb, 4u, tot);
        beta = tot[0] / fmax(rz, 1e-300);
        rz = tot[1];
        const double err = tot[2] / norm;
        it += 1.0;
        const bool more = err > dv.tol && it < dv.maxIter;
        if (x == 0 && tid == 0) {
            sc[SC_BETA] = beta;
            sc[SC_RZ] = rz;
            sc[SC_ERR] = err;
            sc[SC_IT] = it;
            if (!more) {
                sc[SC_DONE] = 1.0;
                atomicAdd(&dv.flags[2], 1);
            }
        }
        if (!more)
            return;
    }
}

}  // namespace pgmb200
