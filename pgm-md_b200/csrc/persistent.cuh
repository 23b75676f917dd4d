// The CG solve of one system in mixed precision as ONE persistent cooperative kernel (one block per SM), for
// grids whose dimensions have at most FFT_MAXK points and the prime factors 2, 3, 5.
//
// Every CG iteration of core/pgm_core.cpp:351-385 (A v = v/alpha - T v; T v = pair + reciprocal + self field)
// runs inside the kernel, with grid barriers between its phases instead of kernel boundaries and graph nodes:
//
//   S  (every block, a chunk of slots)  p = z + beta p; the pair pass's float copy of p and the PME weights
//      (q, e_a = K_a p . recip[:, a]) of each slot;                                               grid barrier
//   F  blocks 0 .. K0-1 own the x-planes of the PME grid: the plane is spread in shared memory from the atoms
//      whose stencil reaches it (64-bit fixed-point shared atomics, so the sums do not depend on their order),
//      transformed along z and y, the x-lines exchanged through L2 (two barriers of the plane blocks), the
//      influence product, transformed back, and the potential gathered at the same atoms: each atom's field
//      sums of this plane go to a slot of their own (one of p per atom), summed later in a fixed order.
//      Blocks K0 .. end run the direct-space field pass of the iteration's direction over the pair records.
//                                                                                                  grid barrier
//   A  (every block) A p rows, the block's share of p . A p;                                        grid barrier
//   U  (every block) alph from the shares (fixed order), x, r, z of its slots, shares of z'.(r' - r), r'.z',
//      max |z'|;                                                                                    grid barrier
//   C  (every block, identically) beta, rz, err, the iteration count and the convergence test.
//
// Every reduction sums in a fixed order, so the solve repeats bit for bit.  Barrier waits are bounded (about
// a second); a block that gives up sets flags[11] and returns, and the host reports the evaluation as failed.
#pragma once

#include "kernels.cuh"

namespace pgmb200 {

constexpr int PCG_THREADS = 512;
constexpr int PCG_MIN_PAIR_BLOCKS = 16;      // blocks left for the pair pass beside the plane blocks
constexpr int PCG_BLOCKS_PER_SM = 1;         // resident blocks per SM (two, at 64 registers, measured slower)
constexpr float PCG_FIX = 4294967296.0f;     // 2^32: the fixed-point scale of the shared-memory spread
constexpr float PCG_UNFIX = 2.3283064365386963e-10f;   // 2^-32

// The spline record of one atom of the plane bins (order P): its slot, b1, b2 and b0 mod K0, and theta and
// dtheta of the three dimensions, c[dim 2P + kind P + j].
template <int P> struct PmeRec {
    int4 idx;
    float c[6 * P];
};

// The atoms that reach plane x: those of b0 = (x + j1) mod K0 for j1 < P, bins b0 nyc .. b0 nyc + nyc - 1 (the
// plane-owner kernels' bins by x-plane and row chunk, contiguous per x-plane; nyc = 1: bins by x-plane only);
// t-th of them -> (j1, record index).
template <int P>
struct PlaneAtoms {
    int start[P], cum[P + 1];
    __device__ __forceinline__ void init(const int* binStart, int x, int K0, int nyc) {
        cum[0] = 0;
#pragma unroll
        for (int j = 0; j < P; j++) {
            const int b = wrapIndex(x + j, K0) * nyc;
            start[j] = binStart[b];
            cum[j + 1] = cum[j] + binStart[b + nyc] - binStart[b];
        }
    }
    __device__ __forceinline__ int total() const { return cum[P]; }
    __device__ __forceinline__ int locate(int t, int& j1) const {
        j1 = 0;
#pragma unroll
        for (int j = 1; j < P; j++)
            j1 += (t >= cum[j]) ? 1 : 0;
        return start[j1] + t - cum[j1];
    }
};

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
    unsigned long long* const plane = (unsigned long long*) (b1 + dv.fftgBuf);
    const C* tw = (const C*) dv.twiddle;
    PlaneAtoms<P> pa;
    if (planeBlock) {
        for (int m = tid; m < K0; m += nT)
            W0[m] = tw[S.twOff[0] + m];
        for (int m = tid; m < K1; m += nT)
            W1[m] = tw[S.twOff[1] + m];
        for (int m = tid; m < K2; m += nT)
            W2[m] = tw[S.twOff[2] + m];
        pa.init(dv.pmeBinStart, x, K0, nyc);
    }
    C* const spec = (C*) dv.spec + S.specOff;
    C* const myPlane = spec + (size_t) x * nline;
    const PmeRec<P>* rec = (const PmeRec<P>*) dv.pmeRec;
    float4* const srcW = dv.srcW;
    float4* const gpart = dv.gpart;
    double* const part = dv.pcgPartial;
    const double cs = 4.0 * S.beta * S.beta * S.beta / (3.0 * SQRT_PI);
    // the block's chunk of slots for the per-atom phases
    const int per = (n + nb - 1) / nb, s0 = x * per, s1 = min(n, s0 + per);
    double rz = sc[SC_RZ], beta = sc[SC_BETA], it = sc[SC_IT];
    const double norm = sc[SC_NORM];
    for (;;) {
        // ---- S: direction p = z + beta p (or the pass's sources); float copy for the pair pass; PME weights
        for (int s = s0 + tid; s < s1; s += nT) {
            const int i = dv.slotAtom[s];
            double d[3];
#pragma unroll
            for (int k = 0; k < 3; k++) {
                if (PASS == 0) {
                    d[k] = dv.z[3 * i + k] + beta * dv.p[3 * i + k];
                    dv.p[3 * i + k] = d[k];
                } else {
                    d[k] = vec[3 * i + k];
                }
            }
            const float qf = PASS == 2 ? (float) dv.q[i] : 0.f;
            ((float4*) dv.dS)[s] = make_float4((float) d[0], (float) d[1], (float) d[2], qf);
            srcW[s] = make_float4(qf, (float) (S.K[0] * (d[0] * S.recip[0] + d[1] * S.recip[3] + d[2] * S.recip[6])),
                                  (float) (S.K[1] * (d[0] * S.recip[1] + d[1] * S.recip[4] + d[2] * S.recip[7])),
                                  (float) (S.K[2] * (d[0] * S.recip[2] + d[1] * S.recip[5] + d[2] * S.recip[8])));
        }
        if (!fftgBarrier(gbar, (unsigned) nb, dv.flags))
            return;
        // ---- F: the plane blocks' reciprocal part, the other blocks' direct part
        if (planeBlock) {
            for (int e = tid; e < K1 * K2; e += nT)
                plane[e] = 0ull;
            __syncthreads();
            for (int t = tid; t < pa.total(); t += nT) {
                int j1;
                const PmeRec<P>& r = rec[pa.locate(t, j1)];
                const int4 id = r.idx;
                const float4 w = __ldcg(srcW + id.x);
                float c[4 * P];   // (in registers before the atomics, which would otherwise force reloads)
#pragma unroll
                for (int k = 0; k < 4 * P; k++)
                    c[k] = r.c[2 * P + k];
                const float t1 = r.c[j1], u1 = r.c[P + j1];
                const float qe = w.x * t1 + w.y * u1, e1t = w.z * t1, e2t = w.w * t1;
                int col[P];
#pragma unroll
                for (int j3 = 0; j3 < P; j3++)
                    col[j3] = wrapIndex(id.z - j3, K2);
#pragma unroll
                for (int j2 = 0; j2 < P; j2++) {
                    const float A2 = c[j2] * qe + e1t * c[P + j2], B2 = e2t * c[j2];
                    unsigned long long* row = plane + wrapIndex(id.y - j2, K1) * K2;
#pragma unroll
                    for (int j3 = 0; j3 < P; j3++) {
                        const float v = A2 * c[2 * P + j3] + B2 * c[3 * P + j3];
                        atomicAdd(row + col[j3], (unsigned long long) __float2ll_rn(v * PCG_FIX));
                    }
                }
            }
            __syncthreads();
            // plane x: rows 2p, 2p + 1 as one complex row [pair][z]; z; separation into y-lines [kz][y]; y
            for (int e = tid; e < NP * K2; e += nT) {
                const int pr = qd(e, K2, iK2), z = e - pr * K2;
                C v;
                v.x = __ll2float_rn((long long) plane[2 * pr * K2 + z]) * PCG_UNFIX;
                v.y = (2 * pr + 1 < K1) ? __ll2float_rn((long long) plane[(2 * pr + 1) * K2 + z]) * PCG_UNFIX : 0.f;
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
            // gather at the same atoms: this plane's part of f_a = sum (d theta_a) theta theta phi
            const float* phi = (const float*) Zt;   // row y at [(y / 2) K2 + z] component y & 1
            for (int t = tid; t < pa.total(); t += nT) {
                int j1;
                const PmeRec<P>& r = rec[pa.locate(t, j1)];
                const int4 id = r.idx;
                int col[P];
#pragma unroll
                for (int j3 = 0; j3 < P; j3++)
                    col[j3] = wrapIndex(id.z - j3, K2);
                float A = 0.f, B = 0.f, Cc = 0.f;
#pragma unroll
                for (int j2 = 0; j2 < P; j2++) {
                    const int yy = wrapIndex(id.y - j2, K1);
                    const float* row = phi + 2 * ((yy >> 1) * K2) + (yy & 1);
                    float st = 0.f, su = 0.f;
#pragma unroll
                    for (int j3 = 0; j3 < P; j3++) {
                        const float ph = row[2 * col[j3]];
                        st += r.c[4 * P + j3] * ph;
                        su += r.c[5 * P + j3] * ph;
                    }
                    const float t2 = r.c[2 * P + j2], u2 = r.c[3 * P + j2];
                    A += t2 * st;
                    B += u2 * st;
                    Cc += t2 * su;
                }
                const float t1 = r.c[j1], u1 = r.c[P + j1];
                gpart[(size_t) j1 * n + id.x] = make_float4(u1 * A, t1 * B, t1 * Cc, 0.f);
            }
        } else {
            const int groups = nT / GS;
            pcgPairField<GS, PASS == 2>(dv, (x - K0) * groups + tid / GS, (nb - K0) * groups);
        }
        if (!fftgBarrier(gbar, (unsigned) nb, dv.flags))
            return;
        if (PASS != 0) {   // one field pass: E_rec per atom from the plane shares, then done
            for (int s = s0 + tid; s < s1; s += nT) {
                const int i = dv.slotAtom[s];
                double f[3] = {0.0, 0.0, 0.0};
#pragma unroll
                for (int j1 = 0; j1 < P; j1++) {
                    const float4 g = __ldcg(gpart + (size_t) j1 * n + s);
                    f[0] += g.x;
                    f[1] += g.y;
                    f[2] += g.z;
                }
#pragma unroll
                for (int k = 0; k < 3; k++)
                    dv.Erec[3 * i + k] = -(S.K[0] * S.recip[3 * k] * f[0] + S.K[1] * S.recip[3 * k + 1] * f[1] +
                                           S.K[2] * S.recip[3 * k + 2] * f[2]);
            }
            return;
        }
        // ---- A: rows of A p, the block's share of p . A p
        {
            double v[1] = {0.0};
            for (int s = s0 + tid; s < s1; s += nT) {
                const int i = dv.slotAtom[s];
                double f[3] = {0.0, 0.0, 0.0};
#pragma unroll
                for (int j1 = 0; j1 < P; j1++) {
                    const float4 g = __ldcg(gpart + (size_t) j1 * n + s);
                    f[0] += g.x;
                    f[1] += g.y;
                    f[2] += g.z;
                }
                const double al = dv.alpha[i];
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    const double Erec = -(S.K[0] * S.recip[3 * k] * f[0] + S.K[1] * S.recip[3 * k + 1] * f[1] +
                                          S.K[2] * S.recip[3 * k + 2] * f[2]);
                    const double pk = dv.p[3 * i + k];
                    const double Tp = __ldcg(dv.Epair + 3 * i + k) + Erec + cs * pk;
                    const double apk = (al > 0) ? pk / al - Tp : 0.0;
                    dv.Ap[3 * i + k] = apk;
                    v[0] += pk * apk;
                }
            }
            blockReduce<1>(v, 0u);
            if (tid == 0)
                part[(size_t) x * 4] = v[0];
        }
        if (!fftgBarrier(gbar, (unsigned) nb, dv.flags))
            return;
        // ---- U: alph, x, r, z; shares of z'.(r' - r), r'.z', max|z'|
        {
            double pap[1];
            pcgTotals<1>(part, nb, 0u, pap);
            const double alph = rz / fmax(pap[0], 1e-300);
            double v[3] = {0.0, 0.0, 0.0};
            for (int s = s0 + tid; s < s1; s += nT) {
                const int i = dv.slotAtom[s];
                const double al = dv.alpha[i];
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    const double pk = dv.p[3 * i + k];
                    dv.x[3 * i + k] += alph * pk;
                    const double rold = dv.r[3 * i + k];
                    const double rn = rold - alph * dv.Ap[3 * i + k];
                    const double zn = al * rn;
                    dv.r[3 * i + k] = rn;
                    dv.z[3 * i + k] = zn;
                    v[0] += zn * (rn - rold);
                    v[1] += rn * zn;
                    v[2] = fmax(v[2], fabs(zn));
                }
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
