// Cell-group tile PME spread and gather of the mixed-precision field passes (one system; orders 4, 5, 6, 8).
//
// The atoms are already in cell order (the pair search's cells, a fraction of the list radius wide), so a block
// takes a G x G x G group of cells -- G^2 contiguous runs of slots -- and the grid window its atoms' stencils
// cover: from the smallest base index of its atoms minus p - 1 to the largest, per dimension (offsets from a
// reference point of the group, wrapped to the nearest image, so a group at the box edge and atoms that drifted
// since the list's build need nothing special).
//   spread  the window is a shared-memory tile; a warp per atom adds its p^3 points with shared float atomics
//           (no index wrapping: the tile is the atom's neighbourhood), then the block adds the tile to the grid
//           once, coalesced along z.  Global atomics fall from p^3 per atom to one per tile point (about a
//           quarter as many at G = 4, 22 cells a side);
//   gather  the block reads its window from the grid once (coalesced) and each warp sums its atom's p^3 points
//           from shared memory.
// A window larger than the tile capacity (atoms far from their cells) sends the block through the grid
// directly: global atomics / loads per point, as the warp-per-atom kernels do.
#pragma once

#include "kernels.cuh"

namespace pgmb200 {

constexpr int TL_THREADS = 256;
constexpr int TL_MAX_G = 4;

struct TileBlock {
    int runStart[TL_MAX_G * TL_MAX_G], runCum[TL_MAX_G * TL_MAX_G + 1];
    int ref[3], lo[3], T[3];
    int mn[3], mx[3];
    int ok;
};

__device__ __forceinline__ int nearestImage(int off, int K) {   // off in (-K, K) -> [-K/2, K - K/2)
    off += off < -(K >> 1) ? K : 0;
    off -= off >= K - (K >> 1) ? K : 0;
    return off;
}

// The block's cell group (blockIdx.x over ceil(n_a / G) groups per dimension), its slot runs and its window.
template <int P>
__device__ void tileSetup(const Dev& dv, const SysDev& S, int G, int cap, TileBlock& tb) {
    const int n0 = S.cellN[0], n1 = S.cellN[1], n2 = S.cellN[2];
    const int ng1 = (n1 + G - 1) / G, ng2 = (n2 + G - 1) / G;
    const int g2 = blockIdx.x % ng2, g1 = (blockIdx.x / ng2) % ng1, g0 = blockIdx.x / (ng2 * ng1);
    const int t = threadIdx.x;
    if (t < G * G) {
        const int c0 = g0 * G + t / G, c1 = g1 * G + t % G, cz0 = g2 * G, cz1 = min(n2, cz0 + G);
        int st = 0, len = 0;
        if (c0 < n0 && c1 < n1) {
            const int lin = S.cellOff + (c0 * n1 + c1) * n2;
            st = dv.cellStart[lin + cz0];
            len = dv.cellStart[lin + cz1] - st;
        }
        tb.runStart[t] = st;
        tb.runCum[t + 1] = len;
    }
    if (t < 3) {
        const int gi = t == 0 ? g0 : t == 1 ? g1 : g2;
        tb.ref[t] = (int) floor((double) S.K[t] * (gi * G) / S.cellN[t]);
        tb.mn[t] = INT_MAX;
        tb.mx[t] = INT_MIN;
    }
    __syncthreads();
    if (t == 0) {
        tb.runCum[0] = 0;
        for (int r = 0; r < G * G; r++)
            tb.runCum[r + 1] += tb.runCum[r];
    }
    __syncthreads();
    const int na = tb.runCum[G * G];
    int mn[3] = {INT_MAX, INT_MAX, INT_MAX}, mx[3] = {INT_MIN, INT_MIN, INT_MIN};
    for (int f = t; f < na; f += blockDim.x) {
        int r = 0;
        while (tb.runCum[r + 1] <= f)
            r++;
        const int4 b = dv.baseS[tb.runStart[r] + f - tb.runCum[r]];
        const int bb[3] = {b.x, b.y, b.z};
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const int o = nearestImage(bb[a] - tb.ref[a], S.K[a]);
            mn[a] = min(mn[a], o);
            mx[a] = max(mx[a], o);
        }
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mn[a] = min(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], o));
            mx[a] = max(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], o));
        }
    }
    if ((t & 31) == 0)
        for (int a = 0; a < 3; a++) {
            atomicMin(&tb.mn[a], mn[a]);
            atomicMax(&tb.mx[a], mx[a]);
        }
    __syncthreads();
    if (t == 0) {
        long long vol = 1;
        for (int a = 0; a < 3; a++) {
            tb.lo[a] = tb.mn[a] - (P - 1);
            tb.T[a] = na > 0 ? tb.mx[a] - tb.lo[a] + 1 : 0;
            vol *= tb.T[a];
        }
        // (a window wider than the grid would also fold onto itself, and grids under 2p points would take the
        // window's corners beyond one image: those blocks take the direct path)
        tb.ok = na > 0 && vol <= cap;
        for (int a = 0; a < 3; a++)   // (local offsets are packed in 10 bits each)
            tb.ok = tb.ok && tb.T[a] <= S.K[a] && S.K[a] >= 2 * P && tb.T[a] < 1024;
    }
    __syncthreads();
}

__device__ __forceinline__ int tileSlot(const TileBlock& tb, int f) {
    int r = 0;
    while (tb.runCum[r + 1] <= f)
        r++;
    return tb.runStart[r] + f - tb.runCum[r];
}

constexpr int TL_CHUNK = TL_THREADS;   // atoms staged per round, one per thread

// Word k < 6p of a slot's spline coefficients: k = kind 3p + dim p + j (kind 0 theta, 1 dtheta).
template <int P>
__device__ __forceinline__ float tileCoefWord(const Dev& dv, int slot, int k) {
    const int kind = k / (3 * P), dim = (k / P) % 3, j = k % P;
    return ((const float*) dv.spl)[(size_t) slot * 9 * MAXP + (kind * 3 + dim) * MAXP + j];
}

__device__ __forceinline__ int tilePack(int x, int y, int z) { return x | (y << 10) | (z << 20); }

// Spread (the k_spread contract: mode 0 q and vec, 1 vec only, 2 the CG direction p = z + beta p first,
// vec = p; writes dS = (d, q)), Q[g] += q t1 t2 t3 + e0 u1 t2 t3 + e1 t1 u2 t3 + e2 t1 t2 u3
// (core/pgm_core.cpp:187-207).  The grid is cleared before.  Per round of up to 256 atoms: a thread per atom
// forms its weights (q, e) and local offsets into shared memory (the dependent loads of all the round's atoms in
// flight at once); then a warp per atom adds its points, the next atom's coefficients loading meanwhile.
template <int P>
__global__ void __launch_bounds__(TL_THREADS) k_spread_tiles(Dev dv, int mode, double* vec, int G, int cap) {
    extern __shared__ float tile[];
    __shared__ TileBlock tb;
    __shared__ float4 aw[TL_CHUNK];
    __shared__ int aslot[TL_CHUNK], aoff[TL_CHUNK];
    __shared__ float sc[2][TL_THREADS / (P * P)][6 * P];
    const SysDev& S = dv.sys[0];
    if (mode == 2 && dv.scal[SC_DONE] != 0.0)
        return;   // every block alike
    tileSetup<P>(dv, S, G, cap, tb);
    const int na = tb.runCum[G * G];
    const int T1 = tb.T[1], T2 = tb.T[2], T12 = T1 * T2, vol = tb.T[0] * T12;
    const bool ok = tb.ok;
    if (ok)
        for (int e = threadIdx.x; e < vol; e += blockDim.x)
            tile[e] = 0.f;
    const int K0 = S.K[0], K1 = S.K[1], K2 = S.K[2];
    float* grid = (float*) dv.grid + S.gridOff;
    const double bt = mode == 2 ? dv.scal[SC_BETA] : 0.0;
    for (int c0 = 0; c0 < na; c0 += TL_CHUNK) {
        const int cn = min(TL_CHUNK, na - c0);
        if ((int) threadIdx.x < cn) {
            const int slot = tileSlot(tb, c0 + threadIdx.x);
            const int i = dv.slotAtom[slot];
            double d[3];
#pragma unroll
            for (int k = 0; k < 3; k++) {
                d[k] = mode == 2 ? dv.z[3 * i + k] + bt * vec[3 * i + k] : vec[3 * i + k];
                if (mode == 2)
                    vec[3 * i + k] = d[k];
            }
            const double qv = mode == 0 ? dv.q[i] : 0.0;
            ((float4*) dv.dS)[slot] = make_float4((float) d[0], (float) d[1], (float) d[2], (float) qv);
            float e[3];
#pragma unroll
            for (int k = 0; k < 3; k++)
                e[k] = (float) (S.K[k] * (d[0] * S.recip[k] + d[1] * S.recip[3 + k] + d[2] * S.recip[6 + k]));
            aw[threadIdx.x] = make_float4((float) qv, e[0], e[1], e[2]);
            aslot[threadIdx.x] = slot;
            if (ok) {
                const int4 b = dv.baseS[slot];
                aoff[threadIdx.x] = tilePack(nearestImage(b.x - tb.ref[0], K0) - tb.lo[0],
                                             nearestImage(b.y - tb.ref[1], K1) - tb.lo[1],
                                             nearestImage(b.z - tb.ref[2], K2) - tb.lo[2]);
            }
        }
        __syncthreads();
        // rounds of APR atoms, a thread per (atom, column (j2, j3)) adding the column's p points; the round's
        // coefficient words staged by the same threads (word w of atom a), the next round's loading meanwhile
        constexpr int NCOL = P * P, APR = TL_THREADS / NCOL;
        const int ra = threadIdx.x / NCOL, col = threadIdx.x - ra * NCOL;
        const int j2 = col / P, j3 = col - (col / P) * P;
        // (an atom has 6p coefficient words and p^2 threads: for p < 6 some threads stage two)
        const bool wordT = ra < APR && col < 6 * P, word2 = ra < APR && col + NCOL < 6 * P;
        float cw = 0.f, cw2 = 0.f;
        if (wordT && ra < cn)
            cw = tileCoefWord<P>(dv, aslot[ra], col);
        if (word2 && ra < cn)
            cw2 = tileCoefWord<P>(dv, aslot[ra], col + NCOL);
        for (int r0 = 0, buf = 0; r0 < cn; r0 += APR, buf ^= 1) {
            if (wordT)
                sc[buf][ra][col] = cw;
            if (word2)
                sc[buf][ra][col + NCOL] = cw2;
            __syncthreads();
            if (wordT && r0 + APR + ra < cn)
                cw = tileCoefWord<P>(dv, aslot[r0 + APR + ra], col);
            if (word2 && r0 + APR + ra < cn)
                cw2 = tileCoefWord<P>(dv, aslot[r0 + APR + ra], col + NCOL);
            const int a = r0 + ra;
            if (ra < APR && a < cn) {
                const float* th = sc[buf][ra];
                const float* dth = th + 3 * P;
                const float4 w = aw[a];
                const float t2 = th[P + j2], u2 = dth[P + j2], t3 = th[2 * P + j3], u3 = dth[2 * P + j3];
                const float c23 = t2 * t3;
                const float ac = w.x * c23 + w.z * u2 * t3 + w.w * t2 * u3, bc = w.y * c23;
                if (ok) {
                    const int pk = aoff[a], ox = pk & 1023, oy = (pk >> 10) & 1023, oz = pk >> 20;
                    float* cp = tile + (oy - j2) * T2 + (oz - j3) + ox * T12;
#pragma unroll
                    for (int j1 = 0; j1 < P; j1++)
                        atomicAdd(cp - j1 * T12, ac * th[j1] + bc * dth[j1]);
                } else {
                    const int4 b = dv.baseS[aslot[a]];
                    float* cp = grid + (size_t) wrapIndex(b.y - j2, K1) * K2 + wrapIndex(b.z - j3, K2);
#pragma unroll
                    for (int j1 = 0; j1 < P; j1++)
                        atomicAdd(cp + (size_t) wrapIndex(b.x - j1, K0) * K1 * K2, ac * th[j1] + bc * dth[j1]);
                }
            }
        }
        __syncthreads();   // (the round's staging read before the next round's)
    }
    if (ok) {
        const int x0 = tb.ref[0] + tb.lo[0], y0 = tb.ref[1] + tb.lo[1], z0 = tb.ref[2] + tb.lo[2];
        for (int e = threadIdx.x; e < vol; e += blockDim.x) {
            const float v = tile[e];
            if (v != 0.f) {
                const int ix = e / T12, r = e - ix * T12, iy = r / T2, iz = r - iy * T2;
                atomicAdd(grid + (size_t) wrapIndex(x0 + ix, K0) * K1 * K2 + (size_t) wrapIndex(y0 + iy, K1) * K2 +
                              wrapIndex(z0 + iz, K2), v);
            }
        }
    }
}

// Gather of the reciprocal field of a field pass (the k_gather contract, FINAL false): per slot
// E_rec = -K recip . (sum_g Q[g] (u1 t2 t3, t1 u2 t3, t1 t2 u3)) (core/pgm_core.cpp:241-260).  Rounds of up to
// 256 atoms: a thread per atom stages its slot and offsets; a warp per atom sums its points from the tile (the
// next atom's coefficients loading meanwhile); a thread per atom forms E_rec and, with CGA (as k_gather's), the
// row of A p and p . A p, the block's share summed in atom order and the last block forming alph in block order.
template <int P, bool CGA>
__global__ void __launch_bounds__(TL_THREADS) k_gather_tiles(Dev dv, int gate, int G, int cap) {
    extern __shared__ float tile[];
    __shared__ TileBlock tb;
    __shared__ int aslot[TL_CHUNK], aoff[TL_CHUNK];
    __shared__ double aF[TL_CHUNK][3];
    __shared__ double av[TL_CHUNK];
    __shared__ float sc[2][TL_THREADS / (P * P)][6 * P];
    __shared__ float red[TL_THREADS / (P * P)][P * P][3];
    const SysDev& S = dv.sys[0];
    if ((CGA || gate) && dv.scal[SC_DONE] != 0.0)
        return;   // every block alike
    tileSetup<P>(dv, S, G, cap, tb);
    const int na = tb.runCum[G * G];
    const int T1 = tb.T[1], T2 = tb.T[2], T12 = T1 * T2, vol = tb.T[0] * T12;
    const bool ok = tb.ok;
    const int K0 = S.K[0], K1 = S.K[1], K2 = S.K[2];
    const float* grid = (const float*) dv.grid + S.gridOff;
    if (ok) {
        const int x0 = tb.ref[0] + tb.lo[0], y0 = tb.ref[1] + tb.lo[1], z0 = tb.ref[2] + tb.lo[2];
        for (int e = threadIdx.x; e < vol; e += blockDim.x) {
            const int ix = e / T12, r = e - ix * T12, iy = r / T2, iz = r - iy * T2;
            tile[e] = __ldcg(grid + (size_t) wrapIndex(x0 + ix, K0) * K1 * K2 + (size_t) wrapIndex(y0 + iy, K1) * K2 +
                             wrapIndex(z0 + iz, K2));
        }
    }
    const double cs = 4.0 * S.beta * S.beta * S.beta / (3.0 * SQRT_PI);
    double pap = 0.0;   // CGA (thread 0): the block's p . A p, atom order
    for (int c0 = 0; c0 < na; c0 += TL_CHUNK) {
        const int cn = min(TL_CHUNK, na - c0);
        if ((int) threadIdx.x < cn) {
            const int slot = tileSlot(tb, c0 + threadIdx.x);
            aslot[threadIdx.x] = slot;
            if (ok) {
                const int4 b = dv.baseS[slot];
                aoff[threadIdx.x] = tilePack(nearestImage(b.x - tb.ref[0], K0) - tb.lo[0],
                                             nearestImage(b.y - tb.ref[1], K1) - tb.lo[1],
                                             nearestImage(b.z - tb.ref[2], K2) - tb.lo[2]);
            }
        }
        __syncthreads();   // (also: the tile is loaded)
        // rounds of APR atoms, a thread per (atom, column (j2, j3)) summing the column's p points; each atom's
        // column sums then added in column order (double) by three of the threads
        constexpr int NCOL = P * P, APR = TL_THREADS / NCOL;
        const int ra = threadIdx.x / NCOL, col = threadIdx.x - ra * NCOL;
        const int j2 = col / P, j3 = col - (col / P) * P;
        // (an atom has 6p coefficient words and p^2 threads: for p < 6 some threads stage two)
        const bool wordT = ra < APR && col < 6 * P, word2 = ra < APR && col + NCOL < 6 * P;
        float cw = 0.f, cw2 = 0.f;
        if (wordT && ra < cn)
            cw = tileCoefWord<P>(dv, aslot[ra], col);
        if (word2 && ra < cn)
            cw2 = tileCoefWord<P>(dv, aslot[ra], col + NCOL);
        for (int r0 = 0, buf = 0; r0 < cn; r0 += APR, buf ^= 1) {
            if (wordT)
                sc[buf][ra][col] = cw;
            if (word2)
                sc[buf][ra][col + NCOL] = cw2;
            __syncthreads();
            if (wordT && r0 + APR + ra < cn)
                cw = tileCoefWord<P>(dv, aslot[r0 + APR + ra], col);
            if (word2 && r0 + APR + ra < cn)
                cw2 = tileCoefWord<P>(dv, aslot[r0 + APR + ra], col + NCOL);
            const int a = r0 + ra;
            if (ra < APR && a < cn) {
                const float* th = sc[buf][ra];
                const float* dth = th + 3 * P;
                const float t2 = th[P + j2], u2 = dth[P + j2], t3 = th[2 * P + j3], u3 = dth[2 * P + j3];
                float st = 0.f, su = 0.f;   // sum_j1 t1 Q, sum_j1 u1 Q along the column
                if (ok) {
                    const int pk = aoff[a], ox = pk & 1023, oy = (pk >> 10) & 1023, oz = pk >> 20;
                    const float* cp = tile + (oy - j2) * T2 + (oz - j3) + ox * T12;
#pragma unroll
                    for (int j1 = 0; j1 < P; j1++) {
                        const float ph = cp[-j1 * T12];
                        st += th[j1] * ph;
                        su += dth[j1] * ph;
                    }
                } else {
                    const int4 b = dv.baseS[aslot[a]];
                    const float* cp = grid + (size_t) wrapIndex(b.y - j2, K1) * K2 + wrapIndex(b.z - j3, K2);
#pragma unroll
                    for (int j1 = 0; j1 < P; j1++) {
                        const float ph = __ldcg(cp + (size_t) wrapIndex(b.x - j1, K0) * K1 * K2);
                        st += th[j1] * ph;
                        su += dth[j1] * ph;
                    }
                }
                red[ra][col][0] = t2 * t3 * su;
                red[ra][col][1] = u2 * t3 * st;
                red[ra][col][2] = t2 * u3 * st;
            }
            __syncthreads();
            if ((int) threadIdx.x < 3 * APR) {
                const int rb = threadIdx.x / 3, k = threadIdx.x - rb * 3;
                if (r0 + rb < cn) {
                    double F = 0.0;
                    for (int c = 0; c < NCOL; c++)
                        F += (double) red[rb][c][k];
                    aF[r0 + rb][k] = F;
                }
            }
        }
        __syncthreads();
        if ((int) threadIdx.x < cn) {
            const int t = threadIdx.x;
            const int i = dv.slotAtom[aslot[t]];
            const double al = CGA ? dv.alpha[i] : 0.0;
            double v = 0.0;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const double E = -(K0 * S.recip[3 * k] * aF[t][0] + K1 * S.recip[3 * k + 1] * aF[t][1] +
                                   K2 * S.recip[3 * k + 2] * aF[t][2]);
                dv.Erec[3 * i + k] = E;
                if (CGA) {   // A p = p / alpha - (E_pair + E_rec + cs p) (core/pgm_core.cpp:363)
                    const double pk = dv.p[3 * i + k];
                    const double apk = (al > 0) ? pk / al - (dv.Epair[3 * i + k] + E + cs * pk) : 0.0;
                    dv.Ap[3 * i + k] = apk;
                    v += pk * apk;
                }
            }
            if (CGA)
                av[t] = v;
        }
        if (CGA) {
            __syncthreads();
            if (threadIdx.x == 0)
                for (int t = 0; t < cn; t++)
                    pap += av[t];
        }
        __syncthreads();   // (the round's staging read before the next round's)
    }
    if constexpr (CGA) {
        __shared__ int isLast;
        if (threadIdx.x == 0) {
            dv.gpartial[blockIdx.x] = pap;
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

}   // namespace pgmb200
