// Kernels of the pgm_b200 engine.  One evaluation:
//   prep -> cell scan -> cell scatter -> cell sort -> pair list (+ G1, G2) -> permanent dipoles
//   -> E_perm = field(q, p) [spread || pair pass, FFT, convolution, gather]
//   -> initial guess, A x0 -> CG loop (graph while node) -> final pass (energies, forces, field, strain)
// Every per-atom array is in the caller's atom order; the hot loops run over "slots" (atoms sorted by cell).
#pragma once

#include "common.cuh"

#include <cooperative_groups.h>
#include <type_traits>

namespace pgmb200 {

__device__ __forceinline__ int wrapIndex(int g, int K) {
    g += (g < 0) ? K : 0;
    g -= (g >= K) ? K : 0;
    return g;
}

// The mixed spread's 64-bit fixed point: contributions rounded to multiples of 2^-32 and added as integers, so
// the grid's sums do not depend on the order of the atomics (the evaluation repeats bit for bit); the grid is
// converted to float once before the transforms.
constexpr float GRID_FIX_SCALE = 4294967296.0f;   // 2^32
__device__ __forceinline__ void gridFixAdd(long long* g, float v) {
    atomicAdd((unsigned long long*) g, (unsigned long long) __float2ll_rn(v * GRID_FIX_SCALE));
}
__device__ __forceinline__ float gridFixTake(long long* g) {   // the value, and the word cleared for the next spread
    const long long v = *g;
    *g = 0;
    return (float) ((double) v * (1.0 / 4294967296.0));
}

// The fixed-point grid to the float grid (every point), clearing the fixed-point grid.
__global__ void k_grid_from_fix(Dev dv) {
    const size_t n = (size_t) dv.gridTotal, stride = (size_t) gridDim.x * blockDim.x;
    for (size_t k = (size_t) blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride)
        ((float*) dv.grid)[k] = gridFixTake(dv.gridFix + k);
}

// Block-wide compaction of the systems still iterating (scal[DONE] == 0) into actSys / actOff / actCount, in
// system order; every thread of one block calls it (a system's slots are the contiguous run of its cells).
__device__ __forceinline__ void compactActive(const Dev& dv) {
    __shared__ int wtot[32];
    __shared__ int carry;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if (threadIdx.x == 0)
        carry = 0;
    __syncthreads();
    __shared__ int slotCarry;
    if (threadIdx.x == 0)
        slotCarry = 0;
    __syncthreads();
    for (int base = 0; base < dv.nSys; base += blockDim.x) {
        const int s = base + threadIdx.x;
        const bool act = s < dv.nSys && dv.scal[s * NSCAL + SC_DONE] == 0.0;
        const int cnt = act ? dv.sys[s].atomEnd - dv.sys[s].atomBegin : 0;
        // two exclusive scans (systems and slots) in one pass of warp scans
        int a = act ? 1 : 0, c = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int ya = __shfl_up_sync(0xffffffffu, a, o), yc = __shfl_up_sync(0xffffffffu, c, o);
            if (lane >= o) {
                a += ya;
                c += yc;
            }
        }
        __shared__ int wa[32], wc[32];
        if (lane == 31) {
            wa[wid] = a;
            wc[wid] = c;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int ra = 0, rc = 0;
            for (int w = 0; w < nw; w++) {
                const int ta = wa[w], tc = wc[w];
                wa[w] = ra;
                wc[w] = rc;
                ra += ta;
                rc += tc;
            }
            wtot[0] = ra;
            wtot[1] = rc;
        }
        __syncthreads();
        if (act) {
            const int k = carry + wa[wid] + a - 1;
            dv.actSys[k] = s;
            dv.actOff[k] = slotCarry + wc[wid] + c - cnt;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            carry += wtot[0];
            slotCarry += wtot[1];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        dv.actOff[carry] = slotCarry;
        dv.actCount[0] = carry;
    }
}

// The slot of virtual slot v of the compacted active systems, or -1 beyond them.
__device__ __forceinline__ int activeSlot(const Dev& dv, int v) {
    const int na = dv.actCount[0];
    if (na <= 0 || v >= dv.actOff[na])
        return -1;
    int lo = 0, hi = na - 1;   // the last k with actOff[k] <= v
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (dv.actOff[mid] <= v)
            lo = mid;
        else
            hi = mid - 1;
    }
    const SysDev& S = dv.sys[dv.actSys[lo]];
    return dv.cellStart[S.cellOff] + (v - dv.actOff[lo]);
}

// ------------------------------------------------------------------------------------------------ prep

// Per atom, what & 1: the positions copied in from the caller's device array, the PME base index and fraction
// (core/pgm_core.cpp:134-152: t = s - floor(s), w = K t, base = floor(w), fr = w - base); what & 2 (a pair-list
// build, positions already in posIn): wrap into the primary cell, cell index (with a within-cell rank from an
// atomic counter, made deterministic by k_cell_sort) and the positions of the build.
// posMode 0: dv.posIn (double 3n); 1: device float4 posq4 (dv.posDevice); 2: device double 3n (dv.posDevice).
__global__ void k_prep(Dev dv, double* posCopy, int what) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= dv.nAtoms)
        return;
    const SysDev& S = dv.sys[dv.atomSys[i]];
    const int posMode = (what & 1) ? dv.ctl->posMode : 0;
    double r[3];
    if (posMode == 1) {
        const float4 v = ((const float4*) dv.ctl->posDevice)[i];
        r[0] = v.x;
        r[1] = v.y;
        r[2] = v.z;
    } else if (posMode == 2) {
        const double* pd = (const double*) dv.ctl->posDevice;
        r[0] = pd[3 * i];
        r[1] = pd[3 * i + 1];
        r[2] = pd[3 * i + 2];
    } else {
        r[0] = dv.posIn[3 * i];
        r[1] = dv.posIn[3 * i + 1];
        r[2] = dv.posIn[3 * i + 2];
    }
    if (posMode != 0) {
        posCopy[3 * i] = r[0];
        posCopy[3 * i + 1] = r[1];
        posCopy[3 * i + 2] = r[2];
    }
    int cell[3];
    double pw[3] = {r[0], r[1], r[2]};
    for (int a = 0; a < 3; a++) {
        const double s = __dadd_rn(__dadd_rn(__dmul_rn(r[0], S.recip[a]), __dmul_rn(r[1], S.recip[3 + a])),
                                   __dmul_rn(r[2], S.recip[6 + a]));
        const double fl = floor(s);
        const double t = s - fl;
        if (what & 1) {
            const double w = (double) S.K[a] * t;
            const double base = floor(w);
            dv.pmeBase[3 * i + a] = (int) base;
            dv.pmeFr[3 * i + a] = w - base;
        }
        if (what & 2) {
            dv.wrapN[3 * i + a] = (int) fl;
            int c = (int) floor(t * S.cellN[a]);
            cell[a] = min(max(c, 0), S.cellN[a] - 1);
            for (int k = 0; k < 3; k++)
                pw[k] -= fl * S.H[3 * a + k];
        }
    }
    if (what & 2) {
        const int lin = S.cellOff + (cell[0] * S.cellN[1] + cell[1]) * S.cellN[2] + cell[2];
        dv.cellOf[i] = lin;
        dv.cellRank[i] = atomicAdd(&dv.cellCount[lin], 1);
        // wrapped position kept per atom until the slot copy
        dv.Etot[3 * i] = pw[0];
        dv.Etot[3 * i + 1] = pw[1];
        dv.Etot[3 * i + 2] = pw[2];
        if (dv.posBuild)
            for (int a = 0; a < 3; a++)
                dv.posBuild[3 * i + a] = r[a];
        if (i == 0)
            dv.flags[8] = 1;   // a build
    }
}

// Stale test of the Verlet list (core/cuda/pgm_cuda.cu:1914-1928 decides the same on the host): an atom that has
// moved by more than half the skin since the build, or the host's request (no list yet, another box, skin 0),
// makes flags[6] = 1; the last block then sets the build's conditional node.  Also clears the cell counters for
// a build.
__global__ void k_displace(Dev dv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    bool stale = false;
    if (i < dv.nAtoms) {
        const SysDev& S = dv.sys[dv.atomSys[i]];
        double d2 = 0.0;
        for (int a = 0; a < 3; a++) {
            const double dx = dv.posIn[3 * i + a] - dv.posBuild[3 * i + a];
            d2 += dx * dx;
        }
        stale = !(d2 <= S.skinHalf2);
    }
    for (int c = i; c < dv.totalCells; c += gridDim.x * blockDim.x)
        dv.cellCount[c] = 0;
    if (__syncthreads_or(stale) && threadIdx.x == 0)
        atomicOr(&dv.flags[6], 1);
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&dv.flags[7], 1) == (int) gridDim.x - 1) {
            const int st = (atomicOr(&dv.flags[6], 0) != 0 || dv.ctl->forceRebuild != 0) ? 1 : 0;
            dv.flags[6] = st;
            dv.flags[7] = 0;
            if (dv.useCond)
                cudaGraphSetConditional(dv.listCond, st ? 1u : 0u);
        }
    }
}

// New positions on an existing pair list (finite-difference probes of the adjoint): PME base and fraction of
// the new positions, wrapped positions with the wraps of the list's build (so the list's image shifts still
// apply), slot-order copies refreshed in place.  The pair set is the build's.
__global__ void k_refresh_positions(Dev dv) {
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= dv.nAtoms)
        return;
    const int i = dv.slotAtom[slot];
    const SysDev& S = dv.sys[dv.atomSys[i]];
    const double r[3] = {dv.posIn[3 * i], dv.posIn[3 * i + 1], dv.posIn[3 * i + 2]};
    double pw[3] = {r[0], r[1], r[2]};
    for (int a = 0; a < 3; a++) {
        const double s = __dadd_rn(__dadd_rn(__dmul_rn(r[0], S.recip[a]), __dmul_rn(r[1], S.recip[3 + a])),
                                   __dmul_rn(r[2], S.recip[6 + a]));
        const double t = s - floor(s);
        const double w = (double) S.K[a] * t;
        const double base = floor(w);
        dv.pmeBase[3 * i + a] = (int) base;
        dv.pmeFr[3 * i + a] = w - base;
        const double n = (double) dv.wrapN[3 * i + a];
        for (int k = 0; k < 3; k++)
            pw[k] -= n * S.H[3 * a + k];
    }
    dv.posS[slot] = make_double4(pw[0], pw[1], pw[2], dv.q[i]);
    dv.origS[slot] = make_double4(r[0], r[1], r[2], dv.radius[i]);
}

// Exclusive scan of the cell counts (one block; totalCells + 1 entries written).
__global__ void k_cell_scan(Dev dv) {
    __shared__ int warpSums[32];
    const int nT = blockDim.x, t = threadIdx.x;
    const int n = dv.totalCells;
    const int per = (n + nT - 1) / nT;
    const int b = t * per, e = min(n, b + per);
    int sum = 0;
    for (int k = b; k < e; k++)
        sum += dv.cellCount[k];
    // inclusive warp scan
    int v = sum;
    const int lane = t & 31, w = t >> 5;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o)
            v += y;
    }
    if (lane == 31)
        warpSums[w] = v;
    __syncthreads();
    if (w == 0) {
        int ws = (lane < (nT >> 5)) ? warpSums[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, ws, o);
            if (lane >= o)
                ws += y;
        }
        warpSums[lane] = ws;
    }
    __syncthreads();
    int run = v - sum + (w > 0 ? warpSums[w - 1] : 0);
    for (int k = b; k < e; k++) {
        dv.cellStart[k] = run;
        run += dv.cellCount[k];
    }
    if (t == nT - 1)
        dv.cellStart[n] = run;
}

__global__ void k_cell_scatter(Dev dv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= dv.nAtoms)
        return;
    dv.slotTmp[dv.cellStart[dv.cellOf[i]] + dv.cellRank[i]] = i;
}

// One warp per cell: each atom's place is its rank by atom index among the cell's atoms (deterministic slot
// order whatever order the atomics gave); fills the slot-order copies.
__global__ void k_cell_sort(Dev dv) {
    const int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (c >= dv.totalCells)
        return;
    const int b = dv.cellStart[c], e = dv.cellStart[c + 1], m = e - b;
    for (int base = 0; base < m; base += 32) {
        const int k = base + lane;
        if (k < m) {
            const int v = dv.slotTmp[b + k];
            int rank = 0;
            for (int o = 0; o < m; o++)
                rank += dv.slotTmp[b + o] < v;
            const int sl = b + rank;
            dv.slotAtom[sl] = v;
            dv.posS[sl] = make_double4(dv.Etot[3 * v], dv.Etot[3 * v + 1], dv.Etot[3 * v + 2], dv.q[v]);
            dv.origS[sl] = make_double4(dv.posIn[3 * v], dv.posIn[3 * v + 1], dv.posIn[3 * v + 2], dv.radius[v]);
            dv.wrapS[sl] = make_int4(dv.wrapN[3 * v], dv.wrapN[3 * v + 1], dv.wrapN[3 * v + 2], 0);
            dv.radS[sl] = dv.radius[v];
            if (dv.atomSlot)
                dv.atomSlot[v] = sl;
        }
    }
}

// ------------------------------------------------------------------------------------------------ pair list

// Minimum image of v as minImageExact, with the divisions replaced by products with the inverse box diagonal
// unless the quotient lies within 1e-9 of a half-integer (then the exact division decides): the same image
// counts, hence the same vector, bit for bit.
__device__ __forceinline__ void minImageFast(double* v, const double* H, const double* invDiag, int* k) {
#pragma unroll
    for (int c = 2; c >= 0; c--) {
        const double qd = v[c] * invDiag[c];
        const double fr = fabs(qd - trunc(qd));
        const double kk = (fabs(fr - 0.5) < 1e-9) ? round(__ddiv_rn(v[c], H[4 * c])) : round(qd);
        k[c] = (int) kk;
#pragma unroll
        for (int j = 0; j < 3; j++)
            v[j] = __dsub_rn(v[j], __dmul_rn(kk, H[3 * c + j]));
    }
}

constexpr int LIST_THREADS = 256;
constexpr int LIST_CHUNK = 1024;  // candidates staged in shared memory at a time
constexpr int MAX_RUNS = 343;     // (2m+1)^3 with m <= 3

// System of a global cell index (binary search over the systems' first cells).
__device__ __forceinline__ int systemOfCell(const Dev& dv, int c) {
    int lo = 0, hi = dv.nSys - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (dv.sys[mid].cellOff <= c)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// One block per cell.  The neighbour cells (offsets -m..m per dimension) become at most (2m+1)^3 runs of
// consecutive slots with one image shift each (cells along the last dimension merged); their atoms are
// staged through shared memory in chunks (the image's wrapped position relative to the cell's first atom, in
// float, and the pair entry) and every warp tests them against the cell's atoms it owns, 32 candidates at a
// time:
//   - float prefilter: outside (1 + 1e-5) rl^2 is out, inside (1 - 1e-5) rl^2 with every component inside half a
//     box edge is in (the float differences of positions within a few nm of the cell err by < 1e-6 nm^2, and
//     a pair clearly inside the radius with its cell image inside half a box edge provably gets the same image
//     and side from the reference's rounding);
//   - the rest (a thin shell, or near half a box edge) takes the reference's exact test: minimum image of the
//     original positions, r^2 < rl^2 in double without contraction (core/pgm_core.cpp:64-87), keeping the
//     candidate only at the image that test chose, so every pair enters once.
// Accepted pairs are appended to the Verlet list (radius rl = cutoff + skin) in candidate order
// (deterministic); k_pair_compact then takes the ones within the cutoff at every evaluation.
__global__ void __launch_bounds__(LIST_THREADS, 4) k_build_list(Dev dv) {
    __shared__ int runSlot[MAX_RUNS], runOff[MAX_RUNS + 1], runShift[MAX_RUNS];
    __shared__ float4 cPos[LIST_CHUNK];
    __shared__ uint32_t cEntry[LIST_CHUNK];
    const int c = blockIdx.x, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    constexpr int NW = LIST_THREADS / 32;
    if (c >= dv.totalCells)
        return;
    const int cb = dv.cellStart[c], ce = dv.cellStart[c + 1];
    if (cb == ce)
        return;
    const int s = systemOfCell(dv, c);
    const SysDev& S = dv.sys[s];
    const int lc = c - S.cellOff;
    const int n0 = S.cellN[0], n1 = S.cellN[1], n2 = S.cellN[2];
    const int c2 = lc % n2, c1 = (lc / n2) % n1, c0 = lc / (n2 * n1);
    const int m0 = S.cellM[0], m1 = S.cellM[1], m2 = S.cellM[2];
    const int rows = (2 * m0 + 1) * (2 * m1 + 1), per = 2 * m2 + 1;
    for (int row = tid; row < rows; row += LIST_THREADS) {
        const int d0 = row / (2 * m1 + 1) - m0, d1 = row % (2 * m1 + 1) - m1;
        const int u0 = c0 + d0, u1 = c1 + d1;
        const int w0 = (int) floor((double) u0 / n0), v0 = u0 - w0 * n0;
        const int w1 = (int) floor((double) u1 / n1), v1 = u1 - w1 * n1;
        int r = 0, d2 = -m2;
        while (d2 <= m2) {
            const int u2 = c2 + d2;
            const int w2 = (int) floor((double) u2 / n2), v2 = u2 - w2 * n2;
            int len = 1;
            while (d2 + len <= m2 && v2 + len < n2)
                len++;
            const int cc = S.cellOff + (v0 * n1 + v1) * n2 + v2;
            runSlot[row * per + r] = dv.cellStart[cc];
            runOff[row * per + r] = dv.cellStart[cc + len] - dv.cellStart[cc];   // length, scanned below
            runShift[row * per + r] = (w0 + 4) | ((w1 + 4) << 3) | ((w2 + 4) << 6);
            r++;
            d2 += len;
        }
        for (; r < per; r++) {
            runSlot[row * per + r] = 0;
            runOff[row * per + r] = 0;
            runShift[row * per + r] = 4 | (4 << 3) | (4 << 6);
        }
    }
    const int nr = rows * per;
    __syncthreads();
    if (wid == 0) {   // exclusive scan of the run lengths
        int carry = 0;
        for (int base = 0; base < nr; base += 32) {
            const int k = base + lane;
            const int len = (k < nr) ? runOff[k] : 0;
            int v = len;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, v, o);
                if (lane >= o)
                    v += y;
            }
            if (k < nr)
                runOff[k] = carry + v - len;
            carry += __shfl_sync(0xffffffffu, v, 31);
        }
        if (lane == 0)
            runOff[nr] = carry;
    }
    for (int ii = cb + tid; ii < ce; ii += LIST_THREADS)
        dv.slistCount[ii] = 0;
    __syncthreads();
    const int total = runOff[nr];
    const double4 org = dv.posS[cb];   // the block's origin for the float positions
    const float preF = (float) (S.rl2 * (1.0 + 1e-5)), preLoF = (float) (S.rl2 * (1.0 - 1e-5));
    const float hf0 = (float) (0.5 * S.H[0] * (1.0 - 1e-5)), hf1 = (float) (0.5 * S.H[4] * (1.0 - 1e-5)),
                hf2 = (float) (0.5 * S.H[8] * (1.0 - 1e-5));
    const double invDiag[3] = {1.0 / S.H[0], 1.0 / S.H[4], 1.0 / S.H[8]};
    for (int base = 0; base < total; base += LIST_CHUNK) {
        const int nc = min(LIST_CHUNK, total - base);
        for (int t = tid; t < nc; t += LIST_THREADS) {
            const int k = base + t;
            int lo = 0, hi = nr - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (runOff[mid] <= k)
                    lo = mid;
                else
                    hi = mid - 1;
            }
            const int js = runSlot[lo] + (k - runOff[lo]);
            const int code = runShift[lo];
            const int w0 = (code & 7) - 4, w1 = ((code >> 3) & 7) - 4, w2 = ((code >> 6) & 7) - 4;
            // the candidate's image (wrapped position + w.H) relative to the origin, staged once for the cell
            const double4 pw = dv.posS[js];
            cPos[t] = make_float4((float) (pw.x + (w0 * S.H[0] + w1 * S.H[3] + w2 * S.H[6]) - org.x),
                                  (float) (pw.y + (w1 * S.H[4] + w2 * S.H[7]) - org.y),
                                  (float) (pw.z + w2 * S.H[8] - org.z), 0.0f);
            cEntry[t] = (uint32_t) (js | (code << 23));
        }
        __syncthreads();
        for (int ii = cb + wid; ii < ce; ii += NW) {
            const double4 pwi = dv.posS[ii];
            const float xi = (float) (pwi.x - org.x), yi = (float) (pwi.y - org.y), zi = (float) (pwi.z - org.z);
            uint32_t* row = dv.slist + (size_t) ii * dv.cap;
            int count = dv.slistCount[ii];
            for (int t0 = 0; t0 < nc; t0 += 32) {
                const int t = t0 + lane;
                bool acc = false, unsure = false;
                uint32_t entry = 0;
                if (t < nc) {
                    const float4 pj = cPos[t];
                    entry = cEntry[t];
                    const float y0 = xi - pj.x, y1 = yi - pj.y, y2 = zi - pj.z;
                    const float r2 = y0 * y0 + y1 * y1 + y2 * y2;
                    if ((int) (entry & 0x7FFFFFu) != ii && r2 < preF) {
                        if (r2 < preLoF && fabsf(y0) < hf0 && fabsf(y1) < hf1 && fabsf(y2) < hf2)
                            acc = true;
                        else
                            unsure = true;
                    }
                }
                if (__any_sync(0xffffffffu, unsure) && unsure) {
                    // the reference's exact test on the original positions; kept only at the image it chooses
                    const int js = (int) (entry & 0x7FFFFFu);
                    const int w0 = (int) ((entry >> 23) & 7u) - 4, w1 = (int) ((entry >> 26) & 7u) - 4,
                              w2 = (int) ((entry >> 29) & 7u) - 4;
                    const double4 oi = dv.origS[ii], oj = dv.origS[js];
                    const int4 wi = dv.wrapS[ii], cw = dv.wrapS[js];
                    double x[3] = {__dsub_rn(oi.x, oj.x), __dsub_rn(oi.y, oj.y), __dsub_rn(oi.z, oj.z)};
                    int kk[3];
                    minImageFast(x, S.H, invDiag, kk);
                    if (dot3exact(x) < S.rl2)
                        acc = (kk[0] - (wi.x - cw.x) == w0 && kk[1] - (wi.y - cw.y) == w1 &&
                               kk[2] - (wi.z - cw.z) == w2);
                }
                const unsigned ma = __ballot_sync(0xffffffffu, acc);
                if (acc) {
                    const int pos = count + __popc(ma & ((1u << lane) - 1u));
                    if (pos < dv.cap)
                        row[pos] = entry;
                }
                count += __popc(ma);
            }
            if (lane == 0)
                dv.slistCount[ii] = count;
        }
        __syncthreads();
    }
    for (int ii = cb + tid; ii < ce; ii += LIST_THREADS) {
        const int cnt = dv.slistCount[ii];
        if (cnt > dv.cap) {
            atomicMax(&dv.flags[0], cnt);
            dv.slistCount[ii] = dv.cap;
        }
    }
}

// The Verlet list from the caller's candidates (setCandidates, core/cuda/pgm_cuda.h:68-73) in place of the cell
// search: one warp per slot, the row of atom i = slotAtom[slot] in the caller's order, the entry of candidate
// (j, t) with the image shift w = N_j - N_i - t of the build's wraps N (r = pw + N.H), so that
// x = pw_i - pw_j - w.H = r_i + t.H - r_j.  A shift outside the entry's range (-4..3 per component) sets
// flags[1]; a row beyond the capacity sets flags[0] (the host grows the rows and repeats).  The evaluations'
// compaction then keeps the candidates within the cutoff.
__global__ void k_list_from_candidates(Dev dv) {
    const int slot = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (slot >= dv.nAtoms)
        return;
    const int i = dv.slotAtom[slot];
    const int4 ni = dv.wrapS[slot];
    const int b = dv.candStart[i], cnt = dv.candStart[i + 1] - b;
    uint32_t* row = dv.slist + (size_t) slot * dv.cap;
    for (int k = lane; k < cnt && k < dv.cap; k += 32) {
        const int j = dv.candJ[b + k], tp = dv.candT[b + k];
        const int js = dv.atomSlot[j];
        const int4 nj = dv.wrapS[js];
        const int w0 = nj.x - ni.x - ((tp & 255) - 128), w1 = nj.y - ni.y - (((tp >> 8) & 255) - 128),
                  w2 = nj.z - ni.z - (((tp >> 16) & 255) - 128);
        if (w0 < -4 || w0 > 3 || w1 < -4 || w1 > 3 || w2 < -4 || w2 > 3) {
            atomicOr(&dv.flags[1], 1);
            row[k] = packEntry(slot, 0, 0, 0);   // (never used: the host raises)
        } else {
            row[k] = packEntry(js, w0, w1, w2);
        }
    }
    if (lane == 0) {
        dv.slistCount[slot] = min(cnt, dv.cap);
        if (cnt > dv.cap)
            atomicMax(&dv.flags[0], cnt);
    }
}

// Pair records.  Mixed precision (float): pairA = (x, G1) with x = pw_i - pw_j - w.H rounded to float,
// pairB = (G2, slot of j), so that the field passes stream them and gather only (d_j, q_j).  FP64: pairB =
// (G1, G2), the field passes form x from the slot-order positions (streaming 48-byte double records is slower
// there than the L1-resident position gathers).
template <typename R> struct PairRec { static constexpr bool storeX = false; };
template <> struct PairRec<float> { static constexpr bool storeX = true; };

// The pair records of every listed pair (the list of the evaluation) in precision R with G0..G3 by
// core/pgm_math.h:77-93 via pairKernels, from the current slot-order positions (also after new positions on a
// kept list), one warp per slot, the pairs of its row over the lanes.
// FIELD: also the direct-space field of the charges and dipoles dS (the permanent field pass, core/pgm_core.cpp:
// 274-284: E_i = sum_j (q_j G1 + (d_j . x) G2) x - d_j G1) from the same G1, G2 and x, written to Epair, as
// k_pair_field<R, true> would (per-lane sums in R, across the lanes in double).
template <typename R, bool FIELD = false>
__global__ void __launch_bounds__(256) k_pair_kernels(Dev dv) {
    typedef typename V2T<R>::T R2;
    typedef typename V4T<R>::T R4;
    constexpr bool STORE_X = PairRec<R>::storeX;
    const int slot = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (slot >= dv.nAtoms)
        return;
    const SysDev& S = dv.sys[dv.atomSys[dv.slotAtom[slot]]];
    const double4 pwi = dv.posS[slot];
    const double Ri = dv.radS[slot];
    const uint32_t* row = dv.list + (size_t) slot * dv.cap;
    R4* arow = (R4*) dv.pairA + (size_t) slot * dv.cap;
    R2* brow = (R2*) dv.pairB + (size_t) slot * dv.cap;
    R2* crow = dv.pairC ? (R2*) dv.pairC + (size_t) slot * dv.cap : nullptr;
    const int cnt = dv.listCount[slot];
    const R beta = (R) S.beta;
    R f0 = 0, f1 = 0, f2 = 0;   // (FIELD) the lane's field sums
    const R4* dS = (const R4*) dv.dS;
    for (int t = lane; t < cnt; t += 32) {
        const uint32_t e = row[t];
        const int js = entrySlot(e);
        double sh[3];
        entryShift(e, S.H, sh);
        const double4 pwj = dv.posS[js];
        const double x0 = pwi.x - pwj.x - sh[0], x1 = pwi.y - pwj.y - sh[1], x2 = pwi.z - pwj.z - sh[2];
        const R Rj = (R) dv.radS[js], Rr = (R) Ri;
        const R xr0 = (R) x0, xr1 = (R) x1, xr2 = (R) x2;
        const R r = fsqrt(xr0 * xr0 + xr1 * xr1 + xr2 * xr2);
        const R a = R(1) / fsqrt(R(2) * (Rr * Rr + Rj * Rj));
        R G[4];
        pairKernels<R, 4>(a, beta, r, G);
        if (FIELD) {
            const R4 dj = dS[js];
            const R c = (dj.x * xr0 + dj.y * xr1 + dj.z * xr2) * G[2] + dj.w * G[1];
            f0 += c * xr0 - dj.x * G[1];
            f1 += c * xr1 - dj.y * G[1];
            f2 += c * xr2 - dj.z * G[1];
        }
        R2 vb;
        if constexpr (STORE_X) {
            R4 va;
            va.x = xr0;
            va.y = xr1;
            va.z = xr2;
            va.w = G[1];
            arow[t] = va;
            vb.x = G[2];
            vb.y = slotAsReal(js, R(0));
        } else {
            vb.x = G[1];
            vb.y = G[2];
        }
        brow[t] = vb;
        if (crow) {
            R2 vc;
            vc.x = G[0];
            vc.y = G[3];
            crow[t] = vc;
        }
    }
    if (FIELD) {
        double E0 = f0, E1 = f1, E2 = f2;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            E0 += __shfl_xor_sync(0xffffffffu, E0, o);
            E1 += __shfl_xor_sync(0xffffffffu, E1, o);
            E2 += __shfl_xor_sync(0xffffffffu, E2, o);
        }
        if (lane == 0) {
            const int i = dv.slotAtom[slot];
            dv.Epair[3 * i] = E0;
            dv.Epair[3 * i + 1] = E1;
            dv.Epair[3 * i + 2] = E2;
        }
    }
}

// The pairs of the Verlet list within the cutoff at this evaluation's positions with their records (x rounded to
// R, G0..G3 in precision R by core/pgm_math.h:77-93 via pairKernels, the slot of j): one warp per slot, the
// list's row in candidate order over the lanes, compacted by ballot into the row of the evaluation's list
// (same order, deterministic), then the radial kernels over the kept pairs.  The test is
// the list build's at the cutoff: a prefilter on the wrapped positions, the reference's exact test
// (core/pgm_core.cpp:64-87) only near the cutoff or near half a box edge.  A pair within the cutoff whose exact
// image is not the one stored at the build sets flags[9]: the list is rebuilt and the evaluation repeated.
template <typename R>
__global__ void __launch_bounds__(256, 3) k_pair_compact(Dev dv) {
    typedef typename V2T<R>::T R2;
    typedef typename V4T<R>::T R4;
    constexpr bool STORE_X = PairRec<R>::storeX;
    const int slot = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (slot >= dv.nAtoms)
        return;
    const SysDev& S = dv.sys[dv.atomSys[dv.slotAtom[slot]]];
    const double4 pwi = dv.posS[slot];
    const double Ri = dv.radS[slot];
    const uint32_t* srow = dv.slist + (size_t) slot * dv.cap;
    uint32_t* row = dv.list + (size_t) slot * dv.cap;
    R4* arow = (R4*) dv.pairA + (size_t) slot * dv.cap;
    R2* brow = (R2*) dv.pairB + (size_t) slot * dv.cap;
    R2* crow = (R2*) dv.pairC + (size_t) slot * dv.cap;
    const int cnt = dv.slistCount[slot];
    const R beta = (R) S.beta;
    const double pre = S.rc2 * (1.0 + 1e-10) + 1e-300, preLo = S.rc2 * (1.0 - 1e-10);
    const double half0 = 0.5 * S.H[0] * (1.0 - 1e-10), half1 = 0.5 * S.H[4] * (1.0 - 1e-10),
                 half2 = 0.5 * S.H[8] * (1.0 - 1e-10);
    // test of list entry t (t < cnt): pair geometry x and whether the pair is within the cutoff
    auto test = [&](int t, uint32_t e, double4 pwj, double* x) -> bool {
        double sh[3];
        entryShift(e, S.H, sh);
        x[0] = pwi.x - pwj.x - sh[0];
        x[1] = pwi.y - pwj.y - sh[1];
        x[2] = pwi.z - pwj.z - sh[2];
        const double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
        if (!(r2 < pre))
            return false;
        if (r2 < preLo && fabs(x[0]) < half0 && fabs(x[1]) < half1 && fabs(x[2]) < half2)
            return true;
        const int js = entrySlot(e);
        const double4 oi = dv.origS[slot], oj = dv.origS[js];
        const int4 wi = dv.wrapS[slot], wj = dv.wrapS[js];
        const double invDiag[3] = {1.0 / S.H[0], 1.0 / S.H[4], 1.0 / S.H[8]};
        double xe[3] = {__dsub_rn(oi.x, oj.x), __dsub_rn(oi.y, oj.y), __dsub_rn(oi.z, oj.z)};
        int kk[3];
        minImageFast(xe, S.H, invDiag, kk);
        if (!(dot3exact(xe) < S.rc2))
            return false;
        const int w0 = (int) ((e >> 23) & 7u) - 4, w1 = (int) ((e >> 26) & 7u) - 4, w2 = (int) ((e >> 29) & 7u) - 4;
        const bool same = kk[0] - (wi.x - wj.x) == w0 && kk[1] - (wi.y - wj.y) == w1 && kk[2] - (wi.z - wj.z) == w2;
        if (!same)
            atomicOr(&dv.flags[9], 1);
        return same;
    };
    // append the accepted lanes of a 32-entry chunk in lane (candidate) order
    int count = 0;
    auto append = [&](bool acc, uint32_t e, const double* x) {
        const unsigned ma = __ballot_sync(0xffffffffu, acc);
        if (acc) {
            const int pos = count + __popc(ma & ((1u << lane) - 1u));
            row[pos] = e;
            if constexpr (STORE_X) {
                R4 va;
                va.x = (R) x[0];
                va.y = (R) x[1];
                va.z = (R) x[2];
                va.w = (R) 0;
                arow[pos] = va;
            }
        }
        count += __popc(ma);
    };
    // two chunks per step: both chunks' entries and partner positions are loaded before either is tested
    for (int t0 = 0; t0 < cnt; t0 += 64) {
        const int ta = t0 + lane, tb = t0 + 32 + lane;
        const uint32_t ea = ta < cnt ? srow[ta] : 0u, eb = tb < cnt ? srow[tb] : 0u;
        const double4 pa = dv.posS[ta < cnt ? entrySlot(ea) : slot];
        const double4 pb = dv.posS[tb < cnt ? entrySlot(eb) : slot];
        double xa[3] = {0, 0, 0}, xb[3] = {0, 0, 0};
        const bool acca = ta < cnt && test(ta, ea, pa, xa);
        const bool accb = tb < cnt && test(tb, eb, pb, xb);
        append(acca, ea, xa);
        if (t0 + 32 < cnt)
            append(accb, eb, xb);
    }
    if (lane == 0)
        dv.listCount[slot] = count;
    __syncwarp();
    // G1, G2 of the kept pairs, every lane busy (the radial kernels branch per pair)
    const R Rr = (R) Ri;
    for (int t = lane; t < count; t += 32) {
        const uint32_t e = row[t];
        const int js = entrySlot(e);
        R xr0, xr1, xr2;
        R4 va;
        if constexpr (STORE_X) {
            va = arow[t];
            xr0 = va.x;
            xr1 = va.y;
            xr2 = va.z;
        } else {
            double sh[3];
            entryShift(e, S.H, sh);
            const double4 pwj = dv.posS[js];
            xr0 = (R) (pwi.x - pwj.x - sh[0]);
            xr1 = (R) (pwi.y - pwj.y - sh[1]);
            xr2 = (R) (pwi.z - pwj.z - sh[2]);
        }
        const R Rj = (R) dv.radS[js];
        const R r = fsqrt(xr0 * xr0 + xr1 * xr1 + xr2 * xr2);
        const R a = R(1) / fsqrt(R(2) * (Rr * Rr + Rj * Rj));
        R G[4];
        pairKernels<R, 4>(a, beta, r, G);
        R2 vb;
        if constexpr (STORE_X) {
            va.w = G[1];
            arow[t] = va;
            vb.x = G[2];
            vb.y = slotAsReal(js, R(0));
        } else {
            vb.x = G[1];
            vb.y = G[2];
        }
        brow[t] = vb;
        R2 vc;
        vc.x = G[0];
        vc.y = G[3];
        crow[t] = vc;
    }
}

// ------------------------------------------------------------------------------------------------ dipoles

// Permanent dipoles p_i = sum_m c_m unit(minimage(r_partner - r_atom)) over the dipoles of atom i
// (core/pgm_core.cpp:51-62).
__global__ void k_perm(Dev dv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= dv.nAtoms)
        return;
    const SysDev& S = dv.sys[dv.atomSys[i]];
    double p[3] = {0, 0, 0};
    for (int k = dv.covByAtomOff[i]; k < dv.covByAtomOff[i + 1]; k++) {
        const int m = dv.covByAtom[k];
        const int j = dv.covPartner[m];
        double v[3] = {dv.posIn[3 * j] - dv.posIn[3 * i], dv.posIn[3 * j + 1] - dv.posIn[3 * i + 1],
                       dv.posIn[3 * j + 2] - dv.posIn[3 * i + 2]};
        int kk[3];
        minImageExact(v, S.H, kk);
        const double L = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        for (int a = 0; a < 3; a++)
            p[a] += dv.covStrength[m] * v[a] / L;
    }
    for (int a = 0; a < 3; a++)
        dv.perm[3 * i + a] = p[a];
}

// ------------------------------------------------------------------------------------------------ PME

// Influence function G(m) = exp(-pi^2 m^2/beta^2)/(pi V m^2)/(b1 b2 b3), G(0) = 0 (core/pgm_core.cpp:155-177),
// one value per half-spectrum element, stored in precision R.
template <typename R>
__global__ void k_influence(Dev dv) {
    const int s = blockIdx.y;
    const SysDev& S = dv.sys[s];
    const int K0 = S.K[0], K1 = S.K[1], K2h = S.K[2] / 2 + 1;
    R* infl = (R*) dv.infl + S.specOff;
    const double fac = PI_D * PI_D / (S.beta * S.beta);
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < S.specN; e += gridDim.x * blockDim.x) {
        const int m3 = e % K2h, m2 = (e / K2h) % K1, m1 = e / (K2h * K1);
        const double mm1 = (m1 <= K0 / 2) ? m1 : m1 - K0, mm2 = (m2 <= K1 / 2) ? m2 : m2 - K1, mm3 = m3;
        double g = 0.0;
        if (e != 0) {
            double ms[3];
            for (int k = 0; k < 3; k++)
                ms[k] = mm1 * S.recip[3 * k] + mm2 * S.recip[3 * k + 1] + mm3 * S.recip[3 * k + 2];
            const double m2s = ms[0] * ms[0] + ms[1] * ms[1] + ms[2] * ms[2];
            g = exp(-fac * m2s) / (PI_D * S.volume * m2s) /
                (dv.moduli[S.modOff[0] + m1] * dv.moduli[S.modOff[1] + m2] * dv.moduli[S.modOff[2] + m3]);
        }
        infl[e] = (R) g;
    }
}

// B-spline coefficients of every atom, once per evaluation (positions are fixed during it): slot-ordered
// spl[(slot * 9 + kind * 3 + dim) * MAXP + j], kind 0 theta, 1 dtheta, 2 d2theta (core/pgm_core.cpp:131-150),
// and the base grid index per dimension.  One thread per (slot, dimension).
template <typename R>
__global__ void k_splines(Dev dv) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * dv.nAtoms)
        return;
    const int slot = t / 3, dim = t % 3;
    const int i = dv.slotAtom[slot];
    R th[MAXP], dth[MAXP], d2[MAXP];
    bspline<R>((R) dv.pmeFr[3 * i + dim], dv.order, th, dth, d2);
    R* out = (R*) dv.spl + (size_t) slot * 9 * MAXP;
#pragma unroll
    for (int j = 0; j < MAXP; j++)
        if (j < dv.order) {
            out[(0 * 3 + dim) * MAXP + j] = th[j];
            out[(1 * 3 + dim) * MAXP + j] = dth[j];
            out[(2 * 3 + dim) * MAXP + j] = d2[j];
        }
    ((int*) dv.baseS)[4 * slot + dim] = dv.pmeBase[3 * i + dim];
}

// Spread of charges and dipoles onto the grid: Q[g] += q t1 t2 t3 + e1 u1 t2 t3 + e2 t1 u2 t3 + e3 t1 t2 u3,
// e_a = K_a d . recip[:, a] (core/pgm_core.cpp:187-207).  One warp per slot, p^3 points over the lanes.
// P: the spline order as a compile-time constant (0: the runtime order).
// mode 0: q and vec; 1: vec only; 2: CG direction update p = z + beta p first (vec = p), no charges.
// Also writes the slot-order copy dS = (d, q) in precision R for the pair passes.
template <typename R, int P>
__global__ void __launch_bounds__(256) k_spread(Dev dv, int mode, double* vec) {
    typedef typename V4T<R>::T R4;
    constexpr int PM = P > 0 ? P : MAXP;
    __shared__ R sth[8][3][PM], sdth[8][3][PM];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int slot = blockIdx.x * 8 + wib;
    if (mode == 2 && dv.useActive)   // the CG direction of a batch: the active systems' slots only
        slot = activeSlot(dv, slot);
    if (slot < 0 || slot >= dv.nAtoms)
        return;
    const int i = dv.slotAtom[slot];
    const int s = dv.atomSys[i];
    if (mode == 2 && dv.scal[s * NSCAL + SC_DONE] != 0.0)
        return;
    const SysDev& S = dv.sys[s];
    const int p = P > 0 ? P : dv.order;
    double dl = 0.0;
    int bl = 0;
    if (lane < 3) {
        if (mode == 2) {
            dl = dv.z[3 * i + lane] + dv.scal[s * NSCAL + SC_BETA] * vec[3 * i + lane];
            vec[3 * i + lane] = dl;
        } else {
            dl = vec[3 * i + lane];
        }
        if (P == 0) {
            R t[MAXP], u[MAXP], v[MAXP];
            bspline<R>((R) dv.pmeFr[3 * i + lane], p, t, u, v);
#pragma unroll
            for (int j = 0; j < PM; j++)
                if (j < p) {
                    sth[wib][lane][j] = t[j];
                    sdth[wib][lane][j] = u[j];
                }
        }
        bl = dv.pmeBase[3 * i + lane];
    }
    if (P > 0) {   // the evaluation's precomputed coefficients (k_splines)
        const R* sp = (const R*) dv.spl + (size_t) slot * 9 * MAXP;
        for (int k = lane; k < 6 * PM; k += 32) {
            const int kind = k / (3 * PM), dim = (k / PM) % 3, j = k % PM;
            const R v = sp[(kind * 3 + dim) * MAXP + j];
            if (kind == 0)
                sth[wib][dim][j] = v;
            else
                sdth[wib][dim][j] = v;
        }
    }
    const double d0 = __shfl_sync(0xffffffffu, dl, 0), d1 = __shfl_sync(0xffffffffu, dl, 1),
                 d2 = __shfl_sync(0xffffffffu, dl, 2);
    const int b0 = __shfl_sync(0xffffffffu, bl, 0), b1 = __shfl_sync(0xffffffffu, bl, 1),
              b2 = __shfl_sync(0xffffffffu, bl, 2);
    const double qv = (mode == 0) ? dv.q[i] : 0.0;
    if (lane == 0) {
        R4 o;
        o.x = (R) d0;
        o.y = (R) d1;
        o.z = (R) d2;
        o.w = (R) qv;
        ((R4*) dv.dS)[slot] = o;
    }
    __syncwarp();
    const R e0 = (R) (S.K[0] * (d0 * S.recip[0] + d1 * S.recip[3] + d2 * S.recip[6]));
    const R e1 = (R) (S.K[1] * (d0 * S.recip[1] + d1 * S.recip[4] + d2 * S.recip[7]));
    const R e2 = (R) (S.K[2] * (d0 * S.recip[2] + d1 * S.recip[5] + d2 * S.recip[8]));
    const R qr = (R) qv;
    R* grid = (R*) dv.grid + S.gridOff;
    long long* gfix = std::is_same<R, float>::value && dv.gridFix ? dv.gridFix + S.gridOff : nullptr;
    const int K0 = S.K[0], K1 = S.K[1], K2 = S.K[2];
    if (P > 0) {
        // lane -> (j2, j3), loop over j1: consecutive lanes hit consecutive grid points of one row, and
        // w = t1 (q t2 t3 + e1 u2 t3 + e2 t2 u3) + u1 (e0 t2 t3) costs two products per point
        // full rounds: lane -> column (j2, j3), loop over j1; the columns left over (P^2 mod 32) then have their
        // points spread over the lanes (p = 6: 6 + 1 iterations instead of 2 x 6 with 4 lanes busy in the second)
        constexpr int PP = P > 0 ? P : 1;
        constexpr int NPAIR = PP * PP, FULL = NPAIR / 32, LEFT = NPAIR % 32, LROUNDS = (LEFT * PP + 31) / 32;
        constexpr int LEFTD = LEFT > 0 ? LEFT : 1;   // (a divisor for the leftover rounds, which run only when LEFT > 0)
        const size_t plane = (size_t) K1 * K2;
#pragma unroll
        for (int rd = 0; rd < FULL; rd++) {
            const int pr = lane + 32 * rd;
            const int j2 = pr / PP, j3 = pr % PP;
            const R t2 = sth[wib][1][j2], u2 = sdth[wib][1][j2];
            const R t3 = sth[wib][2][j3], u3 = sdth[wib][2][j3];
            const R c23 = t2 * t3;
            const R a = qr * c23 + e1 * u2 * t3 + e2 * t2 * u3;
            const R b = e0 * c23;
            const size_t col = (size_t) wrapIndex(b1 - j2, K1) * K2 + wrapIndex(b2 - j3, K2);
            if (gfix) {
#pragma unroll
                for (int j1 = 0; j1 < PP; j1++)
                    gridFixAdd(gfix + col + (size_t) wrapIndex(b0 - j1, K0) * plane,
                               (float) (a * sth[wib][0][j1] + b * sdth[wib][0][j1]));
            } else {
#pragma unroll
                for (int j1 = 0; j1 < PP; j1++)
                    atomicAdd(grid + col + (size_t) wrapIndex(b0 - j1, K0) * plane,
                              a * sth[wib][0][j1] + b * sdth[wib][0][j1]);
            }
        }
#pragma unroll
        for (int lr = 0; lr < LROUNDS; lr++) {
            const int k = lane + 32 * lr;
            if (k < LEFT * PP) {
                const int pr = 32 * FULL + k % LEFTD, j1 = k / LEFTD;
                const int j2 = pr / PP, j3 = pr % PP;
                const R t2 = sth[wib][1][j2], u2 = sdth[wib][1][j2];
                const R t3 = sth[wib][2][j3], u3 = sdth[wib][2][j3];
                const R c23 = t2 * t3;
                const R w = (qr * c23 + e1 * u2 * t3 + e2 * t2 * u3) * sth[wib][0][j1] + e0 * c23 * sdth[wib][0][j1];
                const size_t at = (size_t) wrapIndex(b0 - j1, K0) * plane + (size_t) wrapIndex(b1 - j2, K1) * K2 +
                                  wrapIndex(b2 - j3, K2);
                if (gfix)
                    gridFixAdd(gfix + at, (float) w);
                else
                    atomicAdd(grid + at, w);
            }
        }
    } else {
        const int pp = p * p, p3 = pp * p;
        for (int t = lane; t < p3; t += 32) {
            const int j1 = t / pp, j2 = (t / p) % p, j3 = t % p;
            const R t1 = sth[wib][0][j1], u1 = sdth[wib][0][j1];
            const R t2 = sth[wib][1][j2], u2 = sdth[wib][1][j2];
            const R t3 = sth[wib][2][j3], u3 = sdth[wib][2][j3];
            const R w = t3 * (t2 * (qr * t1 + e0 * u1) + e1 * t1 * u2) + e2 * t1 * t2 * u3;
            const int g1 = wrapIndex(b0 - j1, K0), g2 = wrapIndex(b1 - j2, K1), g3 = wrapIndex(b2 - j3, K2);
            const size_t at = ((size_t) g1 * K1 + g2) * K2 + g3;
            if (gfix)
                gridFixAdd(gfix + at, (float) w);
            else
                atomicAdd(&grid[at], w);
        }
    }
}

// Multiplies the spectrum by the influence function.  ENERGY: also the reciprocal energy
// (1/2) sum w G |F|^2 (w = 1 on the m3 = 0 and Nyquist planes, else 2) and its strain derivative
// e (-delta + 2 (pi^2/beta^2 + 1/m^2) m m) per block (core/pgm_core.cpp:214-235).  gateDone: skip systems whose
// CG has converged.
template <typename R, bool ENERGY>
__global__ void __launch_bounds__(256) k_conv(Dev dv, int gateDone) {
    typedef typename CplxT<R>::T C;
    const int s = blockIdx.y;
    if (gateDone && dv.scal[s * NSCAL + SC_DONE] != 0.0)
        return;
    const SysDev& S = dv.sys[s];
    C* spec = (C*) dv.spec + S.specOff;
    const R* infl = (const R*) dv.infl + S.specOff;
    double acc[NCONV];
#pragma unroll
    for (int k = 0; k < NCONV; k++)
        acc[k] = 0.0;
    const int K0 = S.K[0], K1 = S.K[1], K2 = S.K[2], K2h = K2 / 2 + 1;
    const double fac = PI_D * PI_D / (S.beta * S.beta);
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < S.specN; e += gridDim.x * blockDim.x) {
        C F = spec[e];
        const R g = infl[e];
        if (ENERGY && e != 0) {
            const int m3 = e % K2h, m2 = (e / K2h) % K1, m1 = e / (K2h * K1);
            const double w = (m3 == 0 || ((K2 & 1) == 0 && m3 == K2 / 2)) ? 1.0 : 2.0;
            const double nrm = (double) F.x * F.x + (double) F.y * F.y;
            const double en = 0.5 * w * (double) g * nrm;
            acc[0] += en;
            const double mm1 = (m1 <= K0 / 2) ? m1 : m1 - K0, mm2 = (m2 <= K1 / 2) ? m2 : m2 - K1, mm3 = m3;
            double ms[3];
            for (int k = 0; k < 3; k++)
                ms[k] = mm1 * S.recip[3 * k] + mm2 * S.recip[3 * k + 1] + mm3 * S.recip[3 * k + 2];
            const double m2s = ms[0] * ms[0] + ms[1] * ms[1] + ms[2] * ms[2];
            const double c2 = 2.0 * (fac + 1.0 / m2s);
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
                for (int b = 0; b < 3; b++)
                    acc[1 + 3 * a + b] += en * ((a == b ? -1.0 : 0.0) + c2 * ms[a] * ms[b]);
        }
        F.x *= g;
        F.y *= g;
        spec[e] = F;
    }
    if (ENERGY) {
        blockReduce<NCONV>(acc, 0u);
        if (threadIdx.x == 0)
            for (int k = 0; k < NCONV; k++)
                dv.convPartial[(size_t) (dv.convPartialOff[s] + blockIdx.x) * NCONV + k] = acc[k];
    }
}

// ------------------------------------------------------------------------------------------------ cluster transforms

// The 3D real transform pair with the influence product of a field pass in ONE kernel: a cluster of C thread
// blocks per system (C = 1 .. 16, the same for every system of a launch) holds the system's half spectrum in
// its distributed shared memory (grids up to FFT_MAXK points per dimension with only the prime factors 2, 3, 5).  Block `rank` of the cluster owns
// x-planes [rank ppc, rank ppc + ppc):
//   1. its planes' real rows, two at a time as one complex row (x + i y), transform along z (real to half
//      spectrum, separated by Hermitian symmetry) and along y in shared memory;
//   2. (cluster barrier) x-lines (ky, kz), numbered kz K1 + ky, are split over the blocks: each gathers its lines
//      from the owners' shared memory, transforms forward along x, multiplies by the influence function,
//      transforms back and scatters the lines to the owners;
//   3. (cluster barrier) its planes transform back along y and z (half spectrum to real; imaginary parts at
//      kz = 0 and the Nyquist index dropped, as a C2R transform does) into the real grid.
// Unnormalised, the spectrum in cuFFT's R2C / C2R layout F[(kx K1 + ky) (K2/2 + 1) + kz].  Each line transform is
// a mixed-radix Stockham FFT (radices 4, 2, 3, 5; ping-pong buffers, no reordering pass) with twiddles
// W^m = exp(-2 pi i m / K) from a table built on the host.
constexpr int FFT_MAXK = 64;
constexpr int FFTC_MAXC = 16;      // the largest cluster (a non-portable cluster size on sm_100)

__host__ __device__ inline int fftRadices(int n, int* r) {
    int c = 0;
    while (n % 4 == 0) { r[c++] = 4; n /= 4; }
    while (n % 2 == 0) { r[c++] = 2; n /= 2; }
    while (n % 3 == 0) { r[c++] = 3; n /= 3; }
    while (n % 5 == 0) { r[c++] = 5; n /= 5; }
    return n == 1 ? c : -1;
}

// In-register DFT of length RAD, sign DIR (-1 forward, +1 inverse), unnormalised.
template <typename R, int RAD, int DIR>
__device__ __forceinline__ void smallDft(R* xr, R* xi) {
    if (RAD == 2) {
        const R ar = xr[0] + xr[1], ai = xi[0] + xi[1];
        xr[1] = xr[0] - xr[1];
        xi[1] = xi[0] - xi[1];
        xr[0] = ar;
        xi[0] = ai;
    } else if (RAD == 3) {
        const R s = (R) (DIR * 0.86602540378443864676);   // DIR sin(2 pi / 3)
        const R tr = xr[1] + xr[2], ti = xi[1] + xi[2];
        const R ur = xr[0] - (R) 0.5 * tr, ui = xi[0] - (R) 0.5 * ti;
        const R dr = s * (xr[1] - xr[2]), di = s * (xi[1] - xi[2]);   // i s (v1 - v2) = (-di, dr)
        xr[0] += tr;
        xi[0] += ti;
        xr[1] = ur - di;
        xi[1] = ui + dr;
        xr[2] = ur + di;
        xi[2] = ui - dr;
    } else if (RAD == 4) {
        const R ar = xr[0] + xr[2], ai = xi[0] + xi[2], br = xr[0] - xr[2], bi = xi[0] - xi[2];
        const R cr = xr[1] + xr[3], ci = xi[1] + xi[3];
        const R er = xr[1] - xr[3], ei = xi[1] - xi[3];
        const R dr = (R) (-DIR) * ei, di = (R) DIR * er;   // (v1 - v3) DIR i
        xr[0] = ar + cr;
        xi[0] = ai + ci;
        xr[2] = ar - cr;
        xi[2] = ai - ci;
        xr[1] = br + dr;
        xi[1] = bi + di;
        xr[3] = br - dr;
        xi[3] = bi - di;
    } else {   // 5
        const R c1 = (R) 0.30901699437494742410, c2 = (R) -0.80901699437494742410;   // cos(2 pi/5), cos(4 pi/5)
        const R s1 = (R) (DIR * 0.95105651629515357212), s2 = (R) (DIR * 0.58778525229247312917);
        const R a1r = xr[1] + xr[4], a1i = xi[1] + xi[4], a2r = xr[2] + xr[3], a2i = xi[2] + xi[3];
        const R b1r = xr[1] - xr[4], b1i = xi[1] - xi[4], b2r = xr[2] - xr[3], b2i = xi[2] - xi[3];
        const R p1r = xr[0] + c1 * a1r + c2 * a2r, p1i = xi[0] + c1 * a1i + c2 * a2i;
        const R p2r = xr[0] + c2 * a1r + c1 * a2r, p2i = xi[0] + c2 * a1i + c1 * a2i;
        const R q1r = s1 * b1r + s2 * b2r, q1i = s1 * b1i + s2 * b2i;   // y1 = p1 + i q1, y4 = p1 - i q1
        const R q2r = s2 * b1r - s1 * b2r, q2i = s2 * b1i - s1 * b2i;   // y2 = p2 + i q2, y3 = p2 - i q2
        xr[0] += a1r + a2r;
        xi[0] += a1i + a2i;
        xr[1] = p1r - q1i;
        xi[1] = p1i + q1r;
        xr[4] = p1r + q1i;
        xi[4] = p1i - q1r;
        xr[2] = p2r - q2i;
        xi[2] = p2i + q2r;
        xr[3] = p2r + q2i;
        xi[3] = p2i - q2r;
    }
}

// e / K for 0 <= e < 2^20, K >= 1 without an integer division: (e + 1/2) / K lies at least 1/(2K) from an
// integer and the float product errs by at most about 2^-23 (e + 1/2) / K < 1/(8K), so truncation gives the
// exact quotient.
__device__ __forceinline__ int fdiv(int e, float invK) { return __float2int_rz(((float) e + 0.5f) * invK); }

// Butterfly j of a Stockham pass of radix RAD (src = in + line start + j, dst = out + line start + (j / Ns) Ns RAD
// + j mod Ns): reads src[r nb], twiddles by W^(r tws) (tws = (j mod Ns) N / (Ns RAD)), writes dst[r Ns].
template <typename R, int RAD, int DIR>
__device__ __forceinline__ void stockhamButterfly(const typename CplxT<R>::T* src, typename CplxT<R>::T* dst, int nb,
                                                  int Ns, int tws, const typename CplxT<R>::T* tw) {
    typedef typename CplxT<R>::T C;
    R xr[RAD], xi[RAD];
    C v[RAD];
#pragma unroll
    for (int r = 0; r < RAD; r++)
        v[r] = src[r * nb];
    xr[0] = v[0].x;
    xi[0] = v[0].y;
#pragma unroll
    for (int r = 1; r < RAD; r++) {
        const C w = tw[tws * r];
        const R wy = DIR < 0 ? w.y : -w.y;
        xr[r] = v[r].x * w.x - v[r].y * wy;
        xi[r] = v[r].x * wy + v[r].y * w.x;
    }
    smallDft<R, RAD, DIR>(xr, xi);
#pragma unroll
    for (int r = 0; r < RAD; r++) {
        C o;
        o.x = xr[r];
        o.y = xi[r];
        dst[r * Ns] = o;
    }
}

// One Stockham pass of radix RAD over nlines lines of length N (line stride ls), Ns the product of the earlier
// radices and n = N / Ns the length still to transform: butterfly j of a line reads in[j + r N/RAD], twiddles by
// W^(r (j mod Ns) N / (Ns RAD)), and writes out[(j / Ns) Ns RAD + j mod Ns + r Ns].
template <typename R, int RAD, int DIR>
__device__ __forceinline__ void stockhamPass(const typename CplxT<R>::T* in, typename CplxT<R>::T* out, int nlines,
                                             int N, int ls, int Ns, int n, const typename CplxT<R>::T* tw) {
    const int nb = N / RAD, step = n / RAD;
    const float invNb = __frcp_rn((float) nb), invNs = __frcp_rn((float) Ns);
    for (int t = threadIdx.x; t < nlines * nb; t += blockDim.x) {
        const int line = fdiv(t, invNb), j = t - line * nb;
        const int q = fdiv(j, invNs), jn = j - q * Ns;
        stockhamButterfly<R, RAD, DIR>(in + line * ls + j, out + line * ls + q * Ns * RAD + jn, nb, Ns, jn * step,
                                       tw);
    }
}

// Transforms nlines lines of length N held in a (line stride ls); b is scratch of the same size.  Returns the
// buffer holding the result (which of the two depends on N only).  Every thread of the block calls it (it
// synchronises after each pass).
template <typename R, int DIR>
__device__ typename CplxT<R>::T* fftLines(typename CplxT<R>::T* a, typename CplxT<R>::T* b, int nlines, int N, int ls,
                                          const typename CplxT<R>::T* tw) {
    typedef typename CplxT<R>::T C;
    int n = N, Ns = 1;
    while (n > 1) {
        if (n % 4 == 0) {
            stockhamPass<R, 4, DIR>(a, b, nlines, N, ls, Ns, n, tw);
            Ns *= 4;
            n /= 4;
        } else if (n % 2 == 0) {
            stockhamPass<R, 2, DIR>(a, b, nlines, N, ls, Ns, n, tw);
            Ns *= 2;
            n /= 2;
        } else if (n % 3 == 0) {
            stockhamPass<R, 3, DIR>(a, b, nlines, N, ls, Ns, n, tw);
            Ns *= 3;
            n /= 3;
        } else {
            stockhamPass<R, 5, DIR>(a, b, nlines, N, ls, Ns, n, tw);
            Ns *= 5;
            n /= 5;
        }
        __syncthreads();
        C* t = a;
        a = b;
        b = t;
    }
    return a;
}

// The same passes for a compile-time length N: the radix sequence, strides and twiddle steps are constants and
// the index divisions become multiplications.  NREM: the length still to transform, NS the earlier radices.
template <typename R, int DIR, int N, int NREM, int NS>
struct FftPassesC {
    typedef typename CplxT<R>::T C;
    static __device__ __forceinline__ C* run(C* a, C* b, int nlines, int ls, const C* tw) {
        constexpr int RAD = NREM % 4 == 0 ? 4 : NREM % 2 == 0 ? 2 : NREM % 3 == 0 ? 3 : 5;
        constexpr int nb = N / RAD, step = NREM / RAD;
        for (int t = threadIdx.x; t < nlines * nb; t += blockDim.x) {
            const int line = t / nb, j = t - line * nb;
            const int q = j / NS, jn = j - q * NS;
            stockhamButterfly<R, RAD, DIR>(a + line * ls + j, b + line * ls + q * NS * RAD + jn, nb, NS, jn * step,
                                           tw);
        }
        __syncthreads();
        return FftPassesC<R, DIR, N, NREM / RAD, NS * RAD>::run(b, a, nlines, ls, tw);
    }
};
template <typename R, int DIR, int N, int NS>
struct FftPassesC<R, DIR, N, 1, NS> {
    typedef typename CplxT<R>::T C;
    static __device__ __forceinline__ C* run(C* a, C*, int, int, const C*) { return a; }
};

// Line transforms of length N (the compile-time passes when KC > 0, which then equals N).
template <typename R, int DIR, int KC>
__device__ __forceinline__ typename CplxT<R>::T* fftLinesK(typename CplxT<R>::T* a, typename CplxT<R>::T* b,
                                                           int nlines, int N, int ls, const typename CplxT<R>::T* tw) {
    if constexpr (KC > 0)
        return FftPassesC<R, DIR, KC, KC, 1>::run(a, b, nlines, ls, tw);
    else
        return fftLines<R, DIR>(a, b, nlines, N, ls, tw);
}

// Complex elements of each of the three transform buffers of a block of a cluster of C blocks for grid K (max
// of the plane rows, the y-lines and the x-lines it holds).
__host__ __device__ inline int fftcBufferElems(const int* K, int C) {
    const int K2h = K[2] / 2 + 1, P = (K[1] + 1) / 2, ly = K[1] + 1;
    const int ppc = (K[0] + C - 1) / C, lpc = (K[1] * K2h + C - 1) / C;
    int m = ppc * P * K[2];
    m = m > ppc * K2h * ly ? m : ppc * K2h * ly;
    m = m > lpc * (K[0] + 1) ? m : lpc * (K[0] + 1);
    return (m + 1) / 2 * 2;   // 16-byte multiples
}

// Threads per cluster block: 1024 in float (64 registers), 512 in double.
template <typename R> struct FftcThreads { static constexpr int n = 512; };
template <> struct FftcThreads<float> { static constexpr int n = 1024; };

template <typename R>
__global__ void __launch_bounds__(FftcThreads<R>::n) k_fft_cluster(Dev dv, int gateDone) {
    typedef typename CplxT<R>::T C;
    namespace cgx = cooperative_groups;
    cgx::cluster_group cl = cgx::this_cluster();
    const int rank = (int) cl.block_rank();
    const int csize = dv.fftcC;
    const int s = blockIdx.x / csize;
    if (gateDone && dv.scal[s * NSCAL + SC_DONE] != 0.0)
        return;   // the whole cluster (one system)
    const SysDev& S = dv.sys[s];
    const int K0 = S.K[0], K1 = S.K[1], K2 = S.K[2], K2h = K2 / 2 + 1, P = (K1 + 1) / 2, ly = K1 + 1, lx = K0 + 1;
    const int ppc = (K0 + csize - 1) / csize, x0 = rank * ppc;
    const int np = max(0, min(K0, x0 + ppc) - x0);                    // my planes
    const int L = K1 * K2h, lpc = (L + csize - 1) / csize, l0 = rank * lpc;
    const int nl = max(0, min(L, l0 + lpc) - l0);                      // my x-lines
    const int nT = blockDim.x, tid = threadIdx.x;
    // reciprocals for the index maps (fdiv: exact quotients below 2^20)
    const float iK1 = 1.0f / (float) K1, iK2 = 1.0f / (float) K2, iK2h = 1.0f / (float) K2h;
    const float iPK2 = 1.0f / (float) (P * K2), iPK2h = 1.0f / (float) (P * K2h), iNl = 1.0f / (float) max(nl, 1);
    const float iPpc = 1.0f / (float) ppc;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* W0 = (C*) smraw;
    C* W1 = W0 + FFT_MAXK;
    C* W2 = W1 + FFT_MAXK;
    C* const b0 = W2 + FFT_MAXK;
    C* const b1 = b0 + dv.fftcBuf;
    C* const b2 = b1 + dv.fftcBuf;
    const C* tw = (const C*) dv.twiddle;
    for (int m = tid; m < K0; m += nT)
        W0[m] = tw[S.twOff[0] + m];
    for (int m = tid; m < K1; m += nT)
        W1[m] = tw[S.twOff[1] + m];
    for (int m = tid; m < K2; m += nT)
        W2[m] = tw[S.twOff[2] + m];
    R* g = (R*) dv.grid + S.gridOff;
    // 1. my planes: rows 2p, 2p + 1 as one complex row, [plane][pair][z]
    const int rowsN = np * P * K2;
    for (int e = tid; e < rowsN; e += nT) {
        const int pl = fdiv(e, iPK2), rem = e - pl * (P * K2), pr = fdiv(rem, iK2), z = rem - pr * K2;
        const R* gp = g + ((size_t) (x0 + pl) * K1 + 2 * pr) * K2 + z;
        C v;
        v.x = gp[0];
        v.y = (2 * pr + 1 < K1) ? gp[K2] : (R) 0;
        b0[e] = v;
    }
    __syncthreads();
    C* Z = fftLines<R, -1>(b0, b1, np * P, K2, K2, W2);
    C* O = (Z == b0) ? b1 : b0;
    for (int e = tid; e < np * P * K2h; e += nT) {   // separate the two rows; y-lines O[(plane K2h + kz) ly + y]
        const int pl = fdiv(e, iPK2h), rem = e - pl * (P * K2h), pr = fdiv(rem, iK2h), kz = rem - pr * K2h;
        const C* zr = Z + (pl * P + pr) * K2;
        const C zk = zr[kz], zm = zr[kz == 0 ? 0 : K2 - kz];
        C X, Y;   // X = (Z_k + conj Z_-k) / 2, Y = (Z_k - conj Z_-k) / 2i
        X.x = (R) 0.5 * (zk.x + zm.x);
        X.y = (R) 0.5 * (zk.y - zm.y);
        Y.x = (R) 0.5 * (zk.y + zm.y);
        Y.y = (R) 0.5 * (zm.x - zk.x);
        C* o = O + (pl * K2h + kz) * ly + 2 * pr;
        o[0] = X;
        if (2 * pr + 1 < K1)
            o[1] = Y;
    }
    __syncthreads();
    C* F = fftLines<R, -1>(O, Z, np * K2h, K1, ly, W1);
    C* const Fb = (F == b0) ? b0 : b1;   // the same buffer in every block (the pass counts depend on K only)
    C* const Yb = (F == b0) ? b1 : b0;
    cl.sync();
    // 2. my x-lines l = kz K1 + ky: gather, forward along x, influence product, inverse, scatter
    C* const Xb = b2;
    for (int e = tid; e < nl * K0; e += nT) {
        const int x = fdiv(e, iNl), li = e - x * nl, l = l0 + li, kz = fdiv(l, iK1), ky = l - kz * K1;
        const int ow = fdiv(x, iPpc), xp = x - ow * ppc;
        const C* src = cl.map_shared_rank(Fb, ow);
        Xb[li * lx + x] = src[(xp * K2h + kz) * ly + ky];
    }
    __syncthreads();
    C* Fx = fftLines<R, -1>(Xb, Yb, nl, K0, lx, W0);
    const R* infl = (const R*) dv.infl + S.specOff;
    for (int e = tid; e < nl * K0; e += nT) {
        const int x = fdiv(e, iNl), li = e - x * nl, l = l0 + li, kz = fdiv(l, iK1), ky = l - kz * K1;
        const R gk = infl[((size_t) x * K1 + ky) * K2h + kz];
        C& v = Fx[li * lx + x];
        v.x *= gk;
        v.y *= gk;
    }
    __syncthreads();
    C* Gx = fftLines<R, 1>(Fx, Fx == Xb ? Yb : Xb, nl, K0, lx, W0);
    for (int e = tid; e < nl * K0; e += nT) {
        const int x = fdiv(e, iNl), li = e - x * nl, l = l0 + li, kz = fdiv(l, iK1), ky = l - kz * K1;
        const int ow = fdiv(x, iPpc), xp = x - ow * ppc;
        C* dst = cl.map_shared_rank(Fb, ow);
        dst[(xp * K2h + kz) * ly + ky] = Gx[li * lx + x];
    }
    cl.sync();
    // 3. my planes back along y, then z (two real rows from one complex row)
    C* Gy = fftLines<R, 1>(Fb, Yb, np * K2h, K1, ly, W1);
    C* O2 = (Gy == Fb) ? Yb : Fb;
    for (int e = tid; e < rowsN; e += nT) {
        const int pl = fdiv(e, iPK2), rem = e - pl * (P * K2), pr = fdiv(rem, iK2), k = rem - pr * K2;
        const bool upper = k >= K2h;
        const int kk = upper ? K2 - k : k;
        const bool realOnly = (k == 0) || ((K2 & 1) == 0 && k == K2 / 2);
        const C* gy = Gy + (pl * K2h + kk) * ly + 2 * pr;
        C X = gy[0], Y;
        Y.x = 0;
        Y.y = 0;
        if (2 * pr + 1 < K1)
            Y = gy[1];
        if (upper) {
            X.y = -X.y;
            Y.y = -Y.y;
        }
        if (realOnly) {
            X.y = 0;
            Y.y = 0;
        }
        C Zv;   // X + i Y
        Zv.x = X.x - Y.y;
        Zv.y = X.y + Y.x;
        O2[e] = Zv;
    }
    __syncthreads();
    const C* Zt = fftLines<R, 1>(O2, Gy, np * P, K2, K2, W2);
    for (int e = tid; e < rowsN; e += nT) {
        const int pl = fdiv(e, iPK2), rem = e - pl * (P * K2), pr = fdiv(rem, iK2), z = rem - pr * K2;
        R* gp = g + ((size_t) (x0 + pl) * K1 + 2 * pr) * K2 + z;
        gp[0] = Zt[e].x;
        if (2 * pr + 1 < K1)
            gp[K2] = Zt[e].y;
    }
}

// The x-lines of the split transforms: after 2D R2C transforms of every x-plane (cuFFT, spectrum layout
// F[(x K1 + ky) (K2/2 + 1) + kz]), XL_LINES consecutive lines (ky, kz) per block transform forward along x,
// take the influence product and transform back (mixed-radix Stockham passes in shared memory, host-built
// twiddles); 2D C2R transforms of the planes follow.  blockIdx.y: the system.
constexpr int XL_LINES = 16;
constexpr int XL_THREADS = 256;

template <typename R>
__global__ void __launch_bounds__(XL_THREADS) k_xlines(Dev dv, int gateDone) {
    typedef typename CplxT<R>::T C;
    __shared__ C W0[FFT_MAXK];
    __shared__ C A[XL_LINES * (FFT_MAXK + 1)], B[XL_LINES * (FFT_MAXK + 1)];
    const int s = blockIdx.y;
    if (gateDone && dv.scal[s * NSCAL + SC_DONE] != 0.0)
        return;
    const SysDev& S = dv.sys[s];
    const int K0 = S.K[0], nline = S.K[1] * (S.K[2] / 2 + 1), lx = K0 + 1;
    const int line0 = blockIdx.x * XL_LINES;
    if (line0 >= nline)
        return;
    const int nl = min(XL_LINES, nline - line0);
    C* spec = (C*) dv.spec + S.specOff + line0;
    const R* infl = (const R*) dv.infl + S.specOff + line0;
    const C* tw = (const C*) dv.twiddle + S.twOff[0];
    for (int m = threadIdx.x; m < K0; m += blockDim.x)
        W0[m] = tw[m];
    for (int e = threadIdx.x; e < K0 * XL_LINES; e += blockDim.x) {   // consecutive threads: consecutive lines
        const int x = e / XL_LINES, l = e % XL_LINES;
        if (l < nl)
            A[l * lx + x] = spec[(size_t) x * nline + l];
    }
    __syncthreads();
    C* F = fftLines<R, -1>(A, B, nl, K0, lx, W0);
    for (int e = threadIdx.x; e < K0 * XL_LINES; e += blockDim.x) {
        const int x = e / XL_LINES, l = e % XL_LINES;
        if (l < nl) {
            const R g = infl[(size_t) x * nline + l];
            C& v = F[l * lx + x];
            v.x *= g;
            v.y *= g;
        }
    }
    __syncthreads();
    const C* G = fftLines<R, 1>(F, F == A ? B : A, nl, K0, lx, W0);
    for (int e = threadIdx.x; e < K0 * XL_LINES; e += blockDim.x) {
        const int x = e / XL_LINES, l = e % XL_LINES;
        if (l < nl)
            spec[(size_t) x * nline + l] = G[l * lx + x];
    }
}

// ------------------------------------------------------------------------------------------------ grid transforms

// The transform pair with the influence product of a field pass as ONE cooperative kernel: block x of system s
// (blockIdx.y; K0 blocks per system) owns x-plane x and, between two barriers of the system's blocks, a run of
// the x-lines:
//   1. plane x: its real rows two at a time as one complex row (x + i y), forward along z (real to half
//      spectrum, separated by Hermitian symmetry) and along y in shared memory, stored to the spectrum
//      F[(x K1 + ky) (K2/2 + 1) + kz];
//   2. (barrier) lines l = ky (K2/2 + 1) + kz in [x lpb, x lpb + lpb): forward along x, the influence product,
//      back along x, in place in the spectrum;
//   3. (barrier) plane x back along y and z (imaginary parts at kz = 0 and the Nyquist index dropped, as a C2R
//      transform does) into the real grid.
// The same Stockham line transforms as the cluster kernel, with the exchange through L2 instead of distributed
// shared memory, so a 48^3 grid spreads over 48 SMs.  Loads of what other blocks wrote bypass L1 (__ldcg).
// Each barrier waits at most FFTG_SPIN_LIMIT polls; a block that gives up sets flags[11] and returns, and the
// host reports the evaluation as failed.
// Threads per block: 512 in float (64 registers, 2 blocks per SM), 256 in double (84 registers, 3 per SM).
template <typename R> struct FftgThreads { static constexpr int n = 256; };
template <> struct FftgThreads<float> { static constexpr int n = 512; };
constexpr unsigned FFTG_SPIN_LIMIT = 1u << 22;   // polls of an L2 word (a few hundred ns each): about 1 s

// Complex elements of each of the two transform buffers of a block for grid K (max of its plane rows, its
// y-lines and its x-lines).
__host__ __device__ inline int fftgBufferElems(const int* K) {
    const int K2h = K[2] / 2 + 1, P = (K[1] + 1) / 2, ly = K[1] + 1, lx = K[0] + 1;
    const int lpb = (K[1] * K2h + K[0] - 1) / K[0];
    int m = P * K[2];
    m = m > K2h * ly ? m : K2h * ly;
    m = m > lpb * lx ? m : lpb * lx;
    return (m + 1) / 2 * 2;   // 16-byte multiples
}

__device__ __forceinline__ unsigned ldAcquireGpu(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Barrier of nb blocks over an arrival counter that only grows between resets (the flags and barrier words are
// cleared at the start of every call): the blocks of barrier k arrive as numbers k nb .. k nb + nb - 1 and leave
// once the counter has reached (k + 1) nb.  The wait is bounded: false, with flags[11] set, when it gave up.
__device__ __forceinline__ unsigned atomAddReleaseGpu(unsigned* p, unsigned v) {
    unsigned old;
    asm volatile("atom.add.release.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// The arrival is a release (it orders the block's writes before it, made the thread's own by the block barrier
// ahead of it) and the wait an acquire load, so no separate fences are needed.
__device__ __forceinline__ bool fftgBarrier(unsigned* bar, unsigned nb, int* flags) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        const unsigned old = atomAddReleaseGpu(bar, 1u);
        const unsigned target = (old / nb + 1) * nb;
        if (old + 1 != target)
            for (unsigned it = 0; (int) (ldAcquireGpu(bar) - target) < 0; it++)
                if (it >= FFTG_SPIN_LIMIT) {
                    ok = 0;
                    atomicExch(flags + 11, 1);
                    break;
                }
    }
    __syncthreads();
    return ok != 0;
}

// Self-test of the bounded barrier wait: the launch's blocks wait at a barrier that expects one block more than
// there are, so every wait runs out (FFTG_SPIN_LIMIT polls), sets flags[11] and returns.
__global__ void k_barrier_probe(unsigned* bar, int* flags) { fftgBarrier(bar, gridDim.x + 1, flags); }

// KC > 0: every grid of the launch is KC^3 (compile-time passes and index maps); 0: any grid.
// ENERGY (the final pass): also the reciprocal energy (1/2) sum w G |F|^2 and its strain derivative, as k_conv
// sums them, from the x-lines' spectrum before the product; block x writes conv partial x of its system and clears
// partials x + K0, x + 2 K0, ... up to the system's convBlocks (the host requires K0 <= convBlocks).
template <typename R, int KC, bool ENERGY = false>
__global__ void __launch_bounds__(FftgThreads<R>::n) k_fft_grid(Dev dv, int gateDone) {
    typedef typename CplxT<R>::T C;
    const int s = blockIdx.y;
    if ((gateDone & 1) && dv.scal[s * NSCAL + SC_DONE] != 0.0)
        return;   // every block of the system
    // gateDone & 2: the spread went to the fixed-point grid; its plane is converted (and cleared) on the load
    long long* const fx = (gateDone & 2) ? dv.gridFix : nullptr;
    const SysDev& S = dv.sys[s];
    const int K0 = KC > 0 ? KC : S.K[0], K1 = KC > 0 ? KC : S.K[1], K2 = KC > 0 ? KC : S.K[2];
    const int K2h = K2 / 2 + 1, P = (K1 + 1) / 2, ly = K1 + 1, lx = K0 + 1;
    const int x = blockIdx.x;
    if (x >= K0)
        return;   // (a smaller grid than the launch's largest)
    const int nline = K1 * K2h, lpb = (nline + K0 - 1) / K0, l0 = x * lpb;
    const int nl = max(0, min(nline, l0 + lpb) - l0);
    const int nT = blockDim.x, tid = threadIdx.x;
    const float iK2 = __frcp_rn((float) K2), iK2h = __frcp_rn((float) K2h), iLpb = __frcp_rn((float) lpb);
    // e / d: by a constant when the grid is one (the compiler multiplies), else through the float reciprocal
    auto qd = [](int e, int d, float inv) { return KC > 0 ? e / d : fdiv(e, inv); };
    extern __shared__ __align__(16) unsigned char smraw[];
    C* W0 = (C*) smraw;
    C* W1 = W0 + FFT_MAXK;
    C* W2 = W1 + FFT_MAXK;
    C* const b0 = W2 + FFT_MAXK;
    C* const b1 = b0 + dv.fftgBuf;
    const C* tw = (const C*) dv.twiddle;
    for (int m = tid; m < K0; m += nT)
        W0[m] = tw[S.twOff[0] + m];
    for (int m = tid; m < K1; m += nT)
        W1[m] = tw[S.twOff[1] + m];
    for (int m = tid; m < K2; m += nT)
        W2[m] = tw[S.twOff[2] + m];
    R* const gx = (R*) dv.grid + S.gridOff + (size_t) x * K1 * K2;
    C* const spec = (C*) dv.spec + S.specOff;
    C* const plane = spec + (size_t) x * nline;
    unsigned* const bar = dv.fftgBar + 2 * s;
    // 1. plane x: rows 2p, 2p + 1 as one complex row [pair][z]; z; separation into y-lines [kz][y]; y
    long long* const fxx = fx ? fx + S.gridOff + (size_t) x * K1 * K2 : nullptr;
    for (int e = tid; e < P * K2; e += nT) {
        const int pr = qd(e, K2, iK2), z = e - pr * K2;
        C v;
        if (fxx) {
            v.x = (R) gridFixTake(fxx + 2 * pr * K2 + z);
            v.y = (2 * pr + 1 < K1) ? (R) gridFixTake(fxx + (2 * pr + 1) * K2 + z) : (R) 0;
        } else {
            v.x = gx[2 * pr * K2 + z];
            v.y = (2 * pr + 1 < K1) ? gx[(2 * pr + 1) * K2 + z] : (R) 0;
        }
        b0[e] = v;
    }
    __syncthreads();
    C* Z = fftLinesK<R, -1, KC>(b0, b1, P, K2, K2, W2);
    C* O = (Z == b0) ? b1 : b0;
    for (int e = tid; e < P * K2h; e += nT) {
        const int pr = qd(e, K2h, iK2h), kz = e - pr * K2h;
        const C* zr = Z + pr * K2;
        const C zk = zr[kz], zm = zr[kz == 0 ? 0 : K2 - kz];
        C X, Y;   // X = (Z_k + conj Z_-k) / 2, Y = (Z_k - conj Z_-k) / 2i
        X.x = (R) 0.5 * (zk.x + zm.x);
        X.y = (R) 0.5 * (zk.y - zm.y);
        Y.x = (R) 0.5 * (zk.y + zm.y);
        Y.y = (R) 0.5 * (zm.x - zk.x);
        C* o = O + kz * ly + 2 * pr;
        o[0] = X;
        if (2 * pr + 1 < K1)
            o[1] = Y;
    }
    __syncthreads();
    const C* F = fftLinesK<R, -1, KC>(O, Z, K2h, K1, ly, W1);
    for (int e = tid; e < nline; e += nT) {
        const int ky = qd(e, K2h, iK2h), kz = e - ky * K2h;
        plane[e] = F[kz * ly + ky];
    }
    if (!fftgBarrier(bar, (unsigned) K0, dv.flags))
        return;
    // 2. my x-lines: forward along x, influence product, back
    for (int e = tid; e < lpb * K0; e += nT) {   // consecutive threads: consecutive lines of a plane
        const int xx = qd(e, lpb, iLpb), li = e - xx * lpb;
        if (li < nl)
            b0[li * lx + xx] = __ldcg(spec + (size_t) xx * nline + l0 + li);
    }
    __syncthreads();
    C* Fx = fftLinesK<R, -1, KC>(b0, b1, nl, K0, lx, W0);
    const R* infl = (const R*) dv.infl + S.specOff;
    double acc[ENERGY ? NCONV : 1];
#pragma unroll
    for (int k = 0; k < (ENERGY ? NCONV : 1); k++)
        acc[k] = 0.0;
    const double fac = PI_D * PI_D / (S.beta * S.beta);
    for (int e = tid; e < lpb * K0; e += nT) {
        const int xx = qd(e, lpb, iLpb), li = e - xx * lpb;
        if (li < nl) {
            const R gk = infl[(size_t) xx * nline + l0 + li];
            C& v = Fx[li * lx + xx];
            if (ENERGY && (xx != 0 || l0 + li != 0)) {   // (the k = 0 term is left out, as k_conv does)
                const int l = l0 + li, m3 = l % K2h, m2 = l / K2h, m1 = xx;
                const double w = (m3 == 0 || ((K2 & 1) == 0 && m3 == K2 / 2)) ? 1.0 : 2.0;
                const double nrm = (double) v.x * v.x + (double) v.y * v.y;
                const double en = 0.5 * w * (double) gk * nrm;
                acc[0] += en;
                const double mm1 = (m1 <= K0 / 2) ? m1 : m1 - K0, mm2 = (m2 <= K1 / 2) ? m2 : m2 - K1, mm3 = m3;
                double ms[3];
#pragma unroll
                for (int k = 0; k < 3; k++)
                    ms[k] = mm1 * S.recip[3 * k] + mm2 * S.recip[3 * k + 1] + mm3 * S.recip[3 * k + 2];
                const double m2s = ms[0] * ms[0] + ms[1] * ms[1] + ms[2] * ms[2];
                const double c2 = 2.0 * (fac + 1.0 / m2s);
#pragma unroll
                for (int a = 0; a < 3; a++)
#pragma unroll
                    for (int b = 0; b < 3; b++)
                        acc[ENERGY ? 1 + 3 * a + b : 0] += en * ((a == b ? -1.0 : 0.0) + c2 * ms[a] * ms[b]);
            }
            v.x *= gk;
            v.y *= gk;
        }
    }
    if (ENERGY) {
        blockReduce<NCONV>(acc, 0u);
        if (tid == 0)
            for (int k = 0; k < NCONV; k++)
                dv.convPartial[(size_t) (dv.convPartialOff[s] + x) * NCONV + k] = acc[k];
        if (tid < NCONV * 16)
            for (int b = x + K0 * (1 + tid / NCONV); b < S.convBlocks; b += 16 * K0)
                dv.convPartial[(size_t) (dv.convPartialOff[s] + b) * NCONV + tid % NCONV] = 0.0;
    }
    __syncthreads();
    const C* Gx = fftLinesK<R, 1, KC>(Fx, Fx == b0 ? b1 : b0, nl, K0, lx, W0);
    for (int e = tid; e < lpb * K0; e += nT) {
        const int xx = qd(e, lpb, iLpb), li = e - xx * lpb;
        if (li < nl)
            spec[(size_t) xx * nline + l0 + li] = Gx[li * lx + xx];
    }
    if (!fftgBarrier(bar, (unsigned) K0, dv.flags))
        return;
    // 3. plane x back: y-lines [kz][y]; y; two real rows from one complex row; z
    for (int e = tid; e < nline; e += nT) {
        const int ky = qd(e, K2h, iK2h), kz = e - ky * K2h;
        b0[kz * ly + ky] = __ldcg(plane + e);
    }
    __syncthreads();
    C* Gy = fftLinesK<R, 1, KC>(b0, b1, K2h, K1, ly, W1);
    C* O2 = (Gy == b0) ? b1 : b0;
    for (int e = tid; e < P * K2; e += nT) {
        const int pr = qd(e, K2, iK2), k = e - pr * K2;
        const bool upper = k >= K2h;
        const int kk = upper ? K2 - k : k;
        const bool realOnly = (k == 0) || ((K2 & 1) == 0 && k == K2 / 2);
        const C* gy = Gy + kk * ly + 2 * pr;
        C X = gy[0], Y;
        Y.x = 0;
        Y.y = 0;
        if (2 * pr + 1 < K1)
            Y = gy[1];
        if (upper) {
            X.y = -X.y;
            Y.y = -Y.y;
        }
        if (realOnly) {
            X.y = 0;
            Y.y = 0;
        }
        C Zv;   // X + i Y
        Zv.x = X.x - Y.y;
        Zv.y = X.y + Y.x;
        O2[e] = Zv;
    }
    __syncthreads();
    const C* Zt = fftLinesK<R, 1, KC>(O2, Gy, P, K2, K2, W2);
    for (int e = tid; e < P * K2; e += nT) {
        const int pr = qd(e, K2, iK2), z = e - pr * K2;
        gx[2 * pr * K2 + z] = Zt[e].x;
        if (2 * pr + 1 < K1)
            gx[(2 * pr + 1) * K2 + z] = Zt[e].y;
    }
}

// Interpolation from the potential grid: f_a = sum (d theta_a) theta theta phi (the field, E_rec = -sum_a K_a
// recip[:, a] f_a, core/pgm_core.cpp:241-264); FINAL also the second derivatives, the potential and the
// reciprocal forces -K_a recip[k][a] (q f1_a + sum_b e_b f2_ab) (core/pgm_core.cpp:452-487) and E_rec (x) d.
// The gather of slot's atom i (system S) by its warp: E_rec (and with FINAL the reciprocal forces, E_rec (x) d
// and the potential); sth / sdth / sd2 are the warp's shared spline rows.
template <typename R, bool FINAL, int P>
__device__ __forceinline__ void gatherSlot(const Dev& dv, const SysDev& S, int slot, int i, int wib, int lane,
                                           R (*sth)[3][P > 0 ? P : MAXP], R (*sdth)[3][P > 0 ? P : MAXP],
                                           R (*sd2)[3][FINAL ? (P > 0 ? P : MAXP) : 1]) {
    constexpr int PM = P > 0 ? P : MAXP;
    const int p = P > 0 ? P : dv.order;
    int bl = 0;
    if (lane < 3) {
        if (P == 0) {
            R t[MAXP], u[MAXP], v[MAXP];
            bspline<R>((R) dv.pmeFr[3 * i + lane], p, t, u, v);
#pragma unroll
            for (int j = 0; j < PM; j++)
                if (j < p) {
                    sth[wib][lane][j] = t[j];
                    sdth[wib][lane][j] = u[j];
                    if (FINAL)
                        sd2[wib][lane][FINAL ? j : 0] = v[j];
                }
        }
        bl = dv.pmeBase[3 * i + lane];
    }
    if (P > 0) {   // the evaluation's precomputed coefficients (k_splines)
        const R* sp = (const R*) dv.spl + (size_t) slot * 9 * MAXP;
        constexpr int KINDS = FINAL ? 3 : 2;
        for (int k = lane; k < KINDS * 3 * PM; k += 32) {
            const int kind = k / (3 * PM), dim = (k / PM) % 3, j = k % PM;
            const R v = sp[(kind * 3 + dim) * MAXP + j];
            if (kind == 0)
                sth[wib][dim][j] = v;
            else if (kind == 1)
                sdth[wib][dim][j] = v;
            else
                sd2[wib][dim][FINAL ? j : 0] = v;
        }
    }
    const int b0 = __shfl_sync(0xffffffffu, bl, 0), b1 = __shfl_sync(0xffffffffu, bl, 1),
              b2 = __shfl_sync(0xffffffffu, bl, 2);
    __syncwarp();
    const R* grid = (const R*) dv.grid + S.gridOff;
    const int K0 = S.K[0], K1 = S.K[1], K2 = S.K[2];
    R f[3] = {0, 0, 0}, f2[6] = {0, 0, 0, 0, 0, 0}, pot = 0;
    if (P > 0) {
        // lane -> (j2, j3), loop over j1: sums S_t = sum t1 phi, S_u = sum u1 phi (S_v = sum v1 phi), then the
        // products with the lane's t2, t3, u2, u3 (v2, v3)
        // full rounds: lane -> column (j2, j3), loop over j1; the leftover columns' points over the lanes
        constexpr int PP = P > 0 ? P : 1;
        constexpr int NPAIR = PP * PP, FULL = NPAIR / 32, LEFT = NPAIR % 32, LROUNDS = (LEFT * PP + 31) / 32;
        constexpr int LEFTD = LEFT > 0 ? LEFT : 1;   // (a divisor for the leftover rounds, which run only when LEFT > 0)
        const size_t plane = (size_t) K1 * K2;
#pragma unroll
        for (int rd = 0; rd < FULL; rd++) {
            const int pr = lane + 32 * rd;
            const int j2 = pr / PP, j3 = pr % PP;
            const R* col = grid + (size_t) wrapIndex(b1 - j2, K1) * K2 + wrapIndex(b2 - j3, K2);
            R St = 0, Su = 0, Sv = 0;
#pragma unroll
            for (int j1 = 0; j1 < PP; j1++) {
                const R ph = col[(size_t) wrapIndex(b0 - j1, K0) * plane];
                St += sth[wib][0][j1] * ph;
                Su += sdth[wib][0][j1] * ph;
                if (FINAL)
                    Sv += sd2[wib][0][FINAL ? j1 : 0] * ph;
            }
            const R t2 = sth[wib][1][j2], u2 = sdth[wib][1][j2];
            const R t3 = sth[wib][2][j3], u3 = sdth[wib][2][j3];
            f[0] += Su * t2 * t3;
            f[1] += St * u2 * t3;
            f[2] += St * t2 * u3;
            if (FINAL) {
                const R v2 = sd2[wib][1][FINAL ? j2 : 0], v3 = sd2[wib][2][FINAL ? j3 : 0];
                f2[0] += Sv * t2 * t3;
                f2[1] += St * v2 * t3;
                f2[2] += St * t2 * v3;
                f2[3] += Su * u2 * t3;
                f2[4] += Su * t2 * u3;
                f2[5] += St * u2 * u3;
                pot += St * t2 * t3;
            }
        }
#pragma unroll
        for (int lr = 0; lr < LROUNDS; lr++) {
            const int k = lane + 32 * lr;
            if (k < LEFT * PP) {
                const int pr = 32 * FULL + k % LEFTD, j1 = k / LEFTD;
                const int j2 = pr / PP, j3 = pr % PP;
                const R ph = grid[(size_t) wrapIndex(b0 - j1, K0) * plane + (size_t) wrapIndex(b1 - j2, K1) * K2 +
                                  wrapIndex(b2 - j3, K2)];
                const R t1 = sth[wib][0][j1], u1 = sdth[wib][0][j1];
                const R t2 = sth[wib][1][j2], u2 = sdth[wib][1][j2];
                const R t3 = sth[wib][2][j3], u3 = sdth[wib][2][j3];
                f[0] += u1 * t2 * t3 * ph;
                f[1] += t1 * u2 * t3 * ph;
                f[2] += t1 * t2 * u3 * ph;
                if (FINAL) {
                    const R v1 = sd2[wib][0][FINAL ? j1 : 0], v2 = sd2[wib][1][FINAL ? j2 : 0],
                            v3 = sd2[wib][2][FINAL ? j3 : 0];
                    f2[0] += v1 * t2 * t3 * ph;
                    f2[1] += t1 * v2 * t3 * ph;
                    f2[2] += t1 * t2 * v3 * ph;
                    f2[3] += u1 * u2 * t3 * ph;
                    f2[4] += u1 * t2 * u3 * ph;
                    f2[5] += t1 * u2 * u3 * ph;
                    pot += t1 * t2 * t3 * ph;
                }
            }
        }
    } else {
        const int pp = p * p, p3 = pp * p;
        for (int t = lane; t < p3; t += 32) {
            const int j1 = t / pp, j2 = (t / p) % p, j3 = t % p;
            const R t1 = sth[wib][0][j1], u1 = sdth[wib][0][j1];
            const R t2 = sth[wib][1][j2], u2 = sdth[wib][1][j2];
            const R t3 = sth[wib][2][j3], u3 = sdth[wib][2][j3];
            const int g1 = wrapIndex(b0 - j1, K0), g2 = wrapIndex(b1 - j2, K1), g3 = wrapIndex(b2 - j3, K2);
            const R ph = grid[((size_t) g1 * K1 + g2) * K2 + g3];
            f[0] += u1 * t2 * t3 * ph;
            f[1] += t1 * u2 * t3 * ph;
            f[2] += t1 * t2 * u3 * ph;
            if (FINAL) {
                const R v1 = sd2[wib][0][FINAL ? j1 : 0], v2 = sd2[wib][1][FINAL ? j2 : 0], v3 = sd2[wib][2][FINAL ? j3 : 0];
                f2[0] += v1 * t2 * t3 * ph;
                f2[1] += t1 * v2 * t3 * ph;
                f2[2] += t1 * t2 * v3 * ph;
                f2[3] += u1 * u2 * t3 * ph;
                f2[4] += u1 * t2 * u3 * ph;
                f2[5] += t1 * u2 * u3 * ph;
                pot += t1 * t2 * t3 * ph;
            }
        }
    }
    double F[3] = {(double) f[0], (double) f[1], (double) f[2]};
    double F2[7] = {(double) f2[0], (double) f2[1], (double) f2[2], (double) f2[3], (double) f2[4], (double) f2[5],
                    (double) pot};
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int k = 0; k < 3; k++)
            F[k] += __shfl_xor_sync(0xffffffffu, F[k], o);
        if (FINAL)
#pragma unroll
            for (int k = 0; k < 7; k++)
                F2[k] += __shfl_xor_sync(0xffffffffu, F2[k], o);
    }
    if (lane < 3) {
        const int k = lane;
        const double E = -(S.K[0] * S.recip[3 * k] * F[0] + S.K[1] * S.recip[3 * k + 1] * F[1] +
                           S.K[2] * S.recip[3 * k + 2] * F[2]);
        dv.Erec[3 * i + k] = E;
        if (FINAL) {
            const double* d = dv.dtot + 3 * i;
            double e[3];
            for (int a = 0; a < 3; a++)
                e[a] = S.K[a] * (d[0] * S.recip[a] + d[1] * S.recip[3 + a] + d[2] * S.recip[6 + a]);
            const double f2m[3][3] = {{F2[0], F2[3], F2[4]}, {F2[3], F2[1], F2[5]}, {F2[4], F2[5], F2[2]}};
            const double qi = dv.q[i];
            double Fk = 0.0;
            for (int a = 0; a < 3; a++) {
                const double c = qi * F[a] + e[0] * f2m[a][0] + e[1] * f2m[a][1] + e[2] * f2m[a][2];
                Fk -= S.K[a] * S.recip[3 * k + a] * c;
            }
            dv.Frec[3 * i + k] = Fk;
            // E_rec (x) d: fractional dipoles change with the box (core/pgm_core.cpp:446-451)
            for (int b = 0; b < 3; b++)
                dv.fin[(size_t) i * NFIN + 3 + 3 * k + b] = E * d[b];
        }
    }
    if (FINAL && lane == 0)
        dv.potRec[i] = F2[6];
    if (FINAL && lane < 6 && dv.hrec)   // (the potential's Hessian at the atom, for the force-matching adjoint)
        dv.hrec[6 * (size_t) i + lane] = F2[lane];
}

// A warp per slot, reads from the grid (L2).  CGA (the CG iterations of a single-system engine): each atom's
// row of A p = p / alpha - (E_pair + E_rec + cs p) (core/pgm_core.cpp:363) in the epilogue, block partials of
// p . A p, and the last block to finish sums them in block order (deterministic) and sets alph = rz / p.Ap.
template <typename R, bool FINAL, int P, bool CGA>
__global__ void __launch_bounds__(256) k_gather(Dev dv, int gateDone) {
    constexpr int PM = P > 0 ? P : MAXP;
    __shared__ R sth[8][3][PM], sdth[8][3][PM], sd2[8][3][FINAL ? PM : 1];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int slot = blockIdx.x * 8 + wib;
    if constexpr (!CGA) {
        if (gateDone && dv.useActive)   // a batch's CG iteration: the active systems' slots only
            slot = activeSlot(dv, slot);
        if (slot < 0 || slot >= dv.nAtoms)
            return;
        const int i = dv.slotAtom[slot];
        const int s = dv.atomSys[i];
        if (gateDone && dv.scal[s * NSCAL + SC_DONE] != 0.0)
            return;
        gatherSlot<R, FINAL, P>(dv, dv.sys[s], slot, i, wib, lane, sth, sdth, sd2);
    } else {
        double* sc = dv.scal;   // system 0
        if (sc[SC_DONE] != 0.0)
            return;   // every block alike
        const SysDev& S = dv.sys[0];
        double v = 0.0;
        if (slot < dv.nAtoms) {
            const int i = dv.slotAtom[slot];
            gatherSlot<R, FINAL, P>(dv, S, slot, i, wib, lane, sth, sdth, sd2);
            if (lane < 3) {
                const double cs = 4.0 * S.beta * S.beta * S.beta / (3.0 * SQRT_PI);
                const double al = dv.alpha[i];
                const int k = lane;
                const double pk = dv.p[3 * i + k];
                const double Tp = dv.Epair[3 * i + k] + dv.Erec[3 * i + k] + cs * pk;
                const double apk = (al > 0) ? pk / al - Tp : 0.0;
                dv.Ap[3 * i + k] = apk;
                v = pk * apk;
            }
        }
        v += __shfl_down_sync(0xffffffffu, v, 2);
        v += __shfl_down_sync(0xffffffffu, v, 1);   // lane 0: its atom's p . A p (lanes 0, 1, 2; fixed order)
        __shared__ double wsum[8];
        __shared__ int isLast;
        if (lane == 0)
            wsum[wib] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            double b = 0.0;
            for (int w = 0; w < 8; w++)
                b += wsum[w];
            dv.gpartial[blockIdx.x] = b;
            __threadfence();
            isLast = atomicAdd(&dv.flags[10], 1) == (int) gridDim.x - 1;
        }
        __syncthreads();
        if (!isLast)
            return;
        __threadfence();
        double acc[1] = {0.0};   // thread t: blocks t, t + 256, ... in order; then the fixed block tree
        for (int b = threadIdx.x; b < (int) gridDim.x; b += blockDim.x)
            acc[0] += __ldcg(&dv.gpartial[b]);
        blockReduce<1>(acc, 0u);
        if (threadIdx.x == 0) {
            sc[SC_ALPH] = sc[SC_RZ] / fmax(acc[0], 1e-300);
            dv.flags[10] = 0;
        }
    }
}

// ------------------------------------------------------------------------------------------------ pair passes

// Direct field at slot's atom of the dipoles (and with WITHQ the charges) of its list: E_i += q_j x G1 - d_j G1
// + (d_j . x) x G2 (core/pgm_core.cpp:274-284), products in precision R, sums in double.  GS lanes per atom.
// Mixed: the pair records (x, G1, G2, slot of j) stream from the evaluation's list and only (d_j, q_j) is
// gathered; FP64: x from the gathered slot-order positions, (G1, G2) streamed.
// DUAL: one sweep over the records for two source sets, (q, d) from dS (with WITHQ) into Epair and the dipoles
// of dS2 into Epair2, each summed exactly as a pass of its own would sum it.
template <typename R, bool WITHQ, int GS, bool DUAL = false>
__global__ void __launch_bounds__(256) k_pair_field(Dev dv, int gateDone) {
    typedef typename V4T<R>::T R4;
    typedef typename V2T<R>::T R2;
    int g = (blockIdx.x * blockDim.x + threadIdx.x) / GS;
    const int lane = threadIdx.x % GS;
    if (gateDone && dv.useActive)   // a batch's CG iteration: the active systems' slots only
        g = activeSlot(dv, g);
    if (g < 0 || g >= dv.nAtoms)
        return;
    const int slot = g;
    const int i = dv.slotAtom[slot];
    const int s = dv.atomSys[i];
    if (gateDone && dv.scal[s * NSCAL + SC_DONE] != 0.0)
        return;
    const R4* arow = (const R4*) dv.pairA + (size_t) slot * dv.cap;
    const R2* brow = (const R2*) dv.pairB + (size_t) slot * dv.cap;
    const R4* dS = (const R4*) dv.dS;
    const R4* dS2 = (const R4*) dv.dS2;
    const int cnt = dv.listCount[slot];
    R a0 = 0, a1 = 0, a2 = 0;   // per-lane sums in R (about cnt / GS terms each), across lanes in double
    R b0 = 0, b1 = 0, b2 = 0;   // (DUAL: the second set's)
    if constexpr (PairRec<R>::storeX) {
#pragma unroll 4
        for (int t = lane; t < cnt; t += GS) {
            const R4 xg = arow[t];
            const R2 gb = brow[t];
            const int js = realAsSlot(gb.y);
            const R4 dj = dS[js];
            const R djx = dj.x * xg.x + dj.y * xg.y + dj.z * xg.z;
            R c = djx * gb.x;
            if (WITHQ)
                c += dj.w * xg.w;
            a0 += c * xg.x - dj.x * xg.w;
            a1 += c * xg.y - dj.y * xg.w;
            a2 += c * xg.z - dj.z * xg.w;
            if (DUAL) {
                const R4 ej = dS2[js];
                const R c2 = (ej.x * xg.x + ej.y * xg.y + ej.z * xg.z) * gb.x;
                b0 += c2 * xg.x - ej.x * xg.w;
                b1 += c2 * xg.y - ej.y * xg.w;
                b2 += c2 * xg.z - ej.z * xg.w;
            }
        }
    } else {
        const SysDev& S = dv.sys[s];
        const double4 pwi = dv.posS[slot];
        const uint32_t* row = dv.list + (size_t) slot * dv.cap;
#pragma unroll 4
        for (int t = lane; t < cnt; t += GS) {
            const uint32_t e = row[t];
            const R2 G = brow[t];
            const int js = entrySlot(e);
            double sh[3];
            entryShift(e, S.H, sh);
            const double4 pwj = dv.posS[js];
            const R x0 = (R) (pwi.x - pwj.x - sh[0]), x1 = (R) (pwi.y - pwj.y - sh[1]), x2 = (R) (pwi.z - pwj.z - sh[2]);
            const R4 dj = dS[js];
            const R djx = dj.x * x0 + dj.y * x1 + dj.z * x2;
            R c = djx * G.y;
            if (WITHQ)
                c += dj.w * G.x;
            a0 += c * x0 - dj.x * G.x;
            a1 += c * x1 - dj.y * G.x;
            a2 += c * x2 - dj.z * G.x;
            if (DUAL) {
                const R4 ej = dS2[js];
                const R c2 = (ej.x * x0 + ej.y * x1 + ej.z * x2) * G.y;
                b0 += c2 * x0 - ej.x * G.x;
                b1 += c2 * x1 - ej.y * G.x;
                b2 += c2 * x2 - ej.z * G.x;
            }
        }
    }
    double E0 = a0, E1 = a1, E2 = a2;
    double H0 = b0, H1 = b1, H2 = b2;
    const unsigned gm = groupMask<GS>();
#pragma unroll
    for (int o = GS / 2; o > 0; o >>= 1) {
        E0 += __shfl_xor_sync(gm, E0, o, GS);
        E1 += __shfl_xor_sync(gm, E1, o, GS);
        E2 += __shfl_xor_sync(gm, E2, o, GS);
        if (DUAL) {
            H0 += __shfl_xor_sync(gm, H0, o, GS);
            H1 += __shfl_xor_sync(gm, H1, o, GS);
            H2 += __shfl_xor_sync(gm, H2, o, GS);
        }
    }
    if (lane == 0) {
        dv.Epair[3 * i] = E0;
        dv.Epair[3 * i + 1] = E1;
        dv.Epair[3 * i + 2] = E2;
        if (DUAL) {
            dv.Epair2[3 * i] = H0;
            dv.Epair2[3 * i + 1] = H1;
            dv.Epair2[3 * i + 2] = H2;
        }
    }
}

// Final pair pass at fixed d (core/pgm_core.cpp:422-440), per directed pair from i's side: half the pair
// energy, the force on i (-dE/dx), the field at i and half the strain dE/dx (x) x.  G_0..G_3 from the
// evaluation's pair records (x from the records in mixed precision, from the slot-order positions in FP64).
template <typename R, int GS>
__global__ void __launch_bounds__(256) k_pair_final(Dev dv) {
    typedef typename V4T<R>::T R4;
    typedef typename V2T<R>::T R2;
    const int g = (blockIdx.x * blockDim.x + threadIdx.x) / GS, lane = threadIdx.x % GS;
    if (g >= dv.nAtoms)
        return;
    const int slot = g;
    const int i = dv.slotAtom[slot];
    const SysDev& S = dv.sys[dv.atomSys[i]];
    const double4 pwi = dv.posS[slot];
    const uint32_t* row = dv.list + (size_t) slot * dv.cap;
    const R4* arow = (const R4*) dv.pairA + (size_t) slot * dv.cap;
    const R2* brow = (const R2*) dv.pairB + (size_t) slot * dv.cap;
    const R2* crow = (const R2*) dv.pairC + (size_t) slot * dv.cap;
    const R4* dS = (const R4*) dv.dS;
    const R4 di = dS[slot];
    const int cnt = dv.listCount[slot];
    R racc[16];
#pragma unroll
    for (int k = 0; k < 16; k++)
        racc[k] = R(0);   // 0 energy, 1-3 force, 4-6 field, 7-15 strain: per-lane sums in R, across lanes in double
    for (int t = lane; t < cnt; t += GS) {
        R x[3], G[4];
        int js;
        const R2 gc = crow[t];
        G[0] = gc.x;
        G[3] = gc.y;
        if constexpr (PairRec<R>::storeX) {
            const R4 xg = arow[t];
            const R2 gb = brow[t];
            x[0] = xg.x;
            x[1] = xg.y;
            x[2] = xg.z;
            G[1] = xg.w;
            G[2] = gb.x;
            js = realAsSlot(gb.y);
        } else {
            const uint32_t e = row[t];
            js = entrySlot(e);
            double sh[3];
            entryShift(e, S.H, sh);
            const double4 pwj = dv.posS[js];
            x[0] = (R) (pwi.x - pwj.x - sh[0]);
            x[1] = (R) (pwi.y - pwj.y - sh[1]);
            x[2] = (R) (pwi.z - pwj.z - sh[2]);
            const R2 gb = brow[t];
            G[1] = gb.x;
            G[2] = gb.y;
        }
        const R4 dj = dS[js];
        const R qi = di.w, qj = dj.w;
        const R dix = di.x * x[0] + di.y * x[1] + di.z * x[2];
        const R djx = dj.x * x[0] + dj.y * x[1] + dj.z * x[2];
        const R didj = di.x * dj.x + di.y * dj.y + di.z * dj.z;
        const R U = qi * qj * G[0] + (qi * djx - qj * dix) * G[1] + didj * G[1] - dix * djx * G[2];
        const R sc = -qi * qj * G[1] - (qi * djx - qj * dix) * G[2] - didj * G[2] + dix * djx * G[3];
        const R dcomp[3] = {dj.x, dj.y, dj.z}, icomp[3] = {di.x, di.y, di.z};
        racc[0] += R(0.5) * U;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const R dedx = sc * x[k] + (qi * dcomp[k] - qj * icomp[k]) * G[1] - (djx * icomp[k] + dix * dcomp[k]) * G[2];
            racc[1 + k] -= dedx;
            racc[4 + k] += qj * x[k] * G[1] - dcomp[k] * G[1] + djx * x[k] * G[2];
#pragma unroll
            for (int b = 0; b < 3; b++)
                racc[7 + 3 * k + b] += R(0.5) * dedx * x[b];
        }
    }
    double acc[16];
#pragma unroll
    for (int k = 0; k < 16; k++)
        acc[k] = racc[k];
    const unsigned gm = groupMask<GS>();
#pragma unroll
    for (int o = GS / 2; o > 0; o >>= 1)
#pragma unroll
        for (int k = 0; k < 16; k++)
            acc[k] += __shfl_xor_sync(gm, acc[k], o, GS);
    if (lane == 0) {
        dv.fin[(size_t) i * NFIN + 0] = acc[0];
        for (int k = 0; k < 3; k++) {
            dv.Fpair[3 * i + k] = acc[1 + k];
            dv.Epair[3 * i + k] = acc[4 + k];
        }
        for (int k = 0; k < 9; k++)
            dv.spair[(size_t) i * 9 + k] = acc[7 + k];
    }
}

// ------------------------------------------------------------------------------------------------ GVDW

// G(y) = F(y)/y^6 and H(y) = G'(y)/y of the GVDW dispersion (core/gvdw_kernel.h:30-58): the series in y^2 below
// y = 0.6 (coefficients dv.gvC, derived on the host), the closed form F = A^2 + g^2/2 above.
template <typename R>
__device__ __forceinline__ void gvdwG(R y, const double* C, R& G, R& H) {
    const R c0 = R(8.0 / (9.0 * PI_D));
    if (y < R(0.6)) {
        const R y2 = y * y;
        R g = R(0), h = R(0);
#pragma unroll
        for (int k = GVDW_TERMS - 1; k >= 0; k--)
            g = g * y2 + (R) C[k];
#pragma unroll
        for (int k = GVDW_TERMS - 1; k >= 1; k--)
            h = h * y2 + R(2 * k) * (R) C[k];
        G = c0 * g;
        H = c0 * h;
        return;
    }
    const R isp = R(1.0 / SQRT_PI);
    const R y2 = y * y, e = fexp(-y2);
    const R A = ferf(y) - R(2) * isp * y * (R(1) + R(2) * y2 / R(3)) * e;
    const R g = (R(4) / R(3)) * isp * y2 * y * e;
    const R F = A * A + R(0.5) * g * g;
    const R Ap = (R(8) / R(3)) * isp * y2 * y2 * e;
    const R gp = R(4) * isp * y2 * (R(1) - R(2) * y2 / R(3)) * e;
    const R Fp = R(2) * A * Ap + g * gp;
    const R y6 = y2 * y2 * y2;
    G = F / y6;
    H = (Fp / y6 - R(6) * F / (y6 * y)) / y;
}

// The GVDW pass of a single-system engine after the final pair pass: per atom (a warp per slot, its
// evaluation's list over the lanes) the pairs within rvdw that are not skipped and carry a parameter,
// U = A exp(-B y^2) (Gaussian) or A exp(-B y) (Slater) - C6 b^6 G(y) with y = b r, b = 1/sqrt(2 (R_i^2 + R_j^2)),
// A = a_i a_j, C6 = c_i c_j, B = (b_i + b_j)/2 (core/gvdw_kernel.h:64-78, the combination rule of
// core/cuda/pgm_cuda.cu:398-413).  Pair arithmetic in R, sums in double; half the pair energy into fin[13], the
// force -dU/dr x/r and half the strain dU/dx (x) x added to the pair force and strain (those in units of ke).
template <typename R>
__global__ void __launch_bounds__(256) k_gvdw(Dev dv) {
    const int slot = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (slot >= dv.nAtoms)
        return;
    const int i = dv.slotAtom[slot];
    const SysDev& S = dv.sys[0];
    const double4 gi = dv.gv[i];
    const double4 pwi = dv.posS[slot];
    const double Ri = dv.radius[i];
    const uint32_t* row = dv.list + (size_t) slot * dv.cap;
    const int cnt = dv.listCount[slot];
    const int sb = dv.skipStart[i], se = dv.skipStart[i + 1];
    double acc[13];
#pragma unroll
    for (int k = 0; k < 13; k++)
        acc[k] = 0.0;
    if (gi.x != 0.0 || gi.y != 0.0)
        for (int t = lane; t < cnt; t += 32) {
            const uint32_t e = row[t];
            const int js = entrySlot(e);
            double sh[3];
            entryShift(e, S.H, sh);
            const double4 pwj = dv.posS[js];
            const double x0 = pwi.x - pwj.x - sh[0], x1 = pwi.y - pwj.y - sh[1], x2 = pwi.z - pwj.z - sh[2];
            const double r2 = x0 * x0 + x1 * x1 + x2 * x2;
            if (!(r2 < dv.rvdw2))
                continue;
            const int j = dv.slotAtom[js];
            const double4 gj = dv.gv[j];
            const double Aij = gi.x * gj.x, C6 = gi.y * gj.y;
            if (Aij == 0.0 && C6 == 0.0)
                continue;
            bool skip = false;
            for (int k = sb; k < se && !skip; k++)
                skip = dv.skipJ[k] == j;
            if (skip)
                continue;
            const double Rj = dv.radius[j];
            const R bij = R(1) / (R) sqrt(2.0 * (Ri * Ri + Rj * Rj));
            const R r = (R) sqrt(r2), y = bij * r, b2 = bij * bij, b6 = b2 * b2 * b2, B = (R) (0.5 * (gi.z + gj.z));
            R erep, drep;   // drep = (1/r) dU_rep/dr
            if (dv.gvdwSlater) {
                erep = (R) Aij * fexp(-B * y);
                drep = r > R(0) ? -B * bij * erep / r : R(0);
            } else {
                erep = (R) Aij * fexp(-B * y * y);
                drep = R(-2) * B * b2 * erep;
            }
            R G, H;
            gvdwG<R>(y, dv.gvC, G, H);
            const R U = erep - (R) C6 * b6 * G;
            const double dEdR = -(double) (drep - (R) C6 * b6 * b2 * H);   // -(1/r) dU/dr
            const double x[3] = {x0, x1, x2};
            acc[0] += 0.5 * (double) U;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                acc[1 + k] += dEdR * x[k];
#pragma unroll
                for (int b = 0; b < 3; b++)
                    acc[4 + 3 * k + b] -= 0.5 * dEdR * x[k] * x[b];
            }
        }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int k = 0; k < 13; k++)
            acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
    if (lane == 0) {
        const double ike = 1.0 / dv.ke;
        dv.fin[(size_t) i * NFIN + 13] = acc[0];
        for (int k = 0; k < 3; k++)
            dv.Fpair[3 * i + k] += acc[1 + k] * ike;
        for (int k = 0; k < 9; k++)
            dv.spair[(size_t) i * 9 + k] += acc[4 + k] * ike;
    }
}

// ------------------------------------------------------------------------------------------------ CG

// The initial guess x0 of component g = 3 gi + k when it does not depend on b (guess 1: zero; 2: history slot;
// 3: mu3 from history; 4: mu4 from history) (core/pgm_core.cpp:309-329).
__device__ __forceinline__ double historyGuess(const Dev& dv, int guess, size_t g, size_t hs) {
    const int h0 = dv.ctl->h[0], h1 = dv.ctl->h[1], h2 = dv.ctl->h[2], h3 = dv.ctl->h[3];
    switch (guess) {
    case 1: return 0.0;
    case 2: return dv.hist[h0 * hs + g];
    case 3: return 3 * dv.hist[h0 * hs + g] - 3 * dv.hist[h1 * hs + g] + dv.hist[h2 * hs + g];
    default:
        return 4 * dv.hist[h0 * hs + g] - 6 * dv.hist[h1 * hs + g] + 4 * dv.hist[h2 * hs + g] - dv.hist[h3 * hs + g];
    }
}

// x0 of a predicted step before the permanent field (guess >= 1), so that one pair sweep forms E_perm and T x0
// together; k_cg_b then writes the same x0 again.
__global__ void k_cg_guess(Dev dv) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * dv.nAtoms)
        return;
    const int i = t / 3, k = t % 3;
    const int guess = dv.ctl->guess;
    const int gi = dv.globalIndex ? dv.globalIndex[i] : i;
    const double x0 = guess >= 1 ? historyGuess(dv, guess, (size_t) 3 * gi + k, (size_t) 3 * dv.numGlobal) : 0.0;
    dv.x[t] = (guess >= 2 && !(dv.alpha[i] > 0)) ? 0.0 : x0;
}

// b = E_perm (pair + reciprocal + self), norm = mean|alpha b| per system, initial guess x0
// (guess 0: alpha b; 1: zero; 2: history slot; 3: mu3 from history; 4: mu4 from history)
// (core/pgm_core.cpp:297-329).
__global__ void __launch_bounds__(CHUNK) k_cg_b(Dev dv) {
    const int chunk = blockIdx.x;
    const int s = dv.chunkSys[chunk];
    const SysDev& S = dv.sys[s];
    const int i = dv.chunkBegin[chunk] + threadIdx.x;
    double v[1] = {0.0};
    if (i < dv.chunkEnd[chunk]) {
        const double cs = 4.0 * S.beta * S.beta * S.beta / (3.0 * SQRT_PI);
        const double al = dv.alpha[i];
        const int gi = dv.globalIndex ? dv.globalIndex[i] : i;
        const size_t hs = (size_t) 3 * dv.numGlobal;
        const int guess = dv.ctl->guess;
        const bool custom = dv.ctl->customRhs != 0;
        for (int k = 0; k < 3; k++) {
            const double bk = custom ? dv.b[3 * i + k] : dv.Epair[3 * i + k] + dv.Erec[3 * i + k] + cs * dv.perm[3 * i + k];
            dv.b[3 * i + k] = bk;
            v[0] += fabs(al * bk);
            const double x0 = guess == 0 ? al * bk : historyGuess(dv, guess, (size_t) 3 * gi + k, hs);
            dv.x[3 * i + k] = (guess >= 2 && !(al > 0)) ? 0.0 : x0;
        }
    }
    double tot[1];
    if (chunkFinish<1>(dv, chunk, s, v, 0u, tot) && threadIdx.x == 0)
        dv.scal[s * NSCAL + SC_NORM] = tot[0] / (3.0 * (S.atomEnd - S.atomBegin)) + 1e-300;
}

// r = b - A x0 (rows of polarizable atoms), z = alpha r, direction p = 0 (so the first direction is z),
// rz, err (core/pgm_core.cpp:351-361).  A v = v/alpha - T v, T v = pair + reciprocal + self field of v.
__global__ void __launch_bounds__(CHUNK) k_cg_init(Dev dv) {
    const int chunk = blockIdx.x;
    const int s = dv.chunkSys[chunk];
    const SysDev& S = dv.sys[s];
    const int i = dv.chunkBegin[chunk] + threadIdx.x;
    double v[2] = {0.0, 0.0};
    if (i < dv.chunkEnd[chunk]) {
        const double cs = 4.0 * S.beta * S.beta * S.beta / (3.0 * SQRT_PI);
        const double al = dv.alpha[i];
        for (int k = 0; k < 3; k++) {
            const double xk = dv.x[3 * i + k];
            const double Tx = dv.Epair[3 * i + k] + dv.Erec[3 * i + k] + cs * xk;
            const double rk = (al > 0) ? dv.b[3 * i + k] - (xk / al - Tx) : 0.0;
            const double zk = al * rk;
            dv.r[3 * i + k] = rk;
            dv.z[3 * i + k] = zk;
            dv.p[3 * i + k] = 0.0;
            v[0] += rk * zk;
            v[1] = fmax(v[1], fabs(zk));
        }
    }
    double tot[2];
    __shared__ int decides;
    if (threadIdx.x == 0)
        decides = 0;
    if (chunkFinish<2>(dv, chunk, s, v, 2u, tot) && threadIdx.x == 0) {
        double* sc = dv.scal + s * NSCAL;
        sc[SC_RZ] = tot[0];
        sc[SC_ERR] = tot[1] / sc[SC_NORM];
        sc[SC_BETA] = 0.0;
        sc[SC_IT] = 0.0;
        const bool more = sc[SC_ERR] > dv.tol && 0 < dv.maxIter;
        sc[SC_DONE] = more ? 0.0 : 1.0;
        if (!more)
            atomicAdd(&dv.flags[2], 1);
        __threadfence();
        if (atomicAdd(&dv.flags[3], 1) == dv.nSys - 1) {
            // the last system to finish its initialisation decides whether the loop runs at all
            const int ndone = atomicAdd(&dv.flags[2], 0);
            dv.flags[5] = dv.nSys - ndone;
            dv.flags[4] = 0;
            dv.flags[3] = 0;
            if (dv.activeHist && dv.maxIter >= 0)
                dv.activeHist[0] = dv.nSys - ndone;
            if (dv.useCond && dv.loopCond)
                cudaGraphSetConditional(dv.cond, (ndone < dv.nSys) ? 1u : 0u);
            decides = 1;
        }
    }
    __syncthreads();
    if (decides && dv.useActive) {   // (every system's DONE is final: each system's last chunk came first)
        __threadfence();
        compactActive(dv);
    }
}

// FP64 refinement, permanent field: b64 = E_pair + E_rec + cs p (all FP64 arithmetic).
__global__ void k_refine_b(Dev dv, double* b64) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= dv.nAtoms)
        return;
    const SysDev& S = dv.sys[dv.atomSys[i]];
    const double cs = 4.0 * S.beta * S.beta * S.beta / (3.0 * SQRT_PI);
    for (int k = 0; k < 3; k++)
        b64[3 * i + k] = dv.Epair[3 * i + k] + dv.Erec[3 * i + k] + cs * dv.perm[3 * i + k];
}

// FP64 refinement, residual: r = b64 - (x/alpha - T x) with T x from FP64 pair and PME passes (rows of
// polarizable atoms), written to the CG's right-hand side b and to r; per system err = max|alpha r| /
// mean|alpha b64| in scal[SC_ERR], the count of systems within tol in flags[2].
__global__ void __launch_bounds__(CHUNK) k_refine_res(Dev dv, const double* b64) {
    const int chunk = blockIdx.x;
    const int s = dv.chunkSys[chunk];
    const SysDev& S = dv.sys[s];
    const int i = dv.chunkBegin[chunk] + threadIdx.x;
    double v[2] = {0.0, 0.0};
    if (i < dv.chunkEnd[chunk]) {
        const double cs = 4.0 * S.beta * S.beta * S.beta / (3.0 * SQRT_PI);
        const double al = dv.alpha[i];
        for (int k = 0; k < 3; k++) {
            const double xk = dv.x[3 * i + k];
            const double Tx = dv.Epair[3 * i + k] + dv.Erec[3 * i + k] + cs * xk;
            const double rk = (al > 0) ? b64[3 * i + k] - (xk / al - Tx) : 0.0;
            dv.b[3 * i + k] = rk;
            dv.r[3 * i + k] = rk;
            v[0] += fabs(al * b64[3 * i + k]);
            v[1] = fmax(v[1], fabs(al * rk));
        }
    }
    double tot[2];
    if (chunkFinish<2>(dv, chunk, s, v, 2u, tot) && threadIdx.x == 0) {
        const double norm = tot[0] / (3.0 * (S.atomEnd - S.atomBegin)) + 1e-300;
        dv.scal[s * NSCAL + SC_ERR] = tot[1] / norm;
        if (tot[1] / norm <= dv.tol)
            atomicAdd(&dv.flags[2], 1);
    }
}

// x = xsave + delta (the correction solved into x).
__global__ void k_refine_add(Dev dv, const double* xsave) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < 3 * dv.nAtoms)
        dv.x[t] += xsave[t];
}

// Ap = p/alpha - T p and p.Ap, then alph = rz / p.Ap per system (core/pgm_core.cpp:363-364).
__global__ void __launch_bounds__(CHUNK) k_cg_a(Dev dv) {
    const int chunk = blockIdx.x;
    const int s = dv.chunkSys[chunk];
    double* sc = dv.scal + s * NSCAL;
    if (sc[SC_DONE] != 0.0)
        return;
    const SysDev& S = dv.sys[s];
    const int i = dv.chunkBegin[chunk] + threadIdx.x;
    double v[1] = {0.0};
    if (i < dv.chunkEnd[chunk]) {
        const double cs = 4.0 * S.beta * S.beta * S.beta / (3.0 * SQRT_PI);
        const double al = dv.alpha[i];
        for (int k = 0; k < 3; k++) {
            const double pk = dv.p[3 * i + k];
            const double Tp = dv.Epair[3 * i + k] + dv.Erec[3 * i + k] + cs * pk;
            const double apk = (al > 0) ? pk / al - Tp : 0.0;
            dv.Ap[3 * i + k] = apk;
            v[0] += pk * apk;
        }
    }
    double tot[1];
    if (chunkFinish<1>(dv, chunk, s, v, 0u, tot) && threadIdx.x == 0)
        sc[SC_ALPH] = sc[SC_RZ] / fmax(tot[0], 1e-300);
}

// x += alph p, r' = r - alph Ap, z' = alpha r', beta = z'.(r' - r)/rz, rz = r'.z', err = max|alpha r'|/norm,
// convergence (core/pgm_core.cpp:362-385).  Also clears the PME grid for the next spread.
__global__ void __launch_bounds__(CHUNK) k_cg_upd(Dev dv) {
    // grid clearing for the next spread, every block (all systems), in 32-bit words
    {
        const size_t nth = (size_t) gridDim.x * blockDim.x;
        for (size_t k = (size_t) blockIdx.x * blockDim.x + threadIdx.x; k < (size_t) dv.gridWords; k += nth)
            ((uint32_t*) dv.grid)[k] = 0u;
    }
    const int chunk = blockIdx.x;
    const int s = dv.chunkSys[chunk];
    double* sc = dv.scal + s * NSCAL;
    if (sc[SC_DONE] != 0.0)
        return;
    const int i = dv.chunkBegin[chunk] + threadIdx.x;
    double v[3] = {0.0, 0.0, 0.0};
    if (i < dv.chunkEnd[chunk]) {
        const double al = dv.alpha[i], alph = sc[SC_ALPH];
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
    double tot[3];
    __shared__ int decides;
    if (threadIdx.x == 0)
        decides = 0;
    if (chunkFinish<3>(dv, chunk, s, v, 4u, tot) && threadIdx.x == 0) {
        sc[SC_BETA] = tot[0] / fmax(sc[SC_RZ], 1e-300);
        sc[SC_RZ] = tot[1];
        sc[SC_ERR] = tot[2] / sc[SC_NORM];
        sc[SC_IT] += 1.0;
        const bool more = sc[SC_ERR] > dv.tol && sc[SC_IT] < dv.maxIter;
        if (!more) {
            sc[SC_DONE] = 1.0;
            atomicAdd(&dv.flags[2], 1);
        }
        if (dv.nSys == 1) {   // the only system decides alone
            if (dv.useCond)
                cudaGraphSetConditional(dv.cond, more ? 1u : 0u);
        } else {
            __threadfence();
            // the last active system of this iteration to finish decides whether the loop goes on (the count of
            // active systems is read before this system's arrival, so before the last arrival resets it)
            const int expected = atomicAdd(&dv.flags[5], 0);
            const int active = atomicAdd(&dv.flags[4], 1) + 1;
            if (active == expected) {
                const int ndone = atomicAdd(&dv.flags[2], 0);
                dv.flags[5] = dv.nSys - ndone;   // systems active in the next iteration
                dv.flags[4] = 0;
                const int loopIt = ++dv.flags[13];
                if (dv.activeHist && loopIt <= dv.maxIter + 1)
                    dv.activeHist[loopIt] = dv.nSys - ndone;
                if (dv.useCond)
                    cudaGraphSetConditional(dv.cond, (ndone < dv.nSys) ? 1u : 0u);
                decides = 1;
            }
        }
    }
    __syncthreads();
    if (decides && dv.useActive) {   // the next iteration's virtual slots
        __threadfence();
        compactActive(dv);
    }
}

// ------------------------------------------------------------------------------------------------ final

// mu = x + peek alpha r (core/pgm_core.cpp:386-389), d = p + mu, self and polarization energies per atom,
// history push of mu (global order).
__global__ void k_final_prep(Dev dv, int solved) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= dv.nAtoms)
        return;
    const int histSlot = dv.ctl->histSlot;
    const SysDev& S = dv.sys[dv.atomSys[i]];
    const double al = dv.alpha[i];
    double m2 = 0.0, d2 = 0.0;
    const int gi = dv.globalIndex ? dv.globalIndex[i] : i;
    const bool fixedMu = dv.ctl->fixedMu != 0;
    for (int k = 0; k < 3; k++) {
        const double m = fixedMu ? dv.mu[3 * i + k] : solved ? dv.x[3 * i + k] + dv.peek * al * dv.r[3 * i + k] : 0.0;
        dv.mu[3 * i + k] = m;
        const double d = dv.perm[3 * i + k] + m;
        dv.dtot[3 * i + k] = d;
        m2 += m * m;
        d2 += d * d;
        if (histSlot >= 0)
            dv.hist[(size_t) histSlot * 3 * dv.numGlobal + 3 * gi + k] = m;
    }
    const double cs = 4.0 * S.beta * S.beta * S.beta / (3.0 * SQRT_PI);
    const double qi = dv.q[i];
    dv.fin[(size_t) i * NFIN + 1] = -(S.beta / SQRT_PI) * qi * qi - 0.5 * cs * d2;
    dv.fin[(size_t) i * NFIN + 2] = (al > 0) ? m2 / (2.0 * al) : 0.0;
}

// Total field E = E_pair + E_rec + cs d (core/pgm_core.cpp:437-438, 445-448, 494-495).
__global__ void k_final_field(Dev dv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= dv.nAtoms)
        return;
    const SysDev& S = dv.sys[dv.atomSys[i]];
    const double cs = 4.0 * S.beta * S.beta * S.beta / (3.0 * SQRT_PI);
    for (int k = 0; k < 3; k++)
        dv.Etot[3 * i + k] = dv.Epair[3 * i + k] + dv.Erec[3 * i + k] + cs * dv.dtot[3 * i + k];
}

__device__ __forceinline__ void covalentTerm(const Dev& dv, const SysDev& S, int m, double* t, double* v) {
    const int i = dv.covAtom[m], j = dv.covPartner[m];
    v[0] = dv.posIn[3 * j] - dv.posIn[3 * i];
    v[1] = dv.posIn[3 * j + 1] - dv.posIn[3 * i + 1];
    v[2] = dv.posIn[3 * j + 2] - dv.posIn[3 * i + 2];
    int kk[3];
    minImageExact(v, S.H, kk);
    const double L = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    const double u[3] = {v[0] / L, v[1] / L, v[2] / L};
    const double g[3] = {-dv.Etot[3 * i], -dv.Etot[3 * i + 1], -dv.Etot[3 * i + 2]};
    const double gu = g[0] * u[0] + g[1] * u[1] + g[2] * u[2];
    for (int k = 0; k < 3; k++)
        t[k] = dv.covStrength[m] * (g[k] - gu * u[k]) / L;
}

// Forces F = ke (pair + reciprocal + covalent chain rule, core/pgm_core.cpp:511-535), written to the
// outputs; per-system sums of the energies and the strain derivative, finished by the last chunk of each
// system together with the reciprocal energy and strain of the convolution blocks.
__global__ void __launch_bounds__(CHUNK) k_final_forces(Dev dv, int iterationsSolved) {
    const int chunk = blockIdx.x;
    const int s = dv.chunkSys[chunk];
    const SysDev& S = dv.sys[s];
    const int i = dv.chunkBegin[chunk] + threadIdx.x;
    double v[14];
#pragma unroll
    for (int k = 0; k < 14; k++)
        v[k] = 0.0;
    if (i < dv.chunkEnd[chunk]) {
        double F[3];
        for (int k = 0; k < 3; k++)
            F[k] = dv.Fpair[3 * i + k] + dv.Frec[3 * i + k];
        double Sv[9];
        for (int k = 0; k < 9; k++)
            Sv[k] = dv.spair[(size_t) i * 9 + k] + dv.fin[(size_t) i * NFIN + 3 + k];
        for (int c = dv.covByAtomOff[i]; c < dv.covByAtomOff[i + 1]; c++) {
            double t[3], vv[3];
            covalentTerm(dv, S, dv.covByAtom[c], t, vv);
            for (int k = 0; k < 3; k++) {
                F[k] += t[k];
                for (int b = 0; b < 3; b++)
                    Sv[3 * k + b] += t[k] * vv[b];
            }
        }
        for (int c = dv.covByPartnerOff[i]; c < dv.covByPartnerOff[i + 1]; c++) {
            double t[3], vv[3];
            covalentTerm(dv, S, dv.covByPartner[c], t, vv);
            for (int k = 0; k < 3; k++)
                F[k] -= t[k];
        }
        for (int k = 0; k < 3; k++)
            F[k] *= dv.ke;
        for (int k = 0; k < 3; k++)
            dv.forces[3 * i + k] = F[k];
        const Ctl& io = *dv.ctl;
        if (io.forcesOut)
            for (int k = 0; k < 3; k++)
                io.forcesOut[3 * i + k] = F[k];
        if (io.forceFixed)
            for (int k = 0; k < 3; k++)
                atomicAdd((unsigned long long*) &io.forceFixed[i + k * io.fixedStride],
                          (unsigned long long) llrint(F[k] * io.fixedScale));
        v[0] = dv.fin[(size_t) i * NFIN + 0];
        v[1] = dv.fin[(size_t) i * NFIN + 1];
        v[2] = dv.fin[(size_t) i * NFIN + 2];
        for (int k = 0; k < 9; k++)
            v[3 + k] = Sv[k];
        v[12] = dv.q[i];
        v[13] = dv.gvdwOn ? dv.fin[(size_t) i * NFIN + 13] : 0.0;
    }
    double tot[14];
    __shared__ double sconv[NCONV], cgrp[CHUNK / 16][NCONV];
    if (!chunkFinish<14>(dv, chunk, s, v, 0u, tot))
        return;
    {   // the reciprocal-space partials: value k = tid mod 16, block group tid / 16 (fixed order)
        const int k = threadIdx.x & 15, grp = threadIdx.x >> 4;
        if (k < NCONV) {
            double acc = 0.0;
#pragma unroll 4
            for (int bk = grp; bk < S.convBlocks; bk += CHUNK / 16)
                acc += __ldcg(&dv.convPartial[(size_t) (dv.convPartialOff[s] + bk) * NCONV + k]);
            cgrp[grp][k] = acc;
        }
    }
    __syncthreads();
    if (threadIdx.x < NCONV) {
        double acc = 0.0;
        for (int g = 0; g < CHUNK / 16; g++)
            acc += cgrp[g][threadIdx.x];
        sconv[threadIdx.x] = acc;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const double* conv = sconv;
        const double Q = tot[12];
        const double bg = -PI_D * Q * Q / (2.0 * S.volume * S.beta * S.beta);
        double* res = dv.results + (size_t) s * NRES;
        res[0] = dv.ke * tot[0];
        res[1] = dv.ke * conv[0];
        res[2] = dv.ke * tot[1];
        res[3] = dv.ke * bg;
        res[4] = dv.ke * tot[2];
        for (int k = 0; k < 9; k++) {
            double sk = tot[3 + k] + conv[1 + k];
            if (k % 4 == 0)
                sk -= bg;
            res[5 + k] = dv.ke * sk;
        }
        res[14] = iterationsSolved ? dv.scal[s * NSCAL + SC_IT] : 0.0;
        res[15] = iterationsSolved ? dv.scal[s * NSCAL + SC_ERR] : 0.0;
        res[16] = tot[13];   // GVDW [kJ/mol]
    }
}

// Pair parts of the parameter gradients at the final dipoles: dE/dq_i = sum_j q_j G0 + d_j.x G1 (x = r_i - r_j)
// and dE/dR_i = sum_j U(dG/da) da/dR_i with dG_n/da = (2/sqrt(pi)) (2a^2)^n exp(-a^2 r^2), da/dR_i = -2 R_i a^3.
// Double precision.  GS lanes per atom; writes gq[i], gR[i] (before the factor ke).
template <int GS>
__global__ void __launch_bounds__(256) k_pair_grad(Dev dv, double* gq, double* gR) {
    const int g = (blockIdx.x * blockDim.x + threadIdx.x) / GS, lane = threadIdx.x % GS;
    if (g >= dv.nAtoms)
        return;
    const int slot = g;
    const int i = dv.slotAtom[slot];
    const SysDev& S = dv.sys[dv.atomSys[i]];
    const double4 pwi = dv.posS[slot];
    const double Ri = dv.radS[slot];
    const uint32_t* row = dv.list + (size_t) slot * dv.cap;
    const int cnt = dv.listCount[slot];
    const double qi = dv.q[i];
    const double di[3] = {dv.dtot[3 * i], dv.dtot[3 * i + 1], dv.dtot[3 * i + 2]};
    double aq = 0.0, aR = 0.0;
    for (int t = lane; t < cnt; t += GS) {
        const uint32_t e = row[t];
        const int js = entrySlot(e);
        const int j = dv.slotAtom[js];
        double sh[3];
        entryShift(e, S.H, sh);
        const double4 pwj = dv.posS[js];
        const double x[3] = {pwi.x - pwj.x - sh[0], pwi.y - pwj.y - sh[1], pwi.z - pwj.z - sh[2]};
        const double Rj = dv.radS[js];
        const double r = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
        const double a = 1.0 / sqrt(2.0 * (Ri * Ri + Rj * Rj));
        double G[3];
        pairKernels<double, 3>(a, S.beta, r, G);
        const double qj = pwj.w;
        const double dj[3] = {dv.dtot[3 * j], dv.dtot[3 * j + 1], dv.dtot[3 * j + 2]};
        const double dix = di[0] * x[0] + di[1] * x[1] + di[2] * x[2];
        const double djx = dj[0] * x[0] + dj[1] * x[1] + dj[2] * x[2];
        const double didj = di[0] * dj[0] + di[1] * dj[1] + di[2] * dj[2];
        aq += qj * G[0] + djx * G[1];
        const double H0 = (2.0 / SQRT_PI) * exp(-(a * r) * (a * r)), H1 = H0 * 2.0 * a * a, H2 = H1 * 2.0 * a * a;
        const double U = qi * qj * H0 + (qi * djx - qj * dix) * H1 + didj * H1 - dix * djx * H2;
        aR += U * (-2.0 * Ri * a * a * a);
    }
    const unsigned gm = groupMask<GS>();
#pragma unroll
    for (int o = GS / 2; o > 0; o >>= 1) {
        aq += __shfl_xor_sync(gm, aq, o, GS);
        aR += __shfl_xor_sync(gm, aR, o, GS);
    }
    if (lane == 0) {
        gq[i] = aq;
        gR[i] = aR;
    }
}

}  // namespace pgmb200
