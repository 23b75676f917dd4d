// Plane-owner PME spread and gather for one system in mixed precision (any grid size; order 6), the field
// passes of the graph path.  Instead of a warp per atom issuing p^3 global atomics (spread) or loads (gather),
// a block owns a tile of the grid -- x-plane x, rows y0 - (p-1) .. y0 + YCH - 1 -- in shared memory:
//   spread  every atom whose stencil reaches the tile (its base b0 in x .. x + p - 1, its row base b1 in the
//           tile's YCH rows) adds its p^2 points of this plane to the shared tile (shared-memory float atomics);
//           the tile is then added to the grid once, coalesced along z;
//   gather  the tile is read from the grid once; each of the same atoms sums its p^2 points of this plane, and
//           the three field sums go to a slot of their own (one of p per atom), summed in a fixed order by the
//           consumer.
// The atoms are binned once per evaluation by (b0 mod K0, (b1 mod K1) / YCH) with their spline records.
#pragma once

#include "persistent.cuh"

namespace pgmb200 {

constexpr int PL_YCH = 16;       // tile rows owned by a block (plus p - 1 rows of halo below them)
constexpr int PL_THREADS = 256;

__device__ __forceinline__ int planeBin(const int4& b, const SysDev& S, int nyc) {
    return wrapIndex(b.x, S.K[0]) * nyc + wrapIndex(b.y, S.K[1]) / PL_YCH;
}

// Bin counts (cleared before; a block-local histogram in shared memory, then one global add per nonzero bin of
// the block), then their exclusive scan, then the records in bin order.
constexpr int PL_BIN_SLOTS = 2048;   // slots per binning block
constexpr int PL_MAX_SMEM_BINS = 8192;

__global__ void __launch_bounds__(256) k_plane_bin_count(Dev dv, int nyc, int* count) {
    extern __shared__ int hist[];
    const int nbins = dv.sys[0].K[0] * nyc;
    for (int b = threadIdx.x; b < nbins; b += blockDim.x)
        hist[b] = 0;
    __syncthreads();
    const int s0 = blockIdx.x * PL_BIN_SLOTS, s1 = min(dv.nAtoms, s0 + PL_BIN_SLOTS);
    for (int slot = s0 + threadIdx.x; slot < s1; slot += blockDim.x)
        atomicAdd(&hist[planeBin(dv.baseS[slot], dv.sys[0], nyc)], 1);
    __syncthreads();
    for (int b = threadIdx.x; b < nbins; b += blockDim.x)
        if (hist[b])
            atomicAdd(&count[b], hist[b]);
}

__global__ void __launch_bounds__(1024) k_plane_bin_scan(Dev dv, int nbins, int* count) {
    // one block: chunked exclusive scan of count into dv.pmeBinStart (nbins + 1) and count (the fill cursors)
    __shared__ int carry;
    __shared__ int wsum[32];
    if (threadIdx.x == 0)
        carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int base = 0; base < nbins; base += blockDim.x) {
        const int k = base + threadIdx.x;
        const int c = k < nbins ? count[k] : 0;
        int v = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o)
                v += y;
        }
        if (lane == 31)
            wsum[wid] = v;
        __syncthreads();
        if (wid == 0) {
            int s = lane < (int) (blockDim.x >> 5) ? wsum[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o)
                    s += y;
            }
            wsum[lane] = s;
        }
        __syncthreads();
        const int excl = carry + (wid > 0 ? wsum[wid - 1] : 0) + v - c;
        if (k < nbins) {
            dv.pmeBinStart[k] = excl;
            count[k] = excl;
        }
        __syncthreads();
        if (threadIdx.x == 0)
            carry += wsum[(blockDim.x >> 5) - 1];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        dv.pmeBinStart[nbins] = carry;
}

// The records in bin order: a block of 256 slots ranks them per bin in shared memory and claims a run of each
// bin's records with one global add per nonzero bin; then the block writes its records word by word, consecutive
// threads on consecutive words of a record (coalesced), reading the spline words from the slot's record.
constexpr int PL_FILL_SLOTS = 256;

template <int P>
__global__ void __launch_bounds__(PL_FILL_SLOTS) k_plane_bin_fill(Dev dv, int nyc, int* fill) {
    extern __shared__ int hist[];   // nbins counts, then the block's base per bin
    __shared__ int dest[PL_FILL_SLOTS];
    const SysDev& S = dv.sys[0];
    const int nbins = S.K[0] * nyc;
    int* base = hist + nbins;
    for (int b = threadIdx.x; b < nbins; b += blockDim.x)
        hist[b] = 0;
    __syncthreads();
    const int s0 = blockIdx.x * PL_FILL_SLOTS, slot = s0 + threadIdx.x;
    const bool on = slot < dv.nAtoms;
    int bin = 0, rank = 0;
    if (on) {
        bin = planeBin(dv.baseS[slot], S, nyc);
        rank = atomicAdd(&hist[bin], 1);
    }
    __syncthreads();
    for (int b = threadIdx.x; b < nbins; b += blockDim.x)
        base[b] = hist[b] ? atomicAdd(&fill[b], hist[b]) : 0;
    __syncthreads();
    dest[threadIdx.x] = on ? base[bin] + rank : 0;
    __syncthreads();
    constexpr int W = 4 + 6 * P;   // words per record: idx, then c[w], w = dim 2P + kind P + j
    static_assert(sizeof(PmeRec<P>) == W * 4, "record words");
    const int nrec = min(PL_FILL_SLOTS, dv.nAtoms - s0);
    for (int t = threadIdx.x; t < nrec * W; t += blockDim.x) {
        const int r = t / W, w = t - r * W, sl = s0 + r;
        int v;
        if (w < 4) {
            const int4 b = dv.baseS[sl];
            v = w == 0 ? sl : w == 1 ? wrapIndex(b.y, S.K[1]) : w == 2 ? b.z : wrapIndex(b.x, S.K[0]);
        } else {
            const int c = w - 4, dim = c / (2 * P), kind = (c / P) % 2, j = c % P;
            v = __float_as_int(((const float*) dv.spl)[(size_t) sl * 9 * MAXP + (kind * 3 + dim) * MAXP + j]);
        }
        ((int*) dv.pmeRec)[(size_t) dest[r] * W + w] = v;
    }
}

// The sources of a field pass per slot: mode 0 charges and vec, 1 vec only, 2 the CG direction p = z + beta p
// first (vec = p).  Writes the pair passes' copy dS = (d, q) and the PME weights srcW = (q, K_a d . recip[:, a]).
__global__ void k_plane_sources(Dev dv, int mode, double* vec) {
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= dv.nAtoms)
        return;
    const int i = dv.slotAtom[slot];
    const SysDev& S = dv.sys[0];
    double d[3];
    for (int k = 0; k < 3; k++) {
        if (mode == 2) {
            d[k] = dv.z[3 * i + k] + dv.scal[SC_BETA] * vec[3 * i + k];
            vec[3 * i + k] = d[k];
        } else {
            d[k] = vec[3 * i + k];
        }
    }
    const double q = (mode == 0) ? dv.q[i] : 0.0;
    ((float4*) dv.dS)[slot] = make_float4((float) d[0], (float) d[1], (float) d[2], (float) q);
    dv.srcW[slot] = make_float4((float) q, (float) (S.K[0] * (d[0] * S.recip[0] + d[1] * S.recip[3] + d[2] * S.recip[6])),
                                (float) (S.K[1] * (d[0] * S.recip[1] + d[1] * S.recip[4] + d[2] * S.recip[7])),
                                (float) (S.K[2] * (d[0] * S.recip[2] + d[1] * S.recip[5] + d[2] * S.recip[8])));
}

// The atoms of tile (x, yc): bins (x + j1 mod K0, yc), j1 < P, flattened.
template <int P>
__device__ __forceinline__ void planeTileAtoms(const Dev& dv, int x, int yc, int nyc, int K0, int* start, int* cum) {
    cum[0] = 0;
#pragma unroll
    for (int j = 0; j < P; j++) {
        const int b = wrapIndex(x + j, K0) * nyc + yc;
        start[j] = dv.pmeBinStart[b];
        cum[j + 1] = cum[j] + dv.pmeBinStart[b + 1] - dv.pmeBinStart[b];
    }
}

template <int P>
__device__ __forceinline__ int planeLocate(const int* start, const int* cum, int t, int& j1) {
    j1 = 0;
#pragma unroll
    for (int j = 1; j < P; j++)
        j1 += (t >= cum[j]) ? 1 : 0;
    return start[j1] + t - cum[j1];
}

// Spread of the sources srcW onto the grid (which starts cleared): block (x, yc) accumulates its tile in shared
// memory, then adds it to the grid.
template <int P>
__global__ void __launch_bounds__(PL_THREADS) k_spread_planes(Dev dv, int nyc) {
    extern __shared__ __align__(16) float tile[];
    const SysDev& S = dv.sys[0];
    const int K0 = S.K[0], K1 = S.K[1], K2 = S.K[2];
    const int x = blockIdx.x, yc = blockIdx.y, y0 = yc * PL_YCH;
    const int rows = min(PL_YCH, K1 - y0) + P - 1;
    for (int e = threadIdx.x; e < rows * K2; e += blockDim.x)
        tile[e] = 0.f;
    __syncthreads();
    int start[P], cum[P + 1];
    planeTileAtoms<P>(dv, x, yc, nyc, K0, start, cum);
    const PmeRec<P>* rec = (const PmeRec<P>*) dv.pmeRec;
    for (int t = threadIdx.x; t < cum[P]; t += blockDim.x) {
        int j1;
        const PmeRec<P>& r = rec[planeLocate<P>(start, cum, t, j1)];
        const int4 id = r.idx;
        const float4 w = dv.srcW[id.x];
        // the record's coefficients in registers first (the shared atomics below would otherwise make the
        // compiler reload them after every update)
        float c[4 * P];
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
            float* row = tile + (id.y - j2 - y0 + P - 1) * K2;
#pragma unroll
            for (int j3 = 0; j3 < P; j3++)
                atomicAdd(row + col[j3], A2 * c[2 * P + j3] + B2 * c[3 * P + j3]);
        }
    }
    __syncthreads();
    float* g = (float*) dv.grid + S.gridOff + (size_t) x * K1 * K2;
    for (int e = threadIdx.x; e < rows * K2; e += blockDim.x) {
        const float v = tile[e];
        if (v != 0.f) {
            const int r = e / K2, z = e - r * K2;
            atomicAdd(g + (size_t) wrapIndex(y0 - (P - 1) + r, K1) * K2 + z, v);
        }
    }
}

// Gather of the potential grid: block (x, yc) reads its tile, each of its atoms sums this plane's share of the
// field sums f_a = sum (d theta_a) theta theta phi into gpart[j1 n + slot].
template <int P>
__global__ void __launch_bounds__(PL_THREADS) k_gather_planes(Dev dv, int nyc) {
    extern __shared__ __align__(16) float tile[];
    const SysDev& S = dv.sys[0];
    const int K0 = S.K[0], K1 = S.K[1], K2 = S.K[2], n = dv.nAtoms;
    const int x = blockIdx.x, yc = blockIdx.y, y0 = yc * PL_YCH;
    const int rows = min(PL_YCH, K1 - y0) + P - 1;
    const float* g = (const float*) dv.grid + S.gridOff + (size_t) x * K1 * K2;
    for (int e = threadIdx.x; e < rows * K2; e += blockDim.x) {
        const int r = e / K2, z = e - r * K2;
        tile[e] = g[(size_t) wrapIndex(y0 - (P - 1) + r, K1) * K2 + z];
    }
    __syncthreads();
    int start[P], cum[P + 1];
    planeTileAtoms<P>(dv, x, yc, nyc, K0, start, cum);
    const PmeRec<P>* rec = (const PmeRec<P>*) dv.pmeRec;
    for (int t = threadIdx.x; t < cum[P]; t += blockDim.x) {
        int j1;
        const PmeRec<P>& r = rec[planeLocate<P>(start, cum, t, j1)];
        const int4 id = r.idx;
        int col[P];
#pragma unroll
        for (int j3 = 0; j3 < P; j3++)
            col[j3] = wrapIndex(id.z - j3, K2);
        float A = 0.f, B = 0.f, C = 0.f;
#pragma unroll
        for (int j2 = 0; j2 < P; j2++) {
            const float* row = tile + (id.y - j2 - y0 + P - 1) * K2;
            float st = 0.f, su = 0.f;
#pragma unroll
            for (int j3 = 0; j3 < P; j3++) {
                const float ph = row[col[j3]];
                st += r.c[4 * P + j3] * ph;
                su += r.c[5 * P + j3] * ph;
            }
            const float t2 = r.c[2 * P + j2], u2 = r.c[3 * P + j2];
            A += t2 * st;
            B += u2 * st;
            C += t2 * su;
        }
        dv.gpart[(size_t) j1 * n + id.x] = make_float4(r.c[P + j1] * A, r.c[j1] * B, r.c[j1] * C, 0.f);
    }
}

// E_rec of every atom from the plane shares (summed in j1 order): E_k = -sum_a K_a recip[k][a] f_a.
template <int P>
__global__ void k_gather_planes_finish(Dev dv) {
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= dv.nAtoms)
        return;
    const SysDev& S = dv.sys[0];
    double f[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int j1 = 0; j1 < P; j1++) {
        const float4 g = dv.gpart[(size_t) j1 * dv.nAtoms + slot];
        f[0] += g.x;
        f[1] += g.y;
        f[2] += g.z;
    }
    const int i = dv.slotAtom[slot];
    for (int k = 0; k < 3; k++)
        dv.Erec[3 * i + k] = -(S.K[0] * S.recip[3 * k] * f[0] + S.K[1] * S.recip[3 * k + 1] * f[1] +
                               S.K[2] * S.recip[3 * k + 2] * f[2]);
}

}  // namespace pgmb200
