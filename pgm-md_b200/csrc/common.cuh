// Shared device definitions of the pgm_b200 engine: the per-system table, the device-pointer bundle, the
// radial pair kernels in float and double, the B-spline recursion and deterministic block reductions.
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>
#include <stdint.h>

namespace pgmb200 {

constexpr int MAXP = 12;                       // largest B-spline order
constexpr double SQRT_PI = 1.7724538509055160273;
constexpr double PI_D = 3.14159265358979323846;
constexpr int CHUNK = 256;                     // atoms per chunk of the per-system reductions
constexpr int NSCAL = 16;                      // per-system CG scalars
// per-system scalar slots
enum { SC_NORM = 0, SC_RZ, SC_ALPH, SC_BETA, SC_ERR, SC_IT, SC_DONE, SC_PAP };
constexpr int NRES = 17;                       // per-system results: 5 terms, 9 strain, iterations, residual, GVDW
constexpr int GVDW_TERMS = 15;                 // terms of the GVDW G(y) series
constexpr int NFIN = 14;                       // per-atom final sums: epair, eself, epol, strain[9], q, GVDW
constexpr int NCONV = 10;                      // reciprocal energy + 9 strain per conv block

// Per-system constants (host-computed at every evaluation; box-dependent parts included).
struct SysDev {
    double H[9];          // box rows a, b, c
    double recip[9];      // recip[k*3+a] = (H^-1)_{k a}
    double volume, cutoff, rc2, beta;
    double rl2;           // list radius^2: (cutoff + skin)^2, the skin shrunk so that it stays below half the box
    double skinHalf2;     // (skin / 2)^2: an atom moved further since the list's build makes the list stale
    int K[3];
    int atomBegin, atomEnd;
    int cellN[3], cellM[3];
    int cellOff, cellCount;
    long long gridOff, specOff;
    int gridN, specN;
    int modOff[3];
    int chunkFirst, chunkCount;
    int convBlocks;
    int covBegin, covEnd;
    int twOff[3];         // offsets of the twiddle tables of K[0..2] in the engine's table (cluster transforms)
};

// Per-call control, read by the kernels from device memory so that one captured graph serves every call.
struct Ctl {
    int guess;               // 0 alpha b, 1 zero, 2 history[h0], 3 mu3, 4 mu4
    int h[4];                // history slots, newest first
    int histSlot;            // slot the solution is pushed to (-1: none)
    int customRhs;           // 1: the CG solves for the right-hand side already in b (adjoint solves)
    int fixedMu;             // 1: the final pass uses the induced dipoles already in mu (no solve)
    int posMode;             // 0 positions in posIn, 1 device float4 posDevice, 2 device double posDevice
    int fixedStride;
    const void* posDevice;
    long long* forceFixed;   // device 64-bit fixed-point forces (added), or null
    double fixedScale;
    double* forcesOut;       // device double forces (written), or null
    int forceRebuild;        // 1: build the pair list whatever the displacements (no list, box changed, skin 0)
};

// Device pointers of one engine (passed by value to every kernel).
struct Dev {
    int nAtoms, nSys, nChunks, cap, order, totalCells;
    long long gridTotal, gridWords;
    const Ctl* ctl;
    double ke, tol, peek;
    int maxIter;
    const SysDev* sys;
    // per atom, caller order
    const int* atomSys;
    const double* q;
    const double* radius;
    const double* alpha;
    const double* posIn;      // original positions (3n)
    int* wrapN;               // 3n: integer wraps N with pos = pw + N.H
    int* cellOf;              // global cell index
    int* cellRank;
    int* pmeBase;             // 3n
    double* pmeFr;            // 3n
    void* spl;                // slot order: 9 * MAXP spline coefficients (R) per atom
    int4* baseS;              // slot order: base grid indices
    // cells
    int* cellCount;
    int* cellStart;           // totalCells + 1
    // slot order (cell-sorted)
    int* slotAtom;
    int* slotTmp;             // cell-scatter order before the per-cell sort
    double4* posS;            // wrapped position + q
    double4* origS;           // original position + radius
    int4* wrapS;              // wraps N
    double* radS;
    // pair lists: the Verlet list of the last build (radius cutoff + skin) and, per evaluation, the pairs of
    // it within the cutoff with their G1, G2
    uint32_t* slist;          // [slot][cap] Verlet list (cutoff + skin)
    int* slistCount;          // per slot
    int* atomSlot;            // slot of each atom at the last build
    // the caller's pair candidates (setCandidates), per atom i in both directions: partners candJ[k] and
    // integer box shifts candT[k] (8 bits per component, offset 128) for k in [candStart[i], candStart[i + 1]),
    // x = r_i + t.H - r_j; null: the engine's own cell search
    const int* candStart;
    const int* candJ;
    const int* candT;
    double* posBuild;         // 3n positions at the list's build
    uint32_t* list;           // [slot][cap] pairs within the cutoff
    int* listCount;           // per slot
    void* pairA;              // [slot][cap] R4: pair geometry x = r_i - r_j (image) and G1, per evaluation
    void* pairB;              // [slot][cap] R2: G2 and the slot of j (as the bits of an R)
    void* pairC;              // [slot][cap] R2: G0, G3 (the final pass), per evaluation
    int* flags;               // [0]: list overflow, [1]: shift out of range, [2]: all systems done, [3]-[5] CG
                              // bookkeeping, [6]: list stale, [7]: block counter, [8]: list built,
                              // [9]: a pair changed its image since the build (rebuild and repeat),
                              // [10]: block counter of the CG gather, [11]: a grid-transform barrier gave up;
                              // followed by the grid transforms' barriers (2 per system)
    // dipoles
    void* dS;                 // slot-order R4 (dipole xyz, charge w) for the pair passes
    void* dS2;                // the second source set of a dual pair pass (the predicted guess's dipoles)
    long long* gridFix;       // mixed precision: the spread's 64-bit fixed-point grid (null: float atomics on grid)
    double* perm;             // 3n
    double* mu;               // 3n
    double* dtot;             // 3n
    // CG
    double* b;
    double* x;
    double* r;
    double* z;
    double* p;
    double* Ap;
    double* scal;             // nSys * NSCAL
    double* partial;          // nChunks * 16
    double* gpartial;         // per gather block: p . A p partials (the CG gather of a single-system engine)
    int* sysCounter;          // nSys
    int* activeHist;          // batched CG: systems still iterating before iteration k (k = 0 .. iterations);
                              // flags[13] counts the loop's iterations
    // batched CG: the systems still iterating, compacted after every iteration -- actSys[k] their indices in
    // order, actOff[k] the first virtual slot of the k-th (actOff[actCount[0]] = active slots), actCount[0] how
    // many; the iteration's per-slot kernels map virtual slots onto them, so converged systems cost nothing
    int* actSys;
    int* actOff;
    int* actCount;
    int useActive;            // 1: the per-slot CG kernels take virtual slots (batched engines)
    // fields / forces
    double* Epair;            // 3n
    double* Epair2;           // 3n: the dual pair pass's field of dS2
    double* Erec;             // 3n
    double* Fpair;            // 3n
    double* spair;            // 9n pair strain
    double* Frec;             // 3n
    double* Etot;             // 3n
    double* fin;              // n * NFIN per-atom final sums
    double* potRec;           // n
    double* hrec;             // 6n second-derivative sums of the final reciprocal potential (00 11 22 01 02 12)
    double* forces;           // 3n output (double)
    double* results;          // nSys * NRES
    double* convPartial;      // sum over systems of convBlocks * NCONV
    int* convPartialOff;      // per system
    // PME
    void* grid;               // R, gridTotal
    void* spec;               // complex R
    void* infl;               // R, spec size
    const void* twiddle;      // complex R tables exp(-2 pi i m / K), m < K, per distinct K (cluster transforms)
    int fftcBuf;              // complex elements per transform buffer of a cluster block
    int fftcC;                // blocks per cluster
    int fftgBuf;              // complex elements per transform buffer of a grid-transform block
    unsigned* fftgBar;        // per system: arrivals and generation of the grid transforms' barrier
    const double* moduli;
    // covalent
    int ncov;
    const int* covAtom;
    const int* covPartner;
    const double* covStrength;
    const int* covByAtomOff;  // n + 1
    const int* covByAtom;
    const int* covByPartnerOff;
    const int* covByPartner;
    // chunks
    const int* chunkSys;
    const int* chunkBegin;
    const int* chunkEnd;
    // the combination-rule GVDW (setGvdw): per atom (sqrt A, sqrt C6, b, 0), caller order; skipped partners per
    // atom (sorted, both directions); pairs within rvdw2 of the evaluation's list; G(y) series coefficients
    int gvdwOn, gvdwSlater;
    double rvdw2;
    const double4* gv;
    const int* skipStart;
    const int* skipJ;
    double gvC[GVDW_TERMS];
    // history (global order)
    double* hist;             // 4 * 3 * numGlobal
    const int* globalIndex;
    int numGlobal;
    // the persistent CG kernel (mixed, one system): plane bins and spline records of the atoms, per-slot PME
    // weights (q, e0, e1, e2) of the current source, per-(j1, slot) gather sums, block shares, barrier words
    void* pmeRec;
    int* pmeBinStart;
    float4* srcW;
    float4* gpart;
    double* pcgPartial;
    unsigned* pcgBar;
    // graph
    int loopCond;                          // 1: the CG loop is a conditional while node (k_cg_init sets it)
    cudaGraphConditionalHandle cond;       // CG while loop
    cudaGraphConditionalHandle listCond;   // pair-list build if stale
    int useCond;
};

template <typename R> struct V4T;
template <> struct V4T<float> { typedef float4 T; };
template <> struct V4T<double> { typedef double4 T; };
template <typename R> struct V2T;
template <> struct V2T<float> { typedef float2 T; };
template <> struct V2T<double> { typedef double2 T; };
// The slot of j carried in a pair record's R lane: the int's bits in a float, its value in a double.
__device__ __forceinline__ float slotAsReal(int js, float) { return __int_as_float(js); }
__device__ __forceinline__ double slotAsReal(int js, double) { return (double) js; }
__device__ __forceinline__ int realAsSlot(float v) { return __float_as_int(v); }
__device__ __forceinline__ int realAsSlot(double v) { return (int) v; }
template <typename R> struct CplxT;
template <> struct CplxT<float> { typedef cufftComplex T; };
template <> struct CplxT<double> { typedef cufftDoubleComplex T; };

__device__ __forceinline__ float fexp(float x) { return expf(x); }
__device__ __forceinline__ double fexp(double x) { return exp(x); }
__device__ __forceinline__ float ferf(float x) { return erff(x); }
__device__ __forceinline__ double ferf(double x) { return erf(x); }
__device__ __forceinline__ float ferfc(float x) { return erfcf(x); }
__device__ __forceinline__ double ferfc(double x) { return erfc(x); }
__device__ __forceinline__ float fsqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double fsqrt(double x) { return sqrt(x); }

// B_0..B_{NMAX-1} of erf(a r)/r: 15-term series for (a r)^2 < 1, else the upward recursion
// (the formulas of core/pgm_math.h:31-61, evaluated in precision R).
template <typename R, int NMAX>
__device__ __forceinline__ void erfKernels(R a, R r, R* B) {
    const R x = a * r, s = x * x;
    const R c0 = R(2) * a / R(SQRT_PI), a2 = R(2) * a * a;
    if (s < R(1)) {
        R t[15];
        t[0] = R(1);
#pragma unroll
        for (int m = 1; m < 15; m++)
            t[m] = t[m - 1] * (-s) * R(1.0 / m);
        R pw = R(1);
#pragma unroll
        for (int k = 0; k < NMAX; k++) {
            R sum = R(0);
#pragma unroll
            for (int m = 14; m >= 0; m--)
                sum += t[m] * R(1.0 / (2 * m + 2 * k + 1));
            B[k] = c0 * pw * sum;
            pw *= a2;
        }
    } else {
        const R c = c0 * fexp(-s), ir2 = R(1) / (r * r);
        B[0] = ferf(x) / r;
        R pw = R(1);
#pragma unroll
        for (int k = 1; k < NMAX; k++) {
            B[k] = (R(2 * k - 1) * B[k - 1] - pw * c) * ir2;
            pw *= a2;
        }
    }
}

// B_n of erfc(a r)/r by the all-positive recursion (core/pgm_math.h:63-75).
template <typename R, int NMAX>
__device__ __forceinline__ void erfcKernels(R a, R r, R* B) {
    const R x = a * r, c = (R(2) / R(SQRT_PI)) * a * fexp(-x * x), ir2 = R(1) / (r * r), a2 = R(2) * a * a;
    B[0] = ferfc(x) / r;
    R pw = R(1);
#pragma unroll
    for (int k = 1; k < NMAX; k++) {
        B[k] = (R(2 * k - 1) * B[k - 1] + pw * c) * ir2;
        pw *= a2;
    }
}

// PME direct-space pair kernels G_n = B_n[erf(a r)/r] - B_n[erf(beta r)/r], n < NMAX: series difference for
// a r < 1, erfc form Bc(beta) - Bc(a) elsewhere (core/pgm_math.h:77-93).
template <typename R, int NMAX>
__device__ __forceinline__ void pairKernels(R a, R beta, R r, R* G) {
    R B[NMAX];
    if (a * r < R(1)) {
        erfKernels<R, NMAX>(a, r, G);
        erfKernels<R, NMAX>(beta, r, B);
    } else {
        erfcKernels<R, NMAX>(beta, r, G);
        erfcKernels<R, NMAX>(a, r, B);
    }
#pragma unroll
    for (int k = 0; k < NMAX; k++)
        G[k] -= B[k];
}

// Cardinal B-spline values M_p(fr + j), first and second derivatives on points base - j, j < p
// (the recursion of core/pgm_core.cpp:131-150).  Unrolled to MAXP with runtime guards so that the arrays
// stay in registers.
template <typename R>
__device__ __forceinline__ void bspline(R fr, int p, R* th, R* dth, R* d2th) {
    R M[MAXP + 1], M1[MAXP + 1], M2[MAXP + 1];
#pragma unroll
    for (int j = 0; j <= MAXP; j++) {
        M[j] = (j == 0) ? R(1) : R(0);
        M1[j] = M[j];
        M2[j] = M[j];
    }
#pragma unroll
    for (int k = 2; k <= MAXP; k++) {
        if (k <= p) {
            const R inv = R(1) / R(k - 1);
#pragma unroll
            for (int j = k - 1; j >= 0; j--) {
                const R cur = (j < k - 1) ? M[j] : R(0);
                const R prev = (j > 0) ? M[j - 1] : R(0);
                M[j] = ((fr + R(j)) * cur + (R(k) - fr - R(j)) * prev) * inv;
            }
            if (k == p - 2) {
#pragma unroll
                for (int j = 0; j <= MAXP; j++)
                    M2[j] = M[j];
            }
            if (k == p - 1) {
#pragma unroll
                for (int j = 0; j <= MAXP; j++)
                    M1[j] = M[j];
            }
        }
    }
#pragma unroll
    for (int j = 0; j < MAXP; j++) {
        if (j < p) {
            th[j] = M[j];
            dth[j] = M1[j] - (j > 0 ? M1[j - 1] : R(0));
            d2th[j] = M2[j] - R(2) * (j > 0 ? M2[j - 1] : R(0)) + (j > 1 ? M2[j - 2] : R(0));
        }
    }
}

// Minimum image of v in a reduced triclinic box, c then b then a, rounding halves away from zero, every
// product and difference rounded separately (core/pgm_math.h:153-160 evaluated without fused multiply-adds,
// so that the pair set is the reference's bit for bit).  k receives the image counts.
__device__ __forceinline__ void minImageExact(double* v, const double* H, int* k) {
#pragma unroll
    for (int c = 2; c >= 0; c--) {
        const double kk = round(__ddiv_rn(v[c], H[4 * c]));
        k[c] = (int) kk;
#pragma unroll
        for (int j = 0; j < 3; j++)
            v[j] = __dsub_rn(v[j], __dmul_rn(kk, H[3 * c + j]));
    }
}

__device__ __forceinline__ double dot3exact(const double* x) {
    return __dadd_rn(__dadd_rn(__dmul_rn(x[0], x[0]), __dmul_rn(x[1], x[1])), __dmul_rn(x[2], x[2]));
}

// Pair-list entry: slot of j (23 bits) and the image shift w (3 x 3 bits, -4..3) with x = pw_i - pw_j - w.H.
__device__ __forceinline__ uint32_t packEntry(int jslot, int w0, int w1, int w2) {
    return (uint32_t) jslot | ((uint32_t) (w0 + 4) << 23) | ((uint32_t) (w1 + 4) << 26) | ((uint32_t) (w2 + 4) << 29);
}
__device__ __forceinline__ int entrySlot(uint32_t e) { return (int) (e & 0x7FFFFFu); }
__device__ __forceinline__ void entryShift(uint32_t e, const double* H, double* sh) {
    const double w0 = (double) ((int) ((e >> 23) & 7u) - 4), w1 = (double) ((int) ((e >> 26) & 7u) - 4),
                 w2 = (double) ((int) ((e >> 29) & 7u) - 4);
    sh[0] = w0 * H[0] + w1 * H[3] + w2 * H[6];
    sh[1] = w1 * H[4] + w2 * H[7];
    sh[2] = w2 * H[8];
}

// Shuffle mask of the GS-lane group holding this thread (GS a power of two <= 32).
template <int GS> __device__ __forceinline__ unsigned groupMask() {
    return GS == 32 ? 0xffffffffu : (((1u << GS) - 1u) << ((threadIdx.x & 31) & ~(GS - 1)));
}

// Deterministic block reduction of NV doubles (sum, or max where the bit of maxMask is set); valid in
// thread 0.  Fixed shuffle and warp order, so repeated runs give identical bits.
template <int NV>
__device__ __forceinline__ void blockReduce(double* v, unsigned maxMask) {
    __shared__ double red[32][NV];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double other = __shfl_down_sync(0xffffffffu, v[k], o);
            v[k] = ((maxMask >> k) & 1u) ? fmax(v[k], other) : v[k] + other;
        }
    }
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; k++)
            red[warp][k] = v[k];
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) {
            double s = red[0][k];
            for (int w = 1; w < nw; w++)
                s = ((maxMask >> k) & 1u) ? fmax(s, red[w][k]) : s + red[w][k];
            v[k] = s;
        }
    }
    __syncthreads();
}

// Writes this chunk's reduced values and returns true in the last chunk of its system to finish (all
// threads), with the system's totals (chunks summed in chunk order, one value per thread) in tot for every
// thread of that block.
template <int NV>
__device__ __forceinline__ bool chunkFinish(const Dev& dv, int chunk, int s, double* v, unsigned maxMask, double* tot) {
    __shared__ int isLast;
    __shared__ double stot[NV];
    blockReduce<NV>(v, maxMask);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++)
            dv.partial[(size_t) chunk * 16 + k] = v[k];
        // the arrival releases this thread's partials and, for the last chunk, acquires the others' (the block
        // barrier below passes them on to the block's threads)
        int t;
        asm volatile("atom.add.acq_rel.gpu.global.s32 %0, [%1], 1;" : "=r"(t) : "l"(&dv.sysCounter[s]) : "memory");
        isLast = (t == dv.sys[s].chunkCount - 1);
    }
    __syncthreads();
    if (!isLast)
        return false;
    const SysDev& S = dv.sys[s];
    // the system's chunk partials in a fixed order: value k = tid mod 16, chunk group tid / 16 takes chunks
    // group, group + 16, ...; the groups' sums then in group order (deterministic)
    __shared__ double sgrp[CHUNK / 16][NV];
    {
        const int k = threadIdx.x & 15, grp = threadIdx.x >> 4;
        if (k < NV) {
            const bool isMax = (maxMask >> k) & 1u;
            double acc = 0.0;
#pragma unroll 4
            for (int c = grp; c < S.chunkCount; c += CHUNK / 16) {
                const double val = __ldcg(&dv.partial[(size_t) (S.chunkFirst + c) * 16 + k]);
                acc = isMax ? fmax(acc, val) : acc + val;
            }
            sgrp[grp][k] = acc;
        }
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        const int k = threadIdx.x;
        const bool isMax = (maxMask >> k) & 1u;
        double acc = 0.0;
        for (int g = 0; g < CHUNK / 16; g++)
            acc = isMax ? fmax(acc, sgrp[g][k]) : acc + sgrp[g][k];
        stot[k] = acc;
    }
    __syncthreads();
    if (threadIdx.x == 0)
        dv.sysCounter[s] = 0;
#pragma unroll
    for (int k = 0; k < NV; k++)
        tot[k] = stot[k];
    return true;
}

}  // namespace pgmb200
