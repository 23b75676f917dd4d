// pgm_b200 engine: host orchestration of one or many periodic pGM systems on one B200.
//
// One evaluation is one CUDA graph: preparation and the cell list, the pair list, the permanent field, the
// initial guess, the CG loop as a conditional while node (its body: spread || pair pass, FFT chain, gather,
// two CG kernels), and the final pass.  Kernels are in kernels.cuh; the C ABI is in capi.cu.
#include "kernels.cuh"
#include "persistent.cuh"
#include "adjoint.cuh"
#include "planes.cuh"
#include "lines.cuh"
#include "tiles.cuh"
#include "pgm_engine.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

namespace pgmb200 {

#define CU(call)                                                                                             \
    do {                                                                                                     \
        cudaError_t e_ = (call);                                                                             \
        if (e_ != cudaSuccess)                                                                               \
            throw std::runtime_error(std::string("pgm_b200: ") + #call + ": " + cudaGetErrorString(e_));      \
    } while (0)
#define CUFFT(call)                                                                                          \
    do {                                                                                                     \
        cufftResult r_ = (call);                                                                             \
        if (r_ != CUFFT_SUCCESS)                                                                             \
            throw std::runtime_error(std::string("pgm_b200: ") + #call + " failed with cufftResult " +        \
                                     std::to_string((int) r_));                                              \
    } while (0)

namespace {

// Device allocation owned by the engine.
struct Buf {
    void* p = nullptr;
    size_t bytes = 0;
    void ensure(size_t b) {
        if (b <= bytes && p)
            return;
        release();
        if (b == 0)
            b = 16;
        CU(cudaMalloc(&p, b));
        bytes = b;
    }
    void release() {
        if (p)
            cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <class T> T* as() const { return (T*) p; }
};

// The B-spline moduli b(m) = |sum_k M_p(k + 1) exp(2 pi i m k / K)|^2, m < K, of the smooth-PME influence
// function, with the reference's convention that a modulus below 1e-7 (an interpolation zero, odd p at the
// Nyquist index) takes the mean of its two neighbours (core/pgm_math.h:98-126 defines the quantity).
//   * M_p at the integer knots comes from the closed form M_p(x) = 1/(p-1)! sum_{j<x} (-1)^j C(p, j) (x - j)^(p-1),
//     summed exactly in 128-bit integers (p <= 12 keeps every term below 2^63) and divided once, so every
//     knot value is correctly rounded;
//   * M_p(k + 1) vanishes for k >= p - 1, so the transform runs over the support only, and each phase m k is
//     reduced modulo K before it becomes an angle, which keeps the angles exact for large m k.
std::vector<double> bsplineModuli(int K, int p) {
    if (p < 2 || p > MAXP)
        throw std::invalid_argument("pgm_b200: spline order outside 2.." + std::to_string(MAXP));
    auto binom = [](int nn, int kk) {
        __int128 c = 1;
        for (int t = 1; t <= kk; t++)
            c = c * (nn - kk + t) / t;
        return c;
    };
    __int128 factorial = 1;
    for (int t = 2; t < p; t++)
        factorial *= t;
    std::vector<double> knot(p, 0.0);   // knot[x] = M_p(x), x = 1 .. p - 1
    for (int x = 1; x < p; x++) {
        __int128 acc = 0;
        for (int j = 0; j < x; j++) {
            __int128 pw = 1;
            for (int t = 0; t < p - 1; t++)
                pw *= (x - j);
            acc += ((j & 1) ? -1 : 1) * binom(p, j) * pw;
        }
        knot[x] = (double) ((long double) acc / (long double) factorial);
    }
    std::vector<double> modulus(K);
    for (int m = 0; m < K; m++) {
        double re = 0.0, im = 0.0;
        for (int k = 0; k + 1 < p && k < K; k++) {   // (a grid smaller than the support is not aliased)
            const long long phase = ((long long) m * k) % K;
            const double ang = 2.0 * PI_D * (double) phase / (double) K;
            re += knot[k + 1] * std::cos(ang);
            im += knot[k + 1] * std::sin(ang);
        }
        modulus[m] = re * re + im * im;
    }
    std::vector<double> fixed(modulus);
    for (int m = 0; m < K; m++)
        if (modulus[m] < 1e-7)
            fixed[m] = 0.5 * (modulus[m == 0 ? K - 1 : m - 1] + modulus[m + 1 == K ? 0 : m + 1]);
    return fixed;
}

// H^-1 by cofactors and |det H| (core/pgm_core.cpp:94-111).
void boxInverse(const double* H, double* inv, double& volume) {
    const double det = H[0] * (H[4] * H[8] - H[5] * H[7]) - H[1] * (H[3] * H[8] - H[5] * H[6]) +
                       H[2] * (H[3] * H[7] - H[4] * H[6]);
    volume = std::fabs(det);
    inv[0] = (H[4] * H[8] - H[5] * H[7]) / det;
    inv[1] = (H[2] * H[7] - H[1] * H[8]) / det;
    inv[2] = (H[1] * H[5] - H[2] * H[4]) / det;
    inv[3] = (H[5] * H[6] - H[3] * H[8]) / det;
    inv[4] = (H[0] * H[8] - H[2] * H[6]) / det;
    inv[5] = (H[2] * H[3] - H[0] * H[5]) / det;
    inv[6] = (H[3] * H[7] - H[4] * H[6]) / det;
    inv[7] = (H[1] * H[6] - H[0] * H[7]) / det;
    inv[8] = (H[0] * H[4] - H[1] * H[3]) / det;
}

template <class T> void upload(Buf& b, const std::vector<T>& v, cudaStream_t st) {
    b.ensure(std::max<size_t>(v.size() * sizeof(T), 16));
    if (!v.empty())
        CU(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
}

int envInt(const char* name, int def) {
    const char* v = std::getenv(name);
    return v ? std::atoi(v) : def;
}

}  // namespace

struct Engine::Impl {
    Settings s;
    cudaStream_t st = nullptr, side = nullptr;
    cudaStream_t callerStream = nullptr;
    cudaEvent_t evFork = nullptr, evJoin = nullptr, evCaller = nullptr, evDone = nullptr, evPerm = nullptr;
    int devId = 0;

    // systems and atoms (host)
    int n = 0, nsys = 0, numGlobal = 0;
    std::vector<int> atomBegin;                 // nsys + 1
    std::vector<double> sysCutoff, sysBeta;
    std::vector<std::array<int, 3>> sysK;
    std::vector<double> q, radius, alpha;
    std::vector<int> atomSys, globalIdx;
    std::vector<int> covAtom, covPartner;       // global atom indices
    std::vector<double> covStrength;
    std::vector<SysDev> sysHost;
    std::vector<int> chunkSys, chunkBegin, chunkEnd;
    std::vector<double> moduliHost;
    std::map<int, int> moduliOff;
    struct FftGroup {
        int K[3];
        int first, count;   // systems (contiguous in grid storage)
        long long gridOff, specOff;
        cufftHandle r2c = 0, c2r = 0;
        cufftHandle r2c2d = 0, c2r2d = 0;   // 2D plans over the x-planes (split transforms)
    };
    std::vector<FftGroup> groups;
    std::vector<int> sysOrder;   // unused (systems stored in caller order within their group)
    long long gridTotal = 0, specTotal = 0;
    int totalCells = 0, cellCapacity = 0;
    int cap = 0;
    int convBlocks = 1;
    // field-pass transforms: TF_CUFFT cuFFT 3D plans + influence product; TF_CLUSTER one cluster kernel;
    // TF_SPLIT cuFFT 2D plans over the x-planes + one kernel for the x-lines with the influence product;
    // TF_GRID one cooperative kernel, a block per x-plane
    // TF_PCG the grid kernel for the field passes outside the CG loop, and the whole CG loop as one persistent
    //   cooperative kernel (mixed precision, one system)
    enum { TF_CUFFT = 0, TF_CLUSTER = 1, TF_SPLIT = 2, TF_GRID = 3, TF_PCG = 4 };
    int tfMode = TF_CUFFT;     // in use
    int tfWant = TF_CUFFT;     // the caller's choice (setTransforms)
    bool fuseCgA = true;       // single system: A p and alph in the CG gather's epilogue (else a separate kernel)
    bool clusterOk = false;    // the systems' grids and the GPU allow the cluster kernel
    bool splitOk = false;      // the systems' x extents allow the x-line kernel
    bool gridOk = false;       // the systems' grids and the GPU allow the grid-transform kernel
    bool gridEnergyOk = false; // ... and its variant with the reciprocal energy for the final pass
    bool pcgOk = false;        // the persistent CG kernel applies (mixed, one system, grid kernel, order 6)
    bool planesOk = false;     // the plane-owner spread and gather apply (mixed, one system, order 6)
    int pmeWant = 0;           // the caller's choice of spread / gather kernels: 0 a warp per atom, 1 plane tiles,
                               // 2 float4 lines
    int planeNyc = 1;          // row chunks per x-plane of the plane-owner kernels
    size_t planeSmem = 0;
    int pcgBlocks = 0;         // its blocks (one per SM)
    size_t pcgSmem = 0;
    int fftcBuf = 0, fftcC = 16, fftgBuf = 0, maxK0 = 0;
    int fftgKc = 0;            // the grid transforms' compile-time size (every grid fftgKc^3), or 0
    size_t fftgSmem = 0;
    int maxLineBlocks = 0;
    size_t fftcSmem = 0;
    bool configured = false, atomsSet = false;

    // device
    Buf dSys, dAtomSys, dQ, dR, dAlpha, dPosIn, dWrap, dCellOf, dCellRank, dBase, dFr, dCellCount, dCellStart,
        dSlotAtom, dSlotTmp, dPosS, dOrigS, dWrapS, dSpl, dBaseS, dRadS, dList, dListCount, dPairA, dPairB, dPairC, dFlags, dDS, dPerm, dMu, dDtot, dB, dX, dRv, dZ, dP, dAp,
        dDS2, dEpair2, dErec2, dGrid2, dGridFix, dGridFix2,
        dScal, dPartial, dGPartial, dHrec, dFm, dPmeRec, dPmeBins, dSrcW, dGPart, dPcgPartial, dBinCount, dActive, dActSys, dSysCounter, dEpair, dErec, dFpair, dSpair, dFrec, dEtot, dFin, dPot, dForces, dResults,
        dConvPartial, dConvOff, dGrid, dSpec, dInfl, dTwiddle, dModuli, dCovAtom, dCovPartner, dCovStrength, dCovByAtomOff,
        dCovByAtom, dCovByPartnerOff, dCovByPartner, dChunkSys, dChunkBegin, dChunkEnd, dHist, dGlobal, dCtl,
        dGradQ, dGradR, dSList, dSListCount, dPosBuild, dAtomSlot, dCandStart, dCandJ, dCandT, dGv, dSkipStart, dSkipJ;
    // FP64 shadow of the mixed path for the iterative refinement
    Buf dPairBd, dDSd, dGridD, dSpecD, dInflD, dSplD, dB64, dXsave;
    std::vector<std::pair<cufftHandle, cufftHandle>> plans64;
    // pinned host staging
    double* hPos = nullptr;
    float* hPosF = nullptr;
    double* hForces = nullptr;
    double* hResults = nullptr;
    int* hFlags = nullptr;
    Ctl* hCtl = nullptr;
    SysDev* hSys = nullptr;
    size_t hPosCap = 0, hSysCap = 0, hResCap = 0;

    // graph
    cudaGraphExec_t exec = nullptr;
    bool useGraph = true;
    int pairGS = 8;
    int pairSmem = 0;

    // predictor history: NHIST slots, newest at head
    static constexpr int NHIST = 5;
    int histHead = 0, histCount = 0;
    int pendingSlot = -1;

    // Verlet list state: valid once built; kept while the boxes stay those of the build and no atom has moved by
    // more than half the skin (checked on the device at every evaluation)
    bool listValid = false;
    bool externalList = false;   // the caller's candidates (setCandidates) in place of the cell search
    // the combination-rule GVDW (setGvdw)
    bool gvdwOn = false, gvdwSlater = false;
    double rvdw = 0.0;
    double gvC[GVDW_TERMS] = {};
    std::vector<double> buildBoxes;    // nsys * 9, the boxes of the last build
    std::vector<double> launchBoxes;   // nsys * 9, the boxes of the evaluation in flight
    cudaGraph_t listBody = nullptr;    // body of the build's conditional node while capturing
    int graphCells = -1;               // cell count the graph was captured with
    int graphTiles[2] = {-1, -1};      // tile groups and capacity the graph was captured with
    bool graphDual = false;            // the graph's first pass is the dual one (a predicted guess)
    // CG iterations captured ahead of the while node (one system): the fewest iterations of the last 4
    // evaluations, so that an evaluation like those runs its loop without the while node's per-iteration cost
    // and the node only takes what is left (an evaluation that converges earlier gates the rest off).  The graph
    // is captured again after 3 evaluations when fewer iterations would do, or at least two more; one more only
    // after 16 (so that counts that alternate do not recapture every few evaluations).
    int graphUnroll = 0;               // iterations unrolled in the captured graph
    int unrollWant = 0;                // what the next capture unrolls
    int recentIt[4] = {0};             // iteration counts of the last evaluations (ring)
    int recentCount = 0, evalsSinceCapture = 0;
    bool graphLoop = false;            // the captured graph holds the CG loop's while node
    bool unrollStale() const {
        if (!graphLoop || nsys != 1 || evalsSinceCapture < 3 || unrollWant == graphUnroll)
            return false;
        return unrollWant < graphUnroll || unrollWant >= graphUnroll + 2 || evalsSinceCapture >= 16;
    }
    bool capturing = false;

    // last evaluation
    std::vector<double> lastResults;   // nsys * NRES
    bool haveResult = false;
    long builds = 0;
    bool lastBuilt = false;   // the last evaluation built the Verlet list
    std::vector<double> forcesHostCache;
    bool launched = false;
    int launchedMode = 0;

    Impl() {}
    ~Impl() { teardown(); }

    void teardown() {
        if (exec)
            cudaGraphExecDestroy(exec);
        exec = nullptr;
        for (auto& g : groups) {
            if (g.r2c)
                cufftDestroy(g.r2c);
            if (g.c2r)
                cufftDestroy(g.c2r);
            if (g.r2c2d)
                cufftDestroy(g.r2c2d);
            if (g.c2r2d)
                cufftDestroy(g.c2r2d);
        }
        groups.clear();
        for (auto& pl : plans64) {
            cufftDestroy(pl.first);
            cufftDestroy(pl.second);
        }
        plans64.clear();
        Buf* all[] = {&dSys, &dAtomSys, &dQ, &dR, &dAlpha, &dPosIn, &dWrap, &dCellOf, &dCellRank, &dBase, &dFr,
                      &dCellCount, &dCellStart, &dSlotAtom, &dSlotTmp, &dPosS, &dOrigS, &dWrapS, &dSpl, &dBaseS, &dRadS, &dList, &dListCount, &dPairA, &dPairB, &dPairC, &dFlags, &dDS,
                      &dDS2, &dEpair2, &dErec2, &dGrid2, &dGridFix, &dGridFix2,
                      &dPerm, &dMu, &dDtot, &dB, &dX, &dRv, &dZ, &dP, &dAp, &dScal, &dPartial, &dGPartial, &dHrec, &dFm, &dPmeRec, &dPmeBins, &dSrcW, &dGPart,
                      &dPcgPartial, &dBinCount, &dActive, &dActSys, &dSysCounter, &dEpair,
                      &dErec, &dFpair, &dSpair, &dFrec, &dEtot, &dFin, &dPot, &dForces, &dResults, &dConvPartial,
                      &dConvOff, &dGrid, &dSpec, &dInfl, &dTwiddle, &dModuli, &dCovAtom, &dCovPartner, &dCovStrength,
                      &dCovByAtomOff, &dCovByAtom, &dCovByPartnerOff, &dCovByPartner, &dChunkSys, &dChunkBegin,
                      &dChunkEnd, &dHist, &dGlobal, &dCtl, &dGradQ, &dGradR, &dPairBd, &dDSd, &dGridD, &dSpecD,
                      &dInflD, &dSplD, &dB64, &dXsave, &dSList, &dSListCount, &dPosBuild, &dAtomSlot, &dCandStart,
                      &dCandJ, &dCandT, &dGv, &dSkipStart, &dSkipJ};
        for (Buf* b : all)
            b->release();
        if (hPos) cudaFreeHost(hPos);
        if (hPosF) cudaFreeHost(hPosF);
        if (hForces) cudaFreeHost(hForces);
        if (hResults) cudaFreeHost(hResults);
        if (hFlags) cudaFreeHost(hFlags);
        if (hCtl) cudaFreeHost(hCtl);
        if (hSys) cudaFreeHost(hSys);
        hPos = nullptr;
        hPosF = nullptr;
        hForces = nullptr;
        hResults = nullptr;
        hFlags = nullptr;
        hCtl = nullptr;
        hSys = nullptr;
        hPosCap = hSysCap = hResCap = 0;
        if (st) cudaStreamDestroy(st);
        if (side) cudaStreamDestroy(side);
        if (evFork) cudaEventDestroy(evFork);
        if (evJoin) cudaEventDestroy(evJoin);
        if (evCaller) cudaEventDestroy(evCaller);
        if (evDone) cudaEventDestroy(evDone);
        if (evPerm) cudaEventDestroy(evPerm);
        st = side = nullptr;
        evFork = evJoin = evCaller = evDone = evPerm = nullptr;
    }

    bool mixed() const { return s.precision != 0; }
    size_t realSize() const { return mixed() ? sizeof(float) : sizeof(double); }

    void init(const Settings& settings) {
        s = settings;
        if (s.order < 3 || s.order > MAXP)
            throw std::invalid_argument("pgm_b200: PME order must be 3..12");
        if (s.device >= 0)
            CU(cudaSetDevice(s.device));
        CU(cudaGetDevice(&devId));
        CU(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        // the side stream (list build, transforms) carries the critical path beside the pair passes: it runs at
        // the highest priority, in the graph too (node priorities)
        int prLeast = 0, prGreatest = 0;
        CU(cudaDeviceGetStreamPriorityRange(&prLeast, &prGreatest));
        CU(cudaStreamCreateWithPriority(&side, cudaStreamNonBlocking, prGreatest));
        CU(cudaEventCreateWithFlags(&evFork, cudaEventDisableTiming));
        CU(cudaEventCreateWithFlags(&evJoin, cudaEventDisableTiming));
        CU(cudaEventCreateWithFlags(&evCaller, cudaEventDisableTiming));
        CU(cudaEventCreateWithFlags(&evDone, cudaEventDisableTiming));
        CU(cudaEventCreateWithFlags(&evPerm, cudaEventDisableTiming));
        CU(cudaMallocHost((void**) &hFlags, 16 * sizeof(int)));
        CU(cudaMallocHost((void**) &hCtl, sizeof(Ctl)));
        useGraph = envInt("PGM_B200_NO_GRAPH", 0) == 0;
        pairGS = envInt("PGM_B200_PAIR_LANES", 32);
        tfWant = envInt("PGM_B200_TRANSFORMS", TF_CUFFT);
        fuseCgA = envInt("PGM_B200_FUSED_CG", 1) != 0;
        // the field pair pass runs beside the transforms of the same pass: optionally at most pairBlocks of its
        // blocks per SM (a shared-memory reservation it does not use), so that the transform kernels find room
        const int pairBlocks = envInt("PGM_B200_PAIR_BLOCKS", 0);
        int smPerSM = 0, smPerBlock = 0;
        CU(cudaDeviceGetAttribute(&smPerSM, cudaDevAttrMaxSharedMemoryPerMultiprocessor, devId));
        CU(cudaDeviceGetAttribute(&smPerBlock, cudaDevAttrMaxSharedMemoryPerBlockOptin, devId));
        pairSmem = pairBlocks > 0 ? std::min(smPerBlock, smPerSM / (pairBlocks + 1) + 1024) : 0;
        if (pairSmem > 0)
            for (auto f : {(const void*) k_pair_field<float, false, 32>, (const void*) k_pair_field<float, true, 32>,
                           (const void*) k_pair_field<double, false, 32>, (const void*) k_pair_field<double, true, 32>,
                           (const void*) k_pair_field<float, false, 16>, (const void*) k_pair_field<float, true, 16>,
                           (const void*) k_pair_field<double, false, 16>, (const void*) k_pair_field<double, true, 16>,
                           (const void*) k_pair_field<float, false, 8>, (const void*) k_pair_field<float, true, 8>,
                           (const void*) k_pair_field<double, false, 8>, (const void*) k_pair_field<double, true, 8>,
                           (const void*) k_pair_field<float, false, 4>, (const void*) k_pair_field<float, true, 4>,
                           (const void*) k_pair_field<double, false, 4>, (const void*) k_pair_field<double, true, 4>})
                CU(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, pairSmem));
        if (pairGS != 4 && pairGS != 8 && pairGS != 16 && pairGS != 32)
            pairGS = 32;
    }

    void selectDevice() {
        if (s.device >= 0)
            CU(cudaSetDevice(devId));
    }

    // ------------------------------------------------------------------------------------------ topology
    void setAtomsSingle(int nAt, const double* qq, const double* rr, const double* aa, const int* gidx, int nGlobal) {
        if (nAt <= 0 || nAt >= (1 << 23))
            throw std::invalid_argument("pgm_b200: setAtoms needs 1 .. 8388607 atoms");
        const bool sameCount = atomsSet && nsys == 1 && n == nAt;
        externalList = false;   // the candidates and the GVDW parameters hold until the next setAtoms
        gvdwOn = false;
        n = nAt;
        nsys = 1;
        atomBegin = {0, n};
        sysCutoff = {s.cutoff};
        sysBeta = {s.beta};
        sysK = {{s.grid[0], s.grid[1], s.grid[2]}};
        q.assign(qq, qq + n);
        radius.assign(rr, rr + n);
        alpha.assign(aa, aa + n);
        for (double& a : alpha)
            if (a <= 1e-9)
                a = 0.0;   // not polarizable (core/pgm_constants.h:9)
        for (int a = 0; a < 3; a++)
            if (s.grid[a] < s.order)
                throw std::invalid_argument("pgm_b200: PME grid smaller than the spline order");
        atomSys.assign(n, 0);
        numGlobal = gidx ? nGlobal : n;
        globalIdx.clear();
        if (gidx) {
            globalIdx.assign(gidx, gidx + n);
            for (int g : globalIdx)
                if (g < 0 || g >= numGlobal)
                    throw std::invalid_argument("pgm_b200: global index out of range");
        }
        covAtom.clear();
        covPartner.clear();
        covStrength.clear();
        if (!sameCount)
            resetHistoryState();
        atomsSet = true;
        configure();
    }

    void setSystemsBatch(int ns, const int* count, const double* cut, const double* bet, const int* grd,
                         const double* qq, const double* rr, const double* aa, const int* covCount, const int* ca,
                         const int* cp, const double* cs) {
        if (ns <= 0)
            throw std::invalid_argument("pgm_b200: setSystems needs at least one system");
        nsys = ns;
        externalList = false;
        gvdwOn = false;
        atomBegin.assign(ns + 1, 0);
        for (int k = 0; k < ns; k++) {
            if (count[k] <= 0)
                throw std::invalid_argument("pgm_b200: every system needs at least one atom");
            atomBegin[k + 1] = atomBegin[k] + count[k];
        }
        n = atomBegin[ns];
        if (n >= (1 << 23))
            throw std::invalid_argument("pgm_b200: at most 8388607 atoms in all systems together");
        sysCutoff.assign(cut, cut + ns);
        sysBeta.assign(bet, bet + ns);
        sysK.resize(ns);
        for (int k = 0; k < ns; k++)
            for (int a = 0; a < 3; a++) {
                sysK[k][a] = grd[3 * k + a];
                if (sysK[k][a] < s.order)
                    throw std::invalid_argument("pgm_b200: PME grid smaller than the spline order");
            }
        q.assign(qq, qq + n);
        radius.assign(rr, rr + n);
        alpha.assign(aa, aa + n);
        for (double& a : alpha)
            if (a <= 1e-9)
                a = 0.0;
        atomSys.resize(n);
        for (int k = 0; k < ns; k++)
            for (int i = atomBegin[k]; i < atomBegin[k + 1]; i++)
                atomSys[i] = k;
        numGlobal = n;
        globalIdx.clear();
        covAtom.clear();
        covPartner.clear();
        covStrength.clear();
        int m = 0;
        for (int k = 0; k < ns; k++)
            for (int c = 0; c < covCount[k]; c++, m++) {
                const int nk = atomBegin[k + 1] - atomBegin[k];
                if (ca[m] < 0 || ca[m] >= nk || cp[m] < 0 || cp[m] >= nk || ca[m] == cp[m])
                    throw std::invalid_argument("pgm_b200: covalent dipole indices out of range");
                covAtom.push_back(atomBegin[k] + ca[m]);
                covPartner.push_back(atomBegin[k] + cp[m]);
                covStrength.push_back(cs[m]);
            }
        resetHistoryState();
        atomsSet = true;
        configure();
        uploadCovalent();
    }

    void setCovalentSingle(int ncov, const int* a, const int* p, const double* c) {
        if (!atomsSet)
            throw std::logic_error("pgm_b200: setCovalent before setAtoms");
        covAtom.clear();
        covPartner.clear();
        covStrength.clear();
        for (int m = 0; m < ncov; m++) {
            if (a[m] < 0 || a[m] >= n || p[m] < 0 || p[m] >= n || a[m] == p[m])
                throw std::invalid_argument("pgm_b200: covalent dipole indices out of range");
            covAtom.push_back(a[m]);
            covPartner.push_back(p[m]);
            covStrength.push_back(c[m]);
        }
        uploadCovalent();
    }

    void uploadCovalent() {
        const int ncov = (int) covAtom.size();
        std::vector<int> byAtomOff(n + 1, 0), byPartnerOff(n + 1, 0), byAtom(ncov), byPartner(ncov);
        for (int m = 0; m < ncov; m++) {
            byAtomOff[covAtom[m] + 1]++;
            byPartnerOff[covPartner[m] + 1]++;
        }
        for (int i = 0; i < n; i++) {
            byAtomOff[i + 1] += byAtomOff[i];
            byPartnerOff[i + 1] += byPartnerOff[i];
        }
        std::vector<int> fa(byAtomOff.begin(), byAtomOff.end() - 1), fp(byPartnerOff.begin(), byPartnerOff.end() - 1);
        for (int m = 0; m < ncov; m++) {
            byAtom[fa[covAtom[m]]++] = m;
            byPartner[fp[covPartner[m]]++] = m;
        }
        upload(dCovAtom, covAtom, st);
        upload(dCovPartner, covPartner, st);
        upload(dCovStrength, covStrength, st);
        upload(dCovByAtomOff, byAtomOff, st);
        upload(dCovByAtom, byAtom, st);
        upload(dCovByPartnerOff, byPartnerOff, st);
        upload(dCovByPartner, byPartner, st);
        CU(cudaStreamSynchronize(st));
    }

    void resetHistoryState() {
        histHead = 0;
        histCount = 0;
    }

    // Allocations, tables and FFT plans for the current atoms/systems.
    void configure() {
        if (exec) {
            cudaGraphExecDestroy(exec);
            exec = nullptr;
        }
        for (auto& g : groups) {
            if (g.r2c) cufftDestroy(g.r2c);
            if (g.c2r) cufftDestroy(g.c2r);
            if (g.r2c2d) cufftDestroy(g.r2c2d);
            if (g.c2r2d) cufftDestroy(g.c2r2d);
        }
        groups.clear();
        for (auto& pl : plans64) {
            cufftDestroy(pl.first);
            cufftDestroy(pl.second);
        }
        plans64.clear();
        // systems grouped by grid shape; grid storage group after group
        std::map<std::array<int, 3>, std::vector<int>> byShape;
        for (int k = 0; k < nsys; k++)
            byShape[sysK[k]].push_back(k);
        sysHost.assign(nsys, SysDev());
        gridTotal = specTotal = 0;
        moduliHost.clear();
        moduliOff.clear();
        int maxSpec = 0;
        for (auto& kv : byShape) {
            FftGroup g;
            for (int a = 0; a < 3; a++)
                g.K[a] = kv.first[a];
            // every group's grid and spectrum start 256-byte aligned (cuFFT's vector loads need aligned bases)
            gridTotal = (gridTotal + 63) / 64 * 64;
            specTotal = (specTotal + 31) / 32 * 32;
            g.gridOff = gridTotal;
            g.specOff = specTotal;
            g.count = (int) kv.second.size();
            g.first = kv.second[0];
            const int gn = g.K[0] * g.K[1] * g.K[2], sn = g.K[0] * g.K[1] * (g.K[2] / 2 + 1);
            for (int k : kv.second) {
                SysDev& S = sysHost[k];
                for (int a = 0; a < 3; a++)
                    S.K[a] = g.K[a];
                S.gridOff = gridTotal;
                S.specOff = specTotal;
                S.gridN = gn;
                S.specN = sn;
                gridTotal += gn;
                specTotal += sn;
            }
            maxSpec = std::max(maxSpec, sn);
            for (int a = 0; a < 3; a++)
                if (!moduliOff.count(g.K[a])) {
                    moduliOff[g.K[a]] = (int) moduliHost.size();
                    std::vector<double> m = bsplineModuli(g.K[a], s.order);
                    moduliHost.insert(moduliHost.end(), m.begin(), m.end());
                }
            groups.push_back(g);
        }
        // the FFT groups need their systems contiguous in storage: systems of one shape are stored in index
        // order, so a group is contiguous; the plan batch covers gridOff..gridOff + count * gn
        for (auto& g : groups) {
            int dims[3] = {g.K[0], g.K[1], g.K[2]};
            const int gn = g.K[0] * g.K[1] * g.K[2], sn = g.K[0] * g.K[1] * (g.K[2] / 2 + 1);
            CUFFT(cufftPlanMany(&g.r2c, 3, dims, nullptr, 1, gn, nullptr, 1, sn, mixed() ? CUFFT_R2C : CUFFT_D2Z,
                                g.count));
            CUFFT(cufftPlanMany(&g.c2r, 3, dims, nullptr, 1, sn, nullptr, 1, gn, mixed() ? CUFFT_C2R : CUFFT_Z2D,
                                g.count));
            if (refining()) {
                cufftHandle a, b;
                CUFFT(cufftPlanMany(&a, 3, dims, nullptr, 1, gn, nullptr, 1, sn, CUFFT_D2Z, g.count));
                CUFFT(cufftPlanMany(&b, 3, dims, nullptr, 1, sn, nullptr, 1, gn, CUFFT_Z2D, g.count));
                plans64.push_back({a, b});
            }
        }
        if (std::getenv("PGM_B200_TRACE"))
            for (auto& g : groups)
                fprintf(stderr, "pgm_b200 trace: FFT group %dx%dx%d, %d systems from %d, grid offset %lld, spectrum "
                        "offset %lld\n", g.K[0], g.K[1], g.K[2], g.count, g.first, g.gridOff, g.specOff);
        convBlocks = std::max(1, std::min(512, (maxSpec + 255) / 256));
        // the field passes' transform pair with the influence product as one cluster kernel (a cluster per
        // system) when chosen (setTransforms, the autotuner) and every grid has at most FFT_MAXK points per
        // dimension with the prime factors 2, 3, 5 only; else cuFFT plans and the product kernel.  Cluster size:
        // 16 for few systems (parallelism), down to the smallest that fits shared memory for many
        auto smallK = [](int K) {
            int rad[16];
            return K <= FFT_MAXK && fftRadices(K, rad) >= 0;
        };
        clusterOk = true;
        splitOk = true;
        maxK0 = 0;
        for (int k = 0; k < nsys; k++) {
            splitOk = splitOk && smallK(sysK[k][0]);
            for (int a = 0; a < 3; a++)
                clusterOk = clusterOk && smallK(sysK[k][a]);
            maxK0 = std::max(maxK0, sysK[k][0]);
        }
        const bool allSmall = clusterOk;
        gridOk = allSmall;
        if (gridOk) {   // the grid transforms: a block per x-plane of every system, all resident at once
            fftgBuf = 0;
            for (int k = 0; k < nsys; k++)
                fftgBuf = std::max(fftgBuf, fftgBufferElems(sysHost[k].K));
            fftgSmem = (3 * (size_t) FFT_MAXK + 2 * (size_t) fftgBuf) * (mixed() ? 8 : 16);
            fftgKc = sysK[0][0];
            for (int k = 0; k < nsys; k++)
                for (int a = 0; a < 3; a++)
                    fftgKc = sysK[k][a] == fftgKc ? fftgKc : 0;
            if (fftgKc != 32 && fftgKc != 40 && fftgKc != 48 && fftgKc != 64)
                fftgKc = 0;
        }
        if (clusterOk) {
            const size_t csz = mixed() ? 8 : 16;
            int optin = 0;
            CU(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, devId));
            auto smemFor = [&](int C) {
                int m = 0;
                for (int k = 0; k < nsys; k++)
                    m = std::max(m, fftcBufferElems(sysHost[k].K, C));
                return std::make_pair(m, (3 * (size_t) FFT_MAXK + 3 * (size_t) m) * csz);
            };
            int cfit = 1;
            while (cfit < FFTC_MAXC && smemFor(cfit).second > (size_t) optin)
                cfit *= 2;
            int cwant = 1;
            while (cwant < FFTC_MAXC && cwant * nsys < 148)
                cwant *= 2;
            fftcC = std::max(cfit, cwant);
            const auto mb = smemFor(fftcC);
            fftcBuf = mb.first;
            fftcSmem = mb.second;
            clusterOk = fftcSmem <= (size_t) optin;
        }
        if (allSmall || splitOk) {   // twiddle tables of every grid size the kernels transform
            std::map<int, int> twOff;
            std::vector<double> tw;
            for (int k = 0; k < nsys; k++) {
                SysDev& S = sysHost[k];
                for (int a = 0; a < 3; a++) {
                    const int K = S.K[a];
                    S.twOff[a] = -1;
                    if (!smallK(K))
                        continue;
                    if (!twOff.count(K)) {
                        twOff[K] = (int) (tw.size() / 2);
                        for (int m = 0; m < K; m++) {   // exp(-2 pi i m / K), the angle reduced to [-pi, pi]
                            const int mm = (2 * m <= K) ? m : m - K;
                            const double ang = -2.0 * PI_D * mm / K;
                            tw.push_back(std::cos(ang));
                            tw.push_back(std::sin(ang));
                        }
                    }
                    S.twOff[a] = twOff[K];
                }
            }
            if (mixed()) {
                std::vector<float> tf(tw.begin(), tw.end());
                upload(dTwiddle, tf, st);
                if (clusterOk)
                    clusterOk = prepareCluster<float>();
                if (gridOk)
                    gridOk = prepareGrid<float>();
            } else {
                upload(dTwiddle, tw, st);
                if (clusterOk)
                    clusterOk = prepareCluster<double>();
                if (gridOk)
                    gridOk = prepareGrid<double>();
            }
        }
        if (splitOk)
            for (auto& g : groups) {   // 2D transforms of the x-planes: [x][y][z] -> [x][ky][kz]
                int dims[2] = {g.K[1], g.K[2]};
                const int pn = g.K[1] * g.K[2], sn = g.K[1] * (g.K[2] / 2 + 1);
                CUFFT(cufftPlanMany(&g.r2c2d, 2, dims, nullptr, 1, pn, nullptr, 1, sn,
                                    mixed() ? CUFFT_R2C : CUFFT_D2Z, g.count * g.K[0]));
                CUFFT(cufftPlanMany(&g.c2r2d, 2, dims, nullptr, 1, sn, nullptr, 1, pn,
                                    mixed() ? CUFFT_C2R : CUFFT_Z2D, g.count * g.K[0]));
            }
        maxLineBlocks = 0;
        for (int k = 0; k < nsys; k++)
            maxLineBlocks = std::max(maxLineBlocks, (sysK[k][1] * (sysK[k][2] / 2 + 1) + XL_LINES - 1) / XL_LINES);
        preparePlanes();
        preparePersistent();
        selectTransforms();
        // chunks
        chunkSys.clear();
        chunkBegin.clear();
        chunkEnd.clear();
        for (int k = 0; k < nsys; k++) {
            SysDev& S = sysHost[k];
            S.atomBegin = atomBegin[k];
            S.atomEnd = atomBegin[k + 1];
            S.chunkFirst = (int) chunkSys.size();
            for (int b = atomBegin[k]; b < atomBegin[k + 1]; b += CHUNK) {
                chunkSys.push_back(k);
                chunkBegin.push_back(b);
                chunkEnd.push_back(std::min(b + CHUNK, atomBegin[k + 1]));
            }
            S.chunkCount = (int) chunkSys.size() - S.chunkFirst;
            S.convBlocks = convBlocks;
            for (int a = 0; a < 3; a++)
                S.modOff[a] = moduliOff[S.K[a]];
        }
        // capacity of the pair list: density estimate at the first evaluation (grown on overflow)
        cap = 0;
        // device buffers sized by n
        const size_t R = realSize();
        dAtomSys.ensure(n * sizeof(int));
        dQ.ensure(n * 8);
        dR.ensure(n * 8);
        dAlpha.ensure(n * 8);
        dPosIn.ensure(3 * n * 8);
        dWrap.ensure(3 * n * sizeof(int));
        dCellOf.ensure(n * sizeof(int));
        dCellRank.ensure(n * sizeof(int));
        dBase.ensure(3 * n * sizeof(int));
        dFr.ensure(3 * n * 8);
        dSlotAtom.ensure(n * sizeof(int));
        dSlotTmp.ensure(n * sizeof(int));
        dPosS.ensure(n * sizeof(double4));
        dOrigS.ensure(n * sizeof(double4));
        dSpl.ensure((size_t) n * 9 * MAXP * R);
        dBaseS.ensure(n * sizeof(int4));
        dWrapS.ensure(n * sizeof(int4));
        dRadS.ensure(n * 8);
        dListCount.ensure(n * sizeof(int));
        dSListCount.ensure(n * sizeof(int));
        dAtomSlot.ensure(n * sizeof(int));
        dPosBuild.ensure(3 * (size_t) n * 8);
        dFlags.ensure(flagBytes());
        dDS.ensure(n * 4 * R);
        dDS2.ensure(n * 4 * R);
        dEpair2.ensure(3 * n * 8);
        dErec2.ensure(3 * n * 8);
        for (Buf* b : {&dPerm, &dMu, &dDtot, &dB, &dX, &dRv, &dZ, &dP, &dAp, &dEpair, &dErec, &dFpair, &dFrec, &dEtot,
                       &dForces})
            b->ensure(3 * n * 8);
        dSpair.ensure(9 * (size_t) n * 8);
        dFin.ensure((size_t) n * NFIN * 8);
        dPot.ensure(n * 8);
        dHrec.ensure(6 * (size_t) n * 8);
        dGradQ.ensure(n * 8);
        dGradR.ensure(n * 8);
        dScal.ensure(nsys * NSCAL * 8);
        dPartial.ensure(chunkSys.size() * 16 * 8);
        dGPartial.ensure(((size_t) n + 7) / 8 * 8);
        dSysCounter.ensure(nsys * sizeof(int));
        dActive.ensure(((size_t) s.maxIter + 2) * sizeof(int));
        dActSys.ensure((2 * (size_t) nsys + 2) * sizeof(int));   // actSys, actOff, actCount
        CU(cudaMemset(dSysCounter.p, 0, nsys * sizeof(int)));
        dResults.ensure(nsys * NRES * 8);
        dConvPartial.ensure((size_t) nsys * convBlocks * NCONV * 8);
        std::vector<int> convOff(nsys);
        for (int k = 0; k < nsys; k++)
            convOff[k] = k * convBlocks;
        upload(dConvOff, convOff, st);
        dGrid.ensure(gridTotal * R);
        dGrid2.ensure(gridTotal * R);
        if (mixed()) {   // (the fixed-point spread grids start cleared; each conversion clears them again)
            dGridFix.ensure(gridTotal * 8);
            dGridFix2.ensure(gridTotal * 8);
            CU(cudaMemset(dGridFix.p, 0, gridTotal * 8));
            CU(cudaMemset(dGridFix2.p, 0, gridTotal * 8));
        }
        dSpec.ensure(specTotal * 2 * R);
        dInfl.ensure(specTotal * R);
        if (refining()) {
            dGridD.ensure(gridTotal * 8);
            dSpecD.ensure(specTotal * 16);
            dInflD.ensure(specTotal * 8);
            dDSd.ensure(n * sizeof(double4));
            dSplD.ensure((size_t) n * 9 * MAXP * 8);
            dB64.ensure(3 * (size_t) n * 8);
            dXsave.ensure(3 * (size_t) n * 8);
        }
        upload(dModuli, moduliHost, st);
        upload(dChunkSys, chunkSys, st);
        upload(dChunkBegin, chunkBegin, st);
        upload(dChunkEnd, chunkEnd, st);
        upload(dAtomSys, atomSys, st);
        upload(dQ, q, st);
        upload(dR, radius, st);
        upload(dAlpha, alpha, st);
        if (!globalIdx.empty())
            upload(dGlobal, globalIdx, st);
        dHist.ensure((size_t) NHIST * 3 * numGlobal * 8);
        dCtl.ensure(sizeof(Ctl));
        dSys.ensure(nsys * sizeof(SysDev));
        // pinned staging
        if (hPosCap < (size_t) 3 * n) {
            if (hPos) cudaFreeHost(hPos);
            if (hPosF) cudaFreeHost(hPosF);
            if (hForces) cudaFreeHost(hForces);
            CU(cudaMallocHost((void**) &hPos, 3 * (size_t) n * 8));
            CU(cudaMallocHost((void**) &hPosF, 3 * (size_t) n * 4));
            CU(cudaMallocHost((void**) &hForces, 3 * (size_t) n * 8));
            hPosCap = 3 * (size_t) n;
        }
        if (hSysCap < (size_t) nsys) {
            if (hSys) cudaFreeHost(hSys);
            if (hResults) cudaFreeHost(hResults);
            CU(cudaMallocHost((void**) &hSys, nsys * sizeof(SysDev)));
            CU(cudaMallocHost((void**) &hResults, nsys * NRES * 8));
            hSysCap = nsys;
        }
        totalCells = 0;
        cellCapacity = 0;
        // no covalent dipoles until setCovalent
        uploadCovalent();
        haveResult = false;
        listValid = false;
        configured = true;
    }

    // Box-dependent per-system constants; cell grids sized so that cells are at least rc/2 wide in every
    // fractional direction (offsets -2..2 cover the cutoff sphere).  Returns true if the cell storage grew.
    bool setBoxes(const double* boxes) {
        int cells = 0;
        double maxDensity = 0.0;
        for (int k = 0; k < nsys; k++) {
            SysDev& S = sysHost[k];
            const double* H = boxes + 9 * k;
            for (int a = 0; a < 9; a++)
                S.H[a] = H[a];
            if (H[1] != 0 || H[2] != 0 || H[5] != 0)
                throw std::invalid_argument("pgm_b200: box not in the reduced triclinic form (a = (ax,0,0), b = (bx,by,0))");
            if (!(H[0] > 0 && H[4] > 0 && H[8] > 0))
                throw std::invalid_argument("pgm_b200: box diagonal must be positive");
            boxInverse(H, S.recip, S.volume);
            S.cutoff = sysCutoff[k];
            S.rc2 = sysCutoff[k] * sysCutoff[k];
            S.beta = sysBeta[k];
            if (!(S.cutoff > 0) || !(S.beta > 0))
                throw std::invalid_argument("pgm_b200: cutoff and Ewald coefficient must be positive");
            S.cellOff = cells;
            // the Verlet list radius: cutoff + skin, the skin shrunk so that the radius stays within half the
            // smallest plane spacing (minimum image), as core/cuda/pgm_cuda.cu:1930-1940
            double colMax = 0.0;
            for (int a = 0; a < 3; a++)
                colMax = std::max(colMax, std::sqrt(S.recip[a] * S.recip[a] + S.recip[3 + a] * S.recip[3 + a] +
                                                    S.recip[6 + a] * S.recip[6 + a]));
            const double skin = std::max(0.0, std::min(s.skin, 0.5 / colMax - S.cutoff));
            const double rl = S.cutoff + skin;
            S.rl2 = rl * rl;
            S.skinHalf2 = externalList ? 1e300 : 0.25 * skin * skin;   // (the caller's candidates: never stale)
            for (int a = 0; a < 3; a++) {
                const double col = std::sqrt(S.recip[a] * S.recip[a] + S.recip[3 + a] * S.recip[3 + a] +
                                             S.recip[6 + a] * S.recip[6 + a]);
                if (S.cutoff * col > 0.5 * (1.0 + 1e-12))
                    throw std::invalid_argument("pgm_b200: cut-off beyond half the box");
                const double rho = std::min(rl * col, 0.5);   // fractional extent of the list radius along a
                int nc = (int) std::floor(2.0 / rho);
                nc = std::max(1, std::min(nc, 1024));
                S.cellN[a] = nc;
                S.cellM[a] = std::max(1, (int) std::ceil(rho * nc * (1.0 + 1e-12)));
            }
            // at most ~8 cells per atom (very short cutoffs): widen the cells, offsets shrink accordingly
            const int na0 = atomBegin[k + 1] - atomBegin[k];
            while ((long long) S.cellN[0] * S.cellN[1] * S.cellN[2] > 8LL * na0 + 64) {
                int a = 0;
                for (int b = 1; b < 3; b++)
                    if (S.cellN[b] > S.cellN[a])
                        a = b;
                S.cellN[a] = std::max(1, S.cellN[a] / 2);
            }
            for (int a = 0; a < 3; a++) {
                const double col = std::sqrt(S.recip[a] * S.recip[a] + S.recip[3 + a] * S.recip[3 + a] +
                                             S.recip[6 + a] * S.recip[6 + a]);
                S.cellM[a] = std::max(1, (int) std::ceil(rl * col * S.cellN[a] * (1.0 + 1e-12)));
            }
            S.cellCount = S.cellN[0] * S.cellN[1] * S.cellN[2];
            cells += S.cellCount;
            const int na = atomBegin[k + 1] - atomBegin[k];
            maxDensity = std::max(maxDensity, na / S.volume);
        }
        totalCells = cells;
        bool grew = false;
        if (cells + 1 > cellCapacity) {
            cellCapacity = std::max(cells + 1, (int) (cellCapacity * 1.25));
            dCellCount.ensure(cellCapacity * sizeof(int));
            dCellStart.ensure((cellCapacity + 1) * sizeof(int));
            grew = true;
        }
        if (cap == 0) {
            // neighbours within rc at the highest density, +50 % for fluctuations
            double maxNb = 0;
            for (int k = 0; k < nsys; k++) {
                const int na = atomBegin[k + 1] - atomBegin[k];
                const double nb = 4.0 / 3.0 * PI_D * std::pow(std::sqrt(sysHost[k].rl2), 3) * (na / sysHost[k].volume);
                maxNb = std::max(maxNb, std::min(nb * 1.5 + 64.0, (double) na * 27));
            }
            cap = ((int) maxNb + 31) / 32 * 32;
            allocList();
            grew = true;
        }
        return grew;
    }

    void allocList() {
        listValid = false;
        dList.ensure((size_t) n * cap * sizeof(uint32_t));
        dSList.ensure((size_t) n * cap * sizeof(uint32_t));
        if (mixed())   // pair records: (x, G1) + (G2, slot of j) in float; FP64 (G1, G2) only
            dPairA.ensure((size_t) n * cap * 16);
        dPairB.ensure((size_t) n * cap * 2 * realSize());
        dPairC.ensure((size_t) n * cap * 2 * realSize());
        if (refining())
            dPairBd.ensure((size_t) n * cap * 16);
    }

    bool refining() const { return mixed() && s.refine && s.polarizable; }

    // A list kept between builds and compacted to the cutoff at every evaluation: a skin, or the caller's
    // candidates.
    bool verletList() const { return s.skin > 0 || externalList; }

    // The mixed path's device pointers with the FP64 shadow buffers in place of the R-typed ones.
    Dev makeDev64() {
        Dev d = makeDev(false, 0);
        d.pairA = nullptr;
        d.pairB = dPairBd.p;
        d.pairC = nullptr;
        d.dS = dDSd.p;
        d.grid = dGridD.p;
        d.spec = dSpecD.p;
        d.infl = dInflD.p;
        d.spl = dSplD.p;
        d.gridWords = gridTotal * 2;
        return d;
    }

    Dev makeDev(bool forGraph, cudaGraphConditionalHandle h, cudaGraphConditionalHandle listHandle = 0) {
        Dev d;
        std::memset(&d, 0, sizeof(d));
        d.listCond = listHandle;
        d.nAtoms = n;
        d.nSys = nsys;
        d.nChunks = (int) chunkSys.size();
        d.cap = cap;
        d.order = s.order;
        d.totalCells = totalCells;
        d.gridTotal = gridTotal;
        // (with the fixed-point spread the conversion rewrites the float grid and clears the fixed-point one: the
        // CG update clears nothing)
        d.gridFix = spreadFix() ? dGridFix.as<long long>() : nullptr;
        d.gridWords = spreadFix() ? 0 : gridTotal * (long long) (realSize() / 4);
        d.ctl = dCtl.as<Ctl>();
        d.ke = s.ke;
        d.tol = s.tol;
        d.peek = s.peek;
        d.maxIter = s.maxIter;
        d.sys = dSys.as<SysDev>();
        d.atomSys = dAtomSys.as<int>();
        d.q = dQ.as<double>();
        d.radius = dR.as<double>();
        d.alpha = dAlpha.as<double>();
        d.posIn = dPosIn.as<double>();
        d.wrapN = dWrap.as<int>();
        d.cellOf = dCellOf.as<int>();
        d.cellRank = dCellRank.as<int>();
        d.pmeBase = dBase.as<int>();
        d.pmeFr = dFr.as<double>();
        d.cellCount = dCellCount.as<int>();
        d.cellStart = dCellStart.as<int>();
        d.slotAtom = dSlotAtom.as<int>();
        d.slotTmp = dSlotTmp.as<int>();
        d.posS = dPosS.as<double4>();
        d.origS = dOrigS.as<double4>();
        d.spl = dSpl.p;
        d.baseS = dBaseS.as<int4>();
        d.wrapS = dWrapS.as<int4>();
        d.radS = dRadS.as<double>();
        d.list = dList.as<uint32_t>();
        d.listCount = dListCount.as<int>();
        d.slist = dSList.as<uint32_t>();
        d.slistCount = dSListCount.as<int>();
        d.atomSlot = dAtomSlot.as<int>();
        d.gvdwOn = gvdwOn ? 1 : 0;
        if (gvdwOn) {
            d.gvdwSlater = gvdwSlater ? 1 : 0;
            d.rvdw2 = rvdw * rvdw;
            d.gv = dGv.as<double4>();
            d.skipStart = dSkipStart.as<int>();
            d.skipJ = dSkipJ.as<int>();
            for (int k = 0; k < GVDW_TERMS; k++)
                d.gvC[k] = gvC[k];
        }
        if (externalList) {
            d.candStart = dCandStart.as<int>();
            d.candJ = dCandJ.as<int>();
            d.candT = dCandT.as<int>();
        }
        if (!verletList()) {   // no skin: the build writes the evaluation's list itself (no compaction)
            d.slist = d.list;
            d.slistCount = d.listCount;
        }
        d.posBuild = dPosBuild.as<double>();
        d.pairA = dPairA.p;
        d.pairB = dPairB.p;
        d.pairC = dPairC.p;
        d.flags = dFlags.as<int>();
        d.dS = dDS.p;
        d.dS2 = dDS2.p;
        d.perm = dPerm.as<double>();
        d.mu = dMu.as<double>();
        d.dtot = dDtot.as<double>();
        d.b = dB.as<double>();
        d.x = dX.as<double>();
        d.r = dRv.as<double>();
        d.z = dZ.as<double>();
        d.p = dP.as<double>();
        d.Ap = dAp.as<double>();
        d.scal = dScal.as<double>();
        d.partial = dPartial.as<double>();
        d.gpartial = dGPartial.as<double>();
        d.sysCounter = dSysCounter.as<int>();
        d.activeHist = dActive.as<int>();
        d.actSys = dActSys.as<int>();
        d.actOff = d.actSys + nsys;
        d.actCount = d.actOff + nsys + 1;
        d.useActive = nsys > 1 ? 1 : 0;
        d.Epair = dEpair.as<double>();
        d.Epair2 = dEpair2.as<double>();
        d.Erec = dErec.as<double>();
        d.Fpair = dFpair.as<double>();
        d.spair = dSpair.as<double>();
        d.Frec = dFrec.as<double>();
        d.Etot = dEtot.as<double>();
        d.fin = dFin.as<double>();
        d.potRec = dPot.as<double>();
        d.hrec = dHrec.as<double>();
        d.forces = dForces.as<double>();
        d.results = dResults.as<double>();
        d.convPartial = dConvPartial.as<double>();
        d.convPartialOff = dConvOff.as<int>();
        d.grid = dGrid.p;
        d.spec = dSpec.p;
        d.infl = dInfl.p;
        d.twiddle = dTwiddle.p;
        d.fftcBuf = fftcBuf;
        d.fftcC = fftcC;
        d.fftgBuf = fftgBuf;
        d.fftgBar = (unsigned*) (dFlags.as<int>() + 16);
        d.pcgBar = (unsigned*) (dFlags.as<int>() + 16 + 2 * nsys);
        d.pmeRec = dPmeRec.p;
        d.pmeBinStart = dPmeBins.as<int>();
        d.srcW = dSrcW.as<float4>();
        d.gpart = dGPart.as<float4>();
        d.pcgPartial = dPcgPartial.as<double>();
        d.moduli = dModuli.as<double>();
        d.ncov = (int) covAtom.size();
        d.covAtom = dCovAtom.as<int>();
        d.covPartner = dCovPartner.as<int>();
        d.covStrength = dCovStrength.as<double>();
        d.covByAtomOff = dCovByAtomOff.as<int>();
        d.covByAtom = dCovByAtom.as<int>();
        d.covByPartnerOff = dCovByPartnerOff.as<int>();
        d.covByPartner = dCovByPartner.as<int>();
        d.chunkSys = dChunkSys.as<int>();
        d.chunkBegin = dChunkBegin.as<int>();
        d.chunkEnd = dChunkEnd.as<int>();
        d.hist = dHist.as<double>();
        d.globalIndex = globalIdx.empty() ? nullptr : dGlobal.as<int>();
        d.numGlobal = numGlobal;
        d.cond = h;
        d.useCond = forGraph ? 1 : 0;
        d.loopCond = (forGraph && h != 0) ? 1 : 0;
        return d;
    }

    // ------------------------------------------------------------------------------------------ launches
    // fix: the spread before went to the fixed-point grid (converted first)
    template <typename R> void fftChain(cudaStream_t sm, const Dev& d, bool energy, bool gate, bool fix = false) {
        typedef typename CplxT<R>::T C;
        constexpr bool dbl = std::is_same<R, double>::value;
        const bool shadow = dbl && mixed();   // the FP64 refinement's transforms of a mixed engine
        if (fix && !dbl)
            gridFromFix(sm, d);
        for (size_t k = 0; k < groups.size(); k++) {
            auto& g = groups[k];
            const cufftHandle plan = shadow ? plans64[k].first : g.r2c;
            CUFFT(cufftSetStream(plan, sm));
            R* gp = (R*) d.grid + g.gridOff;
            C* sp = (C*) d.spec + g.specOff;
            if (!dbl)
                CUFFT(cufftExecR2C(plan, (cufftReal*) gp, (cufftComplex*) sp));
            else
                CUFFT(cufftExecD2Z(plan, (cufftDoubleReal*) gp, (cufftDoubleComplex*) sp));
        }
        dim3 cg(convBlocks, nsys);
        if (energy)
            k_conv<R, true><<<cg, 256, 0, sm>>>(d, 0);
        else
            k_conv<R, false><<<cg, 256, 0, sm>>>(d, gate ? 1 : 0);
        CU(cudaGetLastError());
        for (size_t k = 0; k < groups.size(); k++) {
            auto& g = groups[k];
            const cufftHandle plan = shadow ? plans64[k].second : g.c2r;
            CUFFT(cufftSetStream(plan, sm));
            R* gp = (R*) d.grid + g.gridOff;
            C* sp = (C*) d.spec + g.specOff;
            if (!dbl)
                CUFFT(cufftExecC2R(plan, (cufftComplex*) sp, (cufftReal*) gp));
            else
                CUFFT(cufftExecZ2D(plan, (cufftDoubleComplex*) sp, (cufftDoubleReal*) gp));
        }
    }

    // Attributes of the cluster transform kernel; false when no cluster of its size fits on this GPU.
    template <typename R> bool prepareCluster() {
        const void* f = (const void*) k_fft_cluster<R>;
        CU(cudaFuncSetAttribute(f, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        CU(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) fftcSmem));
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = fftcC;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(fftcC * nsys);
        cfg.blockDim = dim3(FftcThreads<R>::n);
        cfg.dynamicSmemBytes = fftcSmem;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int clusters = 0;
        if (cudaOccupancyMaxActiveClusters(&clusters, k_fft_cluster<R>, &cfg) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        return clusters > 0;
    }

    // The grid-transform kernel: compiled for one cubic grid size (32, 40, 48, 64), or for any grid; energy: the
    // final pass's variant that also sums the reciprocal energy and strain.
    template <typename R> static void (*fftgKernel(int kc, bool energy = false))(Dev, int) {
        if (energy)
            switch (kc) {
            case 32: return k_fft_grid<R, 32, true>;
            case 40: return k_fft_grid<R, 40, true>;
            case 48: return k_fft_grid<R, 48, true>;
            case 64: return k_fft_grid<R, 64, true>;
            default: return k_fft_grid<R, 0, true>;
            }
        switch (kc) {
        case 32: return k_fft_grid<R, 32>;
        case 40: return k_fft_grid<R, 40>;
        case 48: return k_fft_grid<R, 48>;
        case 64: return k_fft_grid<R, 64>;
        default: return k_fft_grid<R, 0>;
        }
    }

    // Attributes of the grid-transform kernel; false when its blocks (a block per x-plane of every system) cannot
    // all be resident at once on this GPU or a block's shared memory does not fit.
    template <typename R> bool prepareGrid() {
        int optin = 0, sms = 0, coop = 0;
        CU(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, devId));
        CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, devId));
        CU(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, devId));
        if (!coop || fftgSmem > (size_t) optin)
            return false;
        CU(cudaFuncSetAttribute((const void*) fftgKernel<R>(fftgKc), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int) fftgSmem));
        int perSm = 0;
        CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, fftgKernel<R>(fftgKc), FftgThreads<R>::n,
                                                         fftgSmem));
        // the final pass's variant: every block resident too, and a conv partial of its own for each x-plane
        CU(cudaFuncSetAttribute((const void*) fftgKernel<R>(fftgKc, true),
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int) fftgSmem));
        int perSmE = 0;
        CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSmE, fftgKernel<R>(fftgKc, true), FftgThreads<R>::n,
                                                         fftgSmem));
        gridEnergyOk = (long long) perSmE * sms >= (long long) maxK0 * nsys && maxK0 <= convBlocks;
        return (long long) perSm * sms >= (long long) maxK0 * nsys;
    }

    // The transform pair with the influence product of a field pass: one cluster kernel (all systems), or
    // cuFFT plans and the product kernel.  The FP64 shadow of a mixed engine takes the cuFFT path.
    // The persistent CG kernel's conditions and launch shape: mixed precision, one polarizable system, order 6,
    // the grid kernel possible, K0 plane blocks plus at least PCG_MIN_PAIR_BLOCKS pair blocks resident at once
    // (one per SM), and its shared memory.
    void preparePersistent() {
        pcgOk = false;
        if (!mixed() || nsys != 1 || !gridOk || s.order != 6 || !s.polarizable)
            return;
        int sms = 0, coop = 0, optin = 0;
        CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, devId));
        CU(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, devId));
        CU(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, devId));
        const int* K = sysK[0].data();
        pcgSmem = (3 * (size_t) FFT_MAXK + 2 * (size_t) fftgBuf) * 8;
        if (!coop || pcgSmem > (size_t) optin || K[0] + PCG_MIN_PAIR_BLOCKS > sms)
            return;
        PcgKernel kfn = persistentKernel(pairGS);
        CU(cudaFuncSetAttribute((const void*) kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) pcgSmem));
        int perSm = 0;
        CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kfn, PCG_THREADS, pcgSmem));
        if (perSm < 1)
            return;
        pcgBlocks = sms * std::min(perSm, PCG_BLOCKS_PER_SM);   // (the plane blocks, 0 .. K0-1, one per SM)
        pcgOk = true;
        dPcgPartial.ensure((size_t) 2 * pcgBlocks * 4 * 8);
    }

    // The plane-owner spread and gather: mixed precision, one system, order 6; tiles of PL_YCH rows (+ 5 halo
    // rows) of an x-plane in shared memory.
    void preparePlanes() {
        planesOk = false;
        if (!mixed() || nsys != 1 || s.order != 6)
            return;
        const int* K = sysK[0].data();
        planeNyc = (K[1] + PL_YCH - 1) / PL_YCH;
        planeSmem = (size_t) (PL_YCH + 5) * K[2] * sizeof(float);
        int optin = 0;
        CU(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, devId));
        if (planeSmem > (size_t) optin)
            return;
        for (const void* f : {(const void*) k_spread_planes<6>, (const void*) k_gather_planes<6>})
            CU(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) planeSmem));
        const size_t nbins = (size_t) K[0] * planeNyc;
        if (nbins > (size_t) PL_MAX_SMEM_BINS)
            return;   // (the binning kernels keep a block's histogram of every bin in shared memory)
        CU(cudaFuncSetAttribute((const void*) k_plane_bin_count, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int) (nbins * sizeof(int))));
        CU(cudaFuncSetAttribute((const void*) k_plane_bin_fill<6>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int) (2 * nbins * sizeof(int))));
        dPmeRec.ensure((size_t) n * sizeof(PmeRec<6>));
        dPmeBins.ensure((std::max<size_t>(nbins, FFT_MAXK) + 1) * sizeof(int));
        dBinCount.ensure(nbins * sizeof(int));
        dSrcW.ensure((size_t) n * sizeof(float4));
        dGPart.ensure((size_t) 6 * n * sizeof(float4));
        planesOk = true;
    }

    bool planesMode() const { return planesOk && pmeWant == 1; }
    // The mixed spread into the 64-bit fixed-point grid (the warp-per-atom kernels; PGM_B200_FLOAT_GRID=1 keeps
    // float atomics on the float grid, for comparison).
    bool fixMode() const {
        const char* e = std::getenv("PGM_B200_FLOAT_GRID");
        return mixed() && !(e && e[0] == '1');
    }
    // whether the field passes' spread (launchSpread) writes the fixed-point grid: the warp-per-atom kernel only
    bool spreadFix() const { return fixMode() && !planesMode() && !linesMode() && !tilesMode(); }
    void gridFromFix(cudaStream_t sm, const Dev& d) {
        const int blocks = (int) std::min<long long>((gridTotal + 255) / 256, 4 * 148);
        k_grid_from_fix<<<blocks, 256, 0, sm>>>(d);
        CU(cudaGetLastError());
    }

    // the float4 line spread and gather: mixed precision, orders 4, 5, 6 and 8, any number of systems
    bool linesMode() const {
        return pmeWant == 2 && mixed() && (s.order == 4 || s.order == 5 || s.order == 6 || s.order == 8);
    }

    // The cell-group tiles of one system: G cells a side per group (the largest of 4, 3, 2, 1 that leaves at
    // least 100 groups and a tile within 96 KB, else the largest whose tile fits; PGM_B200_TILE_G overrides), the
    // tile capacity in floats (the
    // window of G cells' base indices + 1 for rounding + p - 1 halo + the list skin's drift both ways), and the
    // group count.  groups = 0: no tiling applies.
    void tileGeometry(int& G, int& cap, int& groups) const {
        G = cap = groups = 0;
        if (nsys != 1 || totalCells == 0)
            return;
        const SysDev& S = sysHost[0];
        int win[5][3];
        for (int g = 1; g <= TL_MAX_G; g++)
            for (int a = 0; a < 3; a++) {
                const double col = std::sqrt(S.recip[a] * S.recip[a] + S.recip[3 + a] * S.recip[3 + a] +
                                             S.recip[6 + a] * S.recip[6 + a]);
                const int drift = 1 + (int) std::ceil(s.skin * S.K[a] * col);
                win[g][a] = (S.K[a] * g + S.cellN[a] - 1) / S.cellN[a] + 1 + (s.order - 1) + 2 * drift;
            }
        auto groupsOf = [&](int g) {
            return ((S.cellN[0] + g - 1) / g) * ((S.cellN[1] + g - 1) / g) * ((S.cellN[2] + g - 1) / g);
        };
        auto capOf = [&](int g) { return (long long) win[g][0] * win[g][1] * win[g][2]; };
        int pick = 0;
        if (const char* e = std::getenv("PGM_B200_TILE_G"))
            pick = std::max(1, std::min(TL_MAX_G, std::atoi(e)));
        for (int g = TL_MAX_G; g >= 1 && !pick; g--)
            if (groupsOf(g) >= 100 && capOf(g) * 4 <= 96 * 1024)
                pick = g;
        for (int g = TL_MAX_G; g >= 1 && !pick; g--)   // (small systems: the fewest groups that fit)
            if (capOf(g) * 4 <= 96 * 1024)
                pick = g;
        if (!pick || capOf(pick) * 4 > 200 * 1024 || (size_t) groupsOf(pick) > ((size_t) n + 7) / 8)
            return;   // (the tile beyond shared memory, or more groups than the block partials hold)
        G = pick;
        cap = (int) capOf(pick);
        groups = groupsOf(pick);
    }

    // the cell-group tile spread and gather: mixed precision, one system, orders 4, 5, 6 and 8
    bool tilesMode() const {
        if (pmeWant != 3 || !mixed() || nsys != 1 ||
            !(s.order == 4 || s.order == 5 || s.order == 6 || s.order == 8))
            return false;
        if (totalCells == 0)
            return true;   // (no box yet: the geometry is settled at the first evaluation)
        int G, cap, groups;
        tileGeometry(G, cap, groups);
        return groups > 0;
    }

    template <int P> void launchTiles(cudaStream_t sm, const Dev& d, bool spread, int mode, double* vec, int gate,
                                      bool cga) {
        int G, cap, groups;
        tileGeometry(G, cap, groups);
        const size_t smem = (size_t) cap * sizeof(float);
        static std::once_flag once[4];
        std::call_once(once[P == 4 ? 0 : P == 5 ? 1 : P == 6 ? 2 : 3], [] {
            for (const void* f : {(const void*) k_spread_tiles<P>, (const void*) k_gather_tiles<P, false>,
                                  (const void*) k_gather_tiles<P, true>})
                CU(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        });
        if (spread)
            k_spread_tiles<P><<<groups, TL_THREADS, smem, sm>>>(d, mode, vec, G, cap);
        else if (cga)
            k_gather_tiles<P, true><<<groups, TL_THREADS, smem, sm>>>(d, gate, G, cap);
        else
            k_gather_tiles<P, false><<<groups, TL_THREADS, smem, sm>>>(d, gate, G, cap);
        CU(cudaGetLastError());
    }

    void launchTilesOrder(cudaStream_t sm, const Dev& d, bool spread, int mode, double* vec, int gate, bool cga) {
        switch (s.order) {
        case 4: launchTiles<4>(sm, d, spread, mode, vec, gate, cga); break;
        case 5: launchTiles<5>(sm, d, spread, mode, vec, gate, cga); break;
        case 6: launchTiles<6>(sm, d, spread, mode, vec, gate, cga); break;
        default: launchTiles<8>(sm, d, spread, mode, vec, gate, cga);
        }
    }

    // The plane bins and records of the evaluation (after k_splines).
    void enqueuePlaneBins(cudaStream_t sm, const Dev& d) {
        const int nbins = sysK[0][0] * planeNyc, bb = (n + PL_BIN_SLOTS - 1) / PL_BIN_SLOTS;
        CU(cudaMemsetAsync(dBinCount.p, 0, nbins * sizeof(int), sm));
        k_plane_bin_count<<<bb, 256, nbins * sizeof(int), sm>>>(d, planeNyc, dBinCount.as<int>());
        k_plane_bin_scan<<<1, 1024, 0, sm>>>(d, nbins, dBinCount.as<int>());
        k_plane_bin_fill<6><<<(n + PL_FILL_SLOTS - 1) / PL_FILL_SLOTS, PL_FILL_SLOTS, 2 * nbins * sizeof(int), sm>>>(
            d, planeNyc, dBinCount.as<int>());
        CU(cudaGetLastError());
    }

    // The persistent kernel for the pair lanes (8, 16 or 32; 4 runs as 8) and the grid's compile-time size.
    // pass 0: the CG loop; 1 / 2: one field pass of dipoles (and charges).
    typedef void (*PcgKernel)(Dev, int, const double*);
    PcgKernel persistentKernel(int lanes, int pass = 0) {
        const int kc = fftgKc;
        auto pick = [&](auto gsTag) -> PcgKernel {
            constexpr int GS = decltype(gsTag)::value;
            if (kc == 48)
                return pass == 0 ? k_cg_persistent<6, GS, 48, 0> : pass == 1 ? k_cg_persistent<6, GS, 48, 1>
                                                                             : k_cg_persistent<6, GS, 48, 2>;
            return pass == 0 ? k_cg_persistent<6, GS, 0, 0> : pass == 1 ? k_cg_persistent<6, GS, 0, 1>
                                                                        : k_cg_persistent<6, GS, 0, 2>;
        };
        if (lanes >= 32)
            return pick(std::integral_constant<int, 32>());
        if (lanes >= 16)
            return pick(std::integral_constant<int, 16>());
        return pick(std::integral_constant<int, 8>());
    }

    // The whole CG loop (pass 0), or one field pass of the dipoles vec (1) and the charges (2): one cooperative
    // launch of the persistent kernel (one block per SM).
    void launchPersistent(cudaStream_t sm, const Dev& d, int pass = 0, const double* vec = nullptr) {
        PcgKernel kfn = persistentKernel(pairGS, pass);
        CU(cudaFuncSetAttribute((const void*) kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) pcgSmem));
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeCooperative;
        at[0].val.cooperative = 1;
        cfg.gridDim = dim3(pcgBlocks);
        cfg.blockDim = dim3(PCG_THREADS);
        cfg.dynamicSmemBytes = pcgSmem;
        cfg.stream = sm;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        Dev dp = d;   // (its spread always goes to the fixed-point grid)
        dp.gridFix = dGridFix.as<long long>();
        CU(cudaLaunchKernelEx(&cfg, kfn, dp, planeNyc, vec));
    }

    bool persistentMode() const { return tfMode == TF_PCG; }

    int solveDevice(double tol);
    template <typename R>
    void tangentPass(const Dev& d, const FmBufs& B, const double* dr, const double* dd, const double* dip,
                     const double* quadD, int withQ);

    // The transform mode in use: the caller's choice where the systems' grids allow it, else cuFFT.
    void selectTransforms() {
        int m = TF_CUFFT;
        if (tfWant == TF_CLUSTER && clusterOk)
            m = TF_CLUSTER;
        if (tfWant == TF_SPLIT && splitOk)
            m = TF_SPLIT;
        if (tfWant == TF_GRID && gridOk)
            m = TF_GRID;
        if (tfWant == TF_PCG && pcgOk)
            m = TF_PCG;
        if (m != tfMode && exec) {
            cudaGraphExecDestroy(exec);
            exec = nullptr;
        }
        tfMode = m;
    }

    // Split transforms: 2D R2C of every x-plane (cuFFT), the x-lines with the influence product (one kernel, all
    // systems), 2D C2R.
    template <typename R> void splitChain(cudaStream_t sm, const Dev& d, bool gate) {
        typedef typename CplxT<R>::T C;
        constexpr bool dbl = std::is_same<R, double>::value;
        for (auto& g : groups) {
            CUFFT(cufftSetStream(g.r2c2d, sm));
            R* gp = (R*) d.grid + g.gridOff;
            C* sp = (C*) d.spec + g.specOff;
            if (!dbl)
                CUFFT(cufftExecR2C(g.r2c2d, (cufftReal*) gp, (cufftComplex*) sp));
            else
                CUFFT(cufftExecD2Z(g.r2c2d, (cufftDoubleReal*) gp, (cufftDoubleComplex*) sp));
        }
        k_xlines<R><<<dim3(maxLineBlocks, nsys), XL_THREADS, 0, sm>>>(d, gate ? 1 : 0);
        CU(cudaGetLastError());
        for (auto& g : groups) {
            CUFFT(cufftSetStream(g.c2r2d, sm));
            R* gp = (R*) d.grid + g.gridOff;
            C* sp = (C*) d.spec + g.specOff;
            if (!dbl)
                CUFFT(cufftExecC2R(g.c2r2d, (cufftComplex*) sp, (cufftReal*) gp));
            else
                CUFFT(cufftExecZ2D(g.c2r2d, (cufftDoubleComplex*) sp, (cufftDoubleReal*) gp));
        }
    }

    // The grid-transform kernel (cooperative: the blocks of a system meet at two barriers); energy: the final
    // pass's variant.
    template <typename R> void launchGrid(cudaStream_t sm, const Dev& d, int flags, bool energy) {
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeCooperative;
        at[0].val.cooperative = 1;
        cfg.gridDim = dim3(maxK0, nsys);
        cfg.blockDim = dim3(FftgThreads<R>::n);
        cfg.dynamicSmemBytes = fftgSmem;
        cfg.stream = sm;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        CU(cudaLaunchKernelEx(&cfg, fftgKernel<R>(fftgKc, energy), d, flags));
    }

    // fix: the spread before went to the fixed-point grid (the grid kernel converts on its load, the others after a
    // conversion kernel)
    template <typename R> void transformPair(cudaStream_t sm, const Dev& d, bool gate, bool fix = false) {
        constexpr bool dbl = std::is_same<R, double>::value;
        fix = fix && !dbl && d.gridFix;
        if (dbl == mixed() || tfMode == TF_CUFFT) {   // (the FP64 shadow of a mixed engine: cuFFT)
            fftChain<R>(sm, d, false, gate, fix);
            return;
        }
        if (fix && tfMode != TF_GRID && tfMode != TF_PCG)
            gridFromFix(sm, d);
        if (tfMode == TF_SPLIT) {
            splitChain<R>(sm, d, gate);
            return;
        }
        if (tfMode == TF_GRID || tfMode == TF_PCG) {   // cooperative: the blocks of a system meet at two barriers
            launchGrid<R>(sm, d, (gate ? 1 : 0) | (fix ? 2 : 0), false);
            return;
        }
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = fftcC;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(fftcC * nsys);
        cfg.blockDim = dim3(FftcThreads<R>::n);
        cfg.dynamicSmemBytes = fftcSmem;
        cfg.stream = sm;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        CU(cudaLaunchKernelEx(&cfg, k_fft_cluster<R>, d, gate ? 1 : 0));
    }

    template <typename R> void launchSpread(cudaStream_t sm, const Dev& d, int mode, double* vec) {
        if (std::is_same<R, float>::value && planesMode()) {   // sources per slot, then plane tiles
            k_plane_sources<<<(n + 255) / 256, 256, 0, sm>>>(d, mode, vec);
            k_spread_planes<6><<<dim3(sysK[0][0], planeNyc), PL_THREADS, planeSmem, sm>>>(d, planeNyc);
            CU(cudaGetLastError());
            return;
        }
        if (std::is_same<R, float>::value && tilesMode()) {
            launchTilesOrder(sm, d, true, mode, vec, 0, false);
            return;
        }
        if (std::is_same<R, float>::value && linesMode()) {
            switch (s.order) {
            case 4: k_spread_lines<4><<<lineBlocks<4>(n), 256, 0, sm>>>(d, mode, vec); break;
            case 5: k_spread_lines<5><<<lineBlocks<5>(n), 256, 0, sm>>>(d, mode, vec); break;
            case 6: k_spread_lines<6><<<lineBlocks<6>(n), 256, 0, sm>>>(d, mode, vec); break;
            default: k_spread_lines<8><<<lineBlocks<8>(n), 256, 0, sm>>>(d, mode, vec);
            }
            CU(cudaGetLastError());
            return;
        }
        const int wb = (n + 7) / 8;
        switch (s.order) {
        case 4: k_spread<R, 4><<<wb, 256, 0, sm>>>(d, mode, vec); break;
        case 5: k_spread<R, 5><<<wb, 256, 0, sm>>>(d, mode, vec); break;
        case 6: k_spread<R, 6><<<wb, 256, 0, sm>>>(d, mode, vec); break;
        case 8: k_spread<R, 8><<<wb, 256, 0, sm>>>(d, mode, vec); break;
        default: k_spread<R, 0><<<wb, 256, 0, sm>>>(d, mode, vec);
        }
        CU(cudaGetLastError());
    }

    // CGA: the CG iteration's gather of a single-system engine, with A p and alph in its epilogue.
    template <typename R, bool FINAL, bool CGA = false> void launchGather(cudaStream_t sm, const Dev& d, int gate) {
        if (std::is_same<R, float>::value && !FINAL && !CGA && planesMode()) {   // plane tiles, then E_rec per atom
            k_gather_planes<6><<<dim3(sysK[0][0], planeNyc), PL_THREADS, planeSmem, sm>>>(d, planeNyc);
            k_gather_planes_finish<6><<<(n + 255) / 256, 256, 0, sm>>>(d);
            CU(cudaGetLastError());
            return;
        }
        if (std::is_same<R, float>::value && !FINAL && tilesMode()) {
            launchTilesOrder(sm, d, false, 0, nullptr, gate, CGA);
            return;
        }
        if (std::is_same<R, float>::value && !FINAL && linesMode()) {
            switch (s.order) {
            case 4: k_gather_lines<4, CGA><<<lineBlocks<4>(n), 256, 0, sm>>>(d, gate); break;
            case 5: k_gather_lines<5, CGA><<<lineBlocks<5>(n), 256, 0, sm>>>(d, gate); break;
            case 6: k_gather_lines<6, CGA><<<lineBlocks<6>(n), 256, 0, sm>>>(d, gate); break;
            default: k_gather_lines<8, CGA><<<lineBlocks<8>(n), 256, 0, sm>>>(d, gate);
            }
            CU(cudaGetLastError());
            return;
        }
        const int wb = (n + 7) / 8;
        switch (s.order) {
        case 4: k_gather<R, FINAL, 4, CGA><<<wb, 256, 0, sm>>>(d, gate); break;
        case 5: k_gather<R, FINAL, 5, CGA><<<wb, 256, 0, sm>>>(d, gate); break;
        case 6: k_gather<R, FINAL, 6, CGA><<<wb, 256, 0, sm>>>(d, gate); break;
        case 8: k_gather<R, FINAL, 8, CGA><<<wb, 256, 0, sm>>>(d, gate); break;
        default: k_gather<R, FINAL, 0, CGA><<<wb, 256, 0, sm>>>(d, gate);
        }
        CU(cudaGetLastError());
    }

    template <typename R, bool WITHQ, bool DUAL = false> void pairField(cudaStream_t sm, const Dev& d, int gate) {
        const long long threads = (long long) n * pairGS;
        const int blocks = (int) ((threads + 255) / 256);
        const int sh = pairSmem;
        switch (pairGS) {
        case 4: k_pair_field<R, WITHQ, 4, DUAL><<<blocks, 256, sh, sm>>>(d, gate); break;
        case 16: k_pair_field<R, WITHQ, 16, DUAL><<<blocks, 256, sh, sm>>>(d, gate); break;
        case 8: k_pair_field<R, WITHQ, 8, DUAL><<<blocks, 256, sh, sm>>>(d, gate); break;
        default: k_pair_field<R, WITHQ, 32, DUAL><<<blocks, 256, sh, sm>>>(d, gate);
        }
        CU(cudaGetLastError());
    }

    // A predicted step (guess from history, not from E_perm) with PGM_B200_DUAL=1: the permanent field and T x0
    // from one pair sweep over the records and two PME passes, the second on its own grid (the transforms in
    // sequence: they share the spectrum buffer and the grid kernel's barrier words).  By default the two passes
    // stay apart: since the first pass runs its PME half beside the list work on the high-priority stream, apart
    // is the faster of the two.
    bool dualFirstPass() const {
        const char* e = std::getenv("PGM_B200_DUAL");
        if (!(e && e[0] == '1'))
            return false;
        return s.polarizable && hCtl && hCtl->guess >= 1 && !hCtl->customRhs && !persistentMode() && !refining() &&
               !planesMode() && !tilesMode();
    }

    // field of (q?, vec) at every atom into Epair / Erec: spread on sm, then the pair pass on sm beside the
    // FFT chain on the side stream; joined on sm.
    template <typename R, bool WITHQ, bool CGA = false>
    void fieldPass(cudaStream_t sm, cudaStream_t sd, const Dev& d, int spreadMode, double* vec, bool gate) {
        launchSpread<R>(sm, d, spreadMode, vec);
        CU(cudaEventRecord(evFork, sm));
        CU(cudaStreamWaitEvent(sd, evFork, 0));
        transformPair<R>(sd, d, gate, spreadFix());
        pairField<R, WITHQ>(sm, d, gate ? 1 : 0);
        CU(cudaEventRecord(evJoin, sd));
        CU(cudaStreamWaitEvent(sm, evJoin, 0));
        launchGather<R, false, CGA>(sm, d, gate ? 1 : 0);
    }

    // The evaluation's pair list with its records: the Verlet list compacted to the cutoff, or, without a skin
    // (the build wrote the evaluation's list), the records of every listed pair.
    template <typename R> void pairRecords(cudaStream_t sm, const Dev& d) {
        if (!verletList())
            k_pair_kernels<R><<<(n + 7) / 8, 256, 0, sm>>>(d);
        else
            k_pair_compact<R><<<(n + 7) / 8, 256, 0, sm>>>(d);
        CU(cudaGetLastError());
    }

    // The Verlet list's build: cells, slots, the list at cutoff + skin (positions already in posIn).
    void enqueueBuild(cudaStream_t sm, const Dev& d) {
        enqueueCells(sm, d);
        listKernel(sm, d);
        CU(cudaGetLastError());
    }

    // The first half of a build: wraps, cells and the slot order with its slot-order copies.
    void enqueueCells(cudaStream_t sm, const Dev& d) {
        const int tb = (n + 255) / 256;
        k_prep<<<tb, 256, 0, sm>>>(d, nullptr, 2);
        k_cell_scan<<<1, 1024, 0, sm>>>(d);
        k_cell_scatter<<<tb, 256, 0, sm>>>(d);
        k_cell_sort<<<(totalCells + 7) / 8, 256, 0, sm>>>(d);
        CU(cudaGetLastError());
    }

    // The list's rows at a build (after the cell sort): the caller's candidates, or the cell search.
    void listKernel(cudaStream_t sm, const Dev& d) {
        if (externalList)
            k_list_from_candidates<<<(n + 7) / 8, 256, 0, sm>>>(d);
        else
            k_build_list<<<totalCells, LIST_THREADS, 0, sm>>>(d);
    }

    // The pair-list step of an evaluation: positions in (PME base and fraction), the stale test, the build when
    // stale (a conditional node of the graph, its body captured after the main capture; without graphs a host
    // decision), the slot-order positions with the build's wraps.  Without a skin the list's rows are left to the
    // caller (listKernel after this step, on a stream of its choice: nothing before it reads the list; the
    // refreshed slot copies equal the cell sort's bit for bit), and the call returns true.
    bool enqueueListStep(cudaStream_t sm, const Dev& d) {
        const int tb = (n + 255) / 256;
        k_prep<<<tb, 256, 0, sm>>>(d, dPosIn.as<double>(), 1);
        const bool rowsLeft = !verletList();
        if (rowsLeft) {   // no skin: a build at every evaluation, without the stale test or a conditional node
            CU(cudaMemsetAsync(d.cellCount, 0, (size_t) totalCells * sizeof(int), sm));
            enqueueCells(sm, d);
        } else {
            enqueueStaleBuild(sm, d);
        }
        k_refresh_positions<<<tb, 256, 0, sm>>>(d);
        CU(cudaGetLastError());
        return rowsLeft;
    }

    // Ends the work captured so far on st with a conditional node (IF or WHILE on `cond`): the node follows
    // everything the stream's capture depends on now, and the stream's later captured work follows the node.
    // Returns the node's body graph, filled by a capture of its own once the main capture has ended.
    static cudaGraph_t appendConditional(cudaStream_t st, cudaGraphConditionalHandle cond,
                                         cudaGraphConditionalNodeType kind) {
        cudaStreamCaptureStatus state = cudaStreamCaptureStatusNone;
        cudaGraph_t target = nullptr;
        const cudaGraphNode_t* frontier = nullptr;
        size_t frontierSize = 0;
        CU(cudaStreamGetCaptureInfo(st, &state, nullptr, &target, &frontier, &frontierSize));
        if (state != cudaStreamCaptureStatusActive || !target)
            throw std::runtime_error("pgm_b200: a conditional node outside an active capture");
        cudaGraphNodeParams params = {};
        params.type = cudaGraphNodeTypeConditional;
        params.conditional.handle = cond;
        params.conditional.type = kind;
        params.conditional.size = 1;
        cudaGraphNode_t added = nullptr;
        CU(cudaGraphAddNode(&added, target, frontier, frontierSize, &params));
        CU(cudaStreamUpdateCaptureDependencies(st, &added, 1, cudaStreamSetCaptureDependencies));
        return params.conditional.phGraph_out[0];
    }

    // The stale test and the build when stale (a conditional node of the graph, its body captured after the main
    // capture; without graphs a host decision).
    void enqueueStaleBuild(cudaStream_t sm, const Dev& d) {
        const int tb = (n + 255) / 256;
        k_displace<<<tb, 256, 0, sm>>>(d);
        CU(cudaGetLastError());
        if (capturing) {
            listBody = appendConditional(sm, d.listCond, cudaGraphCondTypeIf);
        } else {
            CU(cudaMemcpyAsync(hFlags, d.flags, 16 * sizeof(int), cudaMemcpyDeviceToHost, sm));
            CU(cudaStreamSynchronize(sm));
            if (hFlags[6])
                enqueueBuild(sm, d);
        }
    }

    template <typename R> void enqueuePre(cudaStream_t sm, cudaStream_t sd, const Dev& d) {
        const int tb = (n + 255) / 256;
        CU(cudaMemsetAsync(d.flags, 0, flagBytes(), sm));
        const bool rowsLeft = enqueueListStep(sm, d);
        if (s.polarizable) {
            // the list's rows when built here, the pairs within the cutoff and their G1, G2 (side stream) beside
            // the permanent field's PME half (main stream).  Without a skin, on the plain first pass, the record
            // kernel also forms the permanent field's direct part (after the permanent spread wrote the sources),
            // in place of a pair pass of its own.
            const bool pcg = std::is_same<R, float>::value && persistentMode();
            if (!dualFirstPass()) {
                // the permanent field's PME half on the side stream, whose higher priority lets the cooperative grid
                // kernel's blocks in ahead of the list build's; on the main stream the list's rows and then the
                // records with the permanent field's direct part (once the spread wrote the sources), or, with a
                // kept list, its compaction and records and then the permanent field's pair pass
                CU(cudaEventRecord(evFork, sm));
                CU(cudaStreamWaitEvent(sd, evFork, 0));
                k_splines<R><<<(3 * n + 255) / 256, 256, 0, sd>>>(d);
                if (std::is_same<R, float>::value && planesMode())
                    enqueuePlaneBins(sd, d);
                k_perm<<<tb, 256, 0, sd>>>(d);
                k_influence<R><<<dim3(convBlocks, nsys), 256, 0, sd>>>(d);
                CU(cudaMemsetAsync(d.grid, 0, gridTotal * realSize(), sd));
                launchSpread<R>(sd, d, 0, d.perm);
                CU(cudaEventRecord(evPerm, sd));
                transformPair<R>(sd, d, false, spreadFix());
                launchGather<R, false>(sd, d, 0);
                CU(cudaEventRecord(evJoin, sd));
                if (rowsLeft) {
                    listKernel(sm, d);
                    CU(cudaStreamWaitEvent(sm, evPerm, 0));
                    k_pair_kernels<R, true><<<(n + 7) / 8, 256, 0, sm>>>(d);
                } else {
                    pairRecords<R>(sm, d);
                    CU(cudaStreamWaitEvent(sm, evPerm, 0));
                    pairField<R, true>(sm, d, 0);
                }
                CU(cudaStreamWaitEvent(sm, evJoin, 0));
                k_cg_b<<<(int) chunkSys.size(), CHUNK, 0, sm>>>(d);
                CU(cudaGetLastError());
                if (pcg) {   // A x0 as one pass of the persistent kernel, then the loop's set-up
                    launchPersistent(sm, d, 1, d.x);
                    k_cg_init<<<(int) chunkSys.size(), CHUNK, 0, sm>>>(d);
                    CU(cudaGetLastError());
                    return;
                }
                CU(cudaMemsetAsync(d.grid, 0, gridTotal * realSize(), sm));
                fieldPass<R, false>(sm, sd, d, 1, d.x, false);
                k_cg_init<<<(int) chunkSys.size(), CHUNK, 0, sm>>>(d);
                CU(cudaGetLastError());
                // the loop's first spread needs a clear grid (each iteration clears it for the next one)
                CU(cudaMemsetAsync(d.grid, 0, gridTotal * realSize(), sm));
                return;
            }
            // a predicted step (dualFirstPass): x0 from the history first; (q, perm) into the grid and dS, x0 into
            // the second grid and dS2, both PME halves on the high-priority side stream (the transforms in sequence:
            // one spectrum buffer, one set of the grid kernel's barrier words); on the main stream the list's rows
            // and records, then one pair sweep for both direct fields once the spreads wrote their sources
            Dev d2 = d;   // the second source set: its grids, its float copy, its reciprocal field
            d2.grid = dGrid2.p;
            d2.gridFix = d.gridFix ? dGridFix2.as<long long>() : nullptr;
            d2.dS = dDS2.p;
            d2.Erec = dErec2.as<double>();
            CU(cudaEventRecord(evFork, sm));
            CU(cudaStreamWaitEvent(sd, evFork, 0));
            k_splines<R><<<(3 * n + 255) / 256, 256, 0, sd>>>(d);
            if (std::is_same<R, float>::value && planesMode())
                enqueuePlaneBins(sd, d);
            k_perm<<<tb, 256, 0, sd>>>(d);
            k_influence<R><<<dim3(convBlocks, nsys), 256, 0, sd>>>(d);
            k_cg_guess<<<(3 * n + 255) / 256, 256, 0, sd>>>(d);
            CU(cudaMemsetAsync(d.grid, 0, gridTotal * realSize(), sd));
            CU(cudaMemsetAsync(d2.grid, 0, gridTotal * realSize(), sd));
            launchSpread<R>(sd, d, 0, d.perm);
            launchSpread<R>(sd, d2, 1, d.x);
            CU(cudaEventRecord(evPerm, sd));
            transformPair<R>(sd, d, false, spreadFix());
            launchGather<R, false>(sd, d, 0);
            transformPair<R>(sd, d2, false, spreadFix());
            launchGather<R, false>(sd, d2, 0);
            CU(cudaEventRecord(evJoin, sd));
            if (rowsLeft)
                listKernel(sm, d);
            pairRecords<R>(sm, d);
            CU(cudaStreamWaitEvent(sm, evPerm, 0));
            pairField<R, true, true>(sm, d, 0);
            CU(cudaStreamWaitEvent(sm, evJoin, 0));
            k_cg_b<<<(int) chunkSys.size(), CHUNK, 0, sm>>>(d);
            Dev d3 = d;   // T x0: the second set's pair and reciprocal fields
            d3.Epair = dEpair2.as<double>();
            d3.Erec = dErec2.as<double>();
            k_cg_init<<<(int) chunkSys.size(), CHUNK, 0, sm>>>(d3);
            CU(cudaGetLastError());
            CU(cudaMemsetAsync(d.grid, 0, gridTotal * realSize(), sm));
        } else {
            if (rowsLeft)
                listKernel(sm, d);
            pairRecords<R>(sm, d);
            k_splines<R><<<(3 * n + 255) / 256, 256, 0, sm>>>(d);
            if (std::is_same<R, float>::value && planesMode())
                enqueuePlaneBins(sm, d);
            k_perm<<<tb, 256, 0, sm>>>(d);
            k_influence<R><<<dim3(convBlocks, nsys), 256, 0, sm>>>(d);
            CU(cudaGetLastError());
        }
    }

    template <typename R> void enqueueIteration(cudaStream_t sm, cudaStream_t sd, const Dev& d) {
        if (nsys == 1 && fuseCgA && !(std::is_same<R, float>::value && planesMode())) {   // A p, alph in the gather
            fieldPass<R, false, true>(sm, sd, d, 2, d.p, true);
        } else {
            fieldPass<R, false>(sm, sd, d, 2, d.p, true);
            k_cg_a<<<(int) chunkSys.size(), CHUNK, 0, sm>>>(d);
        }
        k_cg_upd<<<(int) chunkSys.size(), CHUNK, 0, sm>>>(d);
        CU(cudaGetLastError());
    }

    template <typename R> void enqueuePost(cudaStream_t sm, cudaStream_t sd, const Dev& d) {
        const int tb = (n + 255) / 256;
        CU(cudaMemsetAsync(d.grid, 0, gridTotal * realSize(), sm));
        k_final_prep<<<tb, 256, 0, sm>>>(d, s.polarizable ? 1 : 0);
        launchSpread<R>(sm, d, 0, d.dtot);
        CU(cudaEventRecord(evFork, sm));
        CU(cudaStreamWaitEvent(sd, evFork, 0));
        // the final pass's transforms with the reciprocal energy: the grid kernel's energy variant where the field
        // passes run the grid kernel, else cuFFT and the product kernel
        if ((tfMode == TF_GRID || tfMode == TF_PCG) && gridEnergyOk && std::is_same<R, float>::value == mixed())
            launchGrid<R>(sd, d, (spreadFix() && std::is_same<R, float>::value && d.gridFix) ? 2 : 0, true);
        else
            fftChain<R>(sd, d, true, false, spreadFix());
        {
            const long long threads = (long long) n * pairGS;
            const int blocks = (int) ((threads + 255) / 256);
            switch (pairGS) {
            case 4: k_pair_final<R, 4><<<blocks, 256, 0, sm>>>(d); break;
            case 16: k_pair_final<R, 16><<<blocks, 256, 0, sm>>>(d); break;
            case 32: k_pair_final<R, 32><<<blocks, 256, 0, sm>>>(d); break;
            default: k_pair_final<R, 8><<<blocks, 256, 0, sm>>>(d);
            }
        }
        if (gvdwOn)   // (adds to the final pair pass's force and strain)
            k_gvdw<R><<<(n + 7) / 8, 256, 0, sm>>>(d);
        CU(cudaEventRecord(evJoin, sd));
        CU(cudaStreamWaitEvent(sm, evJoin, 0));
        launchGather<R, true>(sm, d, 0);
        k_final_field<<<tb, 256, 0, sm>>>(d);
        k_final_forces<<<(int) chunkSys.size(), CHUNK, 0, sm>>>(d, s.polarizable ? 1 : 0);
        CU(cudaGetLastError());
    }

    template <typename R> void captureGraph() {
        if (exec) {
            cudaGraphExecDestroy(exec);
            exec = nullptr;
        }
        cudaGraph_t graph;
        CU(cudaGraphCreate(&graph, 0));
        cudaGraphConditionalHandle handle = 0, listHandle = 0;
        const bool loopNode = s.polarizable && !persistentMode();   // (the persistent kernel loops by itself)
        if (loopNode)
            CU(cudaGraphConditionalHandleCreate(&handle, graph, 0, cudaGraphCondAssignDefault));
        if (verletList())   // (a handle without its conditional node makes the instantiation fail)
            CU(cudaGraphConditionalHandleCreate(&listHandle, graph, 0, cudaGraphCondAssignDefault));
        const Dev d = makeDev(true, handle, listHandle);
        CU(cudaStreamBeginCaptureToGraph(st, graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        cudaGraph_t body = nullptr;
        capturing = true;
        listBody = nullptr;
        const int unroll = (loopNode && nsys == 1) ? unrollWant : 0;
        try {
            enqueuePre<R>(st, side, d);
            if (loopNode) {   // the CG loop: unrolled iterations (gated by the system's convergence), then the node
                for (int u = 0; u < unroll; u++)
                    enqueueIteration<R>(st, side, d);
                body = appendConditional(st, handle, cudaGraphCondTypeWhile);
            }
            else if (s.polarizable)
                launchPersistent(st, d);
            enqueuePost<R>(st, side, d);
        } catch (...) {
            capturing = false;
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(st, &g);
            if (g)
                cudaGraphDestroy(g);
            cudaGraphDestroy(graph);
            throw;
        }
        capturing = false;
        CU(cudaStreamEndCapture(st, &graph));
        if (listBody) {   // (no skin: the build is part of the main graph)
            CU(cudaStreamBeginCaptureToGraph(st, listBody, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
            try {
                enqueueBuild(st, d);
            } catch (...) {
                cudaGraph_t g = nullptr;
                cudaStreamEndCapture(st, &g);
                cudaGraphDestroy(graph);
                throw;
            }
            CU(cudaStreamEndCapture(st, &listBody));
        }
        if (body) {
            CU(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
            try {
                enqueueIteration<R>(st, side, d);
            } catch (...) {
                cudaGraph_t g = nullptr;
                cudaStreamEndCapture(st, &g);
                cudaGraphDestroy(graph);
                throw;
            }
            CU(cudaStreamEndCapture(st, &body));
        }
        CU(cudaGraphInstantiate(&exec, graph, cudaGraphInstantiateFlagUseNodePriority));
        graphCells = totalCells;
        graphDual = dualFirstPass();
        graphUnroll = unroll;
        graphLoop = loopNode;
        evalsSinceCapture = 0;
        {
            int G, cap, groups;
            tileGeometry(G, cap, groups);
            graphTiles[0] = groups;
            graphTiles[1] = cap;
        }
        CU(cudaGraphDestroy(graph));
    }

    template <typename R> void runDirect() {
        const Dev d = makeDev(false, 0);
        enqueuePre<R>(st, side, d);
        if (s.polarizable && persistentMode()) {
            launchPersistent(st, d);
        } else if (s.polarizable) {
            static const bool trace = std::getenv("PGM_B200_TRACE") != nullptr;
            for (int it = 0; it <= s.maxIter + 1; it++) {
                CU(cudaMemcpyAsync(hFlags, d.flags, 16 * sizeof(int), cudaMemcpyDeviceToHost, st));
                CU(cudaStreamSynchronize(st));
                if (trace) {
                    double sc[NSCAL];
                    CU(cudaMemcpy(sc, d.scal, sizeof(sc), cudaMemcpyDeviceToHost));
                    fprintf(stderr, "pgm_b200 trace: it %d done %d/%d system 0: norm %.6e rz %.6e alph %.6e beta %.6e "
                            "err %.6e\n", it, hFlags[2], nsys, sc[SC_NORM], sc[SC_RZ], sc[SC_ALPH], sc[SC_BETA],
                            sc[SC_ERR]);
                }
                if (hFlags[2] >= nsys)
                    break;
                enqueueIteration<R>(st, side, d);
            }
        }
        enqueuePost<R>(st, side, d);
    }

    // Mixed path with FP64 iterative refinement: the FP32-operator CG, then up to three rounds of
    //   r = E_perm - (alpha^-1 - T) x   with FP64 pair and PME arithmetic (FP64 G1, G2, splines, grids, D2Z/Z2D),
    //   stop when max|alpha r| / mean|alpha E_perm| <= tol, else solve (alpha^-1 - T) delta = r with the FP32-operator
    //   CG and x += delta;
    // the peek step then uses the FP64 residual.  Direct launches (the rounds depend on host-read residuals).
    void runRefined() {
        static const bool trace = std::getenv("PGM_B200_TRACE") != nullptr;
        const Dev d = makeDev(false, 0);
        const Dev d64 = makeDev64();
        auto cgLoop = [&]() {
            for (int it = 0; it <= s.maxIter + 1; it++) {
                CU(cudaMemcpyAsync(hFlags, d.flags, 16 * sizeof(int), cudaMemcpyDeviceToHost, st));
                CU(cudaStreamSynchronize(st));
                if (hFlags[2] >= nsys)
                    break;
                enqueueIteration<float>(st, side, d);
            }
        };
        enqueuePre<float>(st, side, d);
        cgLoop();
        // FP64 geometry: G1, G2, splines and influence in double
        k_pair_kernels<double><<<(n + 7) / 8, 256, 0, st>>>(d64);
        k_splines<double><<<(3 * n + 255) / 256, 256, 0, st>>>(d64);
        k_influence<double><<<dim3(convBlocks, nsys), 256, 0, st>>>(d64);
        CU(cudaMemsetAsync(d64.grid, 0, gridTotal * 8, st));
        fieldPass<double, true>(st, side, d64, 0, d.perm, false);
        k_refine_b<<<(n + 255) / 256, 256, 0, st>>>(d64, dB64.as<double>());
        CU(cudaGetLastError());
        for (int round = 0; round < 4; round++) {
            CU(cudaMemsetAsync(d64.grid, 0, gridTotal * 8, st));
            CU(cudaMemsetAsync(d.flags + 2, 0, sizeof(int), st));
            fieldPass<double, false>(st, side, d64, 1, d.x, false);
            k_refine_res<<<(int) chunkSys.size(), CHUNK, 0, st>>>(d64, dB64.as<double>());
            CU(cudaMemcpyAsync(hFlags, d.flags, 16 * sizeof(int), cudaMemcpyDeviceToHost, st));
            CU(cudaStreamSynchronize(st));
            if (trace) {
                double sc[NSCAL];
                CU(cudaMemcpy(sc, d.scal, sizeof(sc), cudaMemcpyDeviceToHost));
                fprintf(stderr, "pgm_b200 trace: refinement round %d: FP64 residual %.3e (system 0)\n", round,
                        sc[SC_ERR]);
            }
            if (hFlags[2] >= nsys || round == 3)
                break;
            // correction: (alpha^-1 - T) delta = r with the FP32 operator, from delta = 0
            CU(cudaMemcpyAsync(dXsave.p, d.x, 3 * (size_t) n * 8, cudaMemcpyDeviceToDevice, st));
            hCtl->customRhs = 1;
            hCtl->guess = 1;
            CU(cudaMemcpyAsync(dCtl.p, hCtl, sizeof(Ctl), cudaMemcpyHostToDevice, st));
            CU(cudaMemsetAsync(d.flags, 0, flagBytes(), st));
            k_cg_b<<<(int) chunkSys.size(), CHUNK, 0, st>>>(d);
            CU(cudaMemsetAsync(d.grid, 0, gridTotal * realSize(), st));
            fieldPass<float, false>(st, side, d, 1, d.x, false);
            k_cg_init<<<(int) chunkSys.size(), CHUNK, 0, st>>>(d);
            CU(cudaMemsetAsync(d.grid, 0, gridTotal * realSize(), st));
            cgLoop();
            k_refine_add<<<(3 * n + 255) / 256, 256, 0, st>>>(d, dXsave.as<double>());
            hCtl->customRhs = 0;
            CU(cudaMemcpyAsync(dCtl.p, hCtl, sizeof(Ctl), cudaMemcpyHostToDevice, st));
            CU(cudaGetLastError());
        }
        // r now holds the FP64 residual of x: the final pass's peek uses it
        enqueuePost<float>(st, side, d);
    }

    // ------------------------------------------------------------------------------------------ evaluation
    void prepareControl(bool newStep, int posMode, const void* posDevice, long long* forceFixed, int stride,
                        double fixedScale, double* forcesOut) {
        Ctl& c = *hCtl;
        std::memset(&c, 0, sizeof(c));
        const int h = histCount;
        auto slot = [&](int back) { return (histHead + back) % NHIST; };
        if (!s.polarizable)
            c.guess = 0;
        else if (!newStep && h > 0)
            c.guess = 2;
        else if (s.predictor == 2 && h >= 4)
            c.guess = 4;
        else if (s.predictor >= 1 && h >= 3)
            c.guess = 3;
        else if (s.predictor >= 1 && h >= 1)
            c.guess = 2;
        else
            c.guess = s.zeroGuess ? 1 : 0;
        for (int k = 0; k < 4; k++)
            c.h[k] = slot(k);
        const bool push = s.polarizable && (newStep || h == 0) && nsys == 1;
        pendingSlot = push ? (histHead + NHIST - 1) % NHIST : -1;
        c.histSlot = pendingSlot;
        c.posMode = posMode;
        c.posDevice = posDevice;
        c.forceFixed = forceFixed;
        c.fixedStride = stride;
        c.fixedScale = fixedScale;
        c.forcesOut = forcesOut;
    }

    // Enqueues one evaluation on st (inputs already staged); host waits only in finish().
    void launch(const double* boxes) {
        if (!configured || !atomsSet)
            throw std::logic_error("pgm_b200: compute before setAtoms");
        const bool grew = setBoxes(boxes);
        // the graph's launch shapes hold the cell count (another box can change it without growing the storage)
        // and the tile kernels' groups
        int tG, tCap, tGroups;
        tileGeometry(tG, tCap, tGroups);
        if ((grew || totalCells != graphCells || tGroups != graphTiles[0] || tCap != graphTiles[1] ||
             dualFirstPass() != graphDual || unrollStale()) && exec) {
            cudaGraphExecDestroy(exec);
            exec = nullptr;
        }
        // the Verlet list is built anew when there is none, the boxes changed or the skin is 0; else the device
        // decides from the displacements
        launchBoxes.assign(boxes, boxes + 9 * (size_t) nsys);
        const bool sameBoxes = listValid && buildBoxes == launchBoxes;
        hCtl->forceRebuild = (!sameBoxes || grew || !verletList()) ? 1 : 0;
        std::memcpy(hSys, sysHost.data(), nsys * sizeof(SysDev));
        CU(cudaMemcpyAsync(dSys.p, hSys, nsys * sizeof(SysDev), cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(dCtl.p, hCtl, sizeof(Ctl), cudaMemcpyHostToDevice, st));
        if (refining()) {
            runRefined();
        } else if (useGraph) {
            if (!exec) {
                try {
                    if (mixed())
                        captureGraph<float>();
                    else
                        captureGraph<double>();
                } catch (const std::exception& e) {
                    fprintf(stderr, "pgm_b200: graph capture failed (%s), running without graphs\n", e.what());
                    cudaGetLastError();
                    useGraph = false;
                }
            }
        }
        if (refining())
            ;
        else if (useGraph)
            CU(cudaGraphLaunch(exec, st));
        else if (mixed())
            runDirect<float>();
        else
            runDirect<double>();
        CU(cudaMemcpyAsync(hResults, dResults.p, nsys * NRES * 8, cudaMemcpyDeviceToHost, st));
        CU(cudaMemcpyAsync(hFlags, dFlags.p, 16 * sizeof(int), cudaMemcpyDeviceToHost, st));
        CU(cudaEventRecord(evDone, st));
        launched = true;
    }

    // The flags and the grid transforms' barrier words (cleared together at the start of every call).
    // (16 flags, 2 barrier words per system for the grid transforms, 2 for the persistent CG kernel)
    size_t flagBytes() const { return (16 + 2 * (size_t) nsys + 2) * sizeof(int); }

    // After the flags came back: a grid-transform barrier that gave up leaves the evaluation's results
    // undefined (the barrier words are reset at the next evaluation's start).
    void barrierCheck() const {
        if (hFlags[11])
            throw std::runtime_error("pgm_b200: a grid-transform barrier gave up waiting (blocks not resident "
                                     "together?)");
    }

    // Waits for the launched evaluation; false if it must be repeated (pair-list capacity grown).
    bool finish() {
        CU(cudaEventSynchronize(evDone));
        launched = false;
        if (hFlags[1])
            throw std::runtime_error("pgm_b200: pair image shift beyond 3 boxes (positions far outside the box?)");
        barrierCheck();
        lastBuilt = hFlags[8] != 0;
        if (hFlags[8]) {
            builds++;
            buildBoxes = launchBoxes;
            listValid = true;
        }
        if (hFlags[0] > cap) {
            cap = (hFlags[0] + hFlags[0] / 4 + 31) / 32 * 32;
            allocList();
            if (exec) {
                cudaGraphExecDestroy(exec);
                exec = nullptr;
            }
            return false;
        }
        if (hFlags[9]) {   // a pair within the cutoff changed its image since the build: rebuild and repeat
            listValid = false;
            return false;
        }
        lastResults.assign(hResults, hResults + nsys * NRES);
        haveResult = true;
        if (nsys == 1 && s.polarizable) {   // the unroll of the next capture
            recentIt[recentCount++ % 4] = (int) hResults[14];
            evalsSinceCapture++;
            static const char* env = std::getenv("PGM_B200_UNROLL");   // (a cap; 0 keeps the plain while node)
            const int cap = env ? std::atoi(env) : 16;
            int m = recentIt[0];
            for (int k = 1; k < std::min(recentCount, 4); k++)
                m = std::min(m, recentIt[k]);
            unrollWant = std::max(0, std::min(m, cap));
        }
        if (pendingSlot >= 0) {
            histHead = pendingSlot;
            histCount = std::min(histCount + 1, 4);
            pendingSlot = -1;
        }
        return true;
    }

    Terms termsOf(int k) const {
        Terms t;
        const double* r = lastResults.data() + (size_t) k * NRES;
        t.direct = r[0];
        t.reciprocal = r[1];
        t.self = r[2];
        t.background = r[3];
        t.polarization = r[4];
        t.gvdw = r[16];
        return t;
    }

    void checkPositions(const double* pos, size_t m) {
        for (size_t k = 0; k < m; k++)
            if (!std::isfinite(pos[k]))
                throw std::invalid_argument("pgm_b200: non-finite position");
    }

    // Host double positions, full evaluation, forces to the pinned buffer.
    Terms evalHost(const double* pos, const double* boxes, bool newStep, bool wantForces) {
        // one pass: the finiteness check with the copy into the pinned staging buffer
        const size_t m = 3 * (size_t) n;
        bool finite = true;
        for (size_t k = 0; k < m; k++) {
            const double v = pos[k];
            finite &= std::isfinite(v);
            hPos[k] = v;
        }
        if (!finite)
            throw std::invalid_argument("pgm_b200: non-finite position");
        selectDevice();
        for (int attempt = 0; attempt < 4; attempt++) {
            prepareControl(newStep, 0, nullptr, nullptr, 0, 0.0, nullptr);
            CU(cudaMemcpyAsync(dPosIn.p, hPos, 3 * (size_t) n * 8, cudaMemcpyHostToDevice, st));
            launch(boxes);
            if (wantForces) {
                CU(cudaMemcpyAsync(hForces, dForces.p, 3 * (size_t) n * 8, cudaMemcpyDeviceToHost, st));
                CU(cudaEventRecord(evDone, st));
            }
            if (finish())
                return termsOf(0);
        }
        throw std::runtime_error("pgm_b200: pair list did not fit after growing it");
    }
};

// ---------------------------------------------------------------------------------------------- Engine

Engine::Engine(const Settings& settings) : impl(new Impl) {
    try {
        impl->init(settings);
    } catch (...) {
        delete impl;
        throw;
    }
}

Engine::~Engine() { delete impl; }

void Engine::setAtoms(int n, const double* q, const double* radius, const double* alpha, const int* globalIndex,
                      int numGlobal) {
    impl->selectDevice();
    impl->setAtomsSingle(n, q, radius, alpha, globalIndex, numGlobal);
}

// Self-test of the grid transforms' bounded barrier: one block waits at a barrier that expects two; the wait
// runs out, sets the error flag and returns.  Returns the flag (1: the wait gave up as designed) and the
// device time of the launch.
int Engine::probeBarrierTimeout(double* seconds) {
    Impl& I = *impl;
    I.selectDevice();
    void* mem = nullptr;
    CU(cudaMalloc(&mem, 64 * sizeof(int)));
    int* words = (int*) mem;
    CU(cudaMemsetAsync(words, 0, 64 * sizeof(int), I.st));
    cudaEvent_t a, b;
    CU(cudaEventCreate(&a));
    CU(cudaEventCreate(&b));
    CU(cudaEventRecord(a, I.st));
    k_barrier_probe<<<1, 32, 0, I.st>>>((unsigned*) (words + 16), words);
    CU(cudaGetLastError());
    CU(cudaEventRecord(b, I.st));
    int flags[16];
    CU(cudaMemcpyAsync(flags, words, sizeof(flags), cudaMemcpyDeviceToHost, I.st));
    CU(cudaStreamSynchronize(I.st));
    float ms = 0.0f;
    CU(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    CU(cudaFree(mem));
    if (seconds)
        *seconds = ms * 1e-3;
    return flags[11];
}

// The caller's pair candidates (core/cuda/pgm_cuda.h:68-73): segment sg holds the pairs (segI[sg], candJ[k]),
// k in [segBegin[sg], segBegin[sg + 1]), with x = r_i + t.box - r_j, t = segShift[3 sg .. 3 sg + 2] integer box
// vectors; every pair at most once.  Kept per atom in both directions ((i, j, t) and (j, i, -t)), in the
// caller's order; they replace the engine's cell search until the next setAtoms, and the pairs beyond the
// cutoff are left out at every evaluation.
void Engine::setCandidates(int nseg, const int* segI, const int* segShift, const int* segBegin, const int* candJ) {
    Impl& I = *impl;
    if (!I.atomsSet || I.nsys != 1)
        throw std::logic_error("pgm_b200: setCandidates needs a single-system engine with atoms set");
    if (nseg < 0 || (nseg > 0 && (!segI || !segShift || !segBegin)))
        throw std::invalid_argument("pgm_b200: setCandidates: bad segment arrays");
    I.selectDevice();
    const int n = I.n;
    const int total = nseg > 0 ? segBegin[nseg] : 0;
    if (nseg > 0 && (segBegin[0] != 0 || total < 0 || (total > 0 && !candJ)))
        throw std::invalid_argument("pgm_b200: setCandidates: segBegin must start at 0 and candJ hold its total");
    // every candidate as two directed entries (owner, partner, shift of the partner's image seen from the
    // owner), then grouped by owner with a stable sort, so each row keeps the caller's order
    struct Directed {
        int owner, partner, shift;
    };
    auto packShift = [](const int* t, int sign) {
        return (sign * t[0] + 128) | ((sign * t[1] + 128) << 8) | ((sign * t[2] + 128) << 16);
    };
    std::vector<Directed> entries;
    entries.reserve(2 * (size_t) std::max(total, 0));
    for (int sg = 0; sg < nseg; sg++) {
        const int i = segI[sg];
        const int* t = segShift + 3 * sg;
        if (i < 0 || i >= n || segBegin[sg + 1] < segBegin[sg])
            throw std::invalid_argument("pgm_b200: setCandidates: atom index or segment bounds out of range");
        if (std::abs(t[0]) > 127 || std::abs(t[1]) > 127 || std::abs(t[2]) > 127)
            throw std::invalid_argument("pgm_b200: setCandidates: box shift out of range");
        for (int k = segBegin[sg]; k < segBegin[sg + 1]; k++) {
            if (candJ[k] < 0 || candJ[k] >= n)
                throw std::invalid_argument("pgm_b200: setCandidates: partner index out of range");
            entries.push_back({i, candJ[k], packShift(t, 1)});
            entries.push_back({candJ[k], i, packShift(t, -1)});
        }
    }
    std::stable_sort(entries.begin(), entries.end(),
                     [](const Directed& a, const Directed& b) { return a.owner < b.owner; });
    std::vector<int> start(n + 1, 0), jj(std::max<size_t>(1, entries.size())), tt(jj.size());
    for (size_t k = 0; k < entries.size(); k++) {
        start[entries[k].owner + 1] = (int) k + 1;   // one past the owner's last entry
        jj[k] = entries[k].partner;
        tt[k] = entries[k].shift;
    }
    int longest = 0;
    for (int i = 0; i < n; i++) {   // owners without entries continue from their predecessor
        start[i + 1] = std::max(start[i + 1], start[i]);
        longest = std::max(longest, start[i + 1] - start[i]);
    }
    CU(cudaStreamSynchronize(I.st));
    upload(I.dCandStart, start, I.st);
    upload(I.dCandJ, jj, I.st);
    upload(I.dCandT, tt, I.st);
    CU(cudaStreamSynchronize(I.st));
    if (longest > I.cap) {   // rows for the longest candidate row
        I.cap = (longest + 31) / 32 * 32;
        I.allocList();
    }
    I.externalList = true;
    I.listValid = false;
    if (I.exec) {   // the graph holds the list's shape
        cudaGraphExecDestroy(I.exec);
        I.exec = nullptr;
    }
}

// The series of the GVDW G(y) / G(0) in y^2, c[0..K-1]: with A(y) = (2/sqrt(pi)) sum a_n y^(2n+1) from the series of
// erf and exp (a_0 = a_1 = 0), G pi/4 = y^4 (sum_{n>=2} a_n y^(2n-4))^2 + (2/9) e^(-2 y^2).
void gvdwSeries(double* c, int K) {
    std::vector<double> a(K + 3), coef(K);
    double fact = 1.0;   // n!
    for (int n2 = 0; n2 < K + 3; n2++) {
        if (n2 > 0)
            fact *= n2;
        const double sg = (n2 % 2) ? -1.0 : 1.0;
        double t = sg / (fact * (2 * n2 + 1)) - sg / fact;
        if (n2 >= 1)
            t -= (2.0 / 3.0) * (-sg) / (fact / n2);
        a[n2] = t;
    }
    fact = 1.0;
    for (int k = 0; k < K; k++) {
        if (k > 0)
            fact *= k;
        coef[k] = (2.0 / 9.0) * std::pow(-2.0, k) / fact;
    }
    for (int m1 = 0; m1 < K; m1++)
        for (int m2 = 0; m1 + m2 + 2 < K; m2++)
            coef[m1 + m2 + 2] += a[m1 + 2] * a[m2 + 2];
    for (int k = 0; k < K; k++)
        c[k] = coef[k] / coef[0];
}

// The combination-rule GVDW (core/cuda/pgm_cuda.h:57-65): per atom sqrt(A), sqrt(C6), b (zeros: none),
// repulsion 0 Gaussian, 1 Slater; the pairs within rvdw except the skipped ones (once each), added in the final
// pass (energy Terms::gvdw, forces and strain added to the evaluation's).  rvdw may not exceed the cutoff (the
// pass runs over the evaluation's pair list).  Until the next setAtoms.
void Engine::setGvdw(int repulsion, double rvdw, const double* sqrtA, const double* sqrtC6, const double* b, int nskip,
                     const int* skipI, const int* skipJ) {
    Impl& I = *impl;
    if (!I.atomsSet || I.nsys != 1)
        throw std::logic_error("pgm_b200: setGvdw needs a single-system engine with atoms set");
    if (repulsion != 0 && repulsion != 1)
        throw std::invalid_argument("pgm_b200: GVDW repulsion must be 0 (Gaussian) or 1 (Slater)");
    if (!(rvdw > 0) || rvdw > I.s.cutoff * (1.0 + 1e-12))
        throw std::invalid_argument("pgm_b200: GVDW radius must be positive and at most the cutoff (the pass runs "
                                    "over the evaluation's pair list)");
    const int n = I.n;
    if (!sqrtA || !sqrtC6 || !b || nskip < 0 || (nskip > 0 && (!skipI || !skipJ)))
        throw std::invalid_argument("pgm_b200: setGvdw arguments");
    std::vector<double> gv(4 * (size_t) n);
    for (int i = 0; i < n; i++) {
        if (!std::isfinite(sqrtA[i]) || !std::isfinite(sqrtC6[i]) || !std::isfinite(b[i]))
            throw std::invalid_argument("pgm_b200: non-finite GVDW parameter");
        gv[4 * i] = sqrtA[i];
        gv[4 * i + 1] = sqrtC6[i];
        gv[4 * i + 2] = b[i];
        gv[4 * i + 3] = 0.0;
    }
    // the skipped pairs in both directions, ordered by (atom, partner); row a is the run of atom a
    std::vector<std::pair<int, int>> skipped;
    skipped.reserve(2 * (size_t) nskip);
    for (int k = 0; k < nskip; k++) {
        if (skipI[k] < 0 || skipI[k] >= n || skipJ[k] < 0 || skipJ[k] >= n)
            throw std::invalid_argument("pgm_b200: GVDW skipped pair index out of range");
        skipped.emplace_back(skipI[k], skipJ[k]);
        skipped.emplace_back(skipJ[k], skipI[k]);
    }
    std::sort(skipped.begin(), skipped.end());
    std::vector<int> start(n + 1), part(std::max<size_t>(1, skipped.size()));
    for (int a = 0; a <= n; a++)
        start[a] = (int) (std::lower_bound(skipped.begin(), skipped.end(), std::make_pair(a, INT_MIN)) -
                          skipped.begin());
    for (size_t k = 0; k < skipped.size(); k++)
        part[k] = skipped[k].second;
    gvdwSeries(I.gvC, GVDW_TERMS);
    I.selectDevice();
    CU(cudaStreamSynchronize(I.st));
    upload(I.dGv, gv, I.st);
    upload(I.dSkipStart, start, I.st);
    upload(I.dSkipJ, part, I.st);
    CU(cudaStreamSynchronize(I.st));
    I.gvdwOn = true;
    I.gvdwSlater = repulsion == 1;
    I.rvdw = rvdw;
    if (I.exec) {   // the graph gains the GVDW pass
        cudaGraphExecDestroy(I.exec);
        I.exec = nullptr;
    }
}

void Engine::setCovalent(int ncov, const int* atom, const int* partner, const double* strength) {
    impl->selectDevice();
    impl->setCovalentSingle(ncov, atom, partner, strength);
}

Terms Engine::compute(const double* pos, const double box[3][3], bool newStep, double* f, double* strain) {
    Impl& I = *impl;
    if (I.nsys != 1)
        throw std::logic_error("pgm_b200: compute on a batched engine (use computeBatch)");
    const Terms t = I.evalHost(pos, &box[0][0], newStep, f != nullptr);
    if (f)
        for (int k = 0; k < 3 * I.n; k++)
            f[k] += I.hForces[k];
    if (strain)
        for (int k = 0; k < 9; k++)
            strain[k] += I.lastResults[5 + k];
    return t;
}

Terms Engine::computeF(const float* pos, const double box[3][3], bool newStep, double* strain) {
    Impl& I = *impl;
    if (!I.atomsSet)
        throw std::logic_error("pgm_b200: compute before setAtoms");
    std::vector<double> pd(pos, pos + 3 * (size_t) I.n);
    const Terms t = I.evalHost(pd.data(), &box[0][0], newStep, true);
    I.forcesHostCache.assign(I.hForces, I.hForces + 3 * (size_t) I.n);
    if (strain)
        for (int k = 0; k < 9; k++)
            strain[k] += I.lastResults[5 + k];
    return t;
}

const double* Engine::forces() const { return impl->forcesHostCache.data(); }

void Engine::launchDevice(const void* posq4, const double box[3][3], bool newStep, long long* forceFixed, int stride,
                          double fixedScale, void* stream) {
    Impl& I = *impl;
    I.selectDevice();
    I.callerStream = (cudaStream_t) stream;
    // the caller's work so far comes first
    CU(cudaEventRecord(I.evCaller, I.callerStream));
    CU(cudaStreamWaitEvent(I.st, I.evCaller, 0));
    I.prepareControl(newStep, 1, posq4, forceFixed, stride, fixedScale, nullptr);
    I.launch(&box[0][0]);
}

bool Engine::finishDevice(Terms& terms) {
    Impl& I = *impl;
    if (!I.launched)
        throw std::logic_error("pgm_b200: finishDevice without launchDevice");
    if (!I.finish())
        return false;   // the pair list outgrew its capacity: grown now; the caller repeats the evaluation
    terms = I.termsOf(0);
    return true;
}

void Engine::waitDevice(void* stream) {
    Impl& I = *impl;
    CU(cudaStreamWaitEvent((cudaStream_t) stream, I.evDone, 0));
}

Terms Engine::computeDevice(const void* posq4, const double box[3][3], bool newStep, long long* forceFixed, int stride,
                            double fixedScale, void* stream) {
    launchDevice(posq4, box, newStep, forceFixed, stride, fixedScale, stream);
    Terms t;
    finishDevice(t);
    return t;
}

void Engine::launchResident(const double* posDev, const double box[3][3], bool newStep, double* forcesDev,
                            void* stream) {
    Impl& I = *impl;
    I.selectDevice();
    if (stream) {
        CU(cudaEventRecord(I.evCaller, (cudaStream_t) stream));
        CU(cudaStreamWaitEvent(I.st, I.evCaller, 0));
    }
    I.prepareControl(newStep, 2, posDev, nullptr, 0, 0.0, forcesDev);
    I.launch(&box[0][0]);
}

int Engine::iterations() const { return impl->haveResult ? (int) impl->lastResults[14] : 0; }
double Engine::residual() const { return impl->haveResult ? impl->lastResults[15] : 0.0; }

void Engine::inducedDipoles(double* mu) const {
    CU(cudaMemcpy(mu, impl->dMu.p, 3 * (size_t) impl->n * 8, cudaMemcpyDeviceToHost));
}

void Engine::permanentDipoles(double* p) const {
    CU(cudaMemcpy(p, impl->dPerm.p, 3 * (size_t) impl->n * 8, cudaMemcpyDeviceToHost));
}

void Engine::resetHistory() { impl->resetHistoryState(); }
long Engine::listBuilds() const { return impl->builds; }

int Engine::numCandidates() const {
    std::vector<int> c(impl->n);
    CU(cudaMemcpy(c.data(), impl->dListCount.p, impl->n * sizeof(int), cudaMemcpyDeviceToHost));
    long long s = 0;
    for (int v : c)
        s += v;
    return (int) s;
}

std::array<double, 9> Engine::strainDerivative() const {
    std::array<double, 9> a{};
    if (impl->haveResult)
        for (int k = 0; k < 9; k++)
            a[k] = impl->lastResults[5 + k];
    return a;
}

long long Engine::pairs(int* pi, int* pj, long long cap) {
    Impl& I = *impl;
    std::vector<int> cnt(I.n), slotAtom(I.n);
    std::vector<uint32_t> list((size_t) I.n * I.cap);
    CU(cudaMemcpy(cnt.data(), I.dListCount.p, I.n * sizeof(int), cudaMemcpyDeviceToHost));
    CU(cudaMemcpy(slotAtom.data(), I.dSlotAtom.p, I.n * sizeof(int), cudaMemcpyDeviceToHost));
    CU(cudaMemcpy(list.data(), I.dList.p, list.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    long long m = 0;
    for (int sl = 0; sl < I.n; sl++) {
        const int i = slotAtom[sl];
        for (int t = 0; t < cnt[sl]; t++) {
            const int j = slotAtom[list[(size_t) sl * I.cap + t] & 0x7FFFFFu];
            if (i < j) {
                if (m < cap) {
                    pi[m] = i;
                    pj[m] = j;
                }
                m++;
            }
        }
    }
    return m;
}

long long Engine::historySize() const {
    return (long long) (Impl::NHIST * 3 * (size_t) impl->numGlobal * 8 + 2 * sizeof(int));
}

void Engine::getHistory(void* blob) const {
    Impl& I = *impl;
    int* hdr = (int*) blob;
    hdr[0] = I.histHead;
    hdr[1] = I.histCount;
    CU(cudaMemcpy((char*) blob + 2 * sizeof(int), I.dHist.p, Impl::NHIST * 3 * (size_t) I.numGlobal * 8,
                  cudaMemcpyDeviceToHost));
}

void Engine::setHistory(const void* blob) {
    Impl& I = *impl;
    const int* hdr = (const int*) blob;
    if (hdr[0] < 0 || hdr[0] >= Impl::NHIST || hdr[1] < 0 || hdr[1] > 4)
        throw std::invalid_argument("pgm_b200: history blob header out of range");
    I.histHead = hdr[0];
    I.histCount = hdr[1];
    CU(cudaMemcpy(I.dHist.p, (const char*) blob + 2 * sizeof(int), Impl::NHIST * 3 * (size_t) I.numGlobal * 8,
                  cudaMemcpyHostToDevice));
}

void Engine::field(const double* pos, const double box[3][3], const double* qf, const double* d, double* E) {
    Impl& I = *impl;
    if (!I.atomsSet || I.nsys != 1)
        throw std::logic_error("pgm_b200: field needs a single-system engine with atoms set");
    I.checkPositions(pos, 3 * (size_t) I.n);
    I.selectDevice();
    for (int attempt = 0; attempt < 4; attempt++) {
        I.setBoxes(&box[0][0]);
        I.prepareControl(true, 0, nullptr, nullptr, 0, 0.0, nullptr);
        std::memcpy(I.hSys, I.sysHost.data(), I.nsys * sizeof(SysDev));
        CU(cudaMemcpyAsync(I.dSys.p, I.hSys, I.nsys * sizeof(SysDev), cudaMemcpyHostToDevice, I.st));
        CU(cudaMemcpyAsync(I.dCtl.p, I.hCtl, sizeof(Ctl), cudaMemcpyHostToDevice, I.st));
        CU(cudaMemcpyAsync(I.dPosIn.p, pos, 3 * (size_t) I.n * 8, cudaMemcpyHostToDevice, I.st));
        CU(cudaMemcpyAsync(I.dQ.p, qf, (size_t) I.n * 8, cudaMemcpyHostToDevice, I.st));
        CU(cudaMemcpyAsync(I.dDtot.p, d, 3 * (size_t) I.n * 8, cudaMemcpyHostToDevice, I.st));
        const Dev dv = I.makeDev(false, 0);
        const int tb = (I.n + 255) / 256;
        CU(cudaMemsetAsync(dv.cellCount, 0, (size_t) I.totalCells * sizeof(int), I.st));
        CU(cudaMemsetAsync(dv.flags, 0, I.flagBytes(), I.st));
        I.listValid = false;   // the list below is this call's
        k_prep<<<tb, 256, 0, I.st>>>(dv, I.dPosIn.as<double>(), 3);
        k_cell_scan<<<1, 1024, 0, I.st>>>(dv);
        k_cell_scatter<<<tb, 256, 0, I.st>>>(dv);
        k_cell_sort<<<(I.totalCells + 7) / 8, 256, 0, I.st>>>(dv);
        if (I.mixed()) {
            I.listKernel(I.st, dv);
            k_pair_compact<float><<<(I.n + 7) / 8, 256, 0, I.st>>>(dv);
            k_splines<float><<<(3 * I.n + 255) / 256, 256, 0, I.st>>>(dv);
            k_influence<float><<<dim3(I.convBlocks, I.nsys), 256, 0, I.st>>>(dv);
            CU(cudaMemsetAsync(dv.grid, 0, I.gridTotal * I.realSize(), I.st));
            I.fieldPass<float, true>(I.st, I.side, dv, 0, dv.dtot, false);
        } else {
            I.listKernel(I.st, dv);
            k_pair_compact<double><<<(I.n + 7) / 8, 256, 0, I.st>>>(dv);
            k_splines<double><<<(3 * I.n + 255) / 256, 256, 0, I.st>>>(dv);
            k_influence<double><<<dim3(I.convBlocks, I.nsys), 256, 0, I.st>>>(dv);
            CU(cudaMemsetAsync(dv.grid, 0, I.gridTotal * I.realSize(), I.st));
            I.fieldPass<double, true>(I.st, I.side, dv, 0, dv.dtot, false);
        }
        CU(cudaGetLastError());
        std::vector<double> ep(3 * (size_t) I.n), er(3 * (size_t) I.n);
        CU(cudaMemcpyAsync(ep.data(), I.dEpair.p, ep.size() * 8, cudaMemcpyDeviceToHost, I.st));
        CU(cudaMemcpyAsync(er.data(), I.dErec.p, er.size() * 8, cudaMemcpyDeviceToHost, I.st));
        CU(cudaMemcpyAsync(I.hFlags, I.dFlags.p, 16 * sizeof(int), cudaMemcpyDeviceToHost, I.st));
        CU(cudaMemcpyAsync(I.dQ.p, I.q.data(), (size_t) I.n * 8, cudaMemcpyHostToDevice, I.st));
        CU(cudaStreamSynchronize(I.st));
        I.barrierCheck();
        if (I.hFlags[0] > I.cap) {
            I.cap = (I.hFlags[0] + I.hFlags[0] / 4 + 31) / 32 * 32;
            I.allocList();
            if (I.exec) {
                cudaGraphExecDestroy(I.exec);
                I.exec = nullptr;
            }
            continue;
        }
        const double beta = I.sysBeta[0];
        const double cs = 4.0 * beta * beta * beta / (3.0 * SQRT_PI);
        for (size_t k = 0; k < 3 * (size_t) I.n; k++)
            E[k] = ep[k] + er[k] + cs * d[k];
        I.haveResult = false;
        return;
    }
    throw std::runtime_error("pgm_b200: pair list did not fit after growing it");
}

void Engine::paramGrad(double* dq, double* dradius, double* dalpha, double* dstrength) {
    Impl& I = *impl;
    if (!I.haveResult)
        throw std::logic_error("pgm_b200: paramGrad needs a completed evaluation");
    if (I.gvdwOn)
        throw std::logic_error("pgm_b200: parameter gradients cover the electrostatics only (GVDW is set)");
    I.selectDevice();
    const Dev dv = I.makeDev(false, 0);
    const int blocks = (int) (((long long) I.n * 8 + 255) / 256);
    k_pair_grad<8><<<blocks, 256, 0, I.st>>>(dv, I.dGradQ.as<double>(), I.dGradR.as<double>());
    CU(cudaGetLastError());
    const size_t n = I.n;
    std::vector<double> gq(n), gR(n), pot(n), mu(3 * n), Et(3 * n), pos(3 * n);
    CU(cudaMemcpyAsync(gq.data(), I.dGradQ.p, n * 8, cudaMemcpyDeviceToHost, I.st));
    CU(cudaMemcpyAsync(gR.data(), I.dGradR.p, n * 8, cudaMemcpyDeviceToHost, I.st));
    CU(cudaMemcpyAsync(pot.data(), I.dPot.p, n * 8, cudaMemcpyDeviceToHost, I.st));
    CU(cudaMemcpyAsync(mu.data(), I.dMu.p, 3 * n * 8, cudaMemcpyDeviceToHost, I.st));
    CU(cudaMemcpyAsync(Et.data(), I.dEtot.p, 3 * n * 8, cudaMemcpyDeviceToHost, I.st));
    CU(cudaMemcpyAsync(pos.data(), I.dPosIn.p, 3 * n * 8, cudaMemcpyDeviceToHost, I.st));
    CU(cudaStreamSynchronize(I.st));
    const double ke = I.s.ke;
    std::vector<double> Qs(I.nsys, 0.0);
    for (size_t i = 0; i < n; i++)
        Qs[I.atomSys[i]] += I.q[i];
    for (size_t i = 0; i < n; i++) {
        const SysDev& S = I.sysHost[I.atomSys[i]];
        if (dq)
            dq[i] = ke * (gq[i] + pot[i] - 2.0 * S.beta / SQRT_PI * I.q[i] -
                          PI_D * Qs[I.atomSys[i]] / (S.volume * S.beta * S.beta));
        if (dradius)
            dradius[i] = ke * gR[i];
        if (dalpha) {
            const double a = I.alpha[i];
            const double m2 = mu[3 * i] * mu[3 * i] + mu[3 * i + 1] * mu[3 * i + 1] + mu[3 * i + 2] * mu[3 * i + 2];
            dalpha[i] = a > 0 ? -ke * m2 / (2.0 * a * a) : 0.0;
        }
    }
    if (dstrength)
        for (size_t m = 0; m < I.covAtom.size(); m++) {
            const int i = I.covAtom[m], j = I.covPartner[m];
            const SysDev& S = I.sysHost[I.atomSys[i]];
            double v[3] = {pos[3 * j] - pos[3 * i], pos[3 * j + 1] - pos[3 * i + 1], pos[3 * j + 2] - pos[3 * i + 2]};
            for (int c = 2; c >= 0; c--) {
                const double k = std::round(v[c] / S.H[4 * c]);
                for (int a = 0; a < 3; a++)
                    v[a] -= k * S.H[3 * c + a];
            }
            const double L = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
            dstrength[m] = -ke * (Et[3 * i] * v[0] + Et[3 * i + 1] * v[1] + Et[3 * i + 2] * v[2]) / L;
        }
}

Terms Engine::evaluateFixed(const double* pos, const double box[3][3], const double* mu, bool keepList,
                            double* forces, double* field) {
    Impl& I = *impl;
    if (!I.atomsSet || I.nsys != 1)
        throw std::logic_error("pgm_b200: evaluateFixed needs a single-system engine with atoms set");
    if (keepList && !I.haveResult)
        throw std::logic_error("pgm_b200: evaluateFixed with keepList needs a previous evaluation");
    I.checkPositions(pos, 3 * (size_t) I.n);
    I.selectDevice();
    for (int attempt = 0; attempt < 4; attempt++) {
        if (!keepList)
            I.setBoxes(&box[0][0]);
        else
            for (int a = 0; a < 9; a++)
                if (I.sysHost[0].H[a] != (&box[0][0])[a])
                    throw std::invalid_argument("pgm_b200: evaluateFixed with keepList needs the list's box");
        I.prepareControl(true, 0, nullptr, nullptr, 0, 0.0, nullptr);
        I.hCtl->histSlot = -1;
        I.hCtl->fixedMu = 1;
        I.pendingSlot = -1;
        std::memcpy(I.hSys, I.sysHost.data(), I.nsys * sizeof(SysDev));
        CU(cudaMemcpyAsync(I.dSys.p, I.hSys, I.nsys * sizeof(SysDev), cudaMemcpyHostToDevice, I.st));
        CU(cudaMemcpyAsync(I.dCtl.p, I.hCtl, sizeof(Ctl), cudaMemcpyHostToDevice, I.st));
        CU(cudaMemcpyAsync(I.dPosIn.p, pos, 3 * (size_t) I.n * 8, cudaMemcpyHostToDevice, I.st));
        CU(cudaMemcpyAsync(I.dMu.p, mu, 3 * (size_t) I.n * 8, cudaMemcpyHostToDevice, I.st));
        const Dev d = I.makeDev(false, 0);
        const int tb = (I.n + 255) / 256;
        CU(cudaMemsetAsync(d.flags, 0, I.flagBytes(), I.st));
        auto body = [&](auto tag) {
            typedef decltype(tag) R;
            if (keepList) {
                k_refresh_positions<<<tb, 256, 0, I.st>>>(d);
                k_pair_kernels<R><<<(I.n + 7) / 8, 256, 0, I.st>>>(d);   // records at the new positions
            } else {
                I.listValid = false;   // the list below is this call's
                CU(cudaMemsetAsync(d.cellCount, 0, (size_t) I.totalCells * sizeof(int), I.st));
                k_prep<<<tb, 256, 0, I.st>>>(d, I.dPosIn.as<double>(), 3);
                k_cell_scan<<<1, 1024, 0, I.st>>>(d);
                k_cell_scatter<<<tb, 256, 0, I.st>>>(d);
                k_cell_sort<<<(I.totalCells + 7) / 8, 256, 0, I.st>>>(d);
                I.listKernel(I.st, d);
                k_pair_compact<R><<<(I.n + 7) / 8, 256, 0, I.st>>>(d);
            }
            k_splines<R><<<(3 * I.n + 255) / 256, 256, 0, I.st>>>(d);
            if (std::is_same<R, float>::value && I.planesMode())
                I.enqueuePlaneBins(I.st, d);
            k_perm<<<tb, 256, 0, I.st>>>(d);
            k_influence<R><<<dim3(I.convBlocks, I.nsys), 256, 0, I.st>>>(d);
            CU(cudaGetLastError());
            I.enqueuePost<R>(I.st, I.side, d);
        };
        if (I.mixed())
            body(float());
        else
            body(double());
        CU(cudaMemcpyAsync(I.hResults, I.dResults.p, I.nsys * NRES * 8, cudaMemcpyDeviceToHost, I.st));
        CU(cudaMemcpyAsync(I.hFlags, I.dFlags.p, 16 * sizeof(int), cudaMemcpyDeviceToHost, I.st));
        if (forces)
            CU(cudaMemcpyAsync(forces, I.dForces.p, 3 * (size_t) I.n * 8, cudaMemcpyDeviceToHost, I.st));
        if (field)
            CU(cudaMemcpyAsync(field, I.dEtot.p, 3 * (size_t) I.n * 8, cudaMemcpyDeviceToHost, I.st));
        CU(cudaStreamSynchronize(I.st));
        I.barrierCheck();
        if (I.hFlags[0] > I.cap) {
            if (keepList)
                throw std::logic_error("pgm_b200: list overflow with keepList");
            I.cap = (I.hFlags[0] + I.hFlags[0] / 4 + 31) / 32 * 32;
            I.allocList();
            if (I.exec) {
                cudaGraphExecDestroy(I.exec);
                I.exec = nullptr;
            }
            continue;
        }
        I.lastResults.assign(I.hResults, I.hResults + I.nsys * NRES);
        I.haveResult = true;
        I.hCtl->fixedMu = 0;
        return I.termsOf(0);
    }
    throw std::runtime_error("pgm_b200: pair list did not fit after growing it");
}

// (alpha^-1 - T) x = b for the right-hand side already in b, on the geometry of the last evaluation, every
// system of the engine at once (rows of non-polarizable atoms: 0); the solution in x.  Returns the largest
// iteration count.
int Engine::Impl::solveDevice(double tol) {
    prepareControl(true, 0, nullptr, nullptr, 0, 0.0, nullptr);
    hCtl->histSlot = -1;
    hCtl->customRhs = 1;
    hCtl->guess = 1;
    pendingSlot = -1;
    CU(cudaMemcpyAsync(dCtl.p, hCtl, sizeof(Ctl), cudaMemcpyHostToDevice, st));
    Dev d = makeDev(false, 0);
    d.tol = tol;
    auto run = [&](auto tag) {
        typedef decltype(tag) R;
        CU(cudaMemsetAsync(d.flags, 0, flagBytes(), st));
        k_cg_b<<<(int) chunkSys.size(), CHUNK, 0, st>>>(d);
        CU(cudaMemsetAsync(d.grid, 0, gridTotal * realSize(), st));
        fieldPass<R, false>(st, side, d, 1, d.x, false);
        k_cg_init<<<(int) chunkSys.size(), CHUNK, 0, st>>>(d);
        CU(cudaMemsetAsync(d.grid, 0, gridTotal * realSize(), st));
        for (int it = 0; it <= s.maxIter + 1; it++) {
            CU(cudaMemcpyAsync(hFlags, d.flags, 16 * sizeof(int), cudaMemcpyDeviceToHost, st));
            CU(cudaStreamSynchronize(st));
            barrierCheck();
            if (hFlags[2] >= nsys)
                break;
            enqueueIteration<R>(st, side, d);
        }
    };
    if (mixed())
        run(float());
    else
        run(double());
    std::vector<double> sc((size_t) nsys * NSCAL);
    CU(cudaMemcpyAsync(sc.data(), dScal.p, sc.size() * 8, cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    hCtl->customRhs = 0;
    int most = 0;
    for (int k = 0; k < nsys; k++)
        most = std::max(most, (int) sc[(size_t) k * NSCAL + SC_IT]);
    return most;
}

// One tangent pass: the direct-space derivatives (k_pair_tangent) beside the PME tangent (spread of the tangent
// sources, transforms with the influence product, potential and field gathered), into the pass buffers.
template <typename R>
void Engine::Impl::tangentPass(const Dev& d, const FmBufs& B, const double* dr, const double* dd, const double* dip,
                               const double* quadD, int withQ) {
    const int blocks = (int) (((long long) n * 8 + 255) / 256), wb = (n + 7) / 8;
    k_pair_tangent<8><<<blocks, 256, 0, st>>>(d, dr, dd, B.pphi, B.pE, B.pR);
    CU(cudaMemsetAsync(d.grid, 0, gridTotal * realSize(), st));
    k_spread_tangent<R><<<wb, 256, 0, st>>>(d, dip, quadD, B.w, withQ);
    CU(cudaGetLastError());
    fftChain<R>(st, d, false, false);
    k_gather_tangent<R><<<wb, 256, 0, st>>>(d, B.tphi, B.tE);
    CU(cudaGetLastError());
}

// The force-matching gradient of the last evaluation (see adjoint.cuh): w = 2 (F - F_target) from the
// evaluation's forces, the pass along w, the adjoint solve (alpha^-1 - T) u = -D_w E_tot, the pass along u;
// per-atom dq, dR, dalpha and per-dipole dc = -(w-pass) + (u-pass).  Works on batched engines (every system at
// once).  Returns the loss L = sum |F - F_target|^2 and the adjoint's iterations.
double Engine::forceMatchingGrad(const double* fTarget, double tol, double* dq, double* dradius, double* dalpha,
                                 double* dstrength, int* iterations) {
    Impl& I = *impl;
    if (!I.haveResult)
        throw std::logic_error("pgm_b200: forceMatchingGrad needs a completed evaluation");
    if (I.gvdwOn)
        throw std::logic_error("pgm_b200: parameter gradients cover the electrostatics only (GVDW is set)");
    if (I.s.peek != 0.0)
        throw std::logic_error("pgm_b200: the force-matching adjoint needs peek = 0 (a stationary energy in mu)");
    if (!fTarget || !(tol > 0))
        throw std::invalid_argument("pgm_b200: forceMatchingGrad needs the target forces and tol > 0");
    I.selectDevice();
    const size_t n = I.n, ncov = I.covAtom.size();
    // buffers: w, dp, pphi, pE, pR, tphi, tE, gq, gR, ga, gc, Ed
    const size_t words = 3 * n + 3 * n + n + 3 * n + n + n + 3 * n + n + n + n + std::max<size_t>(ncov, 1) + 3 * n;
    I.dFm.ensure(words * 8);
    double* base = I.dFm.as<double>();
    FmBufs B;
    size_t off = 0;
    auto take = [&](size_t m) {
        double* p = base + off;
        off += m;
        return p;
    };
    B.w = take(3 * n);
    B.dp = take(3 * n);
    B.pphi = take(n);
    B.pE = take(3 * n);
    B.pR = take(n);
    B.tphi = take(n);
    B.tE = take(3 * n);
    B.gq = take(n);
    B.gR = take(n);
    B.ga = take(n);
    B.gc = take(std::max<size_t>(ncov, 1));
    B.Ed = take(3 * n);
    // w = 2 (F - F_target) and the loss, on the host (the forces of the last evaluation)
    std::vector<double> F(3 * n), w(3 * n);
    CU(cudaMemcpyAsync(F.data(), I.dForces.p, 3 * n * 8, cudaMemcpyDeviceToHost, I.st));
    CU(cudaStreamSynchronize(I.st));
    double loss = 0.0;
    for (size_t k = 0; k < 3 * n; k++) {
        const double r = F[k] - fTarget[k];
        loss += r * r;
        w[k] = 2.0 * r;
    }
    CU(cudaMemcpyAsync(B.w, w.data(), 3 * n * 8, cudaMemcpyHostToDevice, I.st));
    const Dev d = I.makeDev(false, 0);
    const int tb = (int) ((n + 255) / 256);
    std::vector<double> gqW(n), gRW(n), gcW(ncov), gqU(n), gRU(n), gaU(n), gcU(ncov);
    auto fetch = [&](std::vector<double>& q_, std::vector<double>& R_, std::vector<double>* a_,
                     std::vector<double>& c_) {
        CU(cudaMemcpyAsync(q_.data(), B.gq, n * 8, cudaMemcpyDeviceToHost, I.st));
        CU(cudaMemcpyAsync(R_.data(), B.gR, n * 8, cudaMemcpyDeviceToHost, I.st));
        if (a_)
            CU(cudaMemcpyAsync(a_->data(), B.ga, n * 8, cudaMemcpyDeviceToHost, I.st));
        if (ncov)
            CU(cudaMemcpyAsync(c_.data(), B.gc, ncov * 8, cudaMemcpyDeviceToHost, I.st));
        CU(cudaStreamSynchronize(I.st));
    };
    // the pass along w (the final pass's fields and Hessian sums are still in place)
    k_fm_dp<<<tb, 256, 0, I.st>>>(d, B.w, B.dp);
    if (I.mixed())
        I.tangentPass<float>(d, B, B.w, B.dp, B.dp, d.dtot, 1);
    else
        I.tangentPass<double>(d, B, B.w, B.dp, B.dp, d.dtot, 1);
    k_fm_assemble_w<<<tb, 256, 0, I.st>>>(d, B);
    if (ncov)
        k_fm_cov<<<(int) ((ncov + 255) / 256), 256, 0, I.st>>>(d, B, 1);
    k_fm_rhs<<<(int) ((3 * n + 255) / 256), 256, 0, I.st>>>(d, B.Ed);
    CU(cudaGetLastError());
    fetch(gqW, gRW, nullptr, gcW);
    // the adjoint solve: u in x
    const int its = I.solveDevice(tol);
    if (iterations)
        *iterations = its;
    // the pass along u
    const double* u = I.dX.as<double>();
    if (I.mixed())
        I.tangentPass<float>(d, B, nullptr, u, u, nullptr, 0);
    else
        I.tangentPass<double>(d, B, nullptr, u, u, nullptr, 0);
    k_fm_assemble_u<<<tb, 256, 0, I.st>>>(d, B, u);
    if (ncov)
        k_fm_cov<<<(int) ((ncov + 255) / 256), 256, 0, I.st>>>(d, B, 0);
    CU(cudaGetLastError());
    fetch(gqU, gRU, &gaU, gcU);
    for (size_t i = 0; i < n; i++) {
        if (dq)
            dq[i] = -gqW[i] + gqU[i];
        if (dradius)
            dradius[i] = -gRW[i] + gRU[i];
        if (dalpha)
            dalpha[i] = gaU[i];
    }
    if (dstrength)
        for (size_t m = 0; m < ncov; m++)
            dstrength[m] = -gcW[m] + gcU[m];
    return loss;
}

int Engine::solve(const double* rhs, double* x, double tol) {
    Impl& I = *impl;
    if (!I.haveResult || I.nsys != 1)
        throw std::logic_error("pgm_b200: solve needs a previous single-system evaluation (its geometry)");
    I.selectDevice();
    I.prepareControl(true, 0, nullptr, nullptr, 0, 0.0, nullptr);
    I.hCtl->histSlot = -1;
    I.hCtl->customRhs = 1;
    I.hCtl->guess = 1;
    I.pendingSlot = -1;
    CU(cudaMemcpyAsync(I.dCtl.p, I.hCtl, sizeof(Ctl), cudaMemcpyHostToDevice, I.st));
    CU(cudaMemcpyAsync(I.dB.p, rhs, 3 * (size_t) I.n * 8, cudaMemcpyHostToDevice, I.st));
    Dev d = I.makeDev(false, 0);
    d.tol = tol;
    auto run = [&](auto tag) {
        typedef decltype(tag) R;
        CU(cudaMemsetAsync(d.flags, 0, I.flagBytes(), I.st));
        k_cg_b<<<(int) I.chunkSys.size(), CHUNK, 0, I.st>>>(d);
        CU(cudaMemsetAsync(d.grid, 0, I.gridTotal * I.realSize(), I.st));
        I.fieldPass<R, false>(I.st, I.side, d, 1, d.x, false);
        k_cg_init<<<(int) I.chunkSys.size(), CHUNK, 0, I.st>>>(d);
        CU(cudaMemsetAsync(d.grid, 0, I.gridTotal * I.realSize(), I.st));
        for (int it = 0; it <= I.s.maxIter + 1; it++) {
            CU(cudaMemcpyAsync(I.hFlags, d.flags, 16 * sizeof(int), cudaMemcpyDeviceToHost, I.st));
            CU(cudaStreamSynchronize(I.st));
            I.barrierCheck();
            if (I.hFlags[2] >= I.nsys)
                break;
            I.enqueueIteration<R>(I.st, I.side, d);
        }
    };
    if (I.mixed())
        run(float());
    else
        run(double());
    double sc[NSCAL];
    CU(cudaMemcpyAsync(x, I.dX.p, 3 * (size_t) I.n * 8, cudaMemcpyDeviceToHost, I.st));
    CU(cudaMemcpyAsync(sc, I.dScal.p, sizeof(sc), cudaMemcpyDeviceToHost, I.st));
    CU(cudaStreamSynchronize(I.st));
    I.hCtl->customRhs = 0;
    return (int) sc[SC_IT];
}

// Systems still iterating before each CG iteration of the last batched evaluation (k = 0 .. its iterations),
// at most cap values; returns how many were written.
int Engine::activeSystems(int* counts, int cap) const {
    const Impl& I = *impl;
    if (!I.haveResult || I.nsys < 2 || !I.s.polarizable)
        return 0;
    int it = 0;
    for (int k = 0; k < I.nsys; k++)
        it = std::max(it, (int) I.lastResults[(size_t) k * NRES + 14]);
    const int m = std::min(cap, std::min(it + 1, I.s.maxIter + 2));
    if (m > 0)
        CU(cudaMemcpy(counts, I.dActive.p, m * sizeof(int), cudaMemcpyDeviceToHost));
    return m;
}

int Engine::kernelLaunches() const {
    const Impl& I = *impl;
    if (!I.haveResult)
        return 0;
    // own kernels per evaluation (the cuFFT transforms not counted): preparation 7, the Verlet list's build 5
    // when it ran; a field pass fp = 4 (spread, the cluster transform kernel or the influence product, pair
    // pass, gather); polarizable: two field passes + 2 before the loop, fp + 2 per CG iteration (fp + 1 for one
    // system); final 7
    int it = 0;
    for (int k = 0; k < I.nsys; k++)
        it = std::max(it, (int) I.lastResults[(size_t) k * NRES + 14]);
    const int fp = 4;
    const int perIt = fp + (I.nsys == 1 && I.fuseCgA ? 1 : 2);   // single system: A p in the gather
    if (I.persistentMode() && I.s.polarizable)   // the bins and one persistent launch for the whole loop
        return 7 + (I.lastBuilt ? 5 : 0) + 2 * fp + 2 + 2 + 7 + (I.gvdwOn ? 1 : 0);
    return 7 + (I.lastBuilt ? 5 : 0) + (I.s.polarizable ? 2 * fp + 2 + perIt * it : 0) + 7 + (I.gvdwOn ? 1 : 0);
}

void Engine::kernelTimes(int reps, double* ms, void* flush, size_t flushBytes) {
    Impl& I = *impl;
    if (!I.haveResult)
        throw std::logic_error("pgm_b200: kernelTimes needs a completed evaluation");
    I.selectDevice();
    const Dev d = I.makeDev(false, 0);
    cudaEvent_t a, b;
    CU(cudaEventCreate(&a));
    CU(cudaEventCreate(&b));
    // warm: reps launches back to back between two events (as inside an evaluation, the inputs stay in L2 where
    // they fit); cold: before every launch the caller's buffer (larger than L2) is overwritten, and only the
    // launch itself lies between the events
    auto timeIt = [&](auto&& fn) {
        fn();
        if (!flush) {
            CU(cudaEventRecord(a, I.st));
            for (int r = 0; r < reps; r++)
                fn();
            CU(cudaEventRecord(b, I.st));
            CU(cudaEventSynchronize(b));
            float t = 0;
            CU(cudaEventElapsedTime(&t, a, b));
            return (double) t / reps;
        }
        double total = 0.0;
        for (int r = 0; r < reps; r++) {
            CU(cudaMemsetAsync(flush, r & 0xff, flushBytes, I.st));
            CU(cudaEventRecord(a, I.st));
            fn();
            CU(cudaEventRecord(b, I.st));
            CU(cudaEventSynchronize(b));
            float t = 0;
            CU(cudaEventElapsedTime(&t, a, b));
            total += t;
        }
        return total / reps;
    };
    auto run = [&](auto tag) {
        typedef decltype(tag) R;
        ms[0] = timeIt([&] {
            I.listKernel(I.st, d);
            I.pairRecords<R>(I.st, d);
        });
        ms[1] = timeIt([&] { I.pairField<R, false>(I.st, d, 0); });
        ms[2] = timeIt([&] { I.launchSpread<R>(I.st, d, 1, d.x); });
        ms[3] = timeIt([&] { I.launchGather<R, false>(I.st, d, 0); });
        ms[4] = timeIt([&] {
            const int blocks = (int) (((long long) I.n * I.pairGS + 255) / 256);
            switch (I.pairGS) {
            case 4: k_pair_final<R, 4><<<blocks, 256, 0, I.st>>>(d); break;
            case 16: k_pair_final<R, 16><<<blocks, 256, 0, I.st>>>(d); break;
            case 32: k_pair_final<R, 32><<<blocks, 256, 0, I.st>>>(d); break;
            default: k_pair_final<R, 8><<<blocks, 256, 0, I.st>>>(d);
            }
        });
        ms[5] = timeIt([&] {
            I.transformPair<R>(I.st, d, false);
        });
        ms[6] = timeIt([&] { k_cg_a<<<(int) I.chunkSys.size(), CHUNK, 0, I.st>>>(d); });
    };
    if (I.mixed())
        run(float());
    else
        run(double());
    if (d.gridFix)   // (the timed spreads added to the fixed-point grid with no conversion after them)
        CU(cudaMemsetAsync(d.gridFix, 0, I.gridTotal * 8, I.st));
    CU(cudaGetLastError());
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    I.haveResult = true;
}

// Median device time [ms] of reps whole evaluations at the last evaluation's positions and boxes (already on
// the device), new step each (the benchmark's step: list, permanent field, the solve from the engine's initial
// guess, final pass), CUDA events around each launch on the engine's stream.  The predictor history is saved
// and restored, so the caller's trajectory state is unchanged.
double Engine::timeEvaluations(int reps) {
    Impl& I = *impl;
    if (!I.haveResult || I.launched)
        throw std::logic_error("pgm_b200: timeEvaluations needs a completed evaluation and no call in flight");
    if (reps <= 0)
        throw std::invalid_argument("pgm_b200: timeEvaluations needs reps > 0");
    I.selectDevice();
    const bool keepHistory = I.numGlobal > 0 && I.dHist.p;
    std::vector<unsigned char> hist(keepHistory ? (size_t) historySize() : 0);
    if (keepHistory)
        getHistory(hist.data());
    const std::vector<double> boxes = I.launchBoxes;
    const std::vector<double> results = I.lastResults;
    cudaEvent_t a, b;
    CU(cudaEventCreate(&a));
    CU(cudaEventCreate(&b));
    std::vector<double> t;
    for (int r = 0; r < reps; r++) {
        for (int attempt = 0; attempt < 4; attempt++) {
            I.prepareControl(true, 0, nullptr, nullptr, 0, 0.0, nullptr);
            CU(cudaEventRecord(a, I.st));
            I.launch(boxes.data());
            CU(cudaEventRecord(b, I.st));
            if (I.finish())
                break;
        }
        CU(cudaEventSynchronize(b));
        float ms = 0;
        CU(cudaEventElapsedTime(&ms, a, b));
        t.push_back(ms);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (keepHistory)
        setHistory(hist.data());
    I.lastResults = results;
    std::sort(t.begin(), t.end());
    return t[t.size() / 2];
}

// The PME spread / gather kernels of the field passes: 0 a warp per atom (every engine), 1 plane-owner tiles in
// shared memory (mixed precision, one system, order 6), 2 float4 lines (mixed precision, orders 4, 5, 6, 8),
// 3 cell-group tiles in shared memory (mixed precision, one system, orders 4, 5, 6, 8); where the choice does not
// apply, 0 runs.
void Engine::setPmeKernels(int kind) {
    if (kind < 0 || kind > 3)
        throw std::invalid_argument(
            "pgm_b200: PME kernels must be 0 (a warp per atom), 1 (plane tiles), 2 (lines) or 3 (cell tiles)");
    Impl& I = *impl;
    if (kind != I.pmeWant && I.exec) {
        cudaGraphExecDestroy(I.exec);
        I.exec = nullptr;
    }
    I.pmeWant = kind;
}

int Engine::pmeKernels() const {
    return impl->planesMode() ? 1 : impl->linesMode() ? 2 : impl->tilesMode() ? 3 : 0;
}

void Engine::setPairLanes(int lanes) {
    if (lanes != 4 && lanes != 8 && lanes != 16 && lanes != 32)
        throw std::invalid_argument("pgm_b200: pair lanes must be 4, 8, 16 or 32");
    if (lanes != impl->pairGS && impl->exec) {
        cudaGraphExecDestroy(impl->exec);
        impl->exec = nullptr;
    }
    impl->pairGS = lanes;
}

int Engine::pairLanes() const { return impl->pairGS; }

void Engine::setTransforms(int mode) {
    if (mode < 0 || mode > 4)
        throw std::invalid_argument("pgm_b200: transforms must be 0 (cuFFT), 1 (cluster kernel), 2 (2D cuFFT + "
                                    "x-line kernel), 3 (grid kernel) or 4 (grid kernel and the persistent CG "
                                    "kernel)");
    impl->tfWant = mode;
    impl->selectTransforms();
}

int Engine::transforms() const { return impl->tfMode; }

void Engine::setSystems(int nsys, const int* atomCount, const double* cutoff, const double* beta, const int* grid,
                        const double* q, const double* radius, const double* alpha, const int* covCount,
                        const int* covAtom, const int* covPartner, const double* strength) {
    impl->selectDevice();
    impl->setSystemsBatch(nsys, atomCount, cutoff, beta, grid, q, radius, alpha, covCount, covAtom, covPartner,
                          strength);
}

void Engine::computeBatch(const double* pos, const double* boxes, double* energies, double* forces, double* strain,
                          int* iterations) {
    Impl& I = *impl;
    I.evalHost(pos, boxes, true, forces != nullptr);
    for (int k = 0; k < I.nsys; k++) {
        const double* r = I.lastResults.data() + (size_t) k * NRES;
        if (energies)
            for (int c = 0; c < 5; c++)
                energies[6 * k + c] = r[c];
        if (energies)
            energies[6 * k + 5] = r[16];
        if (strain)
            for (int c = 0; c < 9; c++)
                strain[9 * k + c] = r[5 + c];
        if (iterations)
            iterations[k] = (int) r[14];
    }
    if (forces)
        std::memcpy(forces, I.hForces, 3 * (size_t) I.n * 8);
}

}  // namespace pgmb200

// ---------------------------------------------------------------------------------------------- no allocation
//
// A pair-list entry point for callers that cannot allocate device memory: MD engines whose memory pool owns
// every byte of the GPU and hands out fixed buffers, hosts that reserve their device memory up front and must
// not grow it, and loops that cannot afford cudaMalloc's implicit synchronisation of the whole device.  It runs
// the engine's own cell-list and pair-list kernels, with their scratch (cell counts and offsets, the
// cell-sorted copies of the atoms) in one statically sized device array instead of engine-owned allocations.
// Every GPU that loads the library holds that array (about 4 MB) until the process exits.
namespace pgmb200 {
namespace {

constexpr int NOALLOC_MAX_ATOMS = 16384;
constexpr int NOALLOC_MAX_CELLS = 8 * NOALLOC_MAX_ATOMS + 64;
constexpr size_t NOALLOC_ATOM_BYTES = 200;   // per-atom scratch, rounded up
constexpr size_t NOALLOC_BYTES = NOALLOC_ATOM_BYTES * NOALLOC_MAX_ATOMS + 8 * (size_t) (NOALLOC_MAX_CELLS + 1) +
                                 sizeof(SysDev) + sizeof(Ctl) + 64 * 16;

// The scratch.  In host code this name is only a stand-in for the device array: its device address comes
// from cudaGetSymbolAddress, once per device (noallocScratch below).
static __device__ __align__(256) unsigned char g_noallocScratch[NOALLOC_BYTES];

// Converts the cell-sorted list entries (slot of j, image shift) into atom indices, in place.
__global__ void k_entries_to_atoms(const int* slotAtom, const int* counts, int* neighbors, int cap, int n) {
    const int slot = blockIdx.x, t0 = threadIdx.x;
    if (slot >= n)
        return;
    const int cnt = counts[slot];
    for (int t = t0; t < cnt; t += blockDim.x) {
        const uint32_t e = (uint32_t) neighbors[(size_t) slot * cap + t];
        neighbors[(size_t) slot * cap + t] = slotAtom[e & 0x7FFFFFu];
    }
}

// The longest row before any clamping: the largest count (rows beyond cap already raised flags[0] to their
// length in the build, so the maximum over both is the longest row either way), into flags[12].
__global__ void k_longest_row(const int* counts, int n, int* flags) {
    int m = 0;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x)
        m = max(m, counts[s]);
    for (int o = 16; o > 0; o >>= 1)
        m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0)
        atomicMax(&flags[12], max(m, flags[0]));
}

// Device address of the scratch on the current device: looked up on the first call on that device, under a
// lock, so that first calls from several host threads do not race on the table.
unsigned char* noallocScratch() {
    static std::mutex lock;
    static unsigned char* addr[64] = {nullptr};
    int dev = 0;
    CU(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64)
        throw std::runtime_error("pgm_b200: device index beyond 63");
    std::lock_guard<std::mutex> guard(lock);
    if (!addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noallocScratch);
        if (e != cudaSuccess || !p)
            throw std::runtime_error(std::string("pgm_b200: cudaGetSymbolAddress of the scratch array failed: ") +
                                     cudaGetErrorString(e));
        addr[dev] = (unsigned char*) p;
    }
    return addr[dev];
}

}  // namespace

int pairListNoAlloc(int n, const double* posDev, const double* box, double cutoff, int cap, int* slotAtomOut,
                    int* countsOut, int* neighborsOut, cudaStream_t st, int* maxCount) {
    if (n <= 0 || n > NOALLOC_MAX_ATOMS)
        throw std::length_error("pgm_b200: pair_list_noalloc handles 1.." + std::to_string(NOALLOC_MAX_ATOMS) +
                                " atoms, got " + std::to_string(n));
    if (cap <= 0 || !posDev || !box || !slotAtomOut || !countsOut || !neighborsOut)
        throw std::invalid_argument("pgm_b200: pair_list_noalloc arguments");
    // the system's constants, as the engine computes them for one system
    SysDev S;
    std::memset(&S, 0, sizeof(S));
    for (int a = 0; a < 9; a++)
        S.H[a] = box[a];
    if (box[1] != 0 || box[2] != 0 || box[5] != 0 || !(box[0] > 0 && box[4] > 0 && box[8] > 0))
        throw std::invalid_argument("pgm_b200: box not in the reduced triclinic form");
    if (!(cutoff > 0))
        throw std::invalid_argument("pgm_b200: cutoff must be positive");
    boxInverse(box, S.recip, S.volume);
    S.cutoff = cutoff;
    S.rc2 = cutoff * cutoff;
    S.rl2 = S.rc2;   // the list at the cutoff itself (no skin)
    S.beta = 1.0;
    S.K[0] = S.K[1] = S.K[2] = 1;
    S.atomBegin = 0;
    S.atomEnd = n;
    double rho[3];
    for (int a = 0; a < 3; a++) {
        rho[a] = cutoff * std::sqrt(S.recip[a] * S.recip[a] + S.recip[3 + a] * S.recip[3 + a] +
                                    S.recip[6 + a] * S.recip[6 + a]);
        if (rho[a] > 0.5 * (1.0 + 1e-12))
            throw std::invalid_argument("pgm_b200: cut-off beyond half the box");
        S.cellN[a] = std::max(1, std::min((int) std::floor(2.0 / rho[a]), 1024));
    }
    while ((long long) S.cellN[0] * S.cellN[1] * S.cellN[2] > 8LL * n + 64) {
        int a = 0;
        for (int b = 1; b < 3; b++)
            if (S.cellN[b] > S.cellN[a])
                a = b;
        S.cellN[a] = std::max(1, S.cellN[a] / 2);
    }
    for (int a = 0; a < 3; a++)
        S.cellM[a] = std::max(1, (int) std::ceil(rho[a] * S.cellN[a] * (1.0 + 1e-12)));
    S.cellCount = S.cellN[0] * S.cellN[1] * S.cellN[2];
    if (S.cellCount > NOALLOC_MAX_CELLS)
        throw std::length_error("pgm_b200: pair_list_noalloc: more cells than its scratch holds");
    // carve the scratch
    unsigned char* base = noallocScratch();
    size_t off = 0;
    auto take = [&](size_t bytes) {
        unsigned char* p = base + off;
        off += (bytes + 255) / 256 * 256;
        return p;
    };
    Dev d;
    std::memset(&d, 0, sizeof(d));
    SysDev* sysD = (SysDev*) take(sizeof(SysDev));
    Ctl* ctlD = (Ctl*) take(sizeof(Ctl));
    int* flags = (int*) take(16 * sizeof(int));
    d.nAtoms = n;
    d.nSys = 1;
    d.cap = cap;
    d.order = 6;
    d.totalCells = S.cellCount;
    d.sys = sysD;
    d.ctl = ctlD;
    d.flags = flags;
    d.posIn = posDev;
    d.atomSys = (const int*) take(n * sizeof(int));
    d.q = (const double*) take(n * 8);
    d.radius = (const double*) take(n * 8);
    d.wrapN = (int*) take(3 * n * sizeof(int));
    d.cellOf = (int*) take(n * sizeof(int));
    d.cellRank = (int*) take(n * sizeof(int));
    d.pmeBase = (int*) take(3 * n * sizeof(int));
    d.pmeFr = (double*) take(3 * n * 8);
    d.Etot = (double*) take(3 * n * 8);
    d.slotTmp = (int*) take(n * sizeof(int));
    d.posS = (double4*) take(n * sizeof(double4));
    d.origS = (double4*) take(n * sizeof(double4));
    d.wrapS = (int4*) take(n * sizeof(int4));
    d.radS = (double*) take(n * 8);
    d.cellCount = (int*) take(S.cellCount * sizeof(int));
    d.cellStart = (int*) take((S.cellCount + 1) * sizeof(int));
    if (off > NOALLOC_BYTES)
        throw std::length_error("pgm_b200: pair_list_noalloc scratch layout exceeds its array");
    d.slotAtom = slotAtomOut;
    d.slistCount = countsOut;
    d.slist = (uint32_t*) neighborsOut;
    Ctl c;
    std::memset(&c, 0, sizeof(c));
    c.posMode = 0;
    c.histSlot = -1;
    // every call shares the scratch and finds the previous call's contents: clear what must start at zero
    CU(cudaMemcpyAsync(sysD, &S, sizeof(S), cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(ctlD, &c, sizeof(c), cudaMemcpyHostToDevice, st));
    CU(cudaMemsetAsync(flags, 0, 16 * sizeof(int), st));
    CU(cudaMemsetAsync((void*) d.atomSys, 0, n * sizeof(int), st));
    CU(cudaMemsetAsync((void*) d.q, 0, n * 8, st));
    CU(cudaMemsetAsync((void*) d.radius, 0, n * 8, st));
    CU(cudaMemsetAsync(d.cellCount, 0, S.cellCount * sizeof(int), st));
    const int tb = (n + 255) / 256;
    k_prep<<<tb, 256, 0, st>>>(d, nullptr, 3);
    k_cell_scan<<<1, 1024, 0, st>>>(d);
    k_cell_scatter<<<tb, 256, 0, st>>>(d);
    k_cell_sort<<<(S.cellCount + 7) / 8, 256, 0, st>>>(d);
    k_build_list<<<S.cellCount, LIST_THREADS, 0, st>>>(d);
    k_entries_to_atoms<<<n, 128, 0, st>>>(slotAtomOut, countsOut, neighborsOut, cap, n);
    k_longest_row<<<std::min((n + 255) / 256, 64), 256, 0, st>>>(countsOut, n, flags);
    CU(cudaGetLastError());
    int hflags[16];
    CU(cudaMemcpyAsync(hflags, flags, sizeof(hflags), cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    if (maxCount)
        *maxCount = hflags[12];
    return hflags[0] > cap ? 1 : 0;
}

}  // namespace pgmb200
