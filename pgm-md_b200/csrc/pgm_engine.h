// pgm_b200 C++ surface: the same methods as the reference GPU engine pgmcuda::Engine
// (core/cuda/pgm_cuda.h:47-127 of larryhuang98/pGM-MD) plus batched systems and parameter gradients.
// The C ABI (include/pgm_b200.h) wraps this class.
#pragma once

#include <array>
#include <string>
#include <vector>

namespace pgmb200 {

// pgmcuda::Settings (core/cuda/pgm_cuda.h:25-39) + precision / initial guess / polarizable.
struct Settings {
    double cutoff = 0.9;
    double beta = 3.5;
    int grid[3] = {36, 36, 36};
    int order = 6;
    double tol = 1e-5;
    int maxIter = 100;
    double peek = 0.65;
    int predictor = 2;
    double ke = 138.935458;
    int device = 0;
    double skin = 0.15;
    int precision = 1;    // 0 FP64, 1 mixed
    int zeroGuess = 0;
    int polarizable = 1;
    int refine = 0;       // mixed: FP64 iterative refinement of the induced dipoles
};

// pgmcuda::Terms (core/cuda/pgm_cuda.h:41-45).
struct Terms {
    double direct = 0, reciprocal = 0, self = 0, background = 0, polarization = 0, gvdw = 0;
    double total() const { return direct + reciprocal + self + background + polarization + gvdw; }
};

// Coefficients c[0..k-1] of the GVDW dispersion's G(y) / G(0) as a series in y^2 (derived from erf and exp).
void gvdwSeries(double* c, int k);

class Engine {
public:
    explicit Engine(const Settings& settings);
    ~Engine();
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    void setAtoms(int n, const double* q, const double* radius, const double* alpha, const int* globalIndex,
                  int numGlobal);
    void setCovalent(int ncov, const int* atom, const int* partner, const double* strength);
    // the caller's pair candidates in place of the own pair search, until the next setAtoms
    void setCandidates(int nseg, const int* segI, const int* segShift, const int* segBegin, const int* candJ);
    // self-test of the grid transforms' bounded barrier wait (1: the wait gave up as designed)
    int probeBarrierTimeout(double* seconds);
    // the combination-rule GVDW van der Waals in the final pair pass, until the next setAtoms
    void setGvdw(int repulsion, double rvdw, const double* sqrtA, const double* sqrtC6, const double* b, int nskip,
                 const int* skipI, const int* skipJ);
    Terms compute(const double* pos, const double box[3][3], bool newStep, double* f, double* strain);
    Terms computeF(const float* pos, const double box[3][3], bool newStep, double* strain);
    void releasePositions() {}
    const double* forces() const;
    Terms computeDevice(const void* posq4, const double box[3][3], bool newStep, long long* forceFixed, int stride,
                        double fixedScale, void* stream);
    void launchDevice(const void* posq4, const double box[3][3], bool newStep, long long* forceFixed, int stride,
                      double fixedScale, void* stream);
    bool finishDevice(Terms& terms);
    void waitDevice(void* stream);
    void launchResident(const double* posDev, const double box[3][3], bool newStep, double* forcesDev, void* stream);
    long lateListChecks() const { return 0; }

    int iterations() const;
    double residual() const;
    void inducedDipoles(double* mu) const;
    void permanentDipoles(double* p) const;
    void resetHistory();
    long listBuilds() const;
    int numCandidates() const;
    std::array<double, 9> strainDerivative() const;
    void field(const double* pos, const double box[3][3], const double* q, const double* d, double* E);
    long long pairs(int* pi, int* pj, long long cap);
    long long historySize() const;
    void getHistory(void* blob) const;
    void setHistory(const void* blob);
    void paramGrad(double* dq, double* dradius, double* dalpha, double* dstrength);
    // Energy, forces and total field at given induced dipoles (no solve); keepList: the previous evaluation's
    // pair list, box and wraps (finite-difference probes).  Then paramGrad gives dE/dtheta at these dipoles.
    Terms evaluateFixed(const double* pos, const double box[3][3], const double* mu, bool keepList, double* forces,
                        double* field);
    // (alpha^-1 - T) x = rhs on the geometry of the last evaluation (rows of non-polarizable atoms: 0);
    // returns the CG iterations.
    int solve(const double* rhs, double* x, double tol);
    // Gradient of the force-matching loss L = sum |F - F_target|^2 of the last evaluation (peek 0) with
    // respect to the per-atom charges, radii, polarizabilities and the per-dipole strengths, by one adjoint
    // solve to tol with analytic tangent passes; batched engines: every system at once.  Returns L.
    double forceMatchingGrad(const double* fTarget, double tol, double* dq, double* dradius, double* dalpha,
                             double* dstrength, int* iterations);

    // measurement: own kernels per evaluation; average durations [ms] of the main kernels relaunched
    // alone (0 pair list, 1 pair field pass, 2 spread, 3 gather, 4 final pair pass, 5 FFT chain, 6 CG update),
    // warm (back to back) or, with a flush buffer larger than L2, cold (the buffer overwritten before each launch)
    int kernelLaunches() const;
    // batched CG: systems still iterating before each iteration of the last evaluation; returns the count
    int activeSystems(int* counts, int cap) const;
    void kernelTimes(int reps, double* ms, void* flush = nullptr, size_t flushBytes = 0);
    // median device time [ms] of reps whole new-step evaluations at the last evaluation's positions
    double timeEvaluations(int reps);
    void setPairLanes(int lanes);
    // field-pass transforms: 0 cuFFT 3D plans + influence product kernel, 1 one cluster kernel per launch,
    // 2 cuFFT 2D plans over the x-planes + one x-line kernel with the influence product, 3 one cooperative kernel
    // with a block per x-plane (1, 2 and 3 where the grids allow them; transforms() tells which runs)
    void setTransforms(int mode);
    // PME spread / gather of the field passes: 0 a warp per atom, 1 plane-owner tiles in shared memory (mixed
    // precision, one system, order 6), 2 float4 lines (mixed precision, orders 4, 5, 6, 8), 3 cell-group tiles
    // (mixed precision, one system, orders 4, 5, 6, 8); pmeKernels() tells which runs
    void setPmeKernels(int kind);
    int pmeKernels() const;
    int transforms() const;
    int pairLanes() const;

    // batched systems
    void setSystems(int nsys, const int* atomCount, const double* cutoff, const double* beta, const int* grid,
                    const double* q, const double* radius, const double* alpha, const int* covCount,
                    const int* covAtom, const int* covPartner, const double* strength);
    void computeBatch(const double* pos, const double* boxes, double* energies, double* forces, double* strain,
                      int* iterations);

    struct Impl;

private:
    Impl* impl;
};

}  // namespace pgmb200
