/*
 * pgm_b200: periodic pGM electrostatics (Gaussian charges, covalent permanent dipoles, Gaussian induced
 * dipoles, smooth PME) on one NVIDIA B200, as a C ABI.
 *
 * The entry points replace the reference's GPU engine interface pgmcuda::Engine
 * (core/cuda/pgm_cuda.h:47-127 of larryhuang98/pGM-MD) one to one, and add batched multi-system
 * evaluation and parameter gradients.  Every call returns PGM_OK (0) or a negative status; the message of
 * the last failure on the calling thread is pgm_last_error().  No call aborts or traps.
 *
 * Units: nm, e, e nm, nm^3; energies kJ/mol, forces kJ/mol/nm, strain derivative kJ/mol (the Coulomb
 * constant is a setting).  Boxes are three rows a, b, c in the reduced triclinic form
 * a = (ax, 0, 0), b = (bx, by, 0), c = (cx, cy, cz), row-major double[9].
 * Threading: one thread at a time per engine (any thread), like the reference engine.
 */
#ifndef PGM_B200_H_
#define PGM_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PGM_OK 0
#define PGM_ERR_ARGUMENT (-1)   /* invalid argument (the reference throws std::invalid_argument) */
#define PGM_ERR_CUDA (-2)       /* CUDA / cuFFT failure (the reference throws std::runtime_error) */
#define PGM_ERR_STATE (-3)      /* call out of order (e.g. compute before set_atoms) */
#define PGM_ERR_CAPACITY (-4)   /* an input beyond a stated maximum */

#define PGM_PRECISION_FP64 0    /* every kernel in double precision */
#define PGM_PRECISION_MIXED 1   /* FP32 pair/PME/matvec arithmetic, FP64 accumulation, CG vectors and scalars */

typedef struct pgm_engine pgm_engine;

/* pgmcuda::Settings (core/cuda/pgm_cuda.h:25-39) plus the precision and the initial guess. */
typedef struct pgm_settings {
    double cutoff;       /* direct-space cutoff [nm] */
    double beta;         /* Ewald coefficient [1/nm] */
    int grid[3];         /* PME grid */
    int order;           /* B-spline order, 3..12 */
    double tol;          /* max|alpha r| / mean|alpha E_perm| */
    int max_iter;
    double peek;         /* final mu += peek alpha r */
    int predictor;       /* 0 none (guess alpha E_perm), 1 mu3, 2 mu4 (history in the global order) */
    double ke;           /* Coulomb constant [kJ mol^-1 nm e^-2] */
    int device;          /* CUDA device; < 0: the device current on the calling thread */
    double skin;         /* Verlet list radius cutoff + skin [nm] (shrunk to stay within half the box); the list is
                            kept while every atom stays within skin/2 of its position at the build and the box
                            is unchanged (checked on the GPU at every evaluation); <= 0: built at every evaluation */
    int precision;       /* PGM_PRECISION_FP64 or PGM_PRECISION_MIXED */
    int zero_guess;      /* 1: initial guess mu = 0 when the predictor has no history (instead of alpha E_perm) */
    int polarizable;     /* 0: no induced dipoles (pgmcore::Settings::polarizable) */
    int refine;          /* mixed precision: 1 = FP64 iterative refinement of the induced dipoles (the residual
                            E_perm - (alpha^-1 - T) mu recomputed with FP64 pair and PME arithmetic, corrections
                            solved with the FP32 operator) */
} pgm_settings;

/* pgmcuda::Terms (core/cuda/pgm_cuda.h:41-45). gvdw is always 0 (combination-rule GVDW is not part of this
 * engine). */
typedef struct pgm_terms {
    double direct, reciprocal, self, background, polarization, gvdw;
} pgm_terms;

/* Fills *s with the reference defaults of pgmcuda::Settings (core/cuda/pgm_cuda.h:25-39). */
void pgm_settings_default(pgm_settings* s);

const char* pgm_last_error(void);
const char* pgm_version(void);

/* pgmcuda::Engine::Engine(const Settings&) (core/cuda/pgm_cuda.h:49). */
int pgm_engine_create(const pgm_settings* s, pgm_engine** out);
/* pgmcuda::Engine::~Engine (core/cuda/pgm_cuda.h:50). */
void pgm_engine_destroy(pgm_engine* e);

/* pgmcuda::Engine::setAtoms (core/cuda/pgm_cuda.h:55-56): atoms in the caller's order; global_index (NULL:
 * identity) keys the predictor history; alpha <= 1e-9 nm^3 is not polarizable (core/pgm_constants.h:9). */
int pgm_engine_set_atoms(pgm_engine* e, int n, const double* q, const double* radius, const double* alpha,
                         const int* global_index, int num_global);
/* pgmcuda::Engine::setCovalent (core/cuda/pgm_cuda.h:67): p_atom += strength unit(r_partner - r_atom). */
int pgm_engine_set_covalent(pgm_engine* e, int ncov, const int* atom, const int* partner, const double* strength);
/* pgmcuda::Engine::setCandidates (core/cuda/pgm_cuda.h:68-73): the caller's pair candidates in place of the
 * engine's own pair search, until the next set_atoms.  Segment s holds the pairs (seg_i[s], cand_j[k]),
 * k in [seg_begin[s], seg_begin[s+1]) (seg_begin has nseg+1 entries, seg_begin[0] = 0), with
 * x = r_i + t.box - r_j, t = seg_shift[3s .. 3s+2] integer box vectors (|t| <= 127); every pair at most once;
 * the pairs beyond the cutoff are left out at every evaluation.  Single-system engines. */
int pgm_engine_set_candidates(pgm_engine* e, int nseg, const int* seg_i, const int* seg_shift, const int* seg_begin,
                              const int* cand_j);
/* Self-test of the failure path of the grid transforms' barriers (no counterpart in the reference): one block
 * waits at a barrier that expects two; the wait gives up after its bounded number of polls, sets the error flag
 * and returns.  *flag = 1 when it did (the expected outcome), *seconds the device time of the launch. */
int pgm_engine_probe_barrier_timeout(pgm_engine* e, int* flag, double* seconds);
/* The coefficients c[0..k-1] (k <= 32) of the GVDW dispersion's G(y)/G(0) = sum c_m y^(2m) that set_gvdw uses
 * below y = 0.6, derived from the series of erf and exp (no counterpart in the reference, which tabulates them in
 * core/gvdw_kernel.h:33-37).  Host only: needs no GPU. */
int pgm_gvdw_series(double* c, int k);
/* pgmcuda::Engine::setGvdw (core/cuda/pgm_cuda.h:57-65): the combination-rule GVDW van der Waals
 * (core/gvdw_kernel.h) for the pairs within rvdw except the skipped ones: per atom sqrt_a = sqrt(A) [kJ/mol]^1/2,
 * sqrt_c6 = sqrt(C6) [kJ/mol nm^6]^1/2, b (zeros: no term), repulsion 0 Gaussian A exp(-B y^2), 1 Slater
 * A exp(-B y) with y = r / sqrt(2 (R_i^2 + R_j^2)); skipped pairs (skip_i[k], skip_j[k]) once each.  Its energy is
 * pgm_terms.gvdw, its forces and strain are added to the evaluation's.  rvdw <= cutoff (the pass runs over the
 * evaluation's pair list).  Single-system engines, until the next set_atoms; parameter gradients (param_grad)
 * are refused while it is set. */
int pgm_engine_set_gvdw(pgm_engine* e, int repulsion, double rvdw, const double* sqrt_a, const double* sqrt_c6,
                        const double* b, int nskip, const int* skip_i, const int* skip_j);

/* pgmcuda::Engine::compute (core/cuda/pgm_cuda.h:79): positions pos (n*3, host), box (9); forces ADDED to
 * f (n*3, may be NULL), strain derivative ADDED to strain (9, may be NULL); terms (may be NULL).
 * new_step: this evaluation starts a new MD step (its solution enters the predictor history). */
int pgm_engine_compute(pgm_engine* e, const double* pos, const double* box, int new_step, double* f,
                       double* strain, pgm_terms* terms);
/* pgmcuda::Engine::computeF (core/cuda/pgm_cuda.h:82): float positions; the forces stay in the engine
 * (pgm_engine_forces). */
int pgm_engine_compute_f(pgm_engine* e, const float* pos, const double* box, int new_step, double* strain,
                         pgm_terms* terms);
/* pgmcuda::Engine::forces (core/cuda/pgm_cuda.h:86): forces of the last compute_f (n*3, valid until the next
 * call). */
const double* pgm_engine_forces(pgm_engine* e);
/* pgmcuda::Engine::releasePositions (core/cuda/pgm_cuda.h:85): no registered memory is kept; accepted. */
int pgm_engine_release_positions(pgm_engine* e);

/* pgmcuda::Engine::launchDevice / finishDevice / waitDevice / computeDevice (core/cuda/pgm_cuda.h:93-111):
 * positions from the device array posq4 (float4, w ignored, caller order); forces added atomically to the
 * device 64-bit fixed-point buffer force_fixed (x of atom i at i, y at i + stride, z at i + 2 stride,
 * scale fixed_scale); stream: the caller's cudaStream_t (its work so far comes first).  finish_device sets
 * *valid = 0 when the evaluation must be repeated (the pair list outgrew its rows and was grown, or a pair
 * within the cutoff changed its image since the list's build and the list is rebuilt), as the reference's
 * finishDevice returns false (core/cuda/pgm_cuda.h:107); else 1. */
int pgm_engine_launch_device(pgm_engine* e, const void* posq4, const double* box, int new_step,
                             long long* force_fixed, int stride, double fixed_scale, void* stream);
int pgm_engine_finish_device(pgm_engine* e, pgm_terms* terms, int* valid);
int pgm_engine_wait_device(pgm_engine* e, void* stream);
int pgm_engine_compute_device(pgm_engine* e, const void* posq4, const double* box, int new_step,
                              long long* force_fixed, int stride, double fixed_scale, void* stream, pgm_terms* terms);
/* Device-resident evaluation for benchmarks and device callers: positions pos_dev (device double n*3),
 * forces written (not added) to forces_dev (device double n*3, may be NULL), no host synchronisation;
 * pgm_engine_finish_device returns its terms.  No counterpart in the reference. */
int pgm_engine_launch_resident(pgm_engine* e, const double* pos_dev, const double* box, int new_step,
                               double* forces_dev, void* stream);

/* Getters of pgmcuda::Engine (core/cuda/pgm_cuda.h:112-122).  list_builds: builds of the Verlet list so far;
 * late_list_checks: always 0 (the stale test runs on the GPU before the list is used); num_candidates: the
 * directed pairs within the cutoff at the last evaluation (the reference counts its list's candidates). */
int pgm_engine_iterations(pgm_engine* e);
double pgm_engine_residual(pgm_engine* e);
int pgm_engine_induced_dipoles(pgm_engine* e, double* mu);
int pgm_engine_permanent_dipoles(pgm_engine* e, double* p);
int pgm_engine_reset_history(pgm_engine* e);
long pgm_engine_list_builds(pgm_engine* e);
long pgm_engine_late_list_checks(pgm_engine* e);
int pgm_engine_num_candidates(pgm_engine* e);

/* pgmcore::Engine::strainDerivative (core/pgm_core.h:67-73) of the last evaluation (9, row-major). */
int pgm_engine_strain(pgm_engine* e, double* strain);
/* pgmcore::Engine::field (core/pgm_core.h:76-77): field [e/nm^2] of charges q (n) and dipoles d (n*3) at
 * the atoms (direct + reciprocal + self) for positions pos and box; E (n*3). */
int pgm_engine_field(pgm_engine* e, const double* pos, const double* box, const double* q, const double* d,
                     double* E);
/* The directed pair list of the last evaluation (both directions, r < cutoff by the reference's minimum
 * image, core/pgm_core.cpp:64-87): pairs i < j written to pi, pj (capacity cap); *npairs = count.  No
 * counterpart in the reference (its list is internal). */
int pgm_engine_pairs(pgm_engine* e, int* pi, int* pj, long long cap, long long* npairs);

/* Predictor history as a blob (checkpoint/resume): size in bytes, get, set.  No counterpart in the
 * reference. */
long long pgm_engine_history_size(pgm_engine* e);
int pgm_engine_get_history(pgm_engine* e, void* blob);
int pgm_engine_set_history(pgm_engine* e, const void* blob);

/* Parameter gradients of the total energy at the solved dipoles of the last evaluation (E is stationary in
 * the induced dipoles; run with peek = 0): dE/dq, dE/dradius, dE/dalpha per atom (n each), dE/dstrength per
 * covalent dipole (ncov).  Any output may be NULL.  No counterpart in the reference. */
int pgm_engine_param_grad(pgm_engine* e, double* dq, double* dradius, double* dalpha, double* dstrength);

/* Adjoint building blocks (no counterpart in the reference).  evaluate_fixed: energy terms, forces (n*3, may be
 * NULL) and the total field (n*3, may be NULL) at the given induced dipoles mu (n*3), without a solve; keep_list
 * reuses the previous evaluation's pair list and box (smooth finite-difference probes).  pgm_engine_param_grad
 * then gives dE/dtheta at those dipoles.  solve: (alpha^-1 - T) x = rhs on the geometry of the last evaluation,
 * to tolerance tol; *iterations (may be NULL) gets the CG iterations. */
int pgm_engine_evaluate_fixed(pgm_engine* e, const double* pos, const double* box, const double* mu, int keep_list,
                              double* forces, double* field, pgm_terms* terms);
int pgm_engine_solve(pgm_engine* e, const double* rhs, double* x, double tol, int* iterations);
/* Gradient of the force-matching loss L = sum |F - F_target|^2 of the last evaluation (run it with peek 0, so
 * that the energy is stationary in the induced dipoles) with respect to every per-atom charge (dq), Gaussian
 * radius (dradius), polarizability (dalpha) and per-dipole covalent strength (dstrength), each may be NULL,
 * by ONE adjoint solve (alpha^-1 - T) u = -D_w E_tot to tol and analytic tangent passes (w = 2 (F - F_target);
 * no iterations unrolled, damping terms recomputed per pair).  f_target: n*3 host forces (batched engines:
 * every system's, concatenated; the gradient covers every system at once).  *loss = L, *iterations = the
 * adjoint's CG iterations (either may be NULL).  No counterpart in the reference, which lists parameter
 * derivatives as not implemented (docs/openmm.md:265). */
int pgm_engine_force_matching_grad(pgm_engine* e, const double* f_target, double tol, double* dq, double* dradius,
                                   double* dalpha, double* dstrength, double* loss, int* iterations);

/* Measurement (no counterpart in the reference): the number of this library's kernels the last evaluation
 * ran (cuFFT transforms not counted); average device durations [ms] over reps launches of the main kernels
 * relaunched alone on the engine's stream after an evaluation: ms[0] pair list build, [1] pair field pass,
 * [2] PME spread, [3] PME gather, [4] final pair pass, [5] FFT chain (r2c, convolution, c2r), [6] CG kernel.
 * pair lanes: lanes per atom of the pair passes (4, 8, 16 or 32; the autotuner's knob). */
int pgm_engine_kernel_launches(pgm_engine* e);
/* Batched engines: the number of systems still iterating before each CG iteration of the last evaluation
 * (counts[k], k = 0 .. its iterations; converged systems retire from the loop); returns how many values were
 * written (at most cap), or a negative status. */
int pgm_engine_active_systems(pgm_engine* e, int* counts, int cap);
int pgm_engine_kernel_times(pgm_engine* e, int reps, double* ms);
/* The same kernels timed cold: before each of the reps launches the caller's device buffer flush_dev
 * (flush_bytes, larger than the 126 MB L2) is overwritten, and only the launch lies between the events. */
int pgm_engine_kernel_times_cold(pgm_engine* e, int reps, void* flush_dev, size_t flush_bytes, double* ms);
/* Median device time [ms] of reps whole new-step evaluations at the last evaluation's positions and boxes
 * (already on the device), the predictor history saved and restored: the autotuner's measure. */
int pgm_engine_time_evaluations(pgm_engine* e, int reps, double* ms);
int pgm_engine_set_pair_lanes(pgm_engine* e, int lanes);
/* PME spread and gather of the field passes (the autotuner's third knob; no counterpart in the reference):
 * 0 a warp per atom with p^3 global atomics / loads; 1 plane-owner tiles -- a block per (x-plane, 16-row chunk)
 * accumulates or reads its tile in shared memory for the atoms whose stencil reaches it (mixed precision, one
 * system, order 6); 2 float4 lines -- a thread per (atom, x-plane of its stencil) adds or loads each z line of
 * the stencil as aligned float4 words (mixed precision, orders 4, 5, 6, 8, batches too); 3 cell-group tiles -- a
 * block per group of the pair search's cells accumulates or reads its atoms' grid window in shared memory (mixed
 * precision, one system, orders 4, 5, 6, 8).  Where the choice does not apply, 0 runs; pgm_engine_pme_kernels
 * tells which runs. */
int pgm_engine_set_pme_kernels(pgm_engine* e, int kind);
int pgm_engine_pme_kernels(pgm_engine* e);
int pgm_engine_pair_lanes(pgm_engine* e);
/* Field-pass transforms (the autotuner's second knob; no counterpart in the reference, which calls cuFFT):
 * 0 cuFFT R2C / C2R 3D plans with an influence-product kernel; 1 one kernel per pass in which a thread-block
 * cluster per system holds the half spectrum in distributed shared memory (grids up to 64 points per dimension
 * with prime factors 2, 3, 5); 2 cuFFT 2D plans over the x-planes with one kernel for the x-lines and the
 * influence product (x extents up to 64 with prime factors 2, 3, 5); 3 one cooperative kernel per pass with a
 * thread block per x-plane of every system, the planes and the x-lines exchanged through L2 between two bounded
 * barriers (grids as for 1, every system's blocks resident together).  pgm_engine_transforms: the kind in use
 * (1, 2 and 3 only where the grids allow them). */
int pgm_engine_set_transforms(pgm_engine* e, int mode);
int pgm_engine_transforms(pgm_engine* e);

/* Batched evaluation: nsys independent systems of uneven sizes in one launch.  Atom arrays are the systems'
 * arrays concatenated; atom_count[s] atoms per system; per-system cutoff, beta and grid (3 ints); covalent
 * indices are local to their system.  The shared settings (order, tol, max_iter, peek, ke, precision) come
 * from the engine's settings.  No counterpart in the reference. */
int pgm_engine_set_systems(pgm_engine* e, int nsys, const int* atom_count, const double* cutoff, const double* beta,
                           const int* grid, const double* q, const double* radius, const double* alpha,
                           const int* cov_count, const int* cov_atom, const int* cov_partner, const double* strength);
/* Positions (concatenated, n_total*3), boxes (nsys*9); energies per system (nsys*6 terms in pgm_terms order,
 * may be NULL), forces (n_total*3, written, may be NULL), strain (nsys*9, written, may be NULL), iterations
 * per system (nsys, may be NULL). */
int pgm_engine_compute_batch(pgm_engine* e, const double* pos, const double* boxes, double* energies, double* forces,
                             double* strain, int* iterations);

/* The directed pair list of one periodic system without allocating anything (no counterpart in the
 * reference).  For callers that cannot allocate device memory: MD engines whose memory pool owns all of the
 * device memory and passes fixed buffers, hosts that reserve their device memory up front, and loops that
 * cannot afford cudaMalloc's implicit synchronisation of the device.  Same list as the engine's (the reference's minimum image and r < cutoff test,
 * core/pgm_core.cpp:64-87), computed by the engine's own kernels; their scratch lives in one static device
 * array of the library (about 4 MB, held by every GPU that loads the library until exit).
 *   n          atoms, 1..16384 (larger: PGM_ERR_CAPACITY); pos_dev device double n*3; box double[9] (host)
 *   outputs    device int arrays: slot_atom_dev[n] (row s of the list belongs to atom slot_atom_dev[s]),
 *              counts_dev[n] (neighbours in row s), neighbors_dev[n*cap] (row s: atom indices j, both
 *              directions, in a deterministic order); rows longer than cap are cut and the call returns
 *              PGM_ERR_CAPACITY.  *max_count (may be NULL) receives the longest row on every call.
 *   stream     cudaStream_t; the call copies its small parameter blocks from host memory to the scratch and
 *              waits for its own work on this stream before returning.
 * The first call on a device looks up the scratch array's device address (under a lock).  Calls share the
 * scratch: calls that overlap on the GPU (other threads, other streams) race and must be serialised by the
 * caller. */
int pgm_pair_list_noalloc(int n, const double* pos_dev, const double* box, double cutoff, int cap, int* slot_atom_dev,
                          int* counts_dev, int* neighbors_dev, void* stream, int* max_count);

#ifdef __cplusplus
}
#endif

#endif
