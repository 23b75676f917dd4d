// C ABI of the pgm_b200 engine (include/pgm_b200.h): exceptions become status codes and a per-thread message.
#include "../../include/pgm_b200.h"
#include "pgm_engine.h"

#include <cuda_runtime.h>

#include <cstring>
#include <new>
#include <stdexcept>
#include <string>

struct pgm_engine {
    pgmb200::Engine* e;
};

namespace {
thread_local std::string g_lastError;

template <class F> int guarded(F&& f) {
    try {
        f();
        return PGM_OK;
    } catch (const std::invalid_argument& ex) {
        g_lastError = ex.what();
        return PGM_ERR_ARGUMENT;
    } catch (const std::logic_error& ex) {
        g_lastError = ex.what();
        return PGM_ERR_STATE;
    } catch (const std::bad_alloc&) {
        g_lastError = "pgm_b200: host allocation failed";
        return PGM_ERR_CAPACITY;
    } catch (const std::exception& ex) {
        g_lastError = ex.what();
        return PGM_ERR_CUDA;
    } catch (...) {
        g_lastError = "pgm_b200: unknown error";
        return PGM_ERR_CUDA;
    }
}

pgmb200::Settings toSettings(const pgm_settings* s) {
    pgmb200::Settings o;
    o.cutoff = s->cutoff;
    o.beta = s->beta;
    for (int a = 0; a < 3; a++)
        o.grid[a] = s->grid[a];
    o.order = s->order;
    o.tol = s->tol;
    o.maxIter = s->max_iter;
    o.peek = s->peek;
    o.predictor = s->predictor;
    o.ke = s->ke;
    o.device = s->device;
    o.skin = s->skin;
    o.precision = s->precision;
    o.zeroGuess = s->zero_guess;
    o.polarizable = s->polarizable;
    o.refine = s->refine;
    return o;
}

void toBox(const double* b, double (&box)[3][3]) {
    for (int a = 0; a < 3; a++)
        for (int c = 0; c < 3; c++)
            box[a][c] = b[3 * a + c];
}

void fill(pgm_terms* t, const pgmb200::Terms& x) {
    if (!t)
        return;
    t->direct = x.direct;
    t->reciprocal = x.reciprocal;
    t->self = x.self;
    t->background = x.background;
    t->polarization = x.polarization;
    t->gvdw = x.gvdw;
}

#define NEED(e)                                                              \
    if (!(e) || !(e)->e) {                                                   \
        g_lastError = "pgm_b200: null engine";                               \
        return PGM_ERR_ARGUMENT;                                             \
    }
}  // namespace

extern "C" {

void pgm_settings_default(pgm_settings* s) {
    if (!s)
        return;
    const pgmb200::Settings d;
    s->cutoff = d.cutoff;
    s->beta = d.beta;
    for (int a = 0; a < 3; a++)
        s->grid[a] = d.grid[a];
    s->order = d.order;
    s->tol = d.tol;
    s->max_iter = d.maxIter;
    s->peek = d.peek;
    s->predictor = d.predictor;
    s->ke = d.ke;
    s->device = d.device;
    s->skin = d.skin;
    s->precision = d.precision;
    s->zero_guess = d.zeroGuess;
    s->polarizable = d.polarizable;
    s->refine = d.refine;
}

const char* pgm_last_error(void) { return g_lastError.c_str(); }
const char* pgm_version(void) { return "pgm_b200 1.0 (sm_100a)"; }

int pgm_engine_create(const pgm_settings* s, pgm_engine** out) {
    if (!s || !out) {
        g_lastError = "pgm_b200: null argument";
        return PGM_ERR_ARGUMENT;
    }
    *out = nullptr;
    return guarded([&] {
        if (s->order < 3 || s->order > 12)
            throw std::invalid_argument("pgm_b200: PME order must be 3..12");
        if (s->precision != PGM_PRECISION_FP64 && s->precision != PGM_PRECISION_MIXED)
            throw std::invalid_argument("pgm_b200: unknown precision");
        if (!(s->tol >= 0) || s->max_iter < 0)
            throw std::invalid_argument("pgm_b200: tolerance and max_iter must be non-negative");
        pgm_engine* h = new pgm_engine{new pgmb200::Engine(toSettings(s))};
        *out = h;
    });
}

void pgm_engine_destroy(pgm_engine* e) {
    if (!e)
        return;
    try {
        delete e->e;
    } catch (...) {
    }
    delete e;
}

int pgm_engine_set_atoms(pgm_engine* e, int n, const double* q, const double* radius, const double* alpha,
                         const int* global_index, int num_global) {
    NEED(e);
    return guarded([&] {
        if (n <= 0 || !q || !radius || !alpha)
            throw std::invalid_argument("pgm_b200: set_atoms needs n > 0 and q, radius, alpha");
        e->e->setAtoms(n, q, radius, alpha, global_index, num_global);
    });
}

int pgm_engine_set_covalent(pgm_engine* e, int ncov, const int* atom, const int* partner, const double* strength) {
    NEED(e);
    return guarded([&] {
        if (ncov < 0 || (ncov > 0 && (!atom || !partner || !strength)))
            throw std::invalid_argument("pgm_b200: set_covalent arguments");
        e->e->setCovalent(ncov, atom, partner, strength);
    });
}

int pgm_gvdw_series(double* c, int k) {
    return guarded([&] {
        if (!c || k < 1 || k > 32)
            throw std::invalid_argument("pgm_b200: gvdw_series needs 1 <= k <= 32 and an output array");
        pgmb200::gvdwSeries(c, k);
    });
}

int pgm_engine_probe_barrier_timeout(pgm_engine* e, int* flag, double* seconds) {
    NEED(e);
    return guarded([&] {
        const int f = e->e->probeBarrierTimeout(seconds);
        if (flag)
            *flag = f;
    });
}

int pgm_engine_set_gvdw(pgm_engine* e, int repulsion, double rvdw, const double* sqrt_a, const double* sqrt_c6,
                        const double* b, int nskip, const int* skip_i, const int* skip_j) {
    NEED(e);
    return guarded([&] { e->e->setGvdw(repulsion, rvdw, sqrt_a, sqrt_c6, b, nskip, skip_i, skip_j); });
}

int pgm_engine_set_candidates(pgm_engine* e, int nseg, const int* seg_i, const int* seg_shift, const int* seg_begin,
                              const int* cand_j) {
    NEED(e);
    return guarded([&] { e->e->setCandidates(nseg, seg_i, seg_shift, seg_begin, cand_j); });
}

int pgm_engine_compute(pgm_engine* e, const double* pos, const double* box, int new_step, double* f, double* strain,
                       pgm_terms* terms) {
    NEED(e);
    return guarded([&] {
        if (!pos || !box)
            throw std::invalid_argument("pgm_b200: compute needs positions and box");
        double b[3][3];
        toBox(box, b);
        fill(terms, e->e->compute(pos, b, new_step != 0, f, strain));
    });
}

int pgm_engine_compute_f(pgm_engine* e, const float* pos, const double* box, int new_step, double* strain,
                         pgm_terms* terms) {
    NEED(e);
    return guarded([&] {
        if (!pos || !box)
            throw std::invalid_argument("pgm_b200: compute_f needs positions and box");
        double b[3][3];
        toBox(box, b);
        fill(terms, e->e->computeF(pos, b, new_step != 0, strain));
    });
}

const double* pgm_engine_forces(pgm_engine* e) { return (e && e->e) ? e->e->forces() : nullptr; }

int pgm_engine_release_positions(pgm_engine* e) {
    NEED(e);
    return guarded([&] { e->e->releasePositions(); });
}

int pgm_engine_launch_device(pgm_engine* e, const void* posq4, const double* box, int new_step, long long* force_fixed,
                             int stride, double fixed_scale, void* stream) {
    NEED(e);
    return guarded([&] {
        if (!posq4 || !box)
            throw std::invalid_argument("pgm_b200: launch_device needs positions and box");
        double b[3][3];
        toBox(box, b);
        e->e->launchDevice(posq4, b, new_step != 0, force_fixed, stride, fixed_scale, stream);
    });
}

int pgm_engine_finish_device(pgm_engine* e, pgm_terms* terms, int* valid) {
    NEED(e);
    return guarded([&] {
        pgmb200::Terms t;
        const bool ok = e->e->finishDevice(t);
        fill(terms, t);
        if (valid)
            *valid = ok ? 1 : 0;
    });
}

int pgm_engine_wait_device(pgm_engine* e, void* stream) {
    NEED(e);
    return guarded([&] { e->e->waitDevice(stream); });
}

int pgm_engine_compute_device(pgm_engine* e, const void* posq4, const double* box, int new_step,
                              long long* force_fixed, int stride, double fixed_scale, void* stream, pgm_terms* terms) {
    NEED(e);
    return guarded([&] {
        double b[3][3];
        toBox(box, b);
        fill(terms, e->e->computeDevice(posq4, b, new_step != 0, force_fixed, stride, fixed_scale, stream));
    });
}

int pgm_engine_launch_resident(pgm_engine* e, const double* pos_dev, const double* box, int new_step,
                               double* forces_dev, void* stream) {
    NEED(e);
    return guarded([&] {
        if (!pos_dev || !box)
            throw std::invalid_argument("pgm_b200: launch_resident needs positions and box");
        double b[3][3];
        toBox(box, b);
        e->e->launchResident(pos_dev, b, new_step != 0, forces_dev, stream);
    });
}

int pgm_engine_iterations(pgm_engine* e) { return (e && e->e) ? e->e->iterations() : -1; }
double pgm_engine_residual(pgm_engine* e) { return (e && e->e) ? e->e->residual() : -1.0; }

int pgm_engine_induced_dipoles(pgm_engine* e, double* mu) {
    NEED(e);
    return guarded([&] { e->e->inducedDipoles(mu); });
}

int pgm_engine_permanent_dipoles(pgm_engine* e, double* p) {
    NEED(e);
    return guarded([&] { e->e->permanentDipoles(p); });
}

int pgm_engine_reset_history(pgm_engine* e) {
    NEED(e);
    return guarded([&] { e->e->resetHistory(); });
}

long pgm_engine_list_builds(pgm_engine* e) { return (e && e->e) ? e->e->listBuilds() : -1; }
long pgm_engine_late_list_checks(pgm_engine* e) { return (e && e->e) ? e->e->lateListChecks() : -1; }
int pgm_engine_num_candidates(pgm_engine* e) {
    if (!e || !e->e)
        return -1;
    int v = -1;
    guarded([&] { v = e->e->numCandidates(); });
    return v;
}

int pgm_engine_strain(pgm_engine* e, double* strain) {
    NEED(e);
    return guarded([&] {
        const auto s = e->e->strainDerivative();
        for (int k = 0; k < 9; k++)
            strain[k] = s[k];
    });
}

int pgm_engine_field(pgm_engine* e, const double* pos, const double* box, const double* q, const double* d,
                     double* E) {
    NEED(e);
    return guarded([&] {
        if (!pos || !box || !q || !d || !E)
            throw std::invalid_argument("pgm_b200: field arguments");
        double b[3][3];
        toBox(box, b);
        e->e->field(pos, b, q, d, E);
    });
}

int pgm_engine_pairs(pgm_engine* e, int* pi, int* pj, long long cap, long long* npairs) {
    NEED(e);
    return guarded([&] {
        const long long m = e->e->pairs(pi, pj, cap);
        if (npairs)
            *npairs = m;
    });
}

long long pgm_engine_history_size(pgm_engine* e) { return (e && e->e) ? e->e->historySize() : -1; }

int pgm_engine_get_history(pgm_engine* e, void* blob) {
    NEED(e);
    return guarded([&] { e->e->getHistory(blob); });
}

int pgm_engine_set_history(pgm_engine* e, const void* blob) {
    NEED(e);
    return guarded([&] { e->e->setHistory(blob); });
}

int pgm_engine_param_grad(pgm_engine* e, double* dq, double* dradius, double* dalpha, double* dstrength) {
    NEED(e);
    return guarded([&] { e->e->paramGrad(dq, dradius, dalpha, dstrength); });
}

int pgm_engine_evaluate_fixed(pgm_engine* e, const double* pos, const double* box, const double* mu, int keep_list,
                              double* forces, double* field, pgm_terms* terms) {
    NEED(e);
    return guarded([&] {
        if (!pos || !box || !mu)
            throw std::invalid_argument("pgm_b200: evaluate_fixed needs positions, box and dipoles");
        double b[3][3];
        toBox(box, b);
        fill(terms, e->e->evaluateFixed(pos, b, mu, keep_list != 0, forces, field));
    });
}

int pgm_engine_solve(pgm_engine* e, const double* rhs, double* x, double tol, int* iterations) {
    NEED(e);
    return guarded([&] {
        if (!rhs || !x || !(tol > 0))
            throw std::invalid_argument("pgm_b200: solve needs rhs, x and tol > 0");
        const int it = e->e->solve(rhs, x, tol);
        if (iterations)
            *iterations = it;
    });
}

int pgm_engine_force_matching_grad(pgm_engine* e, const double* f_target, double tol, double* dq, double* dradius,
                                   double* dalpha, double* dstrength, double* loss, int* iterations) {
    NEED(e);
    return guarded([&] {
        if (!f_target || !(tol > 0))
            throw std::invalid_argument("pgm_b200: force_matching_grad needs f_target and tol > 0");
        const double L = e->e->forceMatchingGrad(f_target, tol, dq, dradius, dalpha, dstrength, iterations);
        if (loss)
            *loss = L;
    });
}

int pgm_engine_active_systems(pgm_engine* e, int* counts, int cap) {
    if (!e || !e->e || !counts || cap < 0)
        return -1;
    try {
        return e->e->activeSystems(counts, cap);
    } catch (const std::exception& ex) {
        g_lastError = ex.what();
        return PGM_ERR_CUDA;
    }
}

int pgm_engine_kernel_launches(pgm_engine* e) { return (e && e->e) ? e->e->kernelLaunches() : -1; }

int pgm_engine_kernel_times(pgm_engine* e, int reps, double* ms) {
    NEED(e);
    return guarded([&] {
        if (reps <= 0 || !ms)
            throw std::invalid_argument("pgm_b200: kernel_times arguments");
        e->e->kernelTimes(reps, ms);
    });
}

int pgm_engine_kernel_times_cold(pgm_engine* e, int reps, void* flush_dev, size_t flush_bytes, double* ms) {
    NEED(e);
    return guarded([&] {
        if (reps <= 0 || !ms || !flush_dev || flush_bytes == 0)
            throw std::invalid_argument("pgm_b200: kernel_times_cold arguments");
        e->e->kernelTimes(reps, ms, flush_dev, flush_bytes);
    });
}

int pgm_engine_time_evaluations(pgm_engine* e, int reps, double* ms) {
    NEED(e);
    return guarded([&] {
        if (reps <= 0 || !ms)
            throw std::invalid_argument("pgm_b200: time_evaluations arguments");
        *ms = e->e->timeEvaluations(reps);
    });
}

int pgm_engine_set_pme_kernels(pgm_engine* e, int kind) {
    NEED(e);
    return guarded([&] { e->e->setPmeKernels(kind); });
}

int pgm_engine_pme_kernels(pgm_engine* e) { return (e && e->e) ? e->e->pmeKernels() : -1; }

int pgm_engine_set_pair_lanes(pgm_engine* e, int lanes) {
    NEED(e);
    return guarded([&] { e->e->setPairLanes(lanes); });
}

int pgm_engine_pair_lanes(pgm_engine* e) { return (e && e->e) ? e->e->pairLanes() : -1; }

int pgm_engine_set_transforms(pgm_engine* e, int mode) {
    NEED(e);
    return guarded([&] { e->e->setTransforms(mode); });
}

int pgm_engine_transforms(pgm_engine* e) { return (e && e->e) ? e->e->transforms() : -1; }

int pgm_engine_set_systems(pgm_engine* e, int nsys, const int* atom_count, const double* cutoff, const double* beta,
                           const int* grid, const double* q, const double* radius, const double* alpha,
                           const int* cov_count, const int* cov_atom, const int* cov_partner, const double* strength) {
    NEED(e);
    return guarded([&] {
        if (nsys <= 0 || !atom_count || !cutoff || !beta || !grid || !q || !radius || !alpha || !cov_count)
            throw std::invalid_argument("pgm_b200: set_systems arguments");
        e->e->setSystems(nsys, atom_count, cutoff, beta, grid, q, radius, alpha, cov_count, cov_atom, cov_partner,
                         strength);
    });
}

int pgm_engine_compute_batch(pgm_engine* e, const double* pos, const double* boxes, double* energies, double* forces,
                             double* strain, int* iterations) {
    NEED(e);
    return guarded([&] {
        if (!pos || !boxes)
            throw std::invalid_argument("pgm_b200: compute_batch needs positions and boxes");
        e->e->computeBatch(pos, boxes, energies, forces, strain, iterations);
    });
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------- no allocation

namespace pgmb200 {
int pairListNoAlloc(int n, const double* posDev, const double* box, double cutoff, int cap, int* slotAtomOut,
                    int* countsOut, int* neighborsOut, cudaStream_t st, int* maxCount);
}

extern "C" int pgm_pair_list_noalloc(int n, const double* pos_dev, const double* box, double cutoff, int cap,
                                     int* slot_atom_dev, int* counts_dev, int* neighbors_dev, void* stream,
                                     int* max_count) {
    try {
        const int over = pgmb200::pairListNoAlloc(n, pos_dev, box, cutoff, cap, slot_atom_dev, counts_dev,
                                                  neighbors_dev, (cudaStream_t) stream, max_count);
        if (over) {
            g_lastError = "pgm_b200: pair_list_noalloc: an atom has more neighbours than cap (see max_count)";
            return PGM_ERR_CAPACITY;
        }
        return PGM_OK;
    } catch (const std::length_error& ex) {
        g_lastError = ex.what();
        return PGM_ERR_CAPACITY;
    } catch (const std::invalid_argument& ex) {
        g_lastError = ex.what();
        return PGM_ERR_ARGUMENT;
    } catch (const std::exception& ex) {
        g_lastError = ex.what();
        return PGM_ERR_CUDA;
    }
}
