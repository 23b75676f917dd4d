// C entry points over the reference FP64 engine pgmcore::Engine (core/pgm_core.h:47-115), so that the
// tests and the CPU-baseline leg of bench.py can run the reference itself through ctypes.
// TEST INFRASTRUCTURE ONLY: built into oracle/_ref/ by oracle/Makefile from the reference's own sources;
// the CUDA engine never links it.
#include "pgm_core.h"

#include <cstring>
#include <exception>
#include <vector>

using pgmcore::V3;

namespace {
struct Handle {
    pgmcore::Engine* eng;
    int n;
    std::vector<V3> forces;
};
thread_local char lastError[512];
}  // namespace

extern "C" {

const char* ref_last_error() { return lastError; }

void* ref_create(int n, const double* q, const double* radius, const double* alpha, int ncov, const int* covAtom,
                 const int* covPartner, const double* covStrength, double cutoff, double beta, const int* grid,
                 int order, double tol, int maxIter, double peek, int predictor, double ke, int polarizable) {
    try {
        pgmcore::Topology top;
        top.q.assign(q, q + n);
        top.radius.assign(radius, radius + n);
        top.alpha.assign(alpha, alpha + n);
        top.covAtom.assign(covAtom, covAtom + ncov);
        top.covPartner.assign(covPartner, covPartner + ncov);
        top.covStrength.assign(covStrength, covStrength + ncov);
        pgmcore::Settings s;
        s.periodic = true;
        s.cutoff = cutoff;
        s.beta = beta;
        for (int a = 0; a < 3; a++)
            s.grid[a] = grid[a];
        s.order = order;
        s.tol = tol;
        s.maxIter = maxIter;
        s.peek = peek;
        s.predictor = predictor;
        s.ke = ke;
        s.polarizable = polarizable != 0;
        Handle* h = new Handle{new pgmcore::Engine(top, s), n, {}};
        return h;
    } catch (const std::exception& e) {
        std::strncpy(lastError, e.what(), sizeof(lastError) - 1);
        return nullptr;
    }
}

void ref_destroy(void* p) {
    Handle* h = static_cast<Handle*>(p);
    if (h) {
        delete h->eng;
        delete h;
    }
}

// Energy [kJ/mol]; forces (n*3, may be null) overwritten with the forces of this evaluation.
double ref_compute(void* p, const double* pos, const double* box9, double* forces) {
    Handle* h = static_cast<Handle*>(p);
    std::vector<V3> x(h->n);
    for (int i = 0; i < h->n; i++)
        x[i] = V3{pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    V3 box[3];
    for (int a = 0; a < 3; a++)
        box[a] = V3{box9[3 * a], box9[3 * a + 1], box9[3 * a + 2]};
    if (!forces)
        return h->eng->compute(x, box, nullptr);
    h->forces.assign(h->n, V3{0, 0, 0});
    double e = h->eng->compute(x, box, &h->forces);
    for (int i = 0; i < h->n; i++)
        for (int k = 0; k < 3; k++)
            forces[3 * i + k] = h->forces[i][k];
    return e;
}

void ref_terms(void* p, double* t5) {
    const pgmcore::EnergyTerms& t = static_cast<Handle*>(p)->eng->terms();
    t5[0] = t.direct;
    t5[1] = t.reciprocal;
    t5[2] = t.self;
    t5[3] = t.background;
    t5[4] = t.polarization;
}

void ref_strain(void* p, double* s9) {
    const auto& s = static_cast<Handle*>(p)->eng->strainDerivative();
    for (int k = 0; k < 9; k++)
        s9[k] = s[k];
}

static void copyV3(const std::vector<V3>& v, double* out) {
    for (size_t i = 0; i < v.size(); i++)
        for (int k = 0; k < 3; k++)
            out[3 * i + k] = v[i][k];
}

void ref_induced(void* p, double* mu) { copyV3(static_cast<Handle*>(p)->eng->inducedDipoles(), mu); }
void ref_permanent(void* p, double* d) { copyV3(static_cast<Handle*>(p)->eng->permanentDipoles(), d); }
int ref_iterations(void* p) { return static_cast<Handle*>(p)->eng->iterations(); }
double ref_residual(void* p) { return static_cast<Handle*>(p)->eng->residual(); }
void ref_set_history_key(void* p, long long key) { static_cast<Handle*>(p)->eng->setHistoryKey(key); }
void ref_reset_history(void* p) { static_cast<Handle*>(p)->eng->resetHistory(); }

// Field [e/nm^2] of charges q and dipoles d (n*3) at the geometry pos/box (core/pgm_core.h:77-79).
void ref_field(void* p, const double* pos, const double* box9, const double* q, const double* d, double* E) {
    Handle* h = static_cast<Handle*>(p);
    std::vector<V3> x(h->n), dv(h->n);
    for (int i = 0; i < h->n; i++) {
        x[i] = V3{pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
        dv[i] = V3{d[3 * i], d[3 * i + 1], d[3 * i + 2]};
    }
    V3 box[3];
    for (int a = 0; a < 3; a++)
        box[a] = V3{box9[3 * a], box9[3 * a + 1], box9[3 * a + 2]};
    h->eng->setGeometry(x, box);
    std::vector<double> qv(q, q + h->n);
    copyV3(h->eng->field(qv, dv), E);
}

}  // extern "C"
