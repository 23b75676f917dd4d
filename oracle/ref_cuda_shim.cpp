// C entry points over the reference GPU engine pgmcuda::Engine (core/cuda/pgm_cuda.h:47-127), so that the
// comparison leg of bench.py can time the reference's own CUDA engine on the same GPU as pgm_b200.
// TEST INFRASTRUCTURE ONLY: built into oracle/_ref/ by oracle/Makefile from the reference's own sources
// (core/cuda/pgm_cuda.cu, unchanged); pgm_b200 never links it.
#include "cuda/pgm_cuda.h"

#include <cstring>
#include <exception>

namespace {
thread_local char lastError[512];

int fail(const std::exception& e) {
    std::strncpy(lastError, e.what(), sizeof(lastError) - 1);
    return -1;
}

void terms6(const pgmcuda::Terms& t, double* out) {
    if (!out)
        return;
    out[0] = t.direct;
    out[1] = t.reciprocal;
    out[2] = t.self;
    out[3] = t.background;
    out[4] = t.polarization;
    out[5] = t.total();
}

void box3(const double* box9, double box[3][3]) {
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
            box[a][b] = box9[3 * a + b];
}
}  // namespace

extern "C" {

const char* refcuda_last_error() { return lastError; }

void* refcuda_create(double cutoff, double beta, const int* grid, int order, double tol, int maxIter, double peek,
                     int predictor, double ke, int device, double skin) {
    try {
        pgmcuda::Settings s;
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
        s.device = device;
        s.skin = skin;
        return new pgmcuda::Engine(s);
    } catch (const std::exception& e) {
        fail(e);
        return nullptr;
    }
}

void refcuda_destroy(void* p) { delete static_cast<pgmcuda::Engine*>(p); }

int refcuda_set_atoms(void* p, int n, const double* q, const double* radius, const double* alpha) {
    try {
        static_cast<pgmcuda::Engine*>(p)->setAtoms(n, q, radius, alpha, nullptr, n);
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

int refcuda_set_covalent(void* p, int ncov, const int* atom, const int* partner, const double* strength) {
    try {
        static_cast<pgmcuda::Engine*>(p)->setCovalent(ncov, atom, partner, strength);
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// Host positions (n*3) in, forces added to f (n*3, may be null), strain (9, may be null); terms: 5 + total.
int refcuda_compute(void* p, const double* pos, const double* box9, int newStep, double* f, double* strain,
                    double* terms) {
    try {
        double box[3][3];
        box3(box9, box);
        terms6(static_cast<pgmcuda::Engine*>(p)->compute(pos, box, newStep != 0, f, strain), terms);
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// Device positions (float4 xyz + w) in, forces added to the device 64-bit fixed-point buffer, on stream.
int refcuda_launch_device(void* p, const void* posq4, const double* box9, int newStep, long long* forceFixed,
                          int stride, double fixedScale, void* stream) {
    try {
        double box[3][3];
        box3(box9, box);
        static_cast<pgmcuda::Engine*>(p)->launchDevice(posq4, box, newStep != 0, forceFixed, stride, fixedScale,
                                                       stream);
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// 1: done; 0: the list was out of date (launch again); -1: error.
int refcuda_finish_device(void* p, double* terms) {
    try {
        pgmcuda::Terms t;
        const bool ok = static_cast<pgmcuda::Engine*>(p)->finishDevice(t);
        terms6(t, terms);
        return ok ? 1 : 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// The caller's stream waits on the GPU for the evaluation in flight.
int refcuda_wait_device(void* p, void* stream) {
    try {
        static_cast<pgmcuda::Engine*>(p)->waitDevice(stream);
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

int refcuda_iterations(void* p) { return static_cast<pgmcuda::Engine*>(p)->iterations(); }

long refcuda_list_builds(void* p) { return static_cast<pgmcuda::Engine*>(p)->listBuilds(); }

}  // extern "C"
