// A pgmcore-style caller of the GPU engine (pgm_core_b200.h): reads a system, evaluates it the way the
// reference's CPU tests drive pgmcore::Engine (compute with forces, terms(), strainDerivative(),
// inducedDipoles(); a second call at the same positions with the same history key; field() of the charges
// alone), and writes what it got.  Built and run by tests/test_capi.py (build) and tests/test_gpu_core_api.py.
//
// input (binary, little endian): int n, int ncov, int grid[3], int order, int precision;
//   double cutoff, beta, tol, ke; double box[9]; double pos[3n], q[n], radius[n], alpha[n];
//   int covAtom[ncov], covPartner[ncov]; double covStrength[ncov]
// output (binary): double energy, terms[5], strain[9], forces[3n], mu[3n], energy2, field[3n]; int iterations,
//   iterations2
#include "pgm_core_b200.h"

#include <cstdio>
#include <vector>

template <class T> static bool rd(FILE* f, T* p, size_t k) { return fread(p, sizeof(T), k, f) == k; }
template <class T> static void wr(FILE* f, const T* p, size_t k) { fwrite(p, sizeof(T), k, f); }

int main(int argc, char** argv) {
    if (argc != 3) {
        fprintf(stderr, "usage: core_engine_check <input> <output>\n");
        return 2;
    }
    FILE* in = fopen(argv[1], "rb");
    if (!in)
        return 2;
    int hdr[7];
    double par[4], box[9];
    if (!rd(in, hdr, 7) || !rd(in, par, 4) || !rd(in, box, 9))
        return 3;
    const int n = hdr[0], ncov = hdr[1];
    pgmb200::CoreSettings s;
    for (int a = 0; a < 3; a++)
        s.grid[a] = hdr[2 + a];
    s.order = hdr[5];
    s.precision = hdr[6];
    s.cutoff = par[0];
    s.beta = par[1];
    s.tol = par[2];
    s.ke = par[3];
    s.maxIter = 1000;
    s.peek = 0.0;
    s.predictor = 0;
    std::vector<double> pos(3 * (size_t) n);
    pgmb200::CoreTopology top;
    top.q.resize(n);
    top.radius.resize(n);
    top.alpha.resize(n);
    top.covAtom.resize(ncov);
    top.covPartner.resize(ncov);
    top.covStrength.resize(ncov);
    if (!rd(in, pos.data(), pos.size()) || !rd(in, top.q.data(), n) || !rd(in, top.radius.data(), n) ||
        !rd(in, top.alpha.data(), n) || !rd(in, top.covAtom.data(), ncov) || !rd(in, top.covPartner.data(), ncov) ||
        !rd(in, top.covStrength.data(), ncov))
        return 3;
    fclose(in);
    std::vector<pgmb200::V3> p(n), F(n, pgmb200::V3{0, 0, 0});
    for (int i = 0; i < n; i++)
        p[i] = pgmb200::V3{pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    pgmb200::V3 B[3];
    for (int r = 0; r < 3; r++)
        B[r] = pgmb200::V3{box[3 * r], box[3 * r + 1], box[3 * r + 2]};
    try {
        pgmb200::CoreEngine eng(top, s);
        eng.setHistoryKey(7);
        const double e = eng.compute(p, B, &F);
        const int it = eng.iterations();
        const pgmb200::CoreTerms t = eng.terms();
        const std::array<double, 9> S = eng.strainDerivative();
        const std::vector<pgmb200::V3> mu = eng.inducedDipoles();
        const double e2 = eng.compute(p, B, nullptr);   // same key: the stored solution, the same energy
        const int it2 = eng.iterations();
        const std::vector<pgmb200::V3> E = eng.field(top.q, std::vector<pgmb200::V3>(n, pgmb200::V3{0, 0, 0}));
        FILE* out = fopen(argv[2], "wb");
        if (!out)
            return 2;
        const double terms[5] = {t.direct, t.reciprocal, t.self, t.background, t.polarization};
        wr(out, &e, 1);
        wr(out, terms, 5);
        wr(out, S.data(), 9);
        for (int i = 0; i < n; i++)
            wr(out, F[i].data(), 3);
        for (int i = 0; i < n; i++)
            wr(out, mu[i].data(), 3);
        wr(out, &e2, 1);
        for (int i = 0; i < n; i++)
            wr(out, E[i].data(), 3);
        wr(out, &it, 1);
        wr(out, &it2, 1);
        fclose(out);
    } catch (const std::exception& ex) {
        fprintf(stderr, "core_engine_check: %s\n", ex.what());
        return 4;
    }
    return 0;
}
