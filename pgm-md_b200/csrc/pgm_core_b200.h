// The FP64-oracle-shaped C++ surface: the methods of the reference CPU engine pgmcore::Engine
// (core/pgm_core.h:47-115 of larryhuang98/pGM-MD) over the pgm_b200 GPU engine, for callers written against
// pgmcore (GROMACS's G3 host code, the reference's own tests).  Header-only; link libpgm_b200.so.
//
//   pgmcore                              here
//   Engine(Topology, Settings)           CoreEngine(Topology, CoreSettings): periodic systems only (the engine
//                                        evaluates the PME form; a non-periodic setting is an invalid_argument)
//   compute(pos, box, forces*)           the energy; forces added to *forces; terms, strain, dipoles kept
//   setHistoryKey(key)                   the same rule: one solution per key; without a key, a call at the
//                                        positions of the previous call reuses its solution (new_step false)
//   terms(), strainDerivative(), permanentDipoles(), inducedDipoles(), iterations(), residual()
//   setTopology(top)                     new parameters of the same atoms; the predictor history is kept
//   resetHistory(), field(q, d), setGeometry(pos, box)
#pragma once

#include "pgm_engine.h"

#include <array>
#include <memory>
#include <stdexcept>
#include <vector>

namespace pgmb200 {

typedef std::array<double, 3> V3;

// pgmcore::Settings (core/pgm_core.h:22-34) with the GPU engine's precision and device.
struct CoreSettings {
    bool periodic = true;
    double cutoff = 0.9;
    double beta = 0.0;
    int grid[3] = {0, 0, 0};
    int order = 6;
    bool polarizable = true;
    double tol = 1e-5;
    int maxIter = 100;
    double peek = 0.65;
    int predictor = 2;
    double ke = 138.935456;
    int precision = 0;   // 0 FP64 (the oracle's arithmetic), 1 mixed
    int device = 0;
};

// pgmcore::Topology (core/pgm_core.h:36-40).
struct CoreTopology {
    std::vector<double> q, radius, alpha;
    std::vector<int> covAtom, covPartner;
    std::vector<double> covStrength;
};

// pgmcore::EnergyTerms (core/pgm_core.h:42-45).
struct CoreTerms {
    double direct = 0, reciprocal = 0, self = 0, background = 0, polarization = 0;
    double total() const { return direct + reciprocal + self + background + polarization; }
};

class CoreEngine {
public:
    CoreEngine(const CoreTopology& top, const CoreSettings& s) : set(s) {
        if (!s.periodic)
            throw std::invalid_argument("pgmcore: the GPU engine evaluates periodic (PME) systems only");
        Settings g;
        g.cutoff = s.cutoff;
        g.beta = s.beta;
        for (int a = 0; a < 3; a++)
            g.grid[a] = s.grid[a];
        g.order = s.order;
        g.tol = s.tol;
        g.maxIter = s.maxIter;
        g.peek = s.peek;
        g.predictor = s.predictor;
        g.ke = s.ke;
        g.device = s.device;
        g.precision = s.precision;
        g.polarizable = s.polarizable ? 1 : 0;
        eng.reset(new Engine(g));
        setTopology(top);
    }

    double compute(const std::vector<V3>& pos, const V3 box[3], std::vector<V3>* forces) {
        if ((int) pos.size() != n)
            throw std::invalid_argument("pgmcore: positions do not match the topology");
        setGeometry(pos, box);
        // the history rule of pgmcore::Engine::setHistoryKey: a new solution per key, or per new positions
        bool newStep;
        if (historyKey >= 0)
            newStep = historyKey != lastKey;
        else
            newStep = !(havePos && flat == lastFlat);
        lastKey = historyKey;
        lastFlat = flat;
        havePos = true;
        std::vector<double> f(forces ? 3 * (size_t) n : 0, 0.0);
        double st[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        const Terms t = eng->compute(flat.data(), hbox, newStep, forces ? f.data() : nullptr, forces ? st : nullptr);
        last.direct = t.direct;
        last.reciprocal = t.reciprocal;
        last.self = t.self;
        last.background = t.background;
        last.polarization = t.polarization;
        if (forces) {
            if ((int) forces->size() != n)
                forces->assign(n, V3{0, 0, 0});
            for (int i = 0; i < n; i++)
                for (int a = 0; a < 3; a++)
                    (*forces)[i][a] += f[3 * i + a];
            for (int k = 0; k < 9; k++)
                strain[k] = st[k];
        }
        std::vector<double> m(3 * (size_t) n);
        eng->inducedDipoles(m.data());
        toV3(m, mu);
        eng->permanentDipoles(m.data());
        toV3(m, perm);
        return last.total();
    }

    void setHistoryKey(long long key) { historyKey = key; }
    const std::vector<V3>& permanentDipoles() const { return perm; }
    const std::vector<V3>& inducedDipoles() const { return mu; }
    int iterations() const { return eng->iterations(); }
    double residual() const { return eng->residual(); }
    const CoreTerms& terms() const { return last; }
    const std::array<double, 9>& strainDerivative() const { return strain; }

    void setTopology(const CoreTopology& top) {
        const int m = (int) top.q.size();
        if ((int) top.radius.size() != m || (int) top.alpha.size() != m || top.covAtom.size() != top.covPartner.size() ||
            top.covAtom.size() != top.covStrength.size())
            throw std::invalid_argument("pgmcore: topology arrays of different lengths");
        if (n && m != n)
            throw std::invalid_argument("pgmcore: setTopology keeps the atoms (same count)");
        n = m;
        std::vector<double> al(top.alpha);
        if (!set.polarizable)
            al.assign(n, 0.0);
        // setAtoms renews the engine's geometry; the history is kept (global index = the atom itself)
        std::vector<unsigned char> hist;
        if (configured) {
            hist.resize((size_t) eng->historySize());
            eng->getHistory(hist.data());
        }
        eng->setAtoms(n, top.q.data(), top.radius.data(), al.data(), nullptr, n);
        eng->setCovalent((int) top.covAtom.size(), top.covAtom.data(), top.covPartner.data(), top.covStrength.data());
        if (configured)
            eng->setHistory(hist.data());
        configured = true;
    }

    void resetHistory() {
        eng->resetHistory();
        havePos = false;
    }

    // Field [e/nm^2] of charges q and dipoles d at every atom (direct + reciprocal + self) at the geometry of
    // the last setGeometry / compute.
    std::vector<V3> field(const std::vector<double>& q, const std::vector<V3>& d) {
        if (!haveGeometry)
            throw std::logic_error("pgmcore: field before setGeometry or compute");
        std::vector<double> dd(3 * (size_t) n), E(3 * (size_t) n);
        for (int i = 0; i < n; i++)
            for (int a = 0; a < 3; a++)
                dd[3 * i + a] = d[i][a];
        eng->field(flat.data(), hbox, q.data(), dd.data(), E.data());
        std::vector<V3> out;
        toV3(E, out);
        return out;
    }

    void setGeometry(const std::vector<V3>& pos, const V3 box[3]) {
        flat.resize(3 * pos.size());
        for (size_t i = 0; i < pos.size(); i++)
            for (int a = 0; a < 3; a++)
                flat[3 * i + a] = pos[i][a];
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++)
                hbox[r][c] = box[r][c];
        haveGeometry = true;
    }

    Engine& gpu() { return *eng; }

private:
    static void toV3(const std::vector<double>& v, std::vector<V3>& out) {
        out.resize(v.size() / 3);
        for (size_t i = 0; i < out.size(); i++)
            out[i] = V3{v[3 * i], v[3 * i + 1], v[3 * i + 2]};
    }

    CoreSettings set;
    std::unique_ptr<Engine> eng;
    int n = 0;
    bool configured = false, havePos = false, haveGeometry = false;
    long long historyKey = -1, lastKey = -1;
    std::vector<double> flat, lastFlat;
    double hbox[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    CoreTerms last;
    std::array<double, 9> strain{};
    std::vector<V3> perm, mu;
};

}  // namespace pgmb200
