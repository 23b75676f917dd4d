// OpenMM CUDA-platform kernel of PGMForce over the pgm_b200 engine; see PgmB200OpenMMKernel.h.
// Mirrors the behaviour of the reference plugin's CudaCalcPGMForceKernel (CudaPGMKernels.cpp:97-188 of
// larryhuang98/pGM-MD) and its factory (CudaPGMKernelFactory.cpp:18-42) through the C ABI.

#include "PgmB200OpenMMKernel.h"

#include "internal/PGMForceImpl.h"
#include "openmm/KernelFactory.h"
#include "openmm/OpenMMException.h"
#include "openmm/common/ComputeForceInfo.h"
#include "openmm/common/ContextSelector.h"
#include "openmm/cuda/CudaPlatform.h"
#include "openmm/internal/ContextImpl.h"

#include <string>

using namespace OpenMM;

namespace PgmB200OpenMM {

// Which particles and covalent groups OpenMM may treat as interchangeable when it reorders molecules.
class PgmB200CalcPGMForceKernel::SameParticles : public ComputeForceInfo {
public:
    explicit SameParticles(const PGMPlugin::PGMForce& f) : f(f) {}
    bool areParticlesIdentical(int a, int b) override {
        double qa, ra, pa, qb, rb, pb;
        f.getParticleParameters(a, qa, ra, pa);
        f.getParticleParameters(b, qb, rb, pb);
        return qa == qb && ra == rb && pa == pb;
    }
    int getNumParticleGroups() override { return f.getNumCovalentDipoles(); }
    void getParticlesInGroup(int g, std::vector<int>& members) override {
        int i, j;
        double c;
        f.getCovalentDipoleParameters(g, i, j, c);
        members = {i, j};
    }
    bool areGroupsIdentical(int g1, int g2) override {
        int i, j;
        double c1, c2;
        f.getCovalentDipoleParameters(g1, i, j, c1);
        f.getCovalentDipoleParameters(g2, i, j, c2);
        return c1 == c2;
    }

private:
    const PGMPlugin::PGMForce& f;
};

class PgmB200CalcPGMForceKernel::OrderChanged : public ComputeContext::ReorderListener {
public:
    explicit OrderChanged(PgmB200CalcPGMForceKernel& k) : k(k) {}
    void execute() override { k.orderStale = true; }

private:
    PgmB200CalcPGMForceKernel& k;
};

// After every force was launched: wait for the engine's evaluation (it ran on OpenMM's stream) and return
// its energy; a stale pair list invalidates the step's forces, so OpenMM computes the step again.
class PgmB200CalcPGMForceKernel::Pending : public ComputeContext::ForcePostComputation {
public:
    explicit Pending(PgmB200CalcPGMForceKernel& k) : k(k) {}
    double computeForceAndEnergy(bool includeForces, bool includeEnergy, int groups) override {
        if (!k.inFlight)
            return 0.0;
        return k.collect(includeEnergy);
    }

private:
    PgmB200CalcPGMForceKernel& k;
};

void PgmB200CalcPGMForceKernel::check(int status, const char* what) {
    if (status != PGM_OK)
        throw OpenMMException(std::string("pgm_b200: ") + what + ": " + pgm_last_error());
}

PgmB200CalcPGMForceKernel::PgmB200CalcPGMForceKernel(std::string name, const Platform& platform, CudaContext& cu,
                                                     const System& system)
    : CalcPGMForceKernel(name, platform), cu(cu) {}

PgmB200CalcPGMForceKernel::~PgmB200CalcPGMForceKernel() {
    if (engine) {
        ContextSelector selector(cu);
        pgm_engine_destroy(engine);
    }
}

void PgmB200CalcPGMForceKernel::initialize(const System& system, const PGMPlugin::PGMForce& force) {
    if (force.getNonbondedMethod() != PGMPlugin::PGMForce::PME)
        throw OpenMMException("pgm_b200: the engine evaluates the periodic (PME) form of PGMForce only");
    ContextSelector selector(cu);
    natoms = force.getNumParticles();
    group = force.getForceGroup();
    mutual = force.getPolarization() == PGMPlugin::PGMForce::Mutual;
    PGMPlugin::PGMForceImpl::calcPMEParameters(system, force, ewald, gridDims[0], gridDims[1], gridDims[2]);
    pgm_settings st;
    pgm_settings_default(&st);
    st.cutoff = force.getCutoffDistance();
    st.beta = ewald;
    for (int a = 0; a < 3; a++)
        st.grid[a] = gridDims[a];
    st.order = force.getPMEOrder();
    st.tol = force.getInducedDipoleTolerance();
    st.max_iter = force.getMaxInducedDipoleIterations();
    st.peek = force.getPeekCoefficient();
    st.predictor = (int) force.getPredictor();   // none, mu3, mu4 in both numberings
    st.ke = force.getCoulombConstant();
    st.device = -1;                               // OpenMM's context, current through the selector
    st.precision = cu.getUseDoublePrecision() ? PGM_PRECISION_FP64 : PGM_PRECISION_MIXED;
    check(pgm_engine_create(&st, &engine), "create");
    readParameters(force);
    cu.addForce(new SameParticles(force));
    cu.addReorderListener(new OrderChanged(*this));
    cu.addPostComputation(new Pending(*this));
}

void PgmB200CalcPGMForceKernel::readParameters(const PGMPlugin::PGMForce& force) {
    if (force.getNumParticles() != natoms)
        throw OpenMMException("updateParametersInContext: the number of particles has changed");
    charge.resize(natoms);
    gaussRadius.resize(natoms);
    polarizability.resize(natoms);
    for (int i = 0; i < natoms; i++)
        force.getParticleParameters(i, charge[i], gaussRadius[i], polarizability[i]);
    std::vector<int> atoms, partners;
    std::vector<double> strength;
    for (int m = 0; m < force.getNumCovalentDipoles(); m++) {
        int i, j;
        double c;
        force.getCovalentDipoleParameters(m, i, j, c);
        atoms.push_back(i);
        partners.push_back(j);
        strength.push_back(c);
    }
    if (!dipoleAtom.empty() && (atoms != dipoleAtom || partners != dipolePartner))
        throw OpenMMException("updateParametersInContext: the covalent dipoles' atoms have changed");
    dipoleAtom = atoms;
    dipolePartner = partners;
    dipoleStrength = strength;
    orderStale = true;
}

// The engine's atoms in OpenMM's local order (local i holds particle getAtomIndex()[i]); the particle index
// keys the predictor history, so the history survives reorderings.
void PgmB200CalcPGMForceKernel::pushAtoms() {
    const std::vector<int>& particleOf = cu.getAtomIndex();
    std::vector<double> q(natoms), R(natoms), al(natoms);
    std::vector<int> localOf(natoms);
    for (int i = 0; i < natoms; i++) {
        const int a = particleOf[i];
        q[i] = charge[a];
        R[i] = gaussRadius[a];
        al[i] = mutual ? polarizability[a] : 0.0;
        localOf[a] = i;
    }
    check(pgm_engine_set_atoms(engine, natoms, q.data(), R.data(), al.data(), particleOf.data(), natoms),
          "set_atoms");
    std::vector<int> ca(dipoleAtom.size()), cp(dipoleAtom.size());
    for (size_t m = 0; m < dipoleAtom.size(); m++) {
        ca[m] = localOf[dipoleAtom[m]];
        cp[m] = localOf[dipolePartner[m]];
    }
    check(pgm_engine_set_covalent(engine, (int) ca.size(), ca.data(), cp.data(), dipoleStrength.data()),
          "set_covalent");
    orderStale = false;
}

double PgmB200CalcPGMForceKernel::execute(ContextImpl& context, bool includeForces, bool includeEnergy) {
    ContextSelector selector(cu);
    if (orderStale)
        pushAtoms();
    Vec3 a, b, c;
    cu.getPeriodicBoxVectors(a, b, c);
    const double box[9] = {a[0], a[1], a[2], b[0], b[1], b[2], c[0], c[1], c[2]};
    const long long step = cu.getStepCount();
    const int newStep = step != previousStep ? 1 : 0;   // a repeat of the same step keeps the history
    previousStep = step;
    check(pgm_engine_launch_device(engine, (const void*) cu.getPosq().getDevicePointer(), box, newStep,
                                   (long long*) cu.getLongForceBuffer().getDevicePointer(),
                                   cu.getPaddedNumAtoms(), (double) 0x100000000LL,
                                   (void*) cu.getCurrentStream()),
          "launch_device");
    inFlight = true;
    wantEnergy = includeEnergy;
    return 0.0;   // the energy comes from the post-computation
}

double PgmB200CalcPGMForceKernel::collect(bool includeEnergy) {
    ContextSelector selector(cu);
    inFlight = false;
    pgm_terms t;
    int valid = 0;
    check(pgm_engine_finish_device(engine, &t, &valid), "finish_device");
    if (!valid) {
        cu.setForcesValid(false);   // the list was grown or rebuilt: OpenMM repeats the step
        return 0.0;
    }
    haveResult = true;
    return (includeEnergy || wantEnergy) ? t.direct + t.reciprocal + t.self + t.background + t.polarization : 0.0;
}

void PgmB200CalcPGMForceKernel::getInducedDipoles(ContextImpl& context, std::vector<Vec3>& dipoles) {
    if (!haveResult)
        context.calcForcesAndEnergy(false, true, 1 << group);
    ContextSelector selector(cu);
    std::vector<double> mu(3 * (size_t) natoms);
    check(pgm_engine_induced_dipoles(engine, mu.data()), "induced_dipoles");
    const std::vector<int>& particleOf = cu.getAtomIndex();
    dipoles.resize(natoms);
    for (int i = 0; i < natoms; i++)
        dipoles[particleOf[i]] = Vec3(mu[3 * i], mu[3 * i + 1], mu[3 * i + 2]);
}

void PgmB200CalcPGMForceKernel::getPermanentDipoles(ContextImpl& context, std::vector<Vec3>& dipoles) {
    context.calcForcesAndEnergy(false, true, 1 << group);   // at the current positions
    ContextSelector selector(cu);
    std::vector<double> p(3 * (size_t) natoms);
    check(pgm_engine_permanent_dipoles(engine, p.data()), "permanent_dipoles");
    const std::vector<int>& particleOf = cu.getAtomIndex();
    dipoles.resize(natoms);
    for (int i = 0; i < natoms; i++)
        dipoles[particleOf[i]] = Vec3(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
}

int PgmB200CalcPGMForceKernel::getInducedDipoleIterations() {
    ContextSelector selector(cu);
    return pgm_engine_iterations(engine);
}

void PgmB200CalcPGMForceKernel::copyParametersToContext(ContextImpl& context, const PGMPlugin::PGMForce& force) {
    readParameters(force);
    cu.invalidateMolecules(new SameParticles(force), true, true);
    ContextSelector selector(cu);
    check(pgm_engine_reset_history(engine), "reset_history");
}

void PgmB200CalcPGMForceKernel::getPMEParameters(double& alpha, int& nx, int& ny, int& nz) const {
    alpha = ewald;
    nx = gridDims[0];
    ny = gridDims[1];
    nz = gridDims[2];
}

// Creates the CUDA platform's PGMForce kernel; GVDWForce stays with the plugin's own factory.
class PgmB200KernelFactory : public KernelFactory {
public:
    KernelImpl* createKernelImpl(std::string name, const Platform& platform, ContextImpl& context) const override {
        CudaContext& cu = *static_cast<CudaPlatform::PlatformData*>(context.getPlatformData())->contexts[0];
        if (name == PGMPlugin::CalcPGMForceKernel::Name())
            return new PgmB200CalcPGMForceKernel(name, platform, cu, context.getSystem());
        throw OpenMMException("pgm_b200: no kernel named '" + name + "'");
    }
};

}  // namespace PgmB200OpenMM

// Loaded after the reference plugin: the CUDA platform's PGMForce kernel becomes this one.
extern "C" OPENMM_EXPORT void registerKernelFactories() {
    try {
        Platform& cuda = Platform::getPlatformByName("CUDA");
        cuda.registerKernelFactory(PGMPlugin::CalcPGMForceKernel::Name(), new PgmB200OpenMM::PgmB200KernelFactory());
    } catch (const std::exception&) {
        // no CUDA platform in this OpenMM build
    }
}

extern "C" OPENMM_EXPORT void registerPlatforms() {}
