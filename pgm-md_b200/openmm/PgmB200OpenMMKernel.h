// OpenMM CUDA-platform kernel of PGMForce over the pgm_b200 engine (C ABI of include/pgm_b200.h).
//
// A drop-in for the reference plugin's CUDA kernel (openmm/platforms/cuda/src/CudaPGMKernels.{h,cpp} and
// CudaPGMKernelFactory.cpp of larryhuang98/pGM-MD): the same kernel name (CalcPGMForceKernel::Name()), the same
// PGMForce parameters, the same use of OpenMM's CUDA context (its posq array, its 64-bit fixed-point force
// buffer, its stream, its atom reordering), and the same repeat of a step whose pair list turned out stale
// (setForcesValid(false)).  Built only against an OpenMM SDK and the reference plugin's API headers
// (Makefile beside this file, OPENMM_DIR and PGM_PLUGIN_DIR).
#pragma once

#include "PGMKernels.h"
#include "openmm/cuda/CudaContext.h"
#include "pgm_b200.h"

#include <memory>
#include <vector>

namespace PgmB200OpenMM {

class PgmB200CalcPGMForceKernel : public PGMPlugin::CalcPGMForceKernel {
public:
    PgmB200CalcPGMForceKernel(std::string name, const OpenMM::Platform& platform, OpenMM::CudaContext& cu,
                              const OpenMM::System& system);
    ~PgmB200CalcPGMForceKernel();
    void initialize(const OpenMM::System& system, const PGMPlugin::PGMForce& force) override;
    double execute(OpenMM::ContextImpl& context, bool includeForces, bool includeEnergy) override;
    void getInducedDipoles(OpenMM::ContextImpl& context, std::vector<OpenMM::Vec3>& dipoles) override;
    void getPermanentDipoles(OpenMM::ContextImpl& context, std::vector<OpenMM::Vec3>& dipoles) override;
    int getInducedDipoleIterations() override;
    void copyParametersToContext(OpenMM::ContextImpl& context, const PGMPlugin::PGMForce& force) override;
    void getPMEParameters(double& alpha, int& nx, int& ny, int& nz) const override;

private:
    class Pending;         // post-computation: waits for the engine and collects its energy
    class OrderChanged;    // reorder listener: the engine's atoms follow OpenMM's local order
    class SameParticles;   // force info: particles and covalent groups OpenMM may exchange
    friend class Pending;
    friend class OrderChanged;

    void readParameters(const PGMPlugin::PGMForce& force);
    void pushAtoms();
    double collect(bool includeEnergy);
    static void check(int status, const char* what);

    OpenMM::CudaContext& cu;
    pgm_engine* engine = nullptr;
    int natoms = 0, group = 0, gridDims[3] = {0, 0, 0};
    double ewald = 0.0;
    bool mutual = true;
    std::vector<double> charge, gaussRadius, polarizability, dipoleStrength;
    std::vector<int> dipoleAtom, dipolePartner;
    bool orderStale = true, inFlight = false, wantEnergy = false, haveResult = false;
    long long previousStep = -1;
};

}  // namespace PgmB200OpenMM
