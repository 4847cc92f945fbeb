// CudaCalcTholeDipoleForceKernel (see CudaTholeDipoleKernels.h).
#include "CudaTholeDipoleKernels.h"

#include <string>

#include "openmm/OpenMMException.h"
#include "openmm/internal/ContextImpl.h"

using namespace TholeDipolePlugin;
using OpenMM::OpenMMException;
using OpenMM::Vec3;

namespace {
// Platform data in one of two shapes (openmm/internal/ContextImpl.h):
// host positions, forces and box vectors as vectors of Vec3 (the layout of
// OpenMM's ReferencePlatform::PlatformData, which
// ReferenceTholeDipoleKernels.cpp:45-68 reads), or the CUDA platform
// context's device buffers (posq, atom index, fixed-point forces).
bool onDevice(OpenMM::ContextImpl& context) {
    return *static_cast<const int*>(context.getPlatformData()) == OpenMM::kDevicePlatformData;
}
OpenMM::HostPlatformData& data(OpenMM::ContextImpl& context) {
    return *static_cast<OpenMM::HostPlatformData*>(context.getPlatformData());
}
OpenMM::DevicePlatformData& device(OpenMM::ContextImpl& context) {
    return *static_cast<OpenMM::DevicePlatformData*>(context.getPlatformData());
}
static_assert(sizeof(Vec3) == 3 * sizeof(double), "Vec3 must be three packed doubles");
}  // namespace

CudaCalcTholeDipoleForceKernel::CudaCalcTholeDipoleForceKernel(std::string name, const OpenMM::Platform& platform,
                                                               const OpenMM::System& system)
    : CalcTholeDipoleForceKernel(name, platform), system_(system) {}

CudaCalcTholeDipoleForceKernel::~CudaCalcTholeDipoleForceKernel() { tdp_destroy(handle_); }

void CudaCalcTholeDipoleForceKernel::check(int status) const {
    if (status != TDP_OK) throw OpenMMException(tdp_last_error(handle_));
}

// ReferenceCalcTholeDipoleKernel::initialize (ReferenceTholeDipoleKernels.cpp:83-158):
// flatten the force's parameters and covalent maps.
void CudaCalcTholeDipoleForceKernel::initialize(const OpenMM::System& system, const TholeDipoleForce& force) {
    int n = force.getNumParticles();
    numParticles_ = n;
    std::vector<double> q(n), dip(3 * n), pol(n), thole(n);
    std::vector<int32_t> type(n), z(n), x(n), y(n), off12(n + 1, 0), off13(n + 1, 0), c12, c13;
    for (int i = 0; i < n; i++) {
        std::vector<double> d;
        int t, az, ax, ay;
        force.getParticleParameters(i, q[i], d, pol[i], thole[i], t, az, ax, ay);
        dip[3 * i] = d[0];
        dip[3 * i + 1] = d[1];
        dip[3 * i + 2] = d[2];
        type[i] = t;
        z[i] = az;
        x[i] = ax;
        y[i] = ay;
        std::vector<std::vector<int> > maps;
        force.getCovalentMaps(i, maps);
        c12.insert(c12.end(), maps[TholeDipoleForce::Covalent12].begin(), maps[TholeDipoleForce::Covalent12].end());
        c13.insert(c13.end(), maps[TholeDipoleForce::Covalent13].begin(), maps[TholeDipoleForce::Covalent13].end());
        off12[i + 1] = (int32_t)c12.size();
        off13[i + 1] = (int32_t)c13.size();
    }
    const std::vector<double>& ex = force.getExtrapolationCoefficients();
    tdp_system_desc desc = {};
    desc.num_particles = n;
    desc.charges = q.data();
    desc.molecular_dipoles = dip.data();
    desc.polarizabilities = pol.data();
    desc.thole_damping = thole.data();
    desc.axis_types = type.data();
    desc.atom_z = z.data();
    desc.atom_x = x.data();
    desc.atom_y = y.data();
    desc.covalent12_offsets = off12.data();
    desc.covalent12_atoms = c12.data();
    desc.covalent13_offsets = off13.data();
    desc.covalent13_atoms = c13.data();
    desc.nonbonded_method = force.getNonbondedMethod();
    desc.polarization_type = force.getPolarizationType();
    desc.cutoff = force.getCutoffDistance();
    desc.ewald_error_tolerance = force.getEwaldErrorTolerance();
    int nx, ny, nz;
    force.getPMEParameters(desc.pme_alpha, nx, ny, nz);
    desc.pme_grid[0] = nx;
    desc.pme_grid[1] = ny;
    desc.pme_grid[2] = nz;
    // The reference copies the Mutual knobs only for Mutual polarization
    // (ReferenceTholeDipoleKernels.cpp:127-134); they are unused otherwise.
    desc.mutual_target_epsilon = force.getMutualInducedTargetEpsilon();
    desc.mutual_max_iterations = force.getMutualInducedMaxIterations();
    desc.num_extrapolation_coefficients = (int32_t)ex.size();
    desc.extrapolation_coefficients = ex.data();
    desc.precision = precision_;
    desc.solver = solver_;
    desc.flags = 0;
    tdp_destroy(handle_);
    handle_ = nullptr;
    if (tdp_create(&desc, &handle_) != TDP_OK) throw OpenMMException(tdp_last_error(nullptr));
    usePme_ = force.getNonbondedMethod() == TholeDipoleForce::PME;
}

void CudaCalcTholeDipoleForceKernel::syncBox(OpenMM::ContextImpl& context) {
    if (!usePme_) return;
    const Vec3* b = onDevice(context) ? device(context).periodicBoxVectors : data(context).periodicBoxVectors;
    double box9[9];
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) box9[3 * r + c] = b[r][c];
    check(tdp_set_box(handle_, box9));
}

const double* CudaCalcTholeDipoleForceKernel::positions(OpenMM::ContextImpl& context) {
    if (onDevice(context)) {
        // The queries run on the coordinates of the context's buffers: one
        // evaluation there (no forces added), after which NULL positions
        // select them.
        const OpenMM::DevicePlatformData& d = device(context);
        check(tdp_compute_openmm(handle_, d.posq, d.posqIsDouble, d.atomIndex, d.paddedNumAtoms, nullptr, nullptr, 0u));
        return nullptr;
    }
    std::vector<Vec3>& pos = *data(context).positions;
    if ((int)pos.size() != numParticles_) throw OpenMMException("TholeDipoleForce: wrong number of positions");
    return reinterpret_cast<const double*>(pos.data());
}

// execute (ReferenceTholeDipoleKernels.cpp:201-215): the forces are added into
// the context's force array and the energy is returned.
double CudaCalcTholeDipoleForceKernel::execute(OpenMM::ContextImpl& context, bool includeForces, bool includeEnergy) {
    syncBox(context);
    double energy = 0.0;
    uint32_t flags = TDP_COMPUTE_ENERGY | (includeForces ? TDP_COMPUTE_FORCES : 0u);
    if (onDevice(context)) {
        // The CUDA platform's buffers: posq in, fixed-point forces added.
        const OpenMM::DevicePlatformData& d = device(context);
        check(tdp_compute_openmm(handle_, d.posq, d.posqIsDouble, d.atomIndex, d.paddedNumAtoms, d.force, &energy,
                                 flags));
        (void)includeEnergy;
        return energy;
    }
    std::vector<Vec3>& forces = *data(context).forces;
    check(tdp_compute(handle_, positions(context), TDP_F64, 0, reinterpret_cast<double*>(forces.data()), TDP_F64,
                      &energy, flags));
    (void)includeEnergy;
    return energy;
}

// copyParametersToContext (ReferenceTholeDipoleKernels.cpp:317-339).
void CudaCalcTholeDipoleForceKernel::copyParametersToContext(OpenMM::ContextImpl& context,
                                                             const TholeDipoleForce& force) {
    int n = force.getNumParticles();
    if (n != numParticles_) throw OpenMMException("updateParametersInContext: The number of particles has changed");
    std::vector<double> q(n), dip(3 * n), pol(n), thole(n);
    std::vector<int32_t> type(n), z(n), x(n), y(n);
    for (int i = 0; i < n; i++) {
        std::vector<double> d;
        int t, az, ax, ay;
        force.getParticleParameters(i, q[i], d, pol[i], thole[i], t, az, ax, ay);
        for (int c = 0; c < 3; c++) dip[3 * i + c] = d[c];
        type[i] = t;
        z[i] = az;
        x[i] = ax;
        y[i] = ay;
    }
    check(tdp_update_params(handle_, n, q.data(), dip.data(), pol.data(), thole.data(), type.data(), z.data(),
                            x.data(), y.data()));
}

// getPMEParameters (ReferenceTholeDipoleKernels.cpp:341-348).
void CudaCalcTholeDipoleForceKernel::getPMEParameters(double& alpha, int& nx, int& ny, int& nz) const {
    int32_t gx, gy, gz;
    check(tdp_get_pme_parameters(handle_, &alpha, &gx, &gy, &gz));
    nx = gx;
    ny = gy;
    nz = gz;
}

void CudaCalcTholeDipoleForceKernel::dipoles(OpenMM::ContextImpl& context, int which, std::vector<Vec3>& out) {
    syncBox(context);
    out.resize(numParticles_);
    check(tdp_get_dipoles(handle_, which, positions(context), TDP_F64, 0, reinterpret_cast<double*>(out.data())));
}

void CudaCalcTholeDipoleForceKernel::getInducedDipoles(OpenMM::ContextImpl& context, std::vector<Vec3>& d) {
    dipoles(context, TDP_DIPOLES_INDUCED, d);
}

void CudaCalcTholeDipoleForceKernel::getLabFramePermanentDipoles(OpenMM::ContextImpl& context, std::vector<Vec3>& d) {
    dipoles(context, TDP_DIPOLES_LAB_PERMANENT, d);
}

void CudaCalcTholeDipoleForceKernel::getTotalDipoles(OpenMM::ContextImpl& context, std::vector<Vec3>& d) {
    dipoles(context, TDP_DIPOLES_TOTAL, d);
}

void CudaCalcTholeDipoleForceKernel::getElectrostaticPotential(OpenMM::ContextImpl& context,
                                                               const std::vector<Vec3>& grid,
                                                               std::vector<double>& out) {
    syncBox(context);
    out.resize(grid.size());
    check(tdp_get_potential(handle_, positions(context), TDP_F64, 0, reinterpret_cast<const double*>(grid.data()),
                            (int32_t)grid.size(), out.data()));
}

// getSystemMultipoleMoments (ReferenceTholeDipoleKernels.cpp:297-315): masses
// come from the System.
void CudaCalcTholeDipoleForceKernel::getSystemMultipoleMoments(OpenMM::ContextImpl& context,
                                                               std::vector<double>& out) {
    syncBox(context);
    const OpenMM::System& system = context.getSystem();
    std::vector<double> masses(system.getNumParticles());
    for (int i = 0; i < system.getNumParticles(); i++) masses[i] = system.getParticleMass(i);
    out.resize(13);
    check(tdp_get_moments(handle_, positions(context), TDP_F64, 0, masses.data(), out.data()));
}
