/* Stand-in for OpenMM's ContextImpl (see standin/openmm/Vec3.h).
 *
 * Platform data comes in the two shapes a TholeDipoleForce kernel meets:
 *  - HostPlatformData: host positions, forces and box vectors, the layout of
 *    OpenMM's ReferencePlatform::PlatformData (ReferenceTholeDipoleKernels.cpp:45-68);
 *  - DevicePlatformData: the buffers of the CUDA platform's CudaContext --
 *    posq (float4 or double4) in the context's atom order, the atom-index
 *    table, the padded atom count and the 64-bit fixed-point force
 *    accumulator, all device pointers.
 * Both start with the same tag, so a kernel can tell them apart. */
#ifndef TDP_STANDIN_OPENMM_CONTEXTIMPL_H_
#define TDP_STANDIN_OPENMM_CONTEXTIMPL_H_
#include <vector>
#include "openmm/KernelImpl.h"
#include "openmm/System.h"
#include "openmm/Vec3.h"
#include "openmm/internal/ForceImpl.h"
namespace OpenMM {
enum PlatformDataKind { kHostPlatformData = 0, kDevicePlatformData = 1 };
struct HostPlatformData {
    int kind = kHostPlatformData;
    std::vector<Vec3>* positions;
    std::vector<Vec3>* forces;
    Vec3* periodicBoxVectors;
};
struct DevicePlatformData {
    int kind = kDevicePlatformData;
    void* posq = nullptr;          // float4 / double4 per slot: x, y, z, q
    int posqIsDouble = 0;
    int* atomIndex = nullptr;      // slot -> atom
    int paddedNumAtoms = 0;
    long long* force = nullptr;    // 3 * paddedNumAtoms, component-major, 2^32 units
    Vec3 periodicBoxVectors[3];
};
class ContextImpl {
public:
    ContextImpl(const System& system, Platform& platform) : system(system), platform(platform) {
        positions.resize(system.getNumParticles());
        forces.resize(system.getNumParticles());
        system.getDefaultPeriodicBoxVectors(box[0], box[1], box[2]);
        data.positions = &positions;
        data.forces = &forces;
        data.periodicBoxVectors = box;
    }
    ~ContextImpl() {
        for (ForceImpl* f : impls) delete f;
    }
    const System& getSystem() const { return system; }
    Platform& getPlatform() { return platform; }
    void* getPlatformData() { return device ? (void*)device : (void*)&data; }
    // Hands the kernels CUDA-context buffers instead of host vectors (NULL: host again).
    void setDevicePlatformData(DevicePlatformData* d) { device = d; }
    // Creates and initializes every Force's implementation (Context creation).
    void initialize() {
        for (int i = 0; i < system.getNumForces(); i++) impls.push_back(system.getForce(i).createImpl());
        for (ForceImpl* f : impls) f->initialize(*this);
    }
    double calcForcesAndEnergy(bool includeForces, bool includeEnergy, int groups) {
        for (Vec3& f : forces) f = Vec3();
        double e = 0.0;
        for (ForceImpl* f : impls) e += f->calcForcesAndEnergy(*this, includeForces, includeEnergy, groups);
        return e;
    }
    ForceImpl& getForceImpl(const Force& force) {
        for (ForceImpl* f : impls)
            if (&f->getOwner() == &force) return *f;
        throw OpenMMException("getImplInContext: the Force is not part of this Context");
    }
    void systemChanged() { changes++; }
    int systemChanges() const { return changes; }
    std::vector<Vec3> positions, forces;
    Vec3 box[3];

private:
    const System& system;
    Platform& platform;
    HostPlatformData data;
    DevicePlatformData* device = nullptr;
    std::vector<ForceImpl*> impls;
    int changes = 0;
};
}  // namespace OpenMM
#endif
