/* Stand-in for OpenMM's ContextImpl (see standin/openmm/Vec3.h).  Its platform
 * data has the shape of OpenMM's ReferencePlatform::PlatformData: host
 * positions, forces and periodic box vectors. */
#ifndef TDP_STANDIN_OPENMM_CONTEXTIMPL_H_
#define TDP_STANDIN_OPENMM_CONTEXTIMPL_H_
#include <vector>
#include "openmm/KernelImpl.h"
#include "openmm/System.h"
#include "openmm/Vec3.h"
namespace OpenMM {
struct HostPlatformData {
    std::vector<Vec3>* positions;
    std::vector<Vec3>* forces;
    Vec3* periodicBoxVectors;
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
    const System& getSystem() const { return system; }
    Platform& getPlatform() { return platform; }
    void* getPlatformData() { return &data; }
    std::vector<Vec3> positions, forces;
    Vec3 box[3];
private:
    const System& system;
    Platform& platform;
    HostPlatformData data;
};
}  // namespace OpenMM
#endif
