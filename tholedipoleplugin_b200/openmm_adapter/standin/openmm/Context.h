/* Stand-in for OpenMM's Context (see standin/openmm/Vec3.h): it creates a
 * ContextImpl, which creates and initializes every Force's ForceImpl on the
 * given Platform -- the path on which a plugin's ForceImpl validates the
 * Force and creates its kernel by name.  Positions go in and energy and
 * forces come out through the ContextImpl (OpenMM does that through State). */
#ifndef TDP_STANDIN_OPENMM_CONTEXT_H_
#define TDP_STANDIN_OPENMM_CONTEXT_H_
#include <vector>
#include "openmm/KernelImpl.h"
#include "openmm/System.h"
#include "openmm/Vec3.h"
namespace OpenMM {
class ContextImpl;
class Context {
public:
    Context(const System& system, Platform& platform);
    ~Context();
    ContextImpl& getImpl() { return *impl; }
    const ContextImpl& getImpl() const { return *impl; }
    void setPositions(const std::vector<Vec3>& positions);
    // Sum over the System's Forces (ContextImpl::calcForcesAndEnergy); forces
    // are those of the last call.
    double calcForcesAndEnergy(bool includeForces = true, bool includeEnergy = true, int groups = -1);
    const std::vector<Vec3>& getForces() const;

private:
    ContextImpl* impl;
};
}  // namespace OpenMM
#endif
