/* Stand-in for OpenMM's Force base class (see standin/openmm/Vec3.h). */
#ifndef TDP_STANDIN_OPENMM_FORCE_H_
#define TDP_STANDIN_OPENMM_FORCE_H_
#ifndef OPENMM_EXPORT
#define OPENMM_EXPORT __attribute__((visibility("default")))
#endif
namespace OpenMM {
class Context;
class ContextImpl;
class ForceImpl;
class Force {
public:
    virtual ~Force() {}
    int getForceGroup() const { return group; }
    void setForceGroup(int g) { group = g; }
    virtual bool usesPeriodicBoundaryConditions() const { return false; }
private:
    int group = 0;
};
}  // namespace OpenMM
#endif
