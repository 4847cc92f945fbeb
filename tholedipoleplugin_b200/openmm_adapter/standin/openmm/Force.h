/* Stand-in for OpenMM's Force base class (see standin/openmm/Vec3.h): force
 * group, name, and the protected hooks a plugin's Force uses to reach its
 * ForceImpl in a Context (createImpl, getImplInContext, getContextImpl). */
#ifndef TDP_STANDIN_OPENMM_FORCE_H_
#define TDP_STANDIN_OPENMM_FORCE_H_
#include <string>
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
    const std::string& getName() const { return name; }
    void setName(const std::string& n) { name = n; }
    virtual bool usesPeriodicBoundaryConditions() const { return false; }

protected:
    friend class ContextImpl;
    // Restated plugin Forces that are never placed in a Context need not
    // override it; OpenMM's own declaration is pure virtual.
    virtual ForceImpl* createImpl() const;
    ForceImpl& getImplInContext(Context& context);
    const ForceImpl& getImplInContext(const Context& context) const;
    ContextImpl& getContextImpl(Context& context);

private:
    int group = 0;
    std::string name;
};
}  // namespace OpenMM
#endif
