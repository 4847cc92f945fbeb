/* Minimal stand-in for OpenMM's Force base class: only the declarations that
 * the reference plugin's TholeDipoleForce.h needs in order to be parsed (the
 * enums it defines are all the oracle uses).  Test infrastructure only. */
#ifndef TDP_SHIM_OPENMM_FORCE_H_
#define TDP_SHIM_OPENMM_FORCE_H_
#ifndef OPENMM_EXPORT
#define OPENMM_EXPORT
#endif
namespace OpenMM {
class Context;
class ContextImpl;
class ForceImpl;
class Force {
public:
    Force() : forceGroup(0) {}
    virtual ~Force() {}
    int getForceGroup() const { return forceGroup; }
    void setForceGroup(int group) { forceGroup = group; }
    virtual bool usesPeriodicBoundaryConditions() const { return false; }
protected:
    virtual ForceImpl* createImpl() const = 0;
    ForceImpl& getImplInContext(Context& context);
    const ForceImpl& getImplInContext(const Context& context) const;
    ContextImpl& getContextImpl(Context& context);
private:
    int forceGroup;
};
}  // namespace OpenMM
#endif
