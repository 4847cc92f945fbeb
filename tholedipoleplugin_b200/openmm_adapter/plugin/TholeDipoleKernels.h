/* CalcTholeDipoleForceKernel: the abstract kernel interface through which the
 * plugin's TholeDipoleForceImpl drives a platform.  Declared with the same
 * name, kernel name string and virtual methods as aehogan/tholedipoleplugin
 * openmmapi/include/TholeDipoleKernels.h:46-122, so that a kernel implementing
 * it here also implements it in the plugin. */
#ifndef TDP_PLUGIN_THOLEDIPOLEKERNELS_H_
#define TDP_PLUGIN_THOLEDIPOLEKERNELS_H_
#include <string>
#include <vector>
#include "TholeDipoleForce.h"
#include "openmm/KernelImpl.h"
#include "openmm/System.h"

namespace OpenMM {
class ContextImpl;
}

namespace TholeDipolePlugin {

class CalcTholeDipoleForceKernel : public OpenMM::KernelImpl {
public:
    static std::string Name() { return "CalcTholeDipoleForce"; }
    CalcTholeDipoleForceKernel(std::string name, const OpenMM::Platform& platform) : OpenMM::KernelImpl(name, platform) {}
    virtual void initialize(const OpenMM::System& system, const TholeDipoleForce& force) = 0;
    virtual double execute(OpenMM::ContextImpl& context, bool includeForces, bool includeEnergy) = 0;
    virtual void copyParametersToContext(OpenMM::ContextImpl& context, const TholeDipoleForce& force) = 0;
    virtual void getPMEParameters(double& alpha, int& nx, int& ny, int& nz) const = 0;
    virtual void getInducedDipoles(OpenMM::ContextImpl& context, std::vector<OpenMM::Vec3>& dipoles) = 0;
    virtual void getLabFramePermanentDipoles(OpenMM::ContextImpl& context, std::vector<OpenMM::Vec3>& dipoles) = 0;
    virtual void getTotalDipoles(OpenMM::ContextImpl& context, std::vector<OpenMM::Vec3>& dipoles) = 0;
    virtual void getElectrostaticPotential(OpenMM::ContextImpl& context, const std::vector<OpenMM::Vec3>& inputGrid,
                                           std::vector<double>& outputElectrostaticPotential) = 0;
    virtual void getSystemMultipoleMoments(OpenMM::ContextImpl& context, std::vector<double>& outputMultipoleMoments) = 0;
};

}  // namespace TholeDipolePlugin
#endif
