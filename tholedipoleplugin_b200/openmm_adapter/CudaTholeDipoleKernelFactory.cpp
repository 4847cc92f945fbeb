// Kernel factory and plugin registration entry points of the B200 kernels,
// following the plugin's CUDA platform registration
// (platforms/cuda/src/CudaTholeDipoleKernelFactory.cpp:44-73): registerPlatforms,
// registerKernelFactories and registerTholeDipoleCudaKernelFactories are the
// C symbols OpenMM's plugin loader and the tests call.
#include <exception>
#include <string>

#include "CudaTholeDipoleKernelFactory.h"
#include "CudaTholeDipoleKernels.h"
#include "openmm/OpenMMException.h"
#include "openmm/internal/ContextImpl.h"

using namespace TholeDipolePlugin;
using namespace OpenMM;

KernelImpl* CudaTholeDipoleKernelFactory::createKernelImpl(std::string name, const Platform& platform,
                                                           ContextImpl& context) const {
    if (name == CalcTholeDipoleForceKernel::Name()) {
        CudaCalcTholeDipoleForceKernel* k = new CudaCalcTholeDipoleForceKernel(name, platform, context.getSystem());
        // The CUDA platform's "Precision" property: "double" selects the FP64
        // form; "single" and "mixed" the mixed form.
        if (platform.getPropertyDefaultValue("Precision") == "double") k->setPrecision(TDP_PRECISION_DOUBLE);
        return k;
    }
    throw OpenMMException((std::string("Tried to create kernel with illegal kernel name '") + name + "'").c_str());
}

extern "C" OPENMM_EXPORT void registerPlatforms() {}

extern "C" OPENMM_EXPORT void registerKernelFactories() {
    try {
        Platform& platform = Platform::getPlatformByName("CUDA");
        platform.registerKernelFactory(CalcTholeDipoleForceKernel::Name(), new CudaTholeDipoleKernelFactory());
    } catch (std::exception&) {
        // No CUDA platform: nothing to register.
    }
}

extern "C" OPENMM_EXPORT void registerTholeDipoleCudaKernelFactories() {
    try {
        Platform::getPlatformByName("CUDA");
    } catch (...) {
        Platform::registerPlatform(new Platform("CUDA"));
    }
    registerKernelFactories();
}
