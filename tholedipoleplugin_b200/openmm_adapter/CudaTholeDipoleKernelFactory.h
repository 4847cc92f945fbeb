/* Kernel factory of the B200 kernels (the role of the plugin's
 * platforms/cuda/include/CudaTholeDipoleKernelFactory.h): creates
 * CudaCalcTholeDipoleForceKernel for the kernel name "CalcTholeDipoleForce"
 * and throws for any other name. */
#ifndef TDP_CUDA_THOLEDIPOLE_KERNEL_FACTORY_H_
#define TDP_CUDA_THOLEDIPOLE_KERNEL_FACTORY_H_
#include <string>
#include "openmm/KernelImpl.h"

namespace TholeDipolePlugin {
class CudaTholeDipoleKernelFactory : public OpenMM::KernelFactory {
public:
    OpenMM::KernelImpl* createKernelImpl(std::string name, const OpenMM::Platform& platform,
                                         OpenMM::ContextImpl& context) const override;
};
}  // namespace TholeDipolePlugin
#endif
