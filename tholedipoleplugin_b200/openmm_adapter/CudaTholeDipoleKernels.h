/* CudaCalcTholeDipoleForceKernel: the B200 implementation of the plugin's
 * CalcTholeDipoleForceKernel (openmmapi/include/TholeDipoleKernels.h:46-122),
 * a thin C++ shell over the C ABI of include/tholedipole_b200.h.  It takes the
 * place of ReferenceCalcTholeDipoleForceKernel
 * (platforms/reference/src/ReferenceTholeDipoleKernels.cpp) and of the
 * non-functional common-compute kernel: same methods, same argument meaning,
 * errors as OpenMMException with the reference's messages. */
#ifndef TDP_CUDA_THOLEDIPOLE_KERNELS_H_
#define TDP_CUDA_THOLEDIPOLE_KERNELS_H_
#include <vector>

#include "TholeDipoleKernels.h"
#include "tholedipole_b200.h"

namespace TholeDipolePlugin {

class CudaCalcTholeDipoleForceKernel : public CalcTholeDipoleForceKernel {
public:
    CudaCalcTholeDipoleForceKernel(std::string name, const OpenMM::Platform& platform, const OpenMM::System& system);
    ~CudaCalcTholeDipoleForceKernel() override;
    void initialize(const OpenMM::System& system, const TholeDipoleForce& force) override;
    double execute(OpenMM::ContextImpl& context, bool includeForces, bool includeEnergy) override;
    void copyParametersToContext(OpenMM::ContextImpl& context, const TholeDipoleForce& force) override;
    void getPMEParameters(double& alpha, int& nx, int& ny, int& nz) const override;
    void getInducedDipoles(OpenMM::ContextImpl& context, std::vector<OpenMM::Vec3>& dipoles) override;
    void getLabFramePermanentDipoles(OpenMM::ContextImpl& context, std::vector<OpenMM::Vec3>& dipoles) override;
    void getTotalDipoles(OpenMM::ContextImpl& context, std::vector<OpenMM::Vec3>& dipoles) override;
    void getElectrostaticPotential(OpenMM::ContextImpl& context, const std::vector<OpenMM::Vec3>& inputGrid,
                                   std::vector<double>& outputElectrostaticPotential) override;
    void getSystemMultipoleMoments(OpenMM::ContextImpl& context, std::vector<double>& outputMultipoleMoments) override;

    /* Options of this platform (the CUDA platform's properties): precision
     * "mixed" (default) or "double"; solver "cg" (default) or "jacobi". */
    void setPrecision(int precision) { precision_ = precision; }
    void setSolver(int solver) { solver_ = solver; }
    tdp_handle* handle() const { return handle_; }

private:
    void check(int status) const;
    void syncBox(OpenMM::ContextImpl& context);
    const double* positions(OpenMM::ContextImpl& context);
    void dipoles(OpenMM::ContextImpl& context, int which, std::vector<OpenMM::Vec3>& out);

    const OpenMM::System& system_;
    tdp_handle* handle_ = nullptr;
    int numParticles_ = 0;
    bool usePme_ = false;
    int precision_ = TDP_PRECISION_MIXED;
    int solver_ = TDP_SOLVER_CG;
};

}  // namespace TholeDipolePlugin
#endif
