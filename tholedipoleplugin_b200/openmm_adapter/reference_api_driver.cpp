// Test driver of the adapter built against the plugin's own public API: the
// reference's openmmapi/include headers and its openmmapi/src/TholeDipoleForce.cpp
// and TholeDipoleForceImpl.cpp, compiled unmodified (oracle/Makefile, target
// api), over the OpenMM stand-in.  It goes the way an OpenMM program goes: a
// Context creates TholeDipoleForceImpl, whose initialize validates the Force
// (TholeDipoleForceImpl.cpp:52-108) and creates the kernel by name through the
// registered CUDA kernel factory; energies come from calcForcesAndEnergy with
// force-group gating (:114-118) and the queries through the Force's own
// Context methods.  Not part of the library.
//
// Usage: reference_api_driver INPUT [mixed|double] [validate]
// Input: the text description of driver_input.h.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <exception>
#include <vector>

#include "TholeDipoleForce.h"
#include "driver_input.h"
#include "openmm/Context.h"
#include "openmm/OpenMMException.h"
#include "openmm/internal/ContextImpl.h"

using namespace TholeDipolePlugin;
using namespace OpenMM;
using tdp_driver::print_vecs;

extern "C" void registerTholeDipoleCudaKernelFactories();

static void report(const char* tag, const char* path, void (*mutate)(tdp_driver::Input&)) {
    tdp_driver::Input in;
    tdp_driver::read_input(path, in);
    mutate(in);
    try {
        Context context(in.system, Platform::getPlatformByName("CUDA"));
        printf("%s none\n", tag);
    } catch (const OpenMMException& ex) {
        printf("%s %s\n", tag, ex.what());
    }
}

static int check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        fprintf(stderr, "reference_api_driver: %s: %s\n", what, cudaGetErrorString(e));
        return 1;
    }
    return 0;
}

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    try {
        registerTholeDipoleCudaKernelFactories();
        Platform& platform = Platform::getPlatformByName("CUDA");
        platform.setPropertyDefaultValue("Precision", argc > 2 && std::strcmp(argv[2], "double") == 0 ? "double"
                                                                                                       : "mixed");
        if (argc > 3 && std::strcmp(argv[3], "validate") == 0) {
            // The reference ForceImpl's own checks at Context creation.
            report("particles_error", argv[1], [](tdp_driver::Input& in) { in.system.addParticle(1.0); });
            report("cutoff_error", argv[1], [](tdp_driver::Input& in) {
                in.force->setNonbondedMethod(TholeDipoleForce::PME);
                in.force->setCutoffDistance(10.0);
            });
            report("axis_error", argv[1], [](tdp_driver::Input& in) {
                double q, p, t;
                std::vector<double> d;
                int a, z, x, y;
                in.force->getParticleParameters(0, q, d, p, t, a, z, x, y);
                in.force->setParticleParameters(0, q, d, p, t, 7, z, x, y);
            });
            report("zaxis_error", argv[1], [](tdp_driver::Input& in) {
                double q, p, t;
                std::vector<double> d;
                int a, z, x, y;
                in.force->getParticleParameters(0, q, d, p, t, a, z, x, y);
                in.force->setParticleParameters(0, q, d, p, t, TholeDipoleForce::ZThenX, in.n + 5, x, y);
            });
            return 0;
        }
        tdp_driver::Input in;
        tdp_driver::read_input(argv[1], in);
        TholeDipoleForce& force = *in.force;
        const int n = in.n;
        Context context(in.system, platform);
        context.setPositions(in.positions);
        printf("energy %.17g\n", context.calcForcesAndEnergy());
        print_vecs("forces", context.getForces());
        std::vector<Vec3> d;
        force.getInducedDipoles(context, d);
        print_vecs("induced", d);
        force.getLabFramePermanentDipoles(context, d);
        print_vecs("lab", d);
        force.getTotalDipoles(context, d);
        print_vecs("total", d);
        std::vector<double> pot, mom;
        force.getElectrostaticPotential(in.grid, context, pot);
        printf("potential");
        for (double p : pot) printf(" %.17g", p);
        printf("\n");
        force.getSystemMultipoleMoments(context, mom);
        printf("moments");
        for (double m : mom) printf(" %.17g", m);
        printf("\n");
        try {
            double a;
            int nx, ny, nz;
            force.getPMEParametersInContext(context, a, nx, ny, nz);
            printf("pme %.17g %d %d %d\n", a, nx, ny, nz);
        } catch (const OpenMMException& ex) {
            printf("pme_error %s\n", ex.what());
        }
        // Force groups (TholeDipoleForceImpl.cpp:114-118).
        force.setForceGroup(3);
        printf("energy_other_groups %.17g\n", context.calcForcesAndEnergy(true, true, ~(1 << 3)));
        printf("energy_own_group %.17g\n", context.calcForcesAndEnergy(true, true, 1 << 3));
        force.setForceGroup(0);

        // The CUDA platform context's buffers: posq in a permuted order and the
        // fixed-point force accumulator (the slot order reverses the atoms).
        const int padded = ((n + 31) / 32) * 32;
        const bool dbl = platform.getPropertyDefaultValue("Precision") == "double";
        std::vector<int> index(padded, -1);
        for (int k = 0; k < n; k++) index[k] = n - 1 - k;
        std::vector<double> posq_d(4 * (size_t)padded, 0.0);
        std::vector<float> posq_f(4 * (size_t)padded, 0.0f);
        for (int k = 0; k < n; k++) {
            double q, p, t;
            std::vector<double> dm;
            int a, z, x, y;
            force.getParticleParameters(index[k], q, dm, p, t, a, z, x, y);
            for (int c = 0; c < 3; c++) {
                posq_d[4 * k + c] = in.positions[index[k]][c];
                posq_f[4 * k + c] = (float)in.positions[index[k]][c];
            }
            posq_d[4 * k + 3] = q;
            posq_f[4 * k + 3] = (float)q;
        }
        DevicePlatformData dev;
        const size_t posq_bytes = dbl ? posq_d.size() * sizeof(double) : posq_f.size() * sizeof(float);
        if (check_cuda(cudaMalloc(&dev.posq, posq_bytes), "cudaMalloc") ||
            check_cuda(cudaMalloc((void**)&dev.atomIndex, sizeof(int) * padded), "cudaMalloc") ||
            check_cuda(cudaMalloc((void**)&dev.force, sizeof(long long) * 3 * padded), "cudaMalloc"))
            return 5;
        cudaMemcpy(dev.posq, dbl ? (const void*)posq_d.data() : (const void*)posq_f.data(), posq_bytes,
                   cudaMemcpyHostToDevice);
        cudaMemcpy(dev.atomIndex, index.data(), sizeof(int) * padded, cudaMemcpyHostToDevice);
        cudaMemset(dev.force, 0, sizeof(long long) * 3 * padded);
        dev.posqIsDouble = dbl ? 1 : 0;
        dev.paddedNumAtoms = padded;
        context.getImpl().getSystem().getDefaultPeriodicBoxVectors(dev.periodicBoxVectors[0],
                                                                   dev.periodicBoxVectors[1],
                                                                   dev.periodicBoxVectors[2]);
        context.getImpl().setDevicePlatformData(&dev);
        printf("energy_device %.17g\n", context.calcForcesAndEnergy());
        std::vector<long long> acc(3 * (size_t)padded);
        if (check_cuda(cudaMemcpy(acc.data(), dev.force, sizeof(long long) * 3 * padded, cudaMemcpyDeviceToHost),
                       "cudaMemcpy"))
            return 5;
        std::vector<Vec3> fdev(n);
        for (int k = 0; k < n; k++)
            for (int c = 0; c < 3; c++) fdev[index[k]][c] = (double)acc[k + (size_t)c * padded] / 4294967296.0;
        print_vecs("forces_device", fdev);
        force.getInducedDipoles(context, d);
        print_vecs("induced_device", d);
        context.getImpl().setDevicePlatformData(nullptr);
        cudaFree(dev.posq);
        cudaFree(dev.atomIndex);
        cudaFree(dev.force);

        // updateParametersInContext (TholeDipoleForceImpl.cpp:188-191): the
        // parameter change of TestReferenceTholeDipoleForce.cpp:263-271.
        for (int i = 0; i < n; i++) {
            double q, p, t;
            std::vector<double> dp;
            int a, z, x, y;
            force.getParticleParameters(i, q, dp, p, t, a, z, x, y);
            dp[0] *= 0.7;
            force.setParticleParameters(i, 1.1 * q, dp, 1.5 * p, 1.3 * t, a, z, x, y);
        }
        force.updateParametersInContext(context);
        printf("system_changed %d\n", context.getImpl().systemChanges());
        printf("energy_updated %.17g\n", context.calcForcesAndEnergy());
        print_vecs("forces_updated", context.getForces());
    } catch (const std::exception& ex) {
        fprintf(stderr, "reference_api_driver: %s\n", ex.what());
        return 4;
    }
    return 0;
}
