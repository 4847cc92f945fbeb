// Test driver of the OpenMM-facing adapter (not part of the library): builds a
// System and TholeDipoleForce through the plugin API from a text description,
// creates the kernel through the registered CUDA kernel factory, and prints
// what the reference tests query (platforms/reference/tests/
// TestReferenceTholeDipoleForce.cpp): energy and forces, induced / lab-frame /
// total dipoles, potential, multipole moments, the PME-parameter query, the
// updateParametersInContext equivalence (:255-313) and its size check.
//
// Input: the text description of driver_input.h.  Argument 2 selects "mixed"
// or "double".
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <vector>

#include "CudaTholeDipoleKernelFactory.h"
#include "CudaTholeDipoleKernels.h"
#include "driver_input.h"
#include "openmm/internal/ContextImpl.h"

using namespace TholeDipolePlugin;
using namespace OpenMM;

extern "C" void registerTholeDipoleCudaKernelFactories();

using tdp_driver::print_vecs;

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    bool dbl = argc > 2 && std::strcmp(argv[2], "double") == 0;
    tdp_driver::Input input;
    tdp_driver::read_input(argv[1], input);
    System& system = input.system;
    TholeDipoleForce* force = input.force;
    const int n = input.n;
    const std::vector<Vec3>& pos = input.positions;
    const std::vector<Vec3>& grid = input.grid;

    try {
    registerTholeDipoleCudaKernelFactories();
    Platform& platform = Platform::getPlatformByName("CUDA");
    ContextImpl context(system, platform);
    context.positions = pos;
    Kernel kernel = platform.createKernel(CalcTholeDipoleForceKernel::Name(), context);
    CudaCalcTholeDipoleForceKernel& k = kernel.getAs<CudaCalcTholeDipoleForceKernel>();
    if (dbl) k.setPrecision(TDP_PRECISION_DOUBLE);
    k.initialize(system, *force);

    for (Vec3& f : context.forces) f = Vec3();
    double e = k.execute(context, true, true);
    printf("energy %.17g\n", e);
    print_vecs("forces", context.forces);
    std::vector<Vec3> d;
    k.getInducedDipoles(context, d);
    print_vecs("induced", d);
    k.getLabFramePermanentDipoles(context, d);
    print_vecs("lab", d);
    k.getTotalDipoles(context, d);
    print_vecs("total", d);
    std::vector<double> pot, mom;
    k.getElectrostaticPotential(context, grid, pot);
    printf("potential");
    for (double p : pot) printf(" %.17g", p);
    printf("\n");
    k.getSystemMultipoleMoments(context, mom);
    printf("moments");
    for (double m : mom) printf(" %.17g", m);
    printf("\n");
    try {
        double a;
        int nx, ny, nz;
        k.getPMEParameters(a, nx, ny, nz);
        printf("pme %.17g %d %d %d\n", a, nx, ny, nz);
    } catch (const OpenMMException& ex) {
        printf("pme_error %s\n", ex.what());
    }
    // Parameter update: the change of TestReferenceTholeDipoleForce.cpp:263-271.
    for (int i = 0; i < n; i++) {
        double q, pl, th;
        std::vector<double> dp;
        int t, z, x, y;
        force->getParticleParameters(i, q, dp, pl, th, t, z, x, y);
        dp[0] *= 0.7;
        force->setParticleParameters(i, 1.1 * q, dp, 1.5 * pl, 1.3 * th, t, z, x, y);
    }
    k.copyParametersToContext(context, *force);
    for (Vec3& f : context.forces) f = Vec3();
    printf("energy_updated %.17g\n", k.execute(context, true, true));
    print_vecs("forces_updated", context.forces);
    ContextImpl context2(system, platform);
    context2.positions = pos;
    Kernel kernel2 = platform.createKernel(CalcTholeDipoleForceKernel::Name(), context2);
    CudaCalcTholeDipoleForceKernel& k2 = kernel2.getAs<CudaCalcTholeDipoleForceKernel>();
    if (dbl) k2.setPrecision(TDP_PRECISION_DOUBLE);
    k2.initialize(system, *force);
    printf("energy_fresh %.17g\n", k2.execute(context2, true, true));
    print_vecs("forces_fresh", context2.forces);
    try {
        TholeDipoleForce smaller;
        k.copyParametersToContext(context, smaller);
        printf("size_error none\n");
    } catch (const OpenMMException& ex) {
        printf("size_error %s\n", ex.what());
    }
    try {
        CudaTholeDipoleKernelFactory factory;
        delete factory.createKernelImpl("NoSuchKernel", platform, context);
        printf("name_error none\n");
    } catch (const OpenMMException& ex) {
        printf("name_error %s\n", ex.what());
    }
    } catch (const std::exception& ex) {
        fprintf(stderr, "adapter_driver: %s\n", ex.what());
        return 4;
    }
    return 0;
}
