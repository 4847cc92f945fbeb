// Test driver of the OpenMM-facing adapter (not part of the library): builds a
// System and TholeDipoleForce through the plugin API from a text description,
// creates the kernel through the registered CUDA kernel factory, and prints
// what the reference tests query (platforms/reference/tests/
// TestReferenceTholeDipoleForce.cpp): energy and forces, induced / lab-frame /
// total dipoles, potential, multipole moments, the PME-parameter query, the
// updateParametersInContext equivalence (:255-313) and its size check.
//
// Input (whitespace separated): n method polarization cutoff ewald_tol eps
// max_iter n_extrap [coefficients], 9 box numbers, then per particle: q dx dy dz
// polarizability thole axis_type z x y n12 [atoms] n13 [atoms] mass px py pz,
// then n_grid and grid points.  Argument 2 selects "mixed" or "double".
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <vector>

#include "CudaTholeDipoleKernelFactory.h"
#include "CudaTholeDipoleKernels.h"
#include "openmm/internal/ContextImpl.h"

using namespace TholeDipolePlugin;
using namespace OpenMM;

extern "C" void registerTholeDipoleCudaKernelFactories();

static void print_vecs(const char* tag, const std::vector<Vec3>& v) {
    printf("%s", tag);
    for (const Vec3& a : v) printf(" %.17g %.17g %.17g", a[0], a[1], a[2]);
    printf("\n");
}

static void need(std::istream& in, const char* what) {
    if (!in) {
        fprintf(stderr, "adapter_driver: malformed input while reading %s\n", what);
        std::exit(3);
    }
}

static int count(std::istream& in, int lo, int hi, const char* what) {
    int v = -1;
    in >> v;
    need(in, what);
    if (v < lo || v > hi) {
        fprintf(stderr, "adapter_driver: %s = %d outside [%d, %d]\n", what, v, lo, hi);
        std::exit(3);
    }
    return v;
}

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    std::ifstream in(argv[1]);
    if (!in) return 2;
    bool dbl = argc > 2 && std::strcmp(argv[2], "double") == 0;
    int n = count(in, 0, 1000000, "particle count");
    int method = count(in, 0, 1, "nonbonded method");
    int pol = count(in, 0, 2, "polarization type");
    double cutoff, tol, eps;
    in >> cutoff >> tol >> eps;
    need(in, "settings");
    int maxIter = count(in, 0, 1000000, "max iterations");
    int nex = count(in, 0, 64, "extrapolation coefficient count");
    std::vector<double> ex(nex);
    for (double& c : ex) in >> c;
    double box[9];
    for (double& b : box) in >> b;
    need(in, "coefficients and box");
    System system;
    system.setDefaultPeriodicBoxVectors(Vec3(box[0], box[1], box[2]), Vec3(box[3], box[4], box[5]),
                                        Vec3(box[6], box[7], box[8]));
    TholeDipoleForce* force = new TholeDipoleForce();
    force->setNonbondedMethod((TholeDipoleForce::NonbondedMethod)method);
    force->setPolarizationType((TholeDipoleForce::PolarizationType)pol);
    force->setCutoffDistance(cutoff);
    force->setEwaldErrorTolerance(tol);
    force->setMutualInducedTargetEpsilon(eps);
    force->setMutualInducedMaxIterations(maxIter);
    if (nex > 0) force->setExtrapolationCoefficients(ex);
    std::vector<Vec3> pos(n);
    for (int i = 0; i < n; i++) {
        double q, pl, th, mass;
        std::vector<double> d(3);
        int t, z, x, y;
        in >> q >> d[0] >> d[1] >> d[2] >> pl >> th >> t >> z >> x >> y;
        need(in, "particle parameters");
        int idx = force->addParticle(q, d, pl, th, t, z, x, y);
        for (int list = 0; list < 2; list++) {
            int k = count(in, 0, 64, "covalent list length");
            std::vector<int> atoms(k);
            for (int& a : atoms) in >> a;
            need(in, "covalent atoms");
            force->setCovalentMap(idx, list == 0 ? TholeDipoleForce::Covalent12 : TholeDipoleForce::Covalent13, atoms);
        }
        in >> mass >> pos[i][0] >> pos[i][1] >> pos[i][2];
        need(in, "mass and position");
        system.addParticle(mass);
    }
    int ng = count(in, 0, 100000, "grid point count");
    std::vector<Vec3> grid(ng);
    for (Vec3& g : grid) in >> g[0] >> g[1] >> g[2];
    need(in, "grid points");
    system.addForce(force);

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
