// Input reader shared by the adapter's test drivers (not part of the library):
// builds a System and a TholeDipoleForce through the plugin API from a text
// description.  Whitespace separated: n method polarization cutoff ewald_tol
// eps max_iter n_extrap [coefficients], 9 box numbers, then per particle:
// q dx dy dz polarizability thole axis_type z x y n12 [atoms] n13 [atoms]
// mass px py pz, then n_grid and grid points.
#ifndef TDP_ADAPTER_DRIVER_INPUT_H_
#define TDP_ADAPTER_DRIVER_INPUT_H_
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <vector>

#include "TholeDipoleForce.h"
#include "openmm/System.h"
#include "openmm/Vec3.h"

namespace tdp_driver {

inline void need(std::istream& in, const char* what) {
    if (!in) {
        fprintf(stderr, "driver: malformed input while reading %s\n", what);
        std::exit(3);
    }
}

inline int count(std::istream& in, int lo, int hi, const char* what) {
    int v = -1;
    in >> v;
    need(in, what);
    if (v < lo || v > hi) {
        fprintf(stderr, "driver: %s = %d outside [%d, %d]\n", what, v, lo, hi);
        std::exit(3);
    }
    return v;
}

struct Input {
    OpenMM::System system;
    TholeDipolePlugin::TholeDipoleForce* force = nullptr;  // owned by system
    std::vector<OpenMM::Vec3> positions, grid;
    int n = 0;
};

// Fills in (the System takes the Force).
inline void read_input(const char* path, Input& out) {
    using OpenMM::Vec3;
    using TholeDipolePlugin::TholeDipoleForce;
    std::ifstream in(path);
    if (!in) {
        fprintf(stderr, "driver: cannot open %s\n", path);
        std::exit(2);
    }
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
    out.system.setDefaultPeriodicBoxVectors(Vec3(box[0], box[1], box[2]), Vec3(box[3], box[4], box[5]),
                                            Vec3(box[6], box[7], box[8]));
    TholeDipoleForce* force = new TholeDipoleForce();
    force->setNonbondedMethod((TholeDipoleForce::NonbondedMethod)method);
    force->setPolarizationType((TholeDipoleForce::PolarizationType)pol);
    force->setCutoffDistance(cutoff);
    force->setEwaldErrorTolerance(tol);
    force->setMutualInducedTargetEpsilon(eps);
    force->setMutualInducedMaxIterations(maxIter);
    if (nex > 0) force->setExtrapolationCoefficients(ex);
    out.positions.resize(n);
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
        in >> mass >> out.positions[i][0] >> out.positions[i][1] >> out.positions[i][2];
        need(in, "mass and position");
        out.system.addParticle(mass);
    }
    int ng = count(in, 0, 100000, "grid point count");
    out.grid.resize(ng);
    for (Vec3& g : out.grid) in >> g[0] >> g[1] >> g[2];
    need(in, "grid points");
    out.system.addForce(force);
    out.force = force;
    out.n = n;
}

inline void print_vecs(const char* tag, const std::vector<OpenMM::Vec3>& v) {
    printf("%s", tag);
    for (const OpenMM::Vec3& a : v) printf(" %.17g %.17g %.17g", a[0], a[1], a[2]);
    printf("\n");
}

}  // namespace tdp_driver
#endif
