/*
 * ref_driver.cpp -- C entry points around the reference plugin's own
 * ReferenceTholeDipoleForce class (aehogan/tholedipoleplugin,
 * platforms/reference/src/ReferenceTholeDipoleForce.cpp), which oracle/Makefile
 * compiles unmodified from the reference tree into oracle/_ref/libtdp_ref.so.
 * TEST INFRASTRUCTURE ONLY: it pins the restatement in tdp_oracle.c, generates
 * the golden fixtures, and serves as the "reference" CPU baseline of bench.py.
 *
 * The set-up mirrors ReferenceCalcTholeDipoleForceKernel
 * (platforms/reference/src/ReferenceTholeDipoleKernels.cpp:160-215): PME
 * selects ReferencePmeTholeDipoleForce with the box, Mutual copies the target
 * epsilon and iteration cap, Extrapolated copies the coefficients.
 *
 * Deterministic heap word.  The reference's pair routine reads rInvVec[4] of
 * a 4-element std::vector (RTDF.cpp:196 vs :264,277,323,333), i.e. the 8 bytes
 * just past a 32-byte heap block.  This library replaces the global operator
 * new (bound inside the library with -Bsymbolic) so that every block is
 * followed by 32 bytes holding the double `fill` chosen by the caller.  With
 * fill = 0.0 the results equal what a fresh process reads; any other fill
 * exposes how that word enters the forces.
 */
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "ReferenceTholeDipoleForce.h"
#include "tdp_oracle.h"

using namespace TholeDipolePlugin;
using OpenMM::Vec3;
using std::vector;

static double g_fill = 0.0;

void* operator new(std::size_t n) {
    std::size_t body = (n + 7) & ~std::size_t(7);
    unsigned char* p = static_cast<unsigned char*>(std::malloc(body + 32));
    if (!p) throw std::bad_alloc();
    for (int k = 0; k < 4; k++) std::memcpy(p + body + 8 * k, &g_fill, 8);
    return p;
}
void* operator new[](std::size_t n) { return operator new(n); }
void operator delete(void* p) noexcept { std::free(p); }
void operator delete[](void* p) noexcept { std::free(p); }
void operator delete(void* p, std::size_t) noexcept { std::free(p); }
void operator delete[](void* p, std::size_t) noexcept { std::free(p); }

namespace {

struct Inputs {
    vector<Vec3> pos;
    vector<double> charges, dipoles, polarity, tholes;
    vector<int> axisTypes, zs, xs, ys;
    vector<vector<vector<int>>> cov;
};

Inputs load(const tdpo_system* s) {
    Inputs in;
    int n = s->n;
    in.pos.resize(n);
    for (int i = 0; i < n; i++) in.pos[i] = Vec3(s->pos[3 * i], s->pos[3 * i + 1], s->pos[3 * i + 2]);
    in.charges.assign(s->charge, s->charge + n);
    in.dipoles.assign(s->dipole, s->dipole + 3 * n);
    in.polarity.assign(s->polarity, s->polarity + n);
    in.tholes.assign(s->thole, s->thole + n);
    in.axisTypes.resize(n);
    in.zs.resize(n);
    in.xs.resize(n);
    in.ys.resize(n);
    for (int i = 0; i < n; i++) {
        in.axisTypes[i] = s->axis[4 * i];
        in.zs[i] = s->axis[4 * i + 1];
        in.xs[i] = s->axis[4 * i + 2];
        in.ys[i] = s->axis[4 * i + 3];
    }
    in.cov.assign(n, vector<vector<int>>(4));
    for (int i = 0; i < n; i++) {
        if (s->cov12_off) in.cov[i][0].assign(s->cov12 + s->cov12_off[i], s->cov12 + s->cov12_off[i + 1]);
        if (s->cov13_off) in.cov[i][1].assign(s->cov13 + s->cov13_off[i], s->cov13 + s->cov13_off[i + 1]);
    }
    return in;
}

/* Exposes the protected stages of the reference class for stage-level pins.
 * A zero box makes getPeriodicDelta a no-op (RTDF.cpp:1419), i.e. NoCutoff. */
class Probe : public ReferencePmeTholeDipoleForce {
public:
    typedef TholeDipoleParticleData Particle;
    void configureBox(const tdpo_system* s) {
        Vec3 box[3];
        if (s->method == TDPO_PME) {
            box[0] = Vec3(s->box[0], 0, 0);
            box[1] = Vec3(0, s->box[1], 0);
            box[2] = Vec3(0, 0, s->box[2]);
        }
        setPeriodicBoxSize(box);
    }
    void runSetup(const Inputs& in, vector<Particle>& pd) {
        setup(in.pos, in.charges, in.dipoles, in.polarity, in.tholes, in.axisTypes, in.zs, in.xs, in.ys, in.cov, pd);
    }
    const vector<Vec3>& fixedField() const { return _fixedDipoleField; }
    void inducedField(const vector<Particle>& pd, const vector<Vec3>& mu, vector<Vec3>& out) {
        calculateInducedDipoleFields(pd, mu, out);
    }
};

void configure(ReferenceTholeDipoleForce* f, const tdpo_system* s) {
    if (s->polarization == TDPO_MUTUAL) {
        f->setPolarizationType(ReferenceTholeDipoleForce::Mutual);
        f->setMutualInducedDipoleTargetEpsilon(s->target_eps);
        f->setMaximumMutualInducedDipoleIterations(s->max_iter);
    } else if (s->polarization == TDPO_DIRECT) {
        f->setPolarizationType(ReferenceTholeDipoleForce::Direct);
    } else {
        f->setPolarizationType(ReferenceTholeDipoleForce::Extrapolated);
        vector<double> c(s->extrap, s->extrap + (s->n_extrap > 0 ? s->n_extrap : 0));
        f->setExtrapolationCoefficients(c);
    }
}

ReferenceTholeDipoleForce* make(const tdpo_system* s) {
    ReferenceTholeDipoleForce* f;
    if (s->method == TDPO_PME) {
        ReferencePmeTholeDipoleForce* p = new ReferencePmeTholeDipoleForce();
        Vec3 box[3] = {Vec3(s->box[0], 0, 0), Vec3(0, s->box[1], 0), Vec3(0, 0, s->box[2])};
        p->setPeriodicBoxSize(box);
        f = p;
    } else {
        f = new ReferenceTholeDipoleForce(ReferenceTholeDipoleForce::NoCutoff);
    }
    configure(f, s);
    return f;
}

/* Either reference class with its protected induced dipoles readable, so that
 * one calculateForceAndEnergy call yields energy, forces and the dipoles it
 * used (the golden fixtures of the large boxes need only one solve). */
template <class Base>
struct Exposed : Base {
    using Base::Base;
    const vector<Vec3>& induced() const { return this->_inducedDipole; }
};

void stats(const ReferenceTholeDipoleForce* f, tdpo_stats* st) {
    if (!st) return;
    st->iterations = f->getMutualInducedDipoleIterations();
    st->epsilon = f->getMutualInducedDipoleEpsilon();
    st->converged = f->getMutualInducedDipoleConverged();
}

void put(const vector<Vec3>& v, double* out) {
    for (size_t i = 0; i < v.size(); i++)
        for (int c = 0; c < 3; c++) out[3 * i + c] = v[i][c];
}

}  // namespace

extern "C" {

/* Full force/energy evaluation: calculateForceAndEnergy (RTDF.cpp:100-127).
 * forces (n*3) are added to, as the kernel wrapper adds into the context's
 * force array. */
int tdpref_compute(const tdpo_system* s, double fill, double* energy, double* forces,
                   tdpo_stats* st) {
    g_fill = fill;
    try {
        Inputs in = load(s);
        ReferenceTholeDipoleForce* f = make(s);
        vector<Vec3> fv(s->n);
        for (int i = 0; i < s->n; i++) fv[i] = Vec3(forces[3 * i], forces[3 * i + 1], forces[3 * i + 2]);
        *energy = f->calculateForceAndEnergy(in.pos, in.charges, in.dipoles, in.polarity, in.tholes, in.axisTypes,
                                             in.zs, in.xs, in.ys, in.cov, fv);
        stats(f, st);
        put(fv, forces);
        delete f;
    } catch (...) {
        return 1;
    }
    return 0;
}

/* calculateForceAndEnergy (RTDF.cpp:100-127) plus the induced dipoles of the
 * same solve (mu, n*3; zeros for Direct are the reference's own values). */
int tdpref_compute_full(const tdpo_system* s, double fill, double* energy, double* forces, double* mu,
                        tdpo_stats* st) {
    g_fill = fill;
    try {
        Inputs in = load(s);
        ReferenceTholeDipoleForce* f;
        Exposed<ReferenceTholeDipoleForce>* fn = nullptr;
        Exposed<ReferencePmeTholeDipoleForce>* fp = nullptr;
        if (s->method == TDPO_PME) {
            fp = new Exposed<ReferencePmeTholeDipoleForce>();
            Vec3 box[3] = {Vec3(s->box[0], 0, 0), Vec3(0, s->box[1], 0), Vec3(0, 0, s->box[2])};
            fp->setPeriodicBoxSize(box);
            f = fp;
        } else {
            fn = new Exposed<ReferenceTholeDipoleForce>(ReferenceTholeDipoleForce::NoCutoff);
            f = fn;
        }
        configure(f, s);
        vector<Vec3> fv(s->n);
        for (int i = 0; i < s->n; i++) fv[i] = Vec3(forces[3 * i], forces[3 * i + 1], forces[3 * i + 2]);
        *energy = f->calculateForceAndEnergy(in.pos, in.charges, in.dipoles, in.polarity, in.tholes, in.axisTypes,
                                             in.zs, in.xs, in.ys, in.cov, fv);
        stats(f, st);
        put(fv, forces);
        const vector<Vec3>& ind = fp ? fp->induced() : fn->induced();
        for (int i = 0; i < s->n; i++)
            for (int c = 0; c < 3; c++) mu[3 * i + c] = i < (int)ind.size() ? ind[i][c] : 0.0;
        delete f;
    } catch (...) {
        return 1;
    }
    return 0;
}

int tdpref_induced_dipoles(const tdpo_system* s, double fill, double* mu, tdpo_stats* st) {
    g_fill = fill;
    try {
        Inputs in = load(s);
        ReferenceTholeDipoleForce* f = make(s);
        vector<Vec3> out;
        f->calculateInducedDipoles(in.pos, in.charges, in.dipoles, in.polarity, in.tholes, in.axisTypes, in.zs,
                                   in.xs, in.ys, in.cov, out);
        stats(f, st);
        put(out, mu);
        delete f;
    } catch (...) {
        return 1;
    }
    return 0;
}

int tdpref_lab_dipoles(const tdpo_system* s, double* lab) {
    try {
        Inputs in = load(s);
        tdpo_system d = *s;
        d.polarization = TDPO_DIRECT;
        ReferenceTholeDipoleForce* f = make(&d);
        vector<Vec3> out;
        f->calculateLabFramePermanentDipoles(in.pos, in.charges, in.dipoles, in.polarity, in.tholes, in.axisTypes,
                                             in.zs, in.xs, in.ys, in.cov, out);
        put(out, lab);
        delete f;
    } catch (...) {
        return 1;
    }
    return 0;
}

int tdpref_total_dipoles(const tdpo_system* s, double* out3) {
    try {
        Inputs in = load(s);
        ReferenceTholeDipoleForce* f = make(s);
        vector<Vec3> out;
        f->calculateTotalDipoles(in.pos, in.charges, in.dipoles, in.polarity, in.tholes, in.axisTypes, in.zs,
                                 in.xs, in.ys, in.cov, out);
        put(out, out3);
        delete f;
    } catch (...) {
        return 1;
    }
    return 0;
}

/* Fixed (permanent) field: the _fixedDipoleField left by setup() with Direct
 * polarization (RTDF.cpp:715-746). */
int tdpref_fixed_field(const tdpo_system* s, double* field) {
    try {
        Inputs in = load(s);
        Probe p;
        p.configureBox(s);
        p.setPolarizationType(ReferenceTholeDipoleForce::Direct);
        vector<Probe::Particle> pd;
        p.runSetup(in, pd);
        put(p.fixedField(), field);
    } catch (...) {
        return 1;
    }
    return 0;
}

/* One mutual-field pass T*mu: calculateInducedDipoleFields (RTDF.cpp:782-818). */
int tdpref_induced_field(const tdpo_system* s, const double* mu, double* field) {
    try {
        Inputs in = load(s);
        Probe p;
        p.configureBox(s);
        p.setPolarizationType(ReferenceTholeDipoleForce::Direct);
        vector<Probe::Particle> pd;
        p.runSetup(in, pd);
        vector<Vec3> m(s->n), out;
        for (int i = 0; i < s->n; i++) m[i] = Vec3(mu[3 * i], mu[3 * i + 1], mu[3 * i + 2]);
        p.inducedField(pd, m, out);
        put(out, field);
    } catch (...) {
        return 1;
    }
    return 0;
}

int tdpref_potential(const tdpo_system* s, const double* grid, int ngrid, double* out) {
    try {
        Inputs in = load(s);
        ReferenceTholeDipoleForce* f = make(s);
        vector<Vec3> g(ngrid);
        for (int i = 0; i < ngrid; i++) g[i] = Vec3(grid[3 * i], grid[3 * i + 1], grid[3 * i + 2]);
        vector<double> pot;
        f->calculateElectrostaticPotential(in.pos, in.charges, in.dipoles, in.polarity, in.tholes, in.axisTypes,
                                           in.zs, in.xs, in.ys, in.cov, g, pot);
        for (int i = 0; i < ngrid; i++) out[i] = pot[i];
        delete f;
    } catch (...) {
        return 1;
    }
    return 0;
}

int tdpref_moments(const tdpo_system* s, const double* masses, double* out13) {
    try {
        Inputs in = load(s);
        ReferenceTholeDipoleForce* f = make(s);
        vector<double> m(masses, masses + s->n), out;
        f->calculateTholeDipoleSystemMultipoleMoments(m, in.pos, in.charges, in.dipoles, in.polarity, in.tholes,
                                                      in.axisTypes, in.zs, in.xs, in.ys, in.cov, out);
        for (int k = 0; k < 13; k++) out13[k] = out[k];
        delete f;
    } catch (...) {
        return 1;
    }
    return 0;
}

}  // extern "C"
