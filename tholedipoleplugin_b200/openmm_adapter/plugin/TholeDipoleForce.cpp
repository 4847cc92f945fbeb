// TholeDipoleForce parameter container (see plugin/TholeDipoleForce.h).
// Defaults as the plugin's constructor: NoCutoff, Mutual, B-spline order 5,
// cutoff 1 nm, Ewald tolerance 1e-4, 60 iterations, target 1e-5, OPT4
// extrapolation coefficients (openmmapi/src/TholeDipoleForce.cpp:43-51).
#include "TholeDipoleForce.h"

using namespace TholeDipolePlugin;

TholeDipoleForce::TholeDipoleForce()
    : nonbondedMethod(NoCutoff), polarizationType(Mutual), cutoffDistance(1.0), alpha(0.0), pmeBSplineOrder(5), nx(0),
      ny(0), nz(0), mutualInducedMaxIterations(60), extrapolationCoefficients({-0.154, 0.017, 0.658, 0.474}),
      mutualInducedTargetEpsilon(1e-5), ewaldErrorTol(1e-4) {}

void TholeDipoleForce::setNonbondedMethod(NonbondedMethod method) {
    if (method < 0 || method > 1) throw OpenMM::OpenMMException("TholeDipoleForce: Illegal value for nonbonded method");
    nonbondedMethod = method;
}

void TholeDipoleForce::getPMEParameters(double& a, int& x, int& y, int& z) const {
    a = alpha;
    x = nx;
    y = ny;
    z = nz;
}

void TholeDipoleForce::setPMEParameters(double a, int x, int y, int z) {
    alpha = a;
    nx = x;
    ny = y;
    nz = z;
}

int TholeDipoleForce::addParticle(double charge, const std::vector<double>& dip, double pol, double thole, int axisType,
                                  int z, int x, int y) {
    ParticleInfo p;
    p.charge = charge;
    p.molecularDipole = {dip[0], dip[1], dip[2]};
    p.polarizability = pol;
    p.tholeDamping = thole;
    p.axisType = axisType;
    p.multipoleAtomZ = z;
    p.multipoleAtomX = x;
    p.multipoleAtomY = y;
    p.covalentInfo.resize(CovalentEnd);
    particles.push_back(p);
    return (int)particles.size() - 1;
}

void TholeDipoleForce::getParticleParameters(int i, double& charge, std::vector<double>& dip, double& pol,
                                             double& thole, int& axisType, int& z, int& x, int& y) const {
    const ParticleInfo& p = particles.at(i);
    charge = p.charge;
    dip = p.molecularDipole;
    pol = p.polarizability;
    thole = p.tholeDamping;
    axisType = p.axisType;
    z = p.multipoleAtomZ;
    x = p.multipoleAtomX;
    y = p.multipoleAtomY;
}

void TholeDipoleForce::setParticleParameters(int i, double charge, const std::vector<double>& dip, double pol,
                                             double thole, int axisType, int z, int x, int y) {
    ParticleInfo& p = particles.at(i);
    p.charge = charge;
    p.molecularDipole = {dip[0], dip[1], dip[2]};
    p.polarizability = pol;
    p.tholeDamping = thole;
    p.axisType = axisType;
    p.multipoleAtomZ = z;
    p.multipoleAtomX = x;
    p.multipoleAtomY = y;
}

void TholeDipoleForce::setCovalentMap(int i, CovalentType type, const std::vector<int>& atoms) {
    particles.at(i).covalentInfo.at(type) = atoms;
}

void TholeDipoleForce::getCovalentMap(int i, CovalentType type, std::vector<int>& atoms) const {
    atoms = particles.at(i).covalentInfo.at(type);
}

void TholeDipoleForce::getCovalentMaps(int i, std::vector<std::vector<int> >& lists) const {
    lists = particles.at(i).covalentInfo;
}
