/* TholeDipoleForce: the plugin's public Force class, restated for building the
 * CUDA kernel adapter where the plugin's own openmmapi is not compiled in.
 * Same class name, enumerators, defaults, method names and argument order as
 * aehogan/tholedipoleplugin openmmapi/include/TholeDipoleForce.h:54-428 (a
 * drop-in kernel must see the identical interface).  Context-level queries
 * (getInducedDipoles(Context&, ...) and friends) live in the plugin's
 * ForceImpl and are reached through the kernel interface instead. */
#ifndef TDP_PLUGIN_THOLEDIPOLEFORCE_H_
#define TDP_PLUGIN_THOLEDIPOLEFORCE_H_
#include <vector>
#include "openmm/Force.h"
#include "openmm/OpenMMException.h"
#include "openmm/Vec3.h"

namespace TholeDipolePlugin {

class TholeDipoleForce : public OpenMM::Force {
public:
    enum NonbondedMethod { NoCutoff = 0, PME = 1 };
    enum PolarizationType { Direct = 0, Mutual = 1, Extrapolated = 2 };
    enum MultipoleAxisTypes { ZThenX = 0, Bisector = 1, ZBisect = 2, ThreeFold = 3, ZOnly = 4, NoAxisType = 5,
                              LastAxisTypeIndex = 6 };
    enum CovalentType { Covalent12 = 0, Covalent13 = 1, Covalent14 = 2, Covalent15 = 3, CovalentEnd = 4 };

    TholeDipoleForce();
    int getNumParticles() const { return (int)particles.size(); }
    NonbondedMethod getNonbondedMethod() const { return nonbondedMethod; }
    void setNonbondedMethod(NonbondedMethod method);
    PolarizationType getPolarizationType() const { return polarizationType; }
    void setPolarizationType(PolarizationType type) { polarizationType = type; }
    double getCutoffDistance() const { return cutoffDistance; }
    void setCutoffDistance(double distance) { cutoffDistance = distance; }
    void getPMEParameters(double& alpha, int& nx, int& ny, int& nz) const;
    void setPMEParameters(double alpha, int nx, int ny, int nz);
    int getPmeBSplineOrder() const { return pmeBSplineOrder; }
    int addParticle(double charge, const std::vector<double>& molecularDipole, double polarizability,
                    double tholeDamping, int axisType = NoAxisType, int multipoleAtomZ = -1, int multipoleAtomX = -1,
                    int multipoleAtomY = -1);
    void getParticleParameters(int index, double& charge, std::vector<double>& molecularDipole,
                               double& polarizability, double& tholeDamping, int& axisType, int& multipoleAtomZ,
                               int& multipoleAtomX, int& multipoleAtomY) const;
    void setParticleParameters(int index, double charge, const std::vector<double>& molecularDipole,
                               double polarizability, double tholeDamping, int axisType, int multipoleAtomZ,
                               int multipoleAtomX, int multipoleAtomY);
    void setCovalentMap(int index, CovalentType typeId, const std::vector<int>& covalentAtoms);
    void getCovalentMap(int index, CovalentType typeId, std::vector<int>& covalentAtoms) const;
    void getCovalentMaps(int index, std::vector<std::vector<int> >& covalentLists) const;
    int getMutualInducedMaxIterations() const { return mutualInducedMaxIterations; }
    void setMutualInducedMaxIterations(int n) { mutualInducedMaxIterations = n; }
    double getMutualInducedTargetEpsilon() const { return mutualInducedTargetEpsilon; }
    void setMutualInducedTargetEpsilon(double eps) { mutualInducedTargetEpsilon = eps; }
    void setExtrapolationCoefficients(const std::vector<double>& c) { extrapolationCoefficients = c; }
    const std::vector<double>& getExtrapolationCoefficients() const { return extrapolationCoefficients; }
    double getEwaldErrorTolerance() const { return ewaldErrorTol; }
    void setEwaldErrorTolerance(double tol) { ewaldErrorTol = tol; }
    bool usesPeriodicBoundaryConditions() const override { return nonbondedMethod == PME; }

private:
    struct ParticleInfo {
        int axisType, multipoleAtomZ, multipoleAtomX, multipoleAtomY;
        double charge, polarizability, tholeDamping;
        std::vector<double> molecularDipole;
        std::vector<std::vector<int> > covalentInfo;
    };
    NonbondedMethod nonbondedMethod;
    PolarizationType polarizationType;
    double cutoffDistance, alpha;
    int pmeBSplineOrder, nx, ny, nz;
    int mutualInducedMaxIterations;
    std::vector<double> extrapolationCoefficients;
    double mutualInducedTargetEpsilon, ewaldErrorTol;
    std::vector<ParticleInfo> particles;
};

}  // namespace TholeDipolePlugin
#endif
