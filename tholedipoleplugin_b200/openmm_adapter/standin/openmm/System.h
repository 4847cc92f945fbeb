/* Stand-in for OpenMM's System (see standin/openmm/Vec3.h): masses, default box, forces. */
#ifndef TDP_STANDIN_OPENMM_SYSTEM_H_
#define TDP_STANDIN_OPENMM_SYSTEM_H_
#include <vector>
#include "openmm/Force.h"
#include "openmm/Vec3.h"
namespace OpenMM {
class System {
public:
    ~System() { for (Force* f : forces) delete f; }
    int addParticle(double mass) { masses.push_back(mass); return (int)masses.size() - 1; }
    int getNumParticles() const { return (int)masses.size(); }
    double getParticleMass(int i) const { return masses[i]; }
    int addForce(Force* f) { forces.push_back(f); return (int)forces.size() - 1; }
    int getNumForces() const { return (int)forces.size(); }
    const Force& getForce(int i) const { return *forces[i]; }
    Force& getForce(int i) { return *forces[i]; }
    void setDefaultPeriodicBoxVectors(const Vec3& a, const Vec3& b, const Vec3& c) { box[0] = a; box[1] = b; box[2] = c; }
    void getDefaultPeriodicBoxVectors(Vec3& a, Vec3& b, Vec3& c) const { a = box[0]; b = box[1]; c = box[2]; }
private:
    std::vector<double> masses;
    std::vector<Force*> forces;
    Vec3 box[3] = {Vec3(2, 0, 0), Vec3(0, 2, 0), Vec3(0, 0, 2)};
};
}  // namespace OpenMM
#endif
