// Platform registry, Context and Force hooks of the OpenMM stand-in (see
// standin/openmm/Vec3.h).
#include "openmm/Context.h"
#include "openmm/KernelImpl.h"
#include "openmm/internal/ContextImpl.h"
#include "openmm/internal/Messages.h"

namespace OpenMM {
static std::vector<Platform*>& registry() {
    static std::vector<Platform*> r;
    return r;
}
void Platform::registerPlatform(Platform* p) { registry().push_back(p); }
int Platform::getNumPlatforms() { return (int)registry().size(); }
Platform& Platform::getPlatform(int i) { return *registry().at(i); }
Platform& Platform::getPlatformByName(const std::string& name) {
    for (Platform* p : registry())
        if (p->getName() == name) return *p;
    throw OpenMMException("There is no registered Platform called \"" + name + "\"");
}
Kernel Platform::createKernel(const std::string& kernel, ContextImpl& context) const {
    auto it = factories.find(kernel);
    if (it == factories.end()) throw OpenMMException("Called createKernel() on a Platform which does not support the requested kernel");
    return Kernel(it->second->createKernelImpl(kernel, *this, context));
}

const std::string Messages::cutoffTooLarge = "The cutoff distance cannot be greater than half the periodic box size.";

ForceImpl* Force::createImpl() const { throw OpenMMException("this Force cannot be placed in a Context"); }
ForceImpl& Force::getImplInContext(Context& context) { return context.getImpl().getForceImpl(*this); }
const ForceImpl& Force::getImplInContext(const Context& context) const {
    return const_cast<Context&>(context).getImpl().getForceImpl(*this);
}
ContextImpl& Force::getContextImpl(Context& context) { return context.getImpl(); }

Context::Context(const System& system, Platform& platform) : impl(new ContextImpl(system, platform)) {
    try {
        impl->initialize();
    } catch (...) {
        delete impl;
        throw;
    }
}
Context::~Context() { delete impl; }
void Context::setPositions(const std::vector<Vec3>& positions) { impl->positions = positions; }
double Context::calcForcesAndEnergy(bool includeForces, bool includeEnergy, int groups) {
    return impl->calcForcesAndEnergy(includeForces, includeEnergy, groups);
}
const std::vector<Vec3>& Context::getForces() const { return impl->forces; }
}  // namespace OpenMM
