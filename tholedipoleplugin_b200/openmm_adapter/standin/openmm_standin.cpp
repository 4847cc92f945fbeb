// Platform registry of the OpenMM stand-in (see standin/openmm/Vec3.h).
#include "openmm/KernelImpl.h"
#include "openmm/internal/ContextImpl.h"

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
}  // namespace OpenMM
