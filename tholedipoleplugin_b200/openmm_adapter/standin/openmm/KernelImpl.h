/* Stand-ins for OpenMM's KernelImpl, Kernel, KernelFactory and Platform (see
 * standin/openmm/Vec3.h): a named kernel object, and a registry of platforms
 * whose kernel factories create kernels by name. */
#ifndef TDP_STANDIN_OPENMM_KERNELIMPL_H_
#define TDP_STANDIN_OPENMM_KERNELIMPL_H_
#include <map>
#include <memory>
#include <string>
#include <vector>
#include "openmm/OpenMMException.h"
namespace OpenMM {
class Platform;
class ContextImpl;
class KernelImpl {
public:
    KernelImpl(std::string name, const Platform& platform) : name(name), platform(&platform) {}
    virtual ~KernelImpl() {}
    std::string getName() const { return name; }
    const Platform& getPlatform() { return *platform; }
private:
    std::string name;
    const Platform* platform;
};
class Kernel {
public:
    Kernel() {}
    explicit Kernel(KernelImpl* impl) : impl(impl) {}
    template <class T> T& getAs() { return dynamic_cast<T&>(*impl); }
    template <class T> const T& getAs() const { return dynamic_cast<const T&>(*impl); }
    KernelImpl& getImpl() { return *impl; }
private:
    std::shared_ptr<KernelImpl> impl;
};
class KernelFactory {
public:
    virtual ~KernelFactory() {}
    virtual KernelImpl* createKernelImpl(std::string name, const Platform& platform, ContextImpl& context) const = 0;
};
class Platform {
public:
    explicit Platform(std::string name) : name(name) {}
    virtual ~Platform() {}
    const std::string& getName() const { return name; }
    void registerKernelFactory(const std::string& kernel, KernelFactory* factory) { factories[kernel] = factory; }
    // Platform properties (OpenMM's CUDA platform has e.g. "Precision").
    void setPropertyDefaultValue(const std::string& property, const std::string& value) { props[property] = value; }
    std::string getPropertyDefaultValue(const std::string& property) const {
        auto it = props.find(property);
        return it == props.end() ? std::string() : it->second;
    }
    Kernel createKernel(const std::string& kernel, ContextImpl& context) const;
    static void registerPlatform(Platform* p);
    static int getNumPlatforms();
    static Platform& getPlatform(int i);
    static Platform& getPlatformByName(const std::string& name);
private:
    std::string name;
    std::map<std::string, KernelFactory*> factories;
    std::map<std::string, std::string> props;
};
}  // namespace OpenMM
#endif
