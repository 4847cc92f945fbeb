/* Stand-in for OpenMM's OpenMMException (see standin/openmm/Vec3.h). */
#ifndef TDP_STANDIN_OPENMM_EXCEPTION_H_
#define TDP_STANDIN_OPENMM_EXCEPTION_H_
#include <exception>
#include <string>
namespace OpenMM {
class OpenMMException : public std::exception {
public:
    explicit OpenMMException(const std::string& m) : msg(m) {}
    const char* what() const noexcept override { return msg.c_str(); }
private:
    std::string msg;
};
}  // namespace OpenMM
#endif
