/* Minimal stand-in for OpenMM's OpenMMException (a std::exception carrying a
 * message).  Test infrastructure only: lets the reference plugin's physics
 * source compile as a CPU oracle. */
#ifndef TDP_SHIM_OPENMM_EXCEPTION_H_
#define TDP_SHIM_OPENMM_EXCEPTION_H_
#include <exception>
#include <string>
namespace OpenMM {
class OpenMMException : public std::exception {
public:
    explicit OpenMMException(const std::string& message) : message(message) {}
    ~OpenMMException() throw() {}
    const char* what() const throw() { return message.c_str(); }
private:
    std::string message;
};
}  // namespace OpenMM
#endif
