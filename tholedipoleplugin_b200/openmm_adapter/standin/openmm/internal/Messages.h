/* Stand-in for OpenMM's Messages (see standin/openmm/Vec3.h): shared error texts. */
#ifndef TDP_STANDIN_OPENMM_MESSAGES_H_
#define TDP_STANDIN_OPENMM_MESSAGES_H_
#include <string>
namespace OpenMM {
class Messages {
public:
    static const std::string cutoffTooLarge;
};
}  // namespace OpenMM
#endif
