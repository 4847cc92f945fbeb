/* Stand-in for OpenMM's Platform (see standin/openmm/KernelImpl.h). */
#ifndef TDP_STANDIN_OPENMM_PLATFORM_H_
#define TDP_STANDIN_OPENMM_PLATFORM_H_
#include "openmm/KernelImpl.h"
#endif
