/* Stand-in for OpenMM's Kernel handle (see standin/openmm/KernelImpl.h). */
#ifndef TDP_STANDIN_OPENMM_KERNEL_H_
#define TDP_STANDIN_OPENMM_KERNEL_H_
#include "openmm/KernelImpl.h"
#endif
