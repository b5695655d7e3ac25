/* Host shim for curand.h (included by the reference's ir.cuh). Test infrastructure only. */
#ifndef XR_REF_SHIM_CURAND_H
#define XR_REF_SHIM_CURAND_H
#include "curand_kernel.h"
#endif
