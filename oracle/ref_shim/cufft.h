/*
 * Stand-in for cufft.h in the host shim build (TEST INFRASTRUCTURE ONLY): the
 * reference's fdk.cuh declares a cuFFT-based helper (the Hilbert variant,
 * outside the built slice); only its complex type is needed to parse that
 * declaration.  Nothing here is called.
 */
#ifndef XR_REF_SHIM_CUFFT_H
#define XR_REF_SHIM_CUFFT_H

typedef struct {
    float x, y;
} cufftComplex;
typedef int cufftHandle;

#endif
