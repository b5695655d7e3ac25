/* Host shim for curand_kernel.h: only the names the reference's ir.cu
 * mentions (setup_rand, ir.cu:1904-1908).  Test infrastructure only. */
#ifndef XR_REF_SHIM_CURAND_KERNEL_H
#define XR_REF_SHIM_CURAND_KERNEL_H
#include "cuda_runtime.h"
struct curandState { unsigned long long s; };
inline void curand_init(unsigned long long seed, unsigned long long seq, unsigned long long off,
                        curandState *st) {
    st->s = seed ^ (seq * 0x9E3779B97F4A7C15ull) ^ off;
}
inline float curand_uniform(curandState *st) {
    st->s = st->s * 6364136223846793005ull + 1442695040888963407ull;
    return (float)((st->s >> 40) + 1) / 16777217.0f;
}
#endif
