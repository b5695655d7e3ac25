/*
 * Storage types of volumes and sinograms: FP32, BF16 or FP16 in HBM, FP32 in
 * every arithmetic operation.  Loads widen exactly; stores round to nearest
 * even.  The projection / ratio images, normaliser and accumulators stay FP32.
 */
#ifndef XR_STORAGE_CUH
#define XR_STORAGE_CUH

#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace xr {

enum Storage { kF32 = 0, kBF16 = 1, kF16 = 2 };

template <typename T>
__device__ __forceinline__ float ldf(const T *p);
template <>
__device__ __forceinline__ float ldf<float>(const float *p) { return *p; }
template <>
__device__ __forceinline__ float ldf<__nv_bfloat16>(const __nv_bfloat16 *p) { return __bfloat162float(*p); }
template <>
__device__ __forceinline__ float ldf<__half>(const __half *p) { return __half2float(*p); }

/* read-only path (non-coherent cache) */
template <typename T>
__device__ __forceinline__ float ldgf(const T *p);
template <>
__device__ __forceinline__ float ldgf<float>(const float *p) { return __ldg(p); }
template <>
__device__ __forceinline__ float ldgf<__nv_bfloat16>(const __nv_bfloat16 *p) { return __bfloat162float(__ldg(p)); }
template <>
__device__ __forceinline__ float ldgf<__half>(const __half *p) { return __half2float(__ldg(p)); }

template <typename T>
__device__ __forceinline__ void stf(T *p, float v);
template <>
__device__ __forceinline__ void stf<float>(float *p, float v) { *p = v; }
template <>
__device__ __forceinline__ void stf<__nv_bfloat16>(__nv_bfloat16 *p, float v) { *p = __float2bfloat16_rn(v); }
template <>
__device__ __forceinline__ void stf<__half>(__half *p, float v) { *p = __float2half_rn(v); }

inline size_t storage_bytes(int storage) { return storage == kF32 ? 4 : 2; }

}  // namespace xr

#endif
