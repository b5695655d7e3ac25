/*
 * Storage types of volumes and sinograms: FP32, BF16 or FP16 in HBM, FP32 in
 * every arithmetic operation.  Loads widen exactly; stores round to nearest
 * even.  The projection / ratio images, normaliser and accumulators stay FP32.
 */
#ifndef XR_STORAGE_CUH
#define XR_STORAGE_CUH

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

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

/* 32-bit integer mixer ("lowbias32", from C. Wellons' public-domain hash
 * prospector). */
__device__ __forceinline__ uint32_t mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

/* Store of an iterative update.  16-bit types with sr != 0 round
 * stochastically: up with probability (v - lo) / (hi - lo) between the two
 * neighbours lo <= v <= hi, so updates smaller than half a unit in the last
 * place still move the stored value in expectation (nearest rounding
 * returns them unchanged and the iteration stalls).  The uniform draw is a
 * hash of the element index and the FP32 value: deterministic, and fresh
 * whenever the value changes.  BF16 adds the draw's top 16 bits below the
 * kept half of the FP32 pattern (3 % faster back-projection than the
 * comparison form FP16 keeps). */
template <typename T>
__device__ __forceinline__ void stu(T *p, float v, uint32_t key, int sr);
template <>
__device__ __forceinline__ void stu<float>(float *p, float v, uint32_t, int) { *p = v; }
template <>
__device__ __forceinline__ void stu<__nv_bfloat16>(__nv_bfloat16 *p, float v, uint32_t key, int sr) {
    if (!sr) { *p = __float2bfloat16_rn(v); return; }
    /* BF16 is the top half of the FP32 pattern: 16 uniform bits added below
     * it carry into the kept half with probability (low half) / 2^16, i.e.
     * the magnitude rounds up with probability (|v| - |lo|) / (|hi| - |lo|) */
    const uint32_t b = __float_as_uint(v);
    if ((b & 0x7F800000u) == 0x7F800000u) { *p = __float2bfloat16_rn(v); return; }   /* inf, NaN */
    const uint32_t h = mix32(b ^ (key * 0x9E3779B9u));
    *p = __ushort_as_bfloat16((unsigned short)((b + (h >> 16)) >> 16));
}
template <>
__device__ __forceinline__ void stu<__half>(__half *p, float v, uint32_t key, int sr) {
    if (!sr) { *p = __float2half_rn(v); return; }
    const __half lo = __float2half_rd(v), hi = __float2half_ru(v);
    const float flo = __half2float(lo), fhi = __half2float(hi);
    const float t = (float)(mix32(__float_as_uint(v) ^ (key * 0x9E3779B9u)) >> 8) * 5.9604645e-08f;
    *p = (fhi != flo && t * (fhi - flo) < (v - flo)) ? hi : lo;
}

/* Pairs of consecutive elements (the first at an even index): one 64-bit
 * (FP32) or 32-bit (16-bit types) access. */
template <typename T>
__device__ __forceinline__ float2 ld2(const T *p);
template <>
__device__ __forceinline__ float2 ld2<float>(const float *p) { return *reinterpret_cast<const float2 *>(p); }
template <>
__device__ __forceinline__ float2 ld2<__nv_bfloat16>(const __nv_bfloat16 *p) {
    return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(p));
}
template <>
__device__ __forceinline__ float2 ld2<__half>(const __half *p) {
    return __half22float2(*reinterpret_cast<const __half2 *>(p));
}

/* stu of two consecutive elements with their own keys, one store. */
template <typename T>
__device__ __forceinline__ void stu2(T *p, float v0, float v1, uint32_t k0, uint32_t k1, int sr);
template <>
__device__ __forceinline__ void stu2<float>(float *p, float v0, float v1, uint32_t, uint32_t, int) {
    *reinterpret_cast<float2 *>(p) = make_float2(v0, v1);
}
template <typename T>
__device__ __forceinline__ void stu2(T *p, float v0, float v1, uint32_t k0, uint32_t k1, int sr) {
    T r[2];
    stu<T>(&r[0], v0, k0, sr);
    stu<T>(&r[1], v1, k1, sr);
    uint32_t w;
    memcpy(&w, r, sizeof(w));
    *reinterpret_cast<uint32_t *>(p) = w;
}
/* BF16 pairs draw once: one hash of the first element's index and both FP32
 * values gives 32 uniform bits, the top 16 rounding the first element and
 * the bottom 16 the second (each added below the kept half, as in stu), so
 * the pair costs one mixer instead of two.  Infinities and NaNs take the
 * per-element path. */
template <>
__device__ __forceinline__ void stu2<__nv_bfloat16>(__nv_bfloat16 *p, float v0, float v1, uint32_t k0, uint32_t k1,
                                                    int sr) {
    const uint32_t b0 = __float_as_uint(v0), b1 = __float_as_uint(v1);
    if (!sr || (b0 & 0x7F800000u) == 0x7F800000u || (b1 & 0x7F800000u) == 0x7F800000u) {
        __nv_bfloat16 r[2];
        stu<__nv_bfloat16>(&r[0], v0, k0, sr);
        stu<__nv_bfloat16>(&r[1], v1, k1, sr);
        uint32_t w;
        memcpy(&w, r, sizeof(w));
        *reinterpret_cast<uint32_t *>(p) = w;
        return;
    }
    const uint32_t h = mix32(b0 ^ ((b1 << 16) | (b1 >> 16)) ^ (k0 * 0x9E3779B9u));
    const uint32_t w0 = (b0 + (h >> 16)) >> 16, w1 = (b1 + (h & 0xFFFFu)) >> 16;
    *reinterpret_cast<uint32_t *>(p) = (w0 & 0xFFFFu) | (w1 << 16);
}

}  // namespace xr

#endif
