/*
 * Gather of the 2 x 2 texels of a bilinear footprint from a 2D-layered
 * texture (tld4, PTX ISA "tld4"): used by the back-projections that read
 * ratio images or filtered projections through the texture unit.
 */
#ifndef XR_TEX_CUH
#define XR_TEX_CUH

#include <cuda_runtime.h>

namespace xr {

/* The 2 x 2 texels around unnormalised coordinates (x, y) of layer `layer`
 * (component r): (T[y1][x0], T[y1][x1], T[y0][x1], T[y0][x0]) with
 * x0 = floor(x - 0.5), x1 = x0 + 1 and likewise y; coordinates outside the
 * layer clamp to its edge.  With x = i + 1 and y = j + 1 (exact small
 * integers) the footprint is texels i, i + 1 and j, j + 1 exactly. */
__device__ __forceinline__ float4 gather_a2d(cudaTextureObject_t t, int layer, float x, float y) {
    float4 r;
    asm("tld4.r.a2d.v4.f32.f32 {%0, %1, %2, %3}, [%4, {%5, %6, %7, %7}];"
        : "=f"(r.x), "=f"(r.y), "=f"(r.z), "=f"(r.w)
        : "l"(t), "r"(layer), "f"(x), "f"(y));
    return r;
}

}  // namespace xr

#endif
