/*
 * Orientation-parametrised XTT (the reference's forwardOrth / backwardOrth,
 * reconstruct/src/ir.cu:294-423, and forwardOrthByMD / backwardOrthByMD,
 * :154-292): every voxel's scattering basis is rotated by its own Rodrigues
 * rotation, built from two coefficient planes (phi, cos theta) as
 * rodriguesRotation(cos phi, sin phi, 0, cos theta, sqrt(1 - cos^2 theta)), or
 * from the voxel's main direction m (ir.cu:597-623).  With S' = R S_k the weight of
 * channel k stays (|B x S'| |S' . G|)^2 = (S' . G)^2 (|S'|^2 - (B . S')^2),
 * so the projectors keep their quadratic-form structure with per-voxel
 * g_k = (S' . G)^2, |S'|^2 and S' S'^T.
 */
#ifndef XR_ORTH_CUH
#define XR_ORTH_CUH

#include "xr_internal.h"
#include "xr_storage.cuh"

namespace xr {

/* rodriguesRotation (ir.cu:597-623) about (x, y, 0) normalised, by the angle
 * of cosine ct / sine sn; identity when |(x, y)| < 1e-8. */
__device__ __forceinline__ void rodrigues_xy(float x, float y, float ct, float sn, float R[9]) {
    const float l = sqrtf(x * x + y * y);
    if (l < 1e-8f) {
#pragma unroll
        for (int i = 0; i < 9; i++) R[i] = (i % 4 == 0) ? 1.f : 0.f;
        return;
    }
    const float nx = x / l, ny = y / l, nz = 0.0f, oc = 1.0f - ct;
    R[0] = oc * nx * nx + ct;      R[1] = oc * nx * ny - nz * sn; R[2] = oc * nx * nz + ny * sn;
    R[3] = oc * nx * ny + nz * sn; R[4] = oc * ny * ny + ct;      R[5] = oc * ny * nz - nx * sn;
    R[6] = oc * nx * nz - ny * sn; R[7] = oc * ny * nz + nx * sn; R[8] = oc * nz * nz + ct;
}

/* R (row-major) of voxel idx; coef holds the phi plane then the cos plane. */
__device__ __forceinline__ void orth_rotation(const float *coef, size_t n3, size_t idx, float R[9]) {
    const float phi = __ldg(coef + idx), ct = __ldg(coef + n3 + idx);
    rodrigues_xy(cosf(phi), sinf(phi), ct, sqrtf(1.0f - ct * ct), R);
}

/* R of voxel idx from its main direction m (three planes), as
 * forwardOrthByMD / backwardOrthByMD (ir.cu:183-189, :262-268): about
 * (-m1, m0, 0) by the angle of cosine m2 / |m|. */
__device__ __forceinline__ void md_rotation(const float *md, size_t n3, size_t idx, float R[9]) {
    const float m0 = __ldg(md + idx), m1 = __ldg(md + n3 + idx), m2 = __ldg(md + 2 * n3 + idx);
    const float l3 = sqrtf(m0 * m0 + m1 * m1 + m2 * m2);
    rodrigues_xy(-m1, m0, m2 / l3, sqrtf(m0 * m0 + m1 * m1) / l3, R);
}

/* The rotation source of the orientation-parametrised projectors:
 * kind 0 (phi, cos theta) planes, kind 1 main-direction planes. */
__device__ __forceinline__ void src_rotation(const float *coef, int kind, size_t n3, size_t idx, float R[9]) {
    if (kind) md_rotation(coef, n3, idx, R);
    else orth_rotation(coef, n3, idx, R);
}

/* S' = R S_k */
__device__ __forceinline__ void orth_basis(const BasisConst *B, int k, const float R[9], float S[3]) {
    const float s0 = B->S[3 * k], s1 = B->S[3 * k + 1], s2 = B->S[3 * k + 2];
    S[0] = R[0] * s0 + R[1] * s1 + R[2] * s2;
    S[1] = R[3] * s0 + R[4] * s1 + R[5] * s2;
    S[2] = R[6] * s0 + R[7] * s1 + R[8] * s2;
}

/* Forward moments of one voxel and axis with the rotated basis:
 * a0 = sc sum_k g'_k |S'|^2 mu_k, M = sc sum_k g'_k mu_k S' S'^T stored as
 * (xx, yy, zz, 2xy, 2xz, 2yz). */
template <typename T>
__device__ __forceinline__ void orth_moments(const BasisConst *B, int cond, int K, float sc, const T *vol,
                                             const float *coef, int kind, size_t idx, size_t n3, float &a0,
                                             float mm[6]) {
    float R[9];
    src_rotation(coef, kind, n3, idx, R);
    const float G0 = B->G[3 * cond], G1 = B->G[3 * cond + 1], G2 = B->G[3 * cond + 2];
    a0 = 0.f;
#pragma unroll
    for (int e = 0; e < 6; e++) mm[e] = 0.f;
    for (int k = 0; k < K; k++) {
        float S[3];
        orth_basis(B, k, R, S);
        const float h = S[0] * G0 + S[1] * G1 + S[2] * G2;
        const float mu = ldgf<T>(vol + idx + (size_t)k * n3) * (h * h * sc);
        a0 = fmaf(S[0] * S[0] + S[1] * S[1] + S[2] * S[2], mu, a0);
        mm[0] = fmaf(mu * S[0], S[0], mm[0]);
        mm[1] = fmaf(mu * S[1], S[1], mm[1]);
        mm[2] = fmaf(mu * S[2], S[2], mm[2]);
        mm[3] = fmaf(2.f * mu * S[0], S[1], mm[3]);
        mm[4] = fmaf(2.f * mu * S[0], S[2], mm[4]);
        mm[5] = fmaf(2.f * mu * S[1], S[2], mm[5]);
    }
}

}  // namespace xr

#endif
