/*
 * Per-voxel fiber orientation on the GPU (the reference runs it on the host
 * with Eigen in FP32, direction/src/pca.cu:12-55, inside an OpenMP loop at
 * reconstruct.cu:935-942).
 *
 * One thread per voxel: the 3x3 orientation tensor T = (1/K) sum_k
 * (mu_k S_k)(mu_k S_k)^T is formed and diagonalised in FP64 by cyclic Jacobi
 * rotations (Golub & Van Loan, Matrix Computations, section 8.5); the unit
 * eigenvector of the smallest eigenvalue, signed so that its z >= 0, scaled by
 * mean(mu), is the fiber direction md; evalue_i = lambda_i / sum(lambda).
 * The sweep stops on the same off-diagonal criterion as the oracle.
 */
#include <cuda_runtime.h>

#include "xr_internal.h"
#include "xr_eig3.cuh"
#include "xr_storage.cuh"

namespace xr {
namespace {

template <typename TS>
__global__ void k_orientation(long nvox, int K, const BasisConst *B, const TS *mu, float *md, float *ev) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < nvox; i += (long)gridDim.x * blockDim.x) {
        double T[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, mean = 0.0;
        for (int k = 0; k < K; k++) {
            const double m = (double)ldgf<TS>(mu + (long)k * nvox + i);
            const double s0 = m * B->S[3 * k], s1 = m * B->S[3 * k + 1], s2 = m * B->S[3 * k + 2];
            mean += m;
            T[0] += s0 * s0; T[1] += s0 * s1; T[2] += s0 * s2;
            T[4] += s1 * s1; T[5] += s1 * s2; T[8] += s2 * s2;
        }
        T[3] = T[1]; T[6] = T[2]; T[7] = T[5];
        mean /= K;
#pragma unroll
        for (int a = 0; a < 9; a++) T[a] /= K;
        double w[3], V[9];
        jacobi3(T, w, V);
        /* ascending order, stable: index of the smallest eigenvalue */
        int idx[3] = {0, 1, 2};
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int b = a + 1; b < 3; b++)
                if (w[idx[b]] < w[idx[a]]) { const int t = idx[a]; idx[a] = idx[b]; idx[b] = t; }
        const int c0 = idx[0];
        double v0 = V[c0], v1 = V[3 + c0], v2 = V[6 + c0];
        const double nv = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
        v0 /= nv; v1 /= nv; v2 /= nv;
        const double sg = v2 >= 0 ? 1.0 : -1.0;
        md[i] = (float)(sg * mean * v0);
        md[nvox + i] = (float)(sg * mean * v1);
        md[2 * nvox + i] = (float)(sg * mean * v2);
        if (ev) {
            const double tr = w[0] + w[1] + w[2];
            ev[i] = (float)(w[idx[0]] / tr);
            ev[nvox + i] = (float)(w[idx[1]] / tr);
            ev[2 * nvox + i] = (float)(w[idx[2]] / tr);
        }
    }
}

/* calcAngleFromMD, direction/src/pca.cu:67-83. */
__global__ void k_angle_from_md(long nvox, const float *md, float *angle) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < nvox; i += (long)gridDim.x * blockDim.x) {
        const float m0 = md[i], m1 = md[nvox + i], m2 = md[2 * nvox + i];
        const float r = sqrtf(m1 * m1 + m0 * m0);
        if (m1 < 0.f) {
            angle[i] = atan2f(-m1, -m0);
            angle[nvox + i] = atan2f(r, -m2);
        } else {
            angle[i] = atan2f(m1, m0);
            angle[nvox + i] = atan2f(r, m2);
        }
    }
}

/* directionNormalization, direction/src/pca.cu:85-106 (threshold 0.65). */
__global__ void k_direction_normalization(long nvox, float *md) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < nvox; i += (long)gridDim.x * blockDim.x) {
        const float x = md[i], y = md[nvox + i], z = md[2 * nvox + i];
        const float n = sqrtf(x * x + y * y + z * z);
        if (n > 0.65f) {
            md[i] = x / n; md[nvox + i] = y / n; md[2 * nvox + i] = z / n;
        } else {
            md[i] = 0.f; md[nvox + i] = 0.f; md[2 * nvox + i] = 0.f;
        }
    }
}

int grid_for(long n, int threads) {
    long b = (n + threads - 1) / threads;
    if (b > 148 * 16) b = 148 * 16;
    return (int)(b < 1 ? 1 : b);
}

}  // namespace

cudaError_t launch_orientation(long nvox, int K, const BasisConst *d_basis, const void *mu, float *md, float *ev,
                               int storage, cudaStream_t s) {
    const int gr = grid_for(nvox, 128);
    if (storage == kBF16) k_orientation<<<gr, 128, 0, s>>>(nvox, K, d_basis, (const __nv_bfloat16 *)mu, md, ev);
    else if (storage == kF16) k_orientation<<<gr, 128, 0, s>>>(nvox, K, d_basis, (const __half *)mu, md, ev);
    else k_orientation<<<gr, 128, 0, s>>>(nvox, K, d_basis, (const float *)mu, md, ev);
    return cudaGetLastError();
}

cudaError_t launch_angle_from_md(long nvox, const float *md, float *angle, cudaStream_t s) {
    k_angle_from_md<<<grid_for(nvox, 256), 256, 0, s>>>(nvox, md, angle);
    return cudaGetLastError();
}

cudaError_t launch_direction_normalization(long nvox, float *md, cudaStream_t s) {
    k_direction_normalization<<<grid_for(nvox, 256), 256, 0, s>>>(nvox, md);
    return cudaGetLastError();
}

}  // namespace xr
