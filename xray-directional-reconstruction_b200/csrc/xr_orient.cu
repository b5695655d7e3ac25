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
#include "xr_orth.cuh"
#include "xr_storage.cuh"

namespace xr {
namespace {

template <typename TS>
__global__ void k_orientation(long nvox, long i0, long i1, int K, const BasisConst *B, const TS *mu, float *md,
                              float *ev) {
    for (long i = i0 + (long)blockIdx.x * blockDim.x + threadIdx.x; i < i1; i += (long)gridDim.x * blockDim.x) {
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
        /* the reference's std::sqrt(m1 * m1 + m0 * m0), rounded op by op */
        const float r = __fsqrt_rn(__fadd_rn(__fmul_rn(m1, m1), __fmul_rn(m0, m0)));
        if (m1 < 0.f) {
            angle[i] = atan2f(-m1, -m0);
            angle[nvox + i] = atan2f(r, -m2);
        } else {
            angle[i] = atan2f(m1, m0);
            angle[nvox + i] = atan2f(r, m2);
        }
    }
}

/* directionNormalization, direction/src/pca.cu:85-106 (threshold 0.65): the
 * length and the quotients rounded op by op as the reference's host code, so
 * the threshold decision and the results are its own bit for bit. */
__global__ void k_direction_normalization(long nvox, float *md) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < nvox; i += (long)gridDim.x * blockDim.x) {
        const float x = md[i], y = md[nvox + i], z = md[2 * nvox + i];
        const float n = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z)));
        if (n > 0.65f) {
            md[i] = __fdiv_rn(x, n); md[nvox + i] = __fdiv_rn(y, n); md[2 * nvox + i] = __fdiv_rn(z, n);
        } else {
            md[i] = 0.f; md[nvox + i] = 0.f; md[2 * nvox + i] = 0.f;
        }
    }
}

/* Vector3X::normalize (reconstruct/include/vec.h:94-106). */
__device__ __forceinline__ void normalize3(float v[3]) {
    const float l = sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (l > 1e-8f) {
        v[0] /= l; v[1] /= l; v[2] /= l;
    } else {
        v[0] = v[1] = v[2] = 0.f;
    }
}

/* calcNormalVectorThreeDirec, ir.cu:856-974: the plane normal
 * (mu0 S0 - mu1' S1) x (mu0 S0 - mu2' S2) (signs of mu1, mu2 by rot), turned
 * by the voxel's current rotation, z >= 0, becomes the new (phi, cos theta);
 * loss = |(R e_z) x normal|. */
__global__ void k_normal_three(long nvox, const BasisConst *B, const float *vol, float *coef, float *loss, int rot_all,
                               const float *est) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < nvox; i += (long)gridDim.x * blockDim.x) {
        int rot = rot_all;
        if (est) {   /* calcNormalVectorThreeDirecWithEst (ir.cu:976-1071): pattern from estimate plane 1 */
            const float r = est[nvox + i];
            rot = r < 0.5f ? 0 : (r < 1.5f ? 1 : (r < 2.5f ? 2 : 3));
        }
        float R[9];
        orth_rotation(coef, (size_t)nvox, (size_t)i, R);
        const float mu0 = vol[i], m1 = vol[nvox + i], m2 = vol[2 * nvox + i];
        float mu1 = m1, mu2 = m2;
        if (rot == 1) { mu1 = -m1; }
        else if (rot == 2) { mu1 = -m1; mu2 = -m2; }
        else if (rot == 3) { mu2 = -m2; }
        float v1[3], v2[3];
#pragma unroll
        for (int j = 0; j < 3; j++) {
            v1[j] = mu0 * B->S[j] - mu1 * B->S[3 + j];
            v2[j] = mu0 * B->S[j] - mu2 * B->S[6 + j];
        }
        float n[3] = {v1[1] * v2[2] - v1[2] * v2[1], v1[2] * v2[0] - v1[0] * v2[2], v1[0] * v2[1] - v1[1] * v2[0]};
        normalize3(n);
        float r[3] = {R[0] * n[0] + R[1] * n[1] + R[2] * n[2], R[3] * n[0] + R[4] * n[1] + R[5] * n[2],
                      R[6] * n[0] + R[7] * n[1] + R[8] * n[2]};
        if (r[2] < 0.f) { r[0] = -r[0]; r[1] = -r[1]; r[2] = -r[2]; }
        normalize3(r);
        /* (R e_z) x r */
        const float be0 = R[2], be1 = R[5], be2 = R[8];
        const float dx = be1 * r[2] - be2 * r[1], dy = be2 * r[0] - be0 * r[2], dz = be0 * r[1] - be1 * r[0];
        loss[i] = sqrtf(dx * dx + dy * dy + dz * dz);
        /* e_z x r = (-r1, r0, 0) */
        coef[i] = atan2f(r[0], -r[1]);
        coef[nvox + i] = r[2];
    }
}

/* meanFiltFiberMD, ir.cu:1304-1363, for 2 <= x, y, z < N-2: the 27
 * neighbours of the centre c signed by their agreement with it (c.o > 0
 * added, < 0 subtracted, weight w), normalised (zero -> e_z), scaled to |c|. */
__global__ void k_md_filter(int N, const float *md, float *out, float w) {
    const long n3 = (long)N * N * N, M = N - 4;
    const long nint = M > 0 ? M * M * M : 0;
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < nint; t += (long)gridDim.x * blockDim.x) {
        const long x = 2 + t % M, y = 2 + (t / M) % M, z = 2 + t / (M * M);
        const long c = x + N * (y + (long)N * z);
        const float c0 = md[c], c1 = md[n3 + c], c2 = md[2 * n3 + c];
        const float len = sqrtf(c0 * c0 + c1 * c1 + c2 * c2);
        float v[3] = {0.f, 0.f, 0.f};
        for (int i = -1; i < 2; i++)
            for (int j = -1; j < 2; j++)
                for (int k = -1; k < 2; k++) {
                    const long o = (x - i) + N * ((y - j) + (long)N * (z - k));
                    const float o0 = md[o], o1 = md[n3 + o], o2 = md[2 * n3 + o];
                    /* products and sums rounded one by one, as the reference's FP32
                     * code: the sign of d decides between adding and subtracting */
                    const float d = __fadd_rn(__fadd_rn(__fmul_rn(c0, o0), __fmul_rn(c1, o1)), __fmul_rn(c2, o2));
                    if (d > 0.f) {
                        v[0] = __fadd_rn(v[0], __fmul_rn(w, o0));
                        v[1] = __fadd_rn(v[1], __fmul_rn(w, o1));
                        v[2] = __fadd_rn(v[2], __fmul_rn(w, o2));
                    } else if (d < -0.f) {
                        v[0] = __fsub_rn(v[0], __fmul_rn(w, o0));
                        v[1] = __fsub_rn(v[1], __fmul_rn(w, o1));
                        v[2] = __fsub_rn(v[2], __fmul_rn(w, o2));
                    }
                }
        normalize3(v);
        if (sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) < 1e-8f) { v[0] = 0.f; v[1] = 0.f; v[2] = 1.f; }
        out[c] = len * v[0];
        out[n3 + c] = len * v[1];
        out[2 * n3 + c] = len * v[2];
    }
}

/* calcMainDirection (ir.cu:624-710; sign pattern iter) or calcMDWithEst
 * (:712-789; pattern from estimate plane 1): the in-plane magnitudes of mu
 * (planes 0..2) after removing its (+-1, +-1, +-1) component, signed, times
 * half the sum of mu, rotated by the voxel's previous main direction, z >= 0. */
__global__ void k_main_direction(int N, const float *vol, float *md, const float *est, int iter) {
    const long n3 = (long)N * N * N;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += (long)gridDim.x * blockDim.x) {
        const float mu0 = vol[i], mu1 = vol[n3 + i], mu2 = vol[2 * n3 + i];
        float n0 = 0.f, n1 = 0.f, n2 = 0.f;
        if (mu2 + mu1 - mu0 < 0.f) { n0 = -1.f; n1 = 1.f; n2 = 1.f; }
        else if (mu0 + mu2 - mu1 < 0.f) { n0 = 1.f; n1 = -1.f; n2 = 1.f; }
        else if (mu1 + mu0 - mu2 < 0.f) { n0 = 1.f; n1 = 1.f; n2 = -1.f; }
        /* rounded one by one: the square roots below amplify any difference
         * in these near-cancelling sums */
        const float co = __fdiv_rn(__fadd_rn(__fadd_rn(__fmul_rn(mu0, n0), __fmul_rn(mu1, n1)), __fmul_rn(mu2, n2)), 3.f);
        const float v0 = __fsub_rn(mu0, __fmul_rn(co, n0)), v1 = __fsub_rn(mu1, __fmul_rn(co, n1));
        const float v2 = __fsub_rn(mu2, __fmul_rn(co, n2));
        float fx = sqrtf(0.5f * fabsf(v2 + v1 - v0)), fy = sqrtf(0.5f * fabsf(v0 + v2 - v1));
        const float fz = sqrtf(0.5f * fabsf(v1 + v0 - v2));
        int sgn = iter;
        if (est) {
            const float r = est[n3 + i];
            sgn = r < 0.5f ? 0 : (r < 1.5f ? 1 : (r < 2.5f ? 2 : 3));
        }
        if (sgn == 1) fx = -fx;
        else if (sgn == 2) { fx = -fx; fy = -fy; }
        else if (sgn == 3) fy = -fy;
        const float mean = (mu0 + mu1 + mu2) / 2.0f;
        const float m[3] = {mean * fx, mean * fy, mean * fz};
        float R[9];
        md_rotation(md, (size_t)n3, (size_t)i, R);
        float r[3] = {R[0] * m[0] + R[1] * m[1] + R[2] * m[2], R[3] * m[0] + R[4] * m[1] + R[5] * m[2],
                      R[6] * m[0] + R[7] * m[1] + R[8] * m[2]};
        if (r[2] < 0.f) { r[0] = -r[0]; r[1] = -r[1]; r[2] = -r[2]; }
        md[i] = r[0];
        md[n3 + i] = r[1];
        md[2 * n3 + i] = r[2];
    }
}

/* updateEstimation, ir.cu:791-844: loss = mu2^2 + (1 - lo/hi)^2 of the first
 * two channels; where it beats estimate plane 0, planes 0/1 <- (loss, iter). */
__global__ void k_update_estimation(int N, const float *vol, float *est, int iter) {
    const long n3 = (long)N * N * N;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += (long)gridDim.x * blockDim.x) {
        const float mu0 = vol[i], mu1 = vol[n3 + i], mu2 = vol[2 * n3 + i];
        const float lo = mu0 < mu1 ? mu0 : mu1, hi = mu0 < mu1 ? mu1 : mu0;
        const float q = __fsub_rn(1.0f, __fdiv_rn(lo, hi));
        const float loss = __fadd_rn(__fmul_rn(mu2, mu2), __fmul_rn(q, q));
        if (loss < est[i]) {
            est[i] = loss;
            est[n3 + i] = (float)iter;
        }
    }
}

/* meanFiltFiber, ir.cu:1231-1302, for 1 <= x, y, z < N-1: each neighbour's
 * direction from its (phi, cos theta) planes as mu (sin t cos(phi - pi/2),
 * sin t sin(phi - pi/2), cos t), mu the sum of its three coefficients; the
 * pairs (i, 26 - i) within 60 degrees of the centre (|dot| > 0.5) added
 * signed to it (weight w), normalised, z >= 0, back to (phi, cos theta). */
__global__ void k_coef_filter(int N, const float *coef, const float *vol, float *out, float w) {
    const long n3 = (long)N * N * N, M = N - 2;
    const long nint = M > 0 ? M * M * M : 0;
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < nint; t += (long)gridDim.x * blockDim.x) {
        const long x = 1 + t % M, y = 1 + (t / M) % M, z = 1 + t / (M * M);
        float nv[27][3];
        int cnt = 0;
        for (int i = -1; i < 2; i++)
            for (int j = -1; j < 2; j++)
                for (int k = -1; k < 2; k++) {
                    const long o = (x - i) + N * ((y - j) + (long)N * (z - k));
                    const float ct = coef[n3 + o];
                    const float st = sqrtf(1.f - ct * ct);
                    const float phi = __double2float_rn(-1.5707963267948966 + (double)coef[o]);
                    const float mu = __fadd_rn(__fadd_rn(vol[o], vol[n3 + o]), vol[2 * n3 + o]);
                    nv[cnt][0] = mu * (st * cosf(phi));
                    nv[cnt][1] = mu * (st * sinf(phi));
                    nv[cnt][2] = mu * ct;
                    cnt++;
                }
        float c[3] = {nv[13][0], nv[13][1], nv[13][2]};
        for (int i = 0; i < 13; i++) {
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const float *a = nv[h ? 26 - i : i];
                const float d = __fadd_rn(__fadd_rn(__fmul_rn(a[0], nv[13][0]), __fmul_rn(a[1], nv[13][1])),
                                          __fmul_rn(a[2], nv[13][2]));
                if (d > 0.5f) {
                    c[0] = __fadd_rn(c[0], __fmul_rn(w, a[0]));
                    c[1] = __fadd_rn(c[1], __fmul_rn(w, a[1]));
                    c[2] = __fadd_rn(c[2], __fmul_rn(w, a[2]));
                } else if (d < -0.5f) {
                    c[0] = __fsub_rn(c[0], __fmul_rn(w, a[0]));
                    c[1] = __fsub_rn(c[1], __fmul_rn(w, a[1]));
                    c[2] = __fsub_rn(c[2], __fmul_rn(w, a[2]));
                }
            }
        }
        normalize3(c);
        if (c[2] < 0.f) { c[0] = -c[0]; c[1] = -c[1]; c[2] = -c[2]; }
        const long ci = x + N * (y + (long)N * z);
        out[ci] = atan2f(c[0], -c[1]);   /* e_z x c = (-c1, c0, 0) */
        out[n3 + ci] = c[2];
    }
}

/* updateEstimationByCoef, ir.cu:1073-1120: the plane normal of the three
 * coefficients (no signs), z >= 0; where its cosine to e_z exceeds estimate
 * plane 0, planes 0/1 <- (cosine, iter). */
__global__ void k_update_estimation_coef(long nvox, const BasisConst *B, const float *vol, float *est, int iter) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < nvox; i += (long)gridDim.x * blockDim.x) {
        const float mu0 = vol[i], mu1 = vol[nvox + i], mu2 = vol[2 * nvox + i];
        float v1[3], v2[3];
#pragma unroll
        for (int j = 0; j < 3; j++) {
            v1[j] = mu0 * B->S[j] - mu1 * B->S[3 + j];
            v2[j] = mu0 * B->S[j] - mu2 * B->S[6 + j];
        }
        float n[3] = {v1[1] * v2[2] - v1[2] * v2[1], v1[2] * v2[0] - v1[0] * v2[2], v1[0] * v2[1] - v1[1] * v2[0]};
        normalize3(n);
        if (n[2] < 0.f) { n[0] = -n[0]; n[1] = -n[1]; n[2] = -n[2]; }
        normalize3(n);
        if (n[2] > est[i]) {
            est[i] = n[2];
            est[nvox + i] = (float)iter;
        }
    }
}

__global__ void k_fill(long n, float *p, float value) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) p[i] = value;
}

int grid_for(long n, int threads) {
    long b = (n + threads - 1) / threads;
    if (b > 148 * 16) b = 148 * 16;
    return (int)(b < 1 ? 1 : b);
}

}  // namespace

cudaError_t launch_orientation_range(long nvox, long i0, long i1, int K, const BasisConst *d_basis, const void *mu,
                                     float *md, float *ev, int storage, cudaStream_t s) {
    if (i0 < 0) i0 = 0;
    if (i1 > nvox) i1 = nvox;
    if (i1 <= i0) return cudaSuccess;
    const int gr = grid_for(i1 - i0, 128);
    if (storage == kBF16)
        k_orientation<<<gr, 128, 0, s>>>(nvox, i0, i1, K, d_basis, (const __nv_bfloat16 *)mu, md, ev);
    else if (storage == kF16)
        k_orientation<<<gr, 128, 0, s>>>(nvox, i0, i1, K, d_basis, (const __half *)mu, md, ev);
    else
        k_orientation<<<gr, 128, 0, s>>>(nvox, i0, i1, K, d_basis, (const float *)mu, md, ev);
    return cudaGetLastError();
}

cudaError_t launch_orientation(long nvox, int K, const BasisConst *d_basis, const void *mu, float *md, float *ev,
                               int storage, cudaStream_t s) {
    return launch_orientation_range(nvox, 0, nvox, K, d_basis, mu, md, ev, storage, s);
}

cudaError_t launch_md_filter(int N, const float *md, float *out, float coef, cudaStream_t s) {
    const long M = N - 4;
    if (M <= 0) return cudaSuccess;
    k_md_filter<<<grid_for(M * M * M, 256), 256, 0, s>>>(N, md, out, coef);
    return cudaGetLastError();
}

cudaError_t launch_main_direction(int N, const float *vol, float *md, const float *est, int iter, cudaStream_t s) {
    k_main_direction<<<grid_for((long)N * N * N, 256), 256, 0, s>>>(N, vol, md, est, iter);
    return cudaGetLastError();
}

cudaError_t launch_update_estimation(int N, const float *vol, float *est, int iter, cudaStream_t s) {
    k_update_estimation<<<grid_for((long)N * N * N, 256), 256, 0, s>>>(N, vol, est, iter);
    return cudaGetLastError();
}

cudaError_t launch_fill(long n, float *p, float value, cudaStream_t s) {
    k_fill<<<grid_for(n, 256), 256, 0, s>>>(n, p, value);
    return cudaGetLastError();
}

cudaError_t launch_coef_filter(int N, const float *coef, const float *vol, float *out, float w, cudaStream_t s) {
    const long M = N - 2;
    if (M <= 0) return cudaSuccess;
    k_coef_filter<<<grid_for(M * M * M, 128), 128, 0, s>>>(N, coef, vol, out, w);
    return cudaGetLastError();
}

cudaError_t launch_update_estimation_coef(long nvox, const BasisConst *d_basis, const float *vol, float *est, int iter,
                                          cudaStream_t s) {
    k_update_estimation_coef<<<grid_for(nvox, 256), 256, 0, s>>>(nvox, d_basis, vol, est, iter);
    return cudaGetLastError();
}

cudaError_t launch_normal_three(long nvox, const BasisConst *d_basis, const float *vol, float *coef, float *loss,
                                int rot, cudaStream_t s, const float *est) {
    k_normal_three<<<grid_for(nvox, 256), 256, 0, s>>>(nvox, d_basis, vol, coef, loss, rot, est);
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
