/*
 * Regularisers of the reconstruction, on the GPU: total-variation denoising
 * by ADMM (the reference's totalVariationMinimized, solver/src/tvmin.cpp:6-98,
 * host Eigen) and the quadratic-form tensor filter that applies it to the
 * orientation tensor (quadlicFormFilterCPU, reconstruct/src/quadfilt.cpp:11-134,
 * host Eigen).
 *
 * TV-ADMM, for a volume x0 of X x Y x Z voxels (x fastest):
 *   F: forward differences (x+e_c) - x, c = x, y, z, defined only at voxels
 *      with x < X-1 and y < Y-1 and z < Z-1 (all three rows, as the
 *      reference's triplet loop builds them; other rows are zero);
 *   y = u = 1 (3N each, as the reference initialises them);
 *   repeat iter times:
 *      solve (I + rho F^T F) x = F^T (rho y - u) + x0
 *      y = soft(F x + u / rho, lambda / rho);  u += rho (F x - y).
 * The reference solves with Eigen's BiCGSTAB to its default tolerance
 * (machine epsilon, up to 2N iterations).  The matrix is symmetric positive
 * definite, so here it is conjugate gradients, matrix-free (F^T F is a
 * 7-point stencil masked by the definition set of F), FP32 vectors, FP64
 * inner products and step scalars kept on the device, warm-started from the
 * previous x, stopped at ||r|| <= tol ||b||.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/xr.h"
#include "xr_eig3.cuh"

namespace xr {
namespace {

constexpr int kThreads = 256;

struct Dims {
    int X, Y, Z;
    long N;
};

__device__ __forceinline__ bool f_row(int x, int y, int z, const Dims &d) {
    return x < d.X - 1 && y < d.Y - 1 && z < d.Z - 1;
}

/* (I + rho F^T F) p; also returns its dot with p (FP64, block partials). */
__global__ void k_apply_a(Dims d, float rho, const float *p, float *ap, double *part) {
    __shared__ double red[kThreads];
    double acc = 0.0;
    const long XY = (long)d.X * d.Y;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < d.N; i += (long)gridDim.x * blockDim.x) {
        const int x = (int)(i % d.X), y = (int)((i / d.X) % d.Y), z = (int)(i / XY);
        const float pc = p[i];
        float s = 0.f;   /* (F^T F p)[i] */
        if (f_row(x, y, z, d)) {
            /* rows at i: -(p[i+e] - p[i]) for each component */
            s -= (p[i + 1] - pc) + (p[i + d.X] - pc) + (p[i + XY] - pc);
        }
        /* rows at i - e_c (component c) contribute +(p[i] - p[i - e_c]) */
        if (x > 0 && f_row(x - 1, y, z, d)) s += pc - p[i - 1];
        if (y > 0 && f_row(x, y - 1, z, d)) s += pc - p[i - d.X];
        if (z > 0 && f_row(x, y, z - 1, d)) s += pc - p[i - XY];
        const float v = pc + rho * s;
        ap[i] = v;
        acc += (double)pc * v;
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = kThreads / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

/* b = F^T (rho y - u) + x0, with y, u stored as 3 planes of N. */
__global__ void k_rhs(Dims d, float rho, const float *y, const float *u, const float *x0, float *b) {
    const long XY = (long)d.X * d.Y;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < d.N; i += (long)gridDim.x * blockDim.x) {
        const int x = (int)(i % d.X), yy = (int)((i / d.X) % d.Y), z = (int)(i / XY);
        float s = 0.f;
        if (f_row(x, yy, z, d))
            for (int c = 0; c < 3; c++) s -= rho * y[c * d.N + i] - u[c * d.N + i];
        if (x > 0 && f_row(x - 1, yy, z, d)) s += rho * y[i - 1] - u[i - 1];
        if (yy > 0 && f_row(x, yy - 1, z, d)) s += rho * y[d.N + i - d.X] - u[d.N + i - d.X];
        if (z > 0 && f_row(x, yy, z - 1, d)) s += rho * y[2 * d.N + i - XY] - u[2 * d.N + i - XY];
        b[i] = s + x0[i];
    }
}

/* y = soft(Fx + u/rho, lambda/rho); u += rho (Fx - y)  (rows outside the set: Fx = 0) */
__global__ void k_shrink(Dims d, float rho, float lambda, const float *xv, float *y, float *u) {
    const long XY = (long)d.X * d.Y;
    const float thr = lambda / rho;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < d.N; i += (long)gridDim.x * blockDim.x) {
        const int x = (int)(i % d.X), yy = (int)((i / d.X) % d.Y), z = (int)(i / XY);
        float fx[3] = {0.f, 0.f, 0.f};
        if (f_row(x, yy, z, d)) {
            const float c = xv[i];
            fx[0] = xv[i + 1] - c;
            fx[1] = xv[i + d.X] - c;
            fx[2] = xv[i + XY] - c;
        }
        for (int k = 0; k < 3; k++) {
            const long j = k * d.N + i;
            const float zz = fx[k] + u[j] / rho;
            const float yn = zz > 0.f ? fmaxf(zz - thr, 0.f) : fminf(zz + thr, 0.f);
            y[j] = yn;
            u[j] += rho * (fx[k] - yn);
        }
    }
}

/* FP64 dot of two vectors (block partials). */
__global__ void k_dot(long n, const float *a, const float *b, double *part) {
    __shared__ double red[kThreads];
    double acc = 0.0;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        acc += (double)a[i] * b[i];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = kThreads / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

/* s[slot] = sum of nparts partials (one block) */
__global__ void k_sum(const double *part, int nparts, double *s, int slot) {
    __shared__ double red[kThreads];
    double acc = 0.0;
    for (int i = threadIdx.x; i < nparts; i += kThreads) acc += part[i];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = kThreads / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) s[slot] = red[0];
}

/* scalars: [0] rr, [1] pAp, [2] rr_new, [3] bb.  CG step on the device:
 * alpha = rr / pAp; x += alpha p; r -= alpha Ap. */
__global__ void k_cg_xr(long n, const double *s, const float *p, const float *ap, float *x, float *r) {
    const double pap = s[1];
    const float alpha = pap > 0.0 ? (float)(s[0] / pap) : 0.f;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        x[i] += alpha * p[i];
        r[i] -= alpha * ap[i];
    }
}

/* p = r + (rr_new / rr) p; rr = rr_new */
__global__ void k_cg_p(long n, double *s, const float *r, float *p) {
    const double rr = s[0];
    const float beta = rr > 0.0 ? (float)(s[2] / rr) : 0.f;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        p[i] = r[i] + beta * p[i];
}

__global__ void k_copy_scalar(double *s, int dst, int src) {
    if (threadIdx.x == 0 && blockIdx.x == 0) s[dst] = s[src];
}

__global__ void k_fill(long n, float *v, float value) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) v[i] = value;
}

/* r = b - A x (x given): ap = A x first */
__global__ void k_sub(long n, const float *b, const float *ax, float *r) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        r[i] = b[i] - ax[i];
}

/* Quadratic-form tensor per voxel (quadfilt.cpp:17-82): mu = (v1, v2, v0),
 * m = mu0 + mu1 + mu2, R = Rodrigues rotation about n = (cos phi, sin phi, 0)
 * by the angle with cosine c (phi, c = coefficient planes 0, 1),
 * Q = R^T diag(m, m, 0) R; out planes: Q00, Q11, Q22, Q01, Q02, Q12. */
__global__ void k_quad_build(long n, const float *vox, const float *coef, float *q) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const float m = vox[n + i] + vox[2 * n + i] + vox[i];
        const float phi = coef[i], c = coef[n + i];
        const float x = cosf(phi), y = sinf(phi), z = 0.0f, s = sqrtf(1.0f - c * c);
        const float nrm = sqrtf(x * x + y * y + z * z);
        const float nx = x / nrm, ny = y / nrm, nz = z / nrm;
        const float oc = 1.0f - c;
        float R[9] = {oc * nx * nx + c,      oc * nx * ny - nz * s, oc * nx * nz + ny * s,
                      oc * nx * ny + nz * s, oc * ny * ny + c,      oc * ny * nz - nx * s,
                      oc * nx * nz - ny * s, oc * ny * nz + nx * s, oc * nz * nz + c};
        /* Q = R^T diag(m, m, 0) R: Q_ab = m (R0a R0b + R1a R1b) */
        auto qe = [&](int a, int b) { return m * (R[a] * R[b] + R[3 + a] * R[3 + b]); };
        q[i] = qe(0, 0);
        q[n + i] = qe(1, 1);
        q[2 * n + i] = qe(2, 2);
        q[3 * n + i] = qe(0, 1);
        q[4 * n + i] = qe(0, 2);
        q[5 * n + i] = qe(1, 2);
    }
}

/* Decomposition of the filtered tensor (quadfilt.cpp:97-132): smallest
 * eigenvector, normalised, signed so that z >= 0; coefficient planes
 * atan2 of (norm x e_z) and norm . e_z; voxel planes (l1, l2, l0) with
 * l0 <= l1 <= l2. */
__global__ void k_quad_decompose(long n, const float *q, float *vox, float *coef) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        double A[9] = {q[i], q[3 * n + i], q[4 * n + i], q[3 * n + i], q[n + i], q[5 * n + i],
                       q[4 * n + i], q[5 * n + i], q[2 * n + i]};
        double w[3], V[9];
        jacobi3(A, w, V);
        int idx[3];
        order3(w, idx);
        double v0 = V[idx[0]], v1 = V[3 + idx[0]], v2 = V[6 + idx[0]];
        const double nv = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
        v0 /= nv; v1 /= nv; v2 /= nv;
        if (v2 < 0) { v0 = -v0; v1 = -v1; v2 = -v2; }
        /* rotAx = norm x (0, 0, 1) = (v1, -v0, 0) */
        coef[i] = (float)atan2(-v0, v1);
        coef[n + i] = (float)v2;
        vox[i] = (float)w[idx[1]];
        vox[n + i] = (float)w[idx[2]];
        vox[2 * n + i] = (float)w[idx[0]];
    }
}

int grid_of(long n) {
    long b = (n + kThreads - 1) / kThreads;
    if (b > 148 * 8) b = 148 * 8;
    return (int)(b < 1 ? 1 : b);
}

struct TvWork {
    float *y = nullptr, *u = nullptr, *x = nullptr, *b = nullptr, *r = nullptr, *p = nullptr, *ap = nullptr;
    double *part = nullptr, *s = nullptr;
    void release() {
        for (float *q : {y, u, x, b, r, p, ap}) cudaFree(q);
        cudaFree(part);
        cudaFree(s);
    }
};

cudaError_t cg_solve(const Dims &d, float rho, const float *b, float *x, TvWork &w, cudaStream_t st, double tol,
                     int max_it, int *iters, double *rel) {
    const int g = grid_of(d.N);
    double h[4];
    /* r = b - A x ; p = r ; rr = r.r ; bb = b.b */
    k_apply_a<<<g, kThreads, 0, st>>>(d, rho, x, w.ap, w.part);
    k_sub<<<g, kThreads, 0, st>>>(d.N, b, w.ap, w.r);
    cudaMemcpyAsync(w.p, w.r, d.N * sizeof(float), cudaMemcpyDeviceToDevice, st);
    k_dot<<<g, kThreads, 0, st>>>(d.N, w.r, w.r, w.part);
    k_sum<<<1, kThreads, 0, st>>>(w.part, g, w.s, 0);
    k_dot<<<g, kThreads, 0, st>>>(d.N, b, b, w.part);
    k_sum<<<1, kThreads, 0, st>>>(w.part, g, w.s, 3);
    int it = 0;
    for (;;) {
        cudaError_t e = cudaMemcpyAsync(h, w.s, 4 * sizeof(double), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return e;
        const double r_rel = h[3] > 0 ? std::sqrt(h[0] / h[3]) : 0.0;
        if (rel) *rel = r_rel;
        if (r_rel <= tol || it >= max_it) break;
        /* 8 CG steps between convergence checks; the scalars stay on the device */
        for (int k = 0; k < 8; k++, it++) {
            k_apply_a<<<g, kThreads, 0, st>>>(d, rho, w.p, w.ap, w.part);   /* pAp */
            k_sum<<<1, kThreads, 0, st>>>(w.part, g, w.s, 1);
            k_cg_xr<<<g, kThreads, 0, st>>>(d.N, w.s, w.p, w.ap, x, w.r);
            k_dot<<<g, kThreads, 0, st>>>(d.N, w.r, w.r, w.part);
            k_sum<<<1, kThreads, 0, st>>>(w.part, g, w.s, 2);
            k_cg_p<<<g, kThreads, 0, st>>>(d.N, w.s, w.r, w.p);
            k_copy_scalar<<<1, 1, 0, st>>>(w.s, 0, 2);
        }
    }
    if (iters) *iters = it;
    return cudaGetLastError();
}

bool dev_ok() {
    int dev = 0;
    cudaDeviceProp p;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&p, dev) != cudaSuccess) return false;
    return p.major == 10;
}

}  // namespace

/* in place on d_vol; returns the CG iterations of the last solve */
xr_status tv_minimize(float *d_vol, int X, int Y, int Z, float rho, float lambda, int iter, double tol, int max_cg,
                      cudaStream_t st, int *cg_iters, double *cg_rel) {
    if (!d_vol || X < 1 || Y < 1 || Z < 1 || !(rho > 0.f) || lambda < 0.f || iter < 0) return XR_ERR_ARG;
    if (!dev_ok()) return XR_ERR_NODEV;
    Dims d{X, Y, Z, (long)X * Y * Z};
    TvWork w;
    const size_t nb = d.N * sizeof(float);
    cudaError_t e = cudaSuccess;
    for (float **q : {&w.x, &w.b, &w.r, &w.p, &w.ap})
        if (e == cudaSuccess) e = cudaMalloc(q, nb);
    if (e == cudaSuccess) e = cudaMalloc(&w.y, 3 * nb);
    if (e == cudaSuccess) e = cudaMalloc(&w.u, 3 * nb);
    if (e == cudaSuccess) e = cudaMalloc(&w.part, 148 * 8 * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&w.s, 8 * sizeof(double));
    if (e != cudaSuccess) {
        w.release();
        return XR_ERR_OOM;
    }
    const int g = grid_of(3 * d.N);
    k_fill<<<g, kThreads, 0, st>>>(3 * d.N, w.y, 1.0f);   /* yy.setOnes(), uu.setOnes() */
    k_fill<<<g, kThreads, 0, st>>>(3 * d.N, w.u, 1.0f);
    cudaMemcpyAsync(w.x, d_vol, nb, cudaMemcpyDeviceToDevice, st);   /* first guess: x0 */
    int its = 0;
    double rel = 0.0;
    for (int i = 0; i < iter && e == cudaSuccess; i++) {
        k_rhs<<<grid_of(d.N), kThreads, 0, st>>>(d, rho, w.y, w.u, d_vol, w.b);
        e = cg_solve(d, rho, w.b, w.x, w, st, tol, max_cg, &its, &rel);
        if (e == cudaSuccess) {
            k_shrink<<<grid_of(d.N), kThreads, 0, st>>>(d, rho, lambda, w.x, w.y, w.u);
            e = cudaGetLastError();
        }
    }
    if (e == cudaSuccess && iter > 0) e = cudaMemcpyAsync(d_vol, w.x, nb, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    w.release();
    if (cg_iters) *cg_iters = its;
    if (cg_rel) *cg_rel = rel;
    return e == cudaSuccess ? XR_OK : XR_ERR_CUDA;
}

}  // namespace xr

using namespace xr;

extern "C" {

xr_status xr_tv_minimize(void *stream, float *d_vol, int nx, int ny, int nz, float rho, float lambda, int iter) {
    return tv_minimize(d_vol, nx, ny, nz, rho, lambda, iter, 1e-6, 2000, (cudaStream_t)stream, nullptr, nullptr);
}

xr_status xr_quad_form_filter(void *stream, float *d_voxel, float *d_coef, int nx, int ny, int nz, float lambda) {
    if (!d_voxel || !d_coef || nx < 1 || ny < 1 || nz < 1 || lambda < 0.f) return XR_ERR_ARG;
    if (!dev_ok()) return XR_ERR_NODEV;
    cudaStream_t st = (cudaStream_t)stream;
    const long n = (long)nx * ny * nz;
    float *q = nullptr;
    if (cudaMalloc(&q, 6 * n * sizeof(float)) != cudaSuccess) return XR_ERR_OOM;
    k_quad_build<<<grid_of(n), kThreads, 0, st>>>(n, d_voxel, d_coef, q);
    xr_status s = cudaGetLastError() == cudaSuccess ? XR_OK : XR_ERR_CUDA;
    for (int e = 0; e < 6 && s == XR_OK; e++)   /* quadfilt.cpp:93-94: rho 3, 20 iterations */
        s = tv_minimize(q + e * n, nx, ny, nz, 3.0f, lambda, 20, 1e-6, 2000, st, nullptr, nullptr);
    if (s == XR_OK) {
        k_quad_decompose<<<grid_of(n), kThreads, 0, st>>>(n, q, d_voxel, d_coef);
        if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess) s = XR_ERR_CUDA;
    }
    cudaFree(q);
    return s;
}

/* Host-buffer forms: copy in, run on `device`, copy out. */
xr_status xr_tv_minimize_host(int device, float *vol, int nx, int ny, int nz, float rho, float lambda, int iter) {
    if (!vol || nx < 1 || ny < 1 || nz < 1) return XR_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return XR_ERR_NODEV;
    const size_t nb = (size_t)nx * ny * nz * sizeof(float);
    float *d = nullptr;
    if (cudaMalloc(&d, nb) != cudaSuccess) return XR_ERR_OOM;
    xr_status st = cudaMemcpy(d, vol, nb, cudaMemcpyHostToDevice) == cudaSuccess ? XR_OK : XR_ERR_CUDA;
    if (!st) st = xr_tv_minimize(nullptr, d, nx, ny, nz, rho, lambda, iter);
    if (!st && cudaMemcpy(vol, d, nb, cudaMemcpyDeviceToHost) != cudaSuccess) st = XR_ERR_CUDA;
    cudaFree(d);
    return st;
}

xr_status xr_quad_form_filter_host(int device, float *const *voxel, float *const *coef, int nx, int ny, int nz,
                                   float lambda) {
    if (!voxel || !coef || nx < 1 || ny < 1 || nz < 1) return XR_ERR_ARG;
    for (int i = 0; i < 3; i++)
        if (!voxel[i]) return XR_ERR_ARG;
    if (!coef[0] || !coef[1]) return XR_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return XR_ERR_NODEV;
    const size_t n = (size_t)nx * ny * nz, nb = n * sizeof(float);
    float *d = nullptr;
    if (cudaMalloc(&d, 5 * nb) != cudaSuccess) return XR_ERR_OOM;
    xr_status st = XR_OK;
    for (int i = 0; i < 3 && !st; i++)
        if (cudaMemcpy(d + i * n, voxel[i], nb, cudaMemcpyHostToDevice) != cudaSuccess) st = XR_ERR_CUDA;
    for (int i = 0; i < 2 && !st; i++)
        if (cudaMemcpy(d + (3 + i) * n, coef[i], nb, cudaMemcpyHostToDevice) != cudaSuccess) st = XR_ERR_CUDA;
    if (!st) st = xr_quad_form_filter(nullptr, d, d + 3 * n, nx, ny, nz, lambda);
    for (int i = 0; i < 3 && !st; i++)
        if (cudaMemcpy(voxel[i], d + i * n, nb, cudaMemcpyDeviceToHost) != cudaSuccess) st = XR_ERR_CUDA;
    for (int i = 0; i < 2 && !st; i++)
        if (cudaMemcpy(coef[i], d + (3 + i) * n, nb, cudaMemcpyDeviceToHost) != cudaSuccess) st = XR_ERR_CUDA;
    cudaFree(d);
    return st;
}

}  // extern "C"
