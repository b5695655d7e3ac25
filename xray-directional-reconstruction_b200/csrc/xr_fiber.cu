/*
 * The fiber-model projectors (reconstruct/src/fiber.cu).  Every voxel holds a
 * fiber vector F = (mu_0, mu_1, mu_2) and, with K = 4, an isotropic term
 * mu_3; a ray with unit direction B through a grating along G sees the signed
 * projection ps = (B x G) . F + mu_3 (fiber.cu:53-58).  Forward:
 * proj += c * vs * ratio * |ps| per tap (no weight image, no chord
 * normalisation).  Back: channel i gathers w_i = |(B x G)_i| (i < 3) or 1
 * times the 4-tap sum of the ratio image, and its own w_i.  The ray casting is
 * rayCastingFiber's (fiber.cu:228-278): rayCasting's source and rotation, but
 * voxel centres at (2i - N + 1)/2 and the detector v axis along -R e_z.
 *
 * Voxel-parallel kernels over all listed (axis, view) pairs with global
 * float atomics for the forward; the model is a research variant of the
 * reference, kept for completeness, not one of the tuned hot paths.
 */
#include <cuda_runtime.h>

#include "xr_internal.h"

namespace xr {
namespace {

constexpr int kFiberThreads = 256;

__device__ __forceinline__ float fdot_rn(float a0, float a1, float a2, float b0, float b1, float b2) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a0, b0), __fmul_rn(a1, b1)), __fmul_rn(a2, b2));
}

__device__ __forceinline__ float fdiv_det(float a, const GeomConst &g) {
    if (!g.exact_rdet) return __fdiv_rn(a, g.det);
    const float q = __fmul_rn(a, g.rdet);
    const float r = __fmaf_rn(-q, g.det, a);
    return __fmaf_rn(r, g.rdet, q);
}

/* (2i - N + 1) / 2 * vs, in the reference's operation order. */
__device__ __forceinline__ float fiber_base(int i, int N, float vs) {
    return __fmul_rn(__fmul_rn(__fadd_rn(__fsub_rn(__fmul_rn(2.0f, (float)i), (float)N), 1.0f), 0.5f), vs);
}

/* rayCastingFiber: u, v and the unit ray B of voxel (x, y, z) in view frame f. */
__device__ __forceinline__ void fiber_ray(const ViewFrame &f, const GeomConst &g, int x, int y, int z, float &u,
                                          float &v, float B[3]) {
    const float o0 = __fsub_rn(__fsub_rn(fiber_base(x, g.N, g.vs), f.off[0]), f.t[0]);
    const float o1 = __fsub_rn(__fsub_rn(fiber_base(y, g.N, g.vs), f.off[1]), f.t[1]);
    const float o2 = __fsub_rn(__fsub_rn(fiber_base(z, g.N, g.vs), f.off[2]), f.t[2]);
    const float d0 = __fsub_rn(o0, f.src[0]), d1 = __fsub_rn(o1, f.src[1]), d2 = __fsub_rn(o2, f.src[2]);
    const float coeff = __fdiv_rn(-f.ss, fdot_rn(f.src[0], f.src[1], f.src[2], d0, d1, d2));
    const float p0 = __fadd_rn(f.src[0], __fmul_rn(coeff, d0));
    const float p1 = __fadd_rn(f.src[1], __fmul_rn(coeff, d1));
    const float p2 = __fadd_rn(f.src[2], __fmul_rn(coeff, d2));
    u = __fadd_rn(fdiv_det(__fmul_rn(fdot_rn(p0, p1, p2, f.eu[0], f.eu[1], f.eu[2]), g.mag), g), g.half);
    v = __fadd_rn(fdiv_det(__fmul_rn(fdot_rn(p0, p1, p2, -f.ev[0], -f.ev[1], -f.ev[2]), g.mag), g), g.half);
    const float len = __fsqrt_rn(fdot_rn(d0, d1, d2, d0, d1, d2));
    const bool ok = len > 1e-8f;
    B[0] = ok ? __fdiv_rn(d0, len) : 0.f;
    B[1] = ok ? __fdiv_rn(d1, len) : 0.f;
    B[2] = ok ? __fdiv_rn(d2, len) : 0.f;
}

/* Window test and bilinear taps (ir.cu:1501-1509 / fiber.cu:35-41). */
__device__ __forceinline__ bool fiber_taps(const GeomConst &g, float u, float v, int &iu, int &iv, float c[4]) {
    if (!(0.55f < u && u < g.lim && 0.55f < v && v < g.lim)) return false;
    const float ut = __fsub_rn(u, 0.5f), vt = __fsub_rn(v, 0.5f);
    const float fiu = floorf(ut), fiv = floorf(vt);
    iu = (int)fiu;
    iv = (int)fiv;
    const float fu = __fsub_rn(ut, fiu), fv = __fsub_rn(vt, fiv);
    const float gu = __fsub_rn(1.0f, fu), gv = __fsub_rn(1.0f, fv);
    c[0] = __fmul_rn(gu, fv);
    c[1] = __fmul_rn(fu, fv);
    c[2] = __fmul_rn(fu, gv);
    c[3] = __fmul_rn(gu, gv);
    return true;
}

struct FiberArgs {
    GeomConst g;
    const ViewFrame *frames;   /* [C][V] */
    const int *view_list;
    int n_views, n_cond;
    const float *proj;         /* back: ratio images, C blocks */
    float *out;                /* forward: C blocks            */
    float *vol;                /* K (3 or 4) planes of N^3     */
    int art;
    float alpha;
};

__global__ void k_fiber_forward(FiberArgs a) {
    const GeomConst &g = a.g;
    const long N = g.N, N3 = N * N * N;
    const int K = g.K < 4 ? g.K : 4;
    const size_t NdNd = (size_t)g.Nd * g.Nd;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < N3; i += (long)gridDim.x * blockDim.x) {
        const int x = (int)(i % N), y = (int)((i / N) % N), z = (int)(i / (N * N));
        float mu[4];
        for (int k = 0; k < K; k++) mu[k] = a.vol[i + k * N3];
        for (int c = 0; c < a.n_cond; c++) {
            for (int j = 0; j < a.n_views; j++) {
                const ViewFrame &f = a.frames[(size_t)c * g.V + a.view_list[j]];
                float u, v, B[3], w[4];
                int iu, iv;
                fiber_ray(f, g, x, y, z, u, v, B);
                if (!fiber_taps(g, u, v, iu, iv, w)) continue;
                const float bxg[3] = {__fsub_rn(__fmul_rn(B[1], f.ev[2]), __fmul_rn(B[2], f.ev[1])),
                                      __fsub_rn(__fmul_rn(B[2], f.ev[0]), __fmul_rn(B[0], f.ev[2])),
                                      __fsub_rn(__fmul_rn(B[0], f.ev[1]), __fmul_rn(B[1], f.ev[0]))};
                float ps = 0.f;
                for (int k = 0; k < K; k++) ps = __fadd_rn(ps, __fmul_rn(k >= 3 ? 1.0f : bxg[k], mu[k]));
                const float pr = fabsf(ps);
                float *P = a.out + (size_t)c * g.V * NdNd + (size_t)f.view * NdNd + iu + (size_t)g.Nd * iv;
                /* c * vs * ratio * |ps|, left to right (fiber.cu:68-71) */
                atomicAdd(P + g.Nd, __fmul_rn(__fmul_rn(__fmul_rn(w[0], g.vs), g.ratio), pr));
                atomicAdd(P + g.Nd + 1, __fmul_rn(__fmul_rn(__fmul_rn(w[1], g.vs), g.ratio), pr));
                atomicAdd(P + 1, __fmul_rn(__fmul_rn(__fmul_rn(w[2], g.vs), g.ratio), pr));
                atomicAdd(P, __fmul_rn(__fmul_rn(__fmul_rn(w[3], g.vs), g.ratio), pr));
            }
        }
    }
}

/* Back-projection of the listed views of every axis fused with the update of
 * channel 0 (MLEM voxelProduct / ART voxelPlus); fiberModelReconstruct
 * (reconstruct.cu:1322-1347) updates that channel alone. */
__global__ void k_fiber_back(FiberArgs a) {
    const GeomConst &g = a.g;
    const long N = g.N, N3 = N * N * N;
    const size_t NdNd = (size_t)g.Nd * g.Nd;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < N3; i += (long)gridDim.x * blockDim.x) {
        const int x = (int)(i % N), y = (int)((i / N) % N), z = (int)(i / (N * N));
        const float mu0 = a.vol[i];
        float tmp = 0.f, fac = 0.f;   /* channel 0 */
        for (int c = 0; c < a.n_cond; c++) {
            for (int j = 0; j < a.n_views; j++) {
                const ViewFrame &f = a.frames[(size_t)c * g.V + a.view_list[j]];
                float u, v, B[3], w[4];
                int iu, iv;
                fiber_ray(f, g, x, y, z, u, v, B);
                if (!fiber_taps(g, u, v, iu, iv, w)) continue;
                /* w_0 = |(B x G)_0 s| = |(B x G)_0| whatever the sign s of ps */
                const float w0 = fabsf(__fsub_rn(__fmul_rn(B[1], f.ev[2]), __fmul_rn(B[2], f.ev[1])));
                const float *P = a.proj + (size_t)c * g.V * NdNd + (size_t)f.view * NdNd + iu + (size_t)g.Nd * iv;
                float nb = __fmul_rn(__fmul_rn(w0, w[0]), __ldg(P + g.Nd));
                nb = __fadd_rn(nb, __fmul_rn(__fmul_rn(w0, w[1]), __ldg(P + g.Nd + 1)));
                nb = __fadd_rn(nb, __fmul_rn(__fmul_rn(w0, w[2]), __ldg(P + 1)));
                nb = __fadd_rn(nb, __fmul_rn(__fmul_rn(w0, w[3]), __ldg(P)));
                tmp = __fadd_rn(tmp, nb);
                fac = __fadd_rn(fac, w0);
            }
        }
        if (a.art) a.vol[i] = __fadd_rn(mu0, __fmul_rn(a.alpha, tmp));
        else a.vol[i] = (fac == 0.0f) ? 0.0f : __fdiv_rn(__fmul_rn(mu0, tmp), fac);
    }
}

int fiber_grid(long n) {
    long b = (n + kFiberThreads - 1) / kFiberThreads;
    if (b > 148 * 16) b = 148 * 16;
    return (int)(b < 1 ? 1 : b);
}

}  // namespace

cudaError_t launch_fiber_forward(const GeomConst &g, const ViewFrame *frames, const int *view_list, int n_views,
                                 int n_cond, const float *vol, float *out, cudaStream_t s) {
    if (n_views <= 0 || n_cond <= 0) return cudaSuccess;
    FiberArgs a{};
    a.g = g;
    a.frames = frames;
    a.view_list = view_list;
    a.n_views = n_views;
    a.n_cond = n_cond;
    a.vol = const_cast<float *>(vol);
    a.out = out;
    k_fiber_forward<<<fiber_grid((long)g.N * g.N * g.N), kFiberThreads, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_fiber_back(const GeomConst &g, const ViewFrame *frames, const int *view_list, int n_views,
                              int n_cond, const float *proj, float *vol, int art, float alpha, cudaStream_t s) {
    if (n_views <= 0 || n_cond <= 0) return cudaSuccess;
    FiberArgs a{};
    a.g = g;
    a.frames = frames;
    a.view_list = view_list;
    a.n_views = n_views;
    a.n_cond = n_cond;
    a.proj = proj;
    a.vol = vol;
    a.art = art;
    a.alpha = alpha;
    k_fiber_back<<<fiber_grid((long)g.N * g.N * g.N), kFiberThreads, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace xr
