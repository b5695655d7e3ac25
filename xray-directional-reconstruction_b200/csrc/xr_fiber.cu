/*
 * The fiber-model projectors (reconstruct/src/fiber.cu).  Every voxel holds a
 * fiber vector F = (mu_0, mu_1, mu_2) and, with K = 4, an isotropic term
 * mu_3; a ray with unit direction B through a grating along G sees the signed
 * projection ps = (B x G) . F + mu_3 (fiber.cu:52-65).  Forward:
 * proj += c * vs * ratio * |ps| per tap (no weight image, no chord
 * normalisation).  Back: channel i gathers w_i = |(B x G)_i| (i < 3) or 1
 * times the 4-tap sum of the ratio image, and its own w_i.  The ray casting is
 * rayCastingFiber's (fiber.cu:228-278): rayCasting's source and rotation, but
 * voxel centres at (2i - N + 1)/2 and the detector v axis along -R e_z.
 *
 * Forward: a CTA owns a 16 x 8 x 8 brick and a chunk of views; per view it
 * splats its voxels' taps into a shared detector tile (two-word fixed point,
 * xr_tile.cuh) over the brick's footprint and flushes the tile with one float
 * atomic per pixel.  Back: voxel-parallel over all listed (axis, view) pairs,
 * gathers from the L2-resident ratio images, fused with the update; since the
 * reference's driver updates channel 0 alone, only channel 0's sums are formed.
 */
#include <cuda_runtime.h>

#include "xr_internal.h"
#include "xr_tile.cuh"

namespace xr {
namespace {

constexpr int kFiberThreads = 256;                 /* back kernel                    */
constexpr int kFwdThreads = 256;                   /* forward: 16 x 8 x 8 brick      */
constexpr int kBX = 16, kBY = 8, kBZ = 8;
constexpr int kTileCap = 48 * 48;                  /* pixels per shared tile         */

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

struct FiberBackArgs {
    GeomConst g;
    const ViewFrame *frames;   /* [C][V] */
    const int *view_list;
    int n_views, n_cond;
    const float *proj;         /* ratio images, C blocks          */
    float *vol;                /* channel 0 updated in place       */
    int art;
    float alpha;
};

struct FiberFwdArgs {
    GeomConst g;
    const ViewFrame *frames;   /* [C][V] */
    const int *view_list;
    int n_views, vpc;
    const float *vol;          /* min(K, 4) planes of N^3 */
    float *out;                /* C blocks of V*Nd*Nd, accumulated */
    int nbx, nby;              /* bricks along x, y */
};

/* forwardProjFiber of a chunk of views of axis blockIdx.y over one brick. */
__global__ void __launch_bounds__(kFwdThreads, 3) k_fiber_forward(FiberFwdArgs a) {
    extern __shared__ int smem[];
    __shared__ float s_red[kFwdThreads / 32];
    int4 *bbox = reinterpret_cast<int4 *>(smem + 4 * kTileCap);   /* vpc entries */
    ViewFrame *fr = reinterpret_cast<ViewFrame *>(bbox + a.vpc);

    const GeomConst &g = a.g;
    const int N = g.N, Nd = g.Nd;
    const int K = g.K < 4 ? g.K : 4;
    const int cond = blockIdx.y;
    const int j0 = blockIdx.z * a.vpc;
    const int nv = min(a.vpc, a.n_views - j0);
    if (nv <= 0) return;

    const int brick = blockIdx.x;
    const int x0 = (brick % a.nbx) * kBX, y0 = ((brick / a.nbx) % a.nby) * kBY, z0 = (brick / (a.nbx * a.nby)) * kBZ;
    const int x1 = min(x0 + kBX, N) - 1, y1 = min(y0 + kBY, N) - 1, z1 = min(z0 + kBZ, N) - 1;

    const int tid = threadIdx.x;
    for (int i = tid; i < 4 * kTileCap; i += kFwdThreads) smem[i] = 0;
    for (int i = tid; i < nv * 5; i += kFwdThreads) {
        const int jj = i / 5, q = i % 5;
        reinterpret_cast<float4 *>(&fr[jj])[q] =
            reinterpret_cast<const float4 *>(&a.frames[(size_t)cond * g.V + a.view_list[j0 + jj]])[q];
    }
    __syncthreads();

    /* footprint of the brick per view: hull of its 8 corner voxels' (u, v),
     * widened by one pixel and clamped to the detector */
    for (int i = tid; i < nv; i += kFwdThreads) {
        const ViewFrame &f = fr[i];
        float umin = 1e30f, umax = -1e30f, vmin = 1e30f, vmax = -1e30f;
        bool ok = true;
        for (int c = 0; c < 8; c++) {
            float u, v, B[3];
            fiber_ray(f, g, (c & 1) ? x1 : x0, (c & 2) ? y1 : y0, (c & 4) ? z1 : z0, u, v, B);
            if (!(fabsf(u) < 1e7f && fabsf(v) < 1e7f)) ok = false;
            umin = fminf(umin, u); umax = fmaxf(umax, u);
            vmin = fminf(vmin, v); vmax = fmaxf(vmax, v);
        }
        int iu0 = (int)floorf(umin - 0.5f) - 1, iu1 = (int)floorf(umax - 0.5f) + 2;
        int iv0 = (int)floorf(vmin - 0.5f) - 1, iv1 = (int)floorf(vmax - 0.5f) + 2;
        iu0 = max(iu0, 0); iv0 = max(iv0, 0);
        iu1 = min(iu1, Nd - 1); iv1 = min(iv1, Nd - 1);
        int W = iu1 - iu0 + 1, H = iv1 - iv0 + 1;
        if (!ok) { W = 1 << 20; H = 1; }              /* every tap to global memory */
        if (iu1 < iu0 || iv1 < iv0) { W = 0; H = 0; } /* off the detector           */
        bbox[i] = make_int4(iu0, iv0, W, H);
    }

    /* this thread's 4 voxels: a warp is 4 (x) x 4 (z) x 2 (y), so its taps
     * spread over several pixels in any view */
    const int lane = tid & 31, w = tid >> 5;
    const int x = x0 + (w & 3) * 4 + (lane & 3);
    const int z = z0 + ((w >> 2) & 1) * 4 + ((lane >> 2) & 3);
    const int yb = y0 + (lane >> 4);
    const long N3 = (long)N * N * N;
    float mu[4][4];
    bool okv[4];
    float bound = 0.f;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int y = yb + 2 * q;
        okv[q] = x <= x1 && z <= z1 && y <= y1;
        float sa = 0.f;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            mu[q][k] = (okv[q] && k < K) ? __ldg(a.vol + (size_t)x + (size_t)N * y + (size_t)N * N * z + k * N3) : 0.f;
            sa += fabsf(mu[q][k]);
        }
        /* |ps| <= |B x G| |F| + |mu_3| <= sum |mu_k| (B, G unit vectors); weights c <= 1 */
        if (okv[q]) bound = fmaxf(bound, sa * g.vs * g.ratio * 1.001f);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) bound = fmaxf(bound, __shfl_xor_sync(0xffffffffu, bound, o));
    if (lane == 0) s_red[w] = bound;
    __syncthreads();
    float S = 0.f;
#pragma unroll
    for (int i = 0; i < kFwdThreads / 32; i++) S = fmaxf(S, s_red[i]);
    if (!(S > 0.f) || !(S < 3e38f)) return;   /* nothing to splat (or non-finite input) */
    const int sh = fix_shift(S);
    const float fscale = ldexpf(1.0f, sh);
    const float finv = ldexpf(1.0f, -sh);

    const size_t NdNd = (size_t)Nd * Nd;
    float *outc = a.out + (size_t)cond * g.V * NdNd;
    for (int jj = 0; jj < nv; jj++) {
        const ViewFrame f = fr[jj];
        const int4 bb = bbox[jj];
        int *T = smem + (jj & 1) * 2 * kTileCap;   /* hi words, lo words after */
        float *P = outc + (size_t)f.view * NdNd;
        const bool use_tile = (bb.z > 0) && (bb.z * bb.w <= kTileCap);
        if (bb.z > 0) {
#pragma unroll
            for (int q = 0; q < 4; q++) {
                if (!okv[q]) continue;
                float u, v, B[3], c[4];
                int iu, iv;
                fiber_ray(f, g, x, yb + 2 * q, z, u, v, B);
                if (!fiber_taps(g, u, v, iu, iv, c)) continue;
                const float bxg[3] = {__fsub_rn(__fmul_rn(B[1], f.ev[2]), __fmul_rn(B[2], f.ev[1])),
                                      __fsub_rn(__fmul_rn(B[2], f.ev[0]), __fmul_rn(B[0], f.ev[2])),
                                      __fsub_rn(__fmul_rn(B[0], f.ev[1]), __fmul_rn(B[1], f.ev[0]))};
                float ps = 0.f;
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if (k < K) ps = __fadd_rn(ps, __fmul_rn(k >= 3 ? 1.0f : bxg[k], mu[q][k]));
                const float pr = fabsf(ps);
                /* c * vs * ratio * |ps|, left to right (fiber.cu:68-75) */
                float wv[4];
#pragma unroll
                for (int t = 0; t < 4; t++) wv[t] = __fmul_rn(__fmul_rn(__fmul_rn(c[t], g.vs), g.ratio), pr);
                const int lu = iu - bb.x, lv = iv - bb.y;
                if (use_tile && lu >= 0 && lu + 1 < bb.z && lv >= 0 && lv + 1 < bb.w) {
                    int *t0 = T + lu + bb.z * lv;
                    fix_add(t0 + bb.z, kTileCap, wv[0] * fscale);
                    fix_add(t0 + bb.z + 1, kTileCap, wv[1] * fscale);
                    fix_add(t0 + 1, kTileCap, wv[2] * fscale);
                    fix_add(t0, kTileCap, wv[3] * fscale);
                } else {
                    float *p0 = P + iu + (size_t)Nd * iv;
                    atomicAdd(p0 + Nd, wv[0]);
                    atomicAdd(p0 + Nd + 1, wv[1]);
                    atomicAdd(p0 + 1, wv[2]);
                    atomicAdd(p0, wv[3]);
                }
            }
        }
        __syncthreads();
        if (use_tile) {   /* one warp per tile row; the tile is cleared behind */
            for (int r = w; r < bb.w; r += kFwdThreads / 32) {
                for (int cc = lane; cc < bb.z; cc += 32) {
                    float t;
                    if (fix_take(T + cc + bb.z * r, kTileCap, finv, t))
                        atomicAdd(P + (bb.x + cc) + (size_t)Nd * (bb.y + r), t);
                }
            }
        }
    }
}

/* Back-projection of the listed views of every axis fused with the update of
 * channel 0 (MLEM voxelProduct / ART voxelPlus); fiberModelReconstruct
 * (reconstruct.cu:1322-1347) updates that channel alone. */
__global__ void k_fiber_back(FiberBackArgs a) {
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
    FiberFwdArgs a{};
    a.g = g;
    a.frames = frames;
    a.view_list = view_list;
    a.n_views = n_views;
    a.vol = vol;
    a.out = out;
    a.nbx = (g.N + kBX - 1) / kBX;
    a.nby = (g.N + kBY - 1) / kBY;
    const int nbz = (g.N + kBZ - 1) / kBZ;
    const long bricks = (long)a.nbx * a.nby * nbz;
    /* views per CTA: the whole list unless that leaves fewer than 2048 CTAs */
    const long ctas = bricks * n_cond;
    const long chunks = ctas >= 2048 ? 1 : (2048 + ctas - 1) / ctas;
    int vpc = (int)((n_views + chunks - 1) / chunks);
    vpc = vpc < 1 ? 1 : (vpc > 64 ? 64 : vpc);
    a.vpc = vpc;
    const dim3 grid((unsigned)bricks, (unsigned)n_cond, (unsigned)((n_views + vpc - 1) / vpc));
    const size_t smem = 4 * kTileCap * sizeof(int) + (size_t)vpc * (sizeof(int4) + sizeof(ViewFrame));
    cudaError_t e = cudaFuncSetAttribute(k_fiber_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_fiber_forward<<<grid, kFwdThreads, smem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_fiber_back(const GeomConst &g, const ViewFrame *frames, const int *view_list, int n_views,
                              int n_cond, const float *proj, float *vol, int art, float alpha, cudaStream_t s) {
    if (n_views <= 0 || n_cond <= 0) return cudaSuccess;
    FiberBackArgs a{};
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
