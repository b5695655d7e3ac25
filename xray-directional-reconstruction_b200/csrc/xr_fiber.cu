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
 * Forward: a CTA owns a brick and a chunk of views; per view it splats its
 * voxels' taps into a shared detector tile (two-word fixed point, xr_tile.cuh)
 * over the brick's footprint and flushes the tile with one float atomic per
 * pixel.  Axes whose grating is a grid axis take the column form (ray set-up
 * once per voxel column and view), the others per-voxel ray casting.  Back: a
 * CTA owns an 8^3 brick, gathers from the L2-resident ratio images axis by
 * axis (column form where it applies) and applies the update; since the
 * reference's driver updates channel 0 alone, only channel 0's sums are formed.
 */
#include <cuda_runtime.h>

#include "xr_internal.h"
#include "xr_tile.cuh"
#include "xr_tex.cuh"

namespace xr {
namespace {

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

struct FiberFwdArgs {
    GeomConst g;
    const ViewFrame *frames;   /* [C][V] */
    const int *view_list;
    int n_views, vpc;
    const int *conds;          /* blockIdx.y -> axis                        */
    const float *magsig;       /* column form: per axis sign(ev[g]) * mag   */
    const float *vol;          /* min(K, 4) planes of N^3 */
    float *out;                /* C blocks of V*Nd*Nd, accumulated */
    int nbx, nby;              /* bricks along x, y (column form: g, a)     */
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
    const int cond = a.conds[blockIdx.y];
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

/* ------------------------------------------------------------------------ */
/* Forward, column form, for axes whose grating G = ev is a grid axis g      */
/* (ev = s e_g with s = +-1, src_g = eu_g = 0, off_g and t_g the same for     */
/* every view; checked on the host).  Along a voxel column parallel to g,     */
/* rayCastingFiber's coeff, u and the (a, b) components of the ray are the    */
/* same bit for bit (the dropped g terms are exact zeros); per voxel only     */
/*     v = ((coeff * o_g) * (-s mag)) / det + Nd/2                            */
/* and |d|^2 = da^2 + db^2 + o_g^2 (summed in x, y, z order) change.  With     */
/* B = d / |d|, B x G has components s (B_b, -B_a) on (a, b) for g = x or z   */
/* and -s (B_b, -B_a) for g = y, zero on g, so                                */
/*     ps = (db t_a - da t_b) / |d| + mu_3,   t = +-s mu  (sign folded in).    */
/* Tap indices, window tests and bilinear weights are the general kernel's,   */
/* bit for bit; 1/|d| is the hardware reciprocal square root and the weight   */
/* c * vs * ratio * |ps| is formed as c * (|ps| * vs * ratio), so each tap    */
/* differs from the reference's by a few ulps.                                */
/* Brick: 16 along g, 16 along a, 8 along b; 512 threads, 4 voxels along g    */
/* each; the warp's 8 columns 4 apart in a and in b.                          */
/* ------------------------------------------------------------------------ */
constexpr int kColThreads = 512;
constexpr int kColTileCap = 64 * 64;

template <int G>
struct FAx {
    static constexpr int A = (G == 0) ? 1 : 0;   /* the two other axes, ascending */
    static constexpr int B = (G == 2) ? 1 : 2;
};

template <int G>
__global__ void __launch_bounds__(kColThreads, 2) k_fiber_fwd_col(FiberFwdArgs a) {
    extern __shared__ int smem[];
    __shared__ float s_red[kColThreads / 32];
    int4 *bbox = reinterpret_cast<int4 *>(smem + 4 * kColTileCap);   /* vpc entries */
    ViewFrame *fr = reinterpret_cast<ViewFrame *>(bbox + a.vpc);
    constexpr int A = FAx<G>::A, B = FAx<G>::B;

    const GeomConst &g = a.g;
    const int N = g.N, Nd = g.Nd;
    const int K = g.K < 4 ? g.K : 4;
    const int cond = a.conds[blockIdx.y];
    const float msig = -a.magsig[cond];           /* detector v along -ev */
    const int j0 = blockIdx.z * a.vpc;
    const int nv = min(a.vpc, a.n_views - j0);
    if (nv <= 0) return;

    const int brick = blockIdx.x;
    const int g0 = (brick % a.nbx) * 16, a0 = ((brick / a.nbx) % a.nby) * 16, b0 = (brick / (a.nbx * a.nby)) * 8;
    const int g1 = min(g0 + 16, N) - 1, a1 = min(a0 + 16, N) - 1, b1 = min(b0 + 8, N) - 1;

    const int tid = threadIdx.x;
    for (int i = tid; i < 4 * kColTileCap; i += kColThreads) smem[i] = 0;
    for (int i = tid; i < nv * 5; i += kColThreads) {
        const int jj = i / 5, q = i % 5;
        reinterpret_cast<float4 *>(&fr[jj])[q] =
            reinterpret_cast<const float4 *>(&a.frames[(size_t)cond * g.V + a.view_list[j0 + jj]])[q];
    }
    __syncthreads();
    /* footprint per view from the brick's 8 corners (general ray casting) */
    for (int i = tid; i < nv; i += kColThreads) {
        const ViewFrame &f = fr[i];
        float umin = 1e30f, umax = -1e30f, vmin = 1e30f, vmax = -1e30f;
        bool ok = true;
        for (int c = 0; c < 8; c++) {
            int cc[3];
            cc[A] = (c & 1) ? a1 : a0;
            cc[B] = (c & 2) ? b1 : b0;
            cc[G] = (c & 4) ? g1 : g0;
            float u, v, Bv[3];
            fiber_ray(f, g, cc[0], cc[1], cc[2], u, v, Bv);
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
        {   /* row stride = 6 mod 8: segments four rows apart fall on other banks */
            const int Wp = W + (((6 - W) % 8) + 8) % 8;
            if (Wp * H <= kColTileCap) W = Wp;
        }
        if (iu1 < iu0 || iv1 < iv0) { W = 0; H = 0; } /* off the detector           */
        bbox[i] = make_int4(iu0, iv0, W, H);
    }

    const int lane = tid & 31, w = tid >> 5;
    const int ia = a0 + (w & 3) + 4 * ((lane >> 2) & 3);
    const int ib = b0 + (w >> 2) + 4 * (lane >> 4);
    const int igb = g0 + (lane & 3) * 4;
    const bool col_ok = ia < N && ib < N;
    const float ba = fiber_base(ia, N, g.vs), bb = fiber_base(ib, N, g.vs);
    const float sgn = (G == 1 ? -1.0f : 1.0f) * (msig < 0.f ? 1.0f : -1.0f);   /* s for g = x, z; -s for y */
    const size_t NN = (size_t)N * N, N3 = NN * N;
    const size_t sgs = (G == 0) ? 1 : (G == 1 ? (size_t)N : NN);
    size_t idx0;
    {
        int cc[3];
        cc[A] = ia; cc[B] = ib; cc[G] = igb;
        idx0 = (size_t)cc[0] + (size_t)N * cc[1] + NN * cc[2];
    }
    float ta[4], tb[4], m3[4], dg[4], dg2[4];
    bool okv[4];
    float bound = 0.f;
    {
        const float offg = fr[0].off[G], tg = fr[0].t[G];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            okv[q] = col_ok && igb + q <= g1;
            /* o_g = (p_g - off_g) - t_g; d_g = o_g - src_g = o_g (src_g = 0) */
            dg[q] = __fsub_rn(__fsub_rn(fiber_base(igb + q, N, g.vs), offg), tg);
            dg2[q] = __fmul_rn(dg[q], dg[q]);
            float mu[4];
#pragma unroll
            for (int k = 0; k < 4; k++)
                mu[k] = (okv[q] && k < K) ? __ldg(a.vol + idx0 + (size_t)q * sgs + k * N3) : 0.f;
            ta[q] = sgn * mu[A];
            tb[q] = sgn * mu[B];
            m3[q] = mu[3];
            if (okv[q])
                bound = fmaxf(bound, (fabsf(mu[0]) + fabsf(mu[1]) + fabsf(mu[2]) + fabsf(mu[3])) * g.vs * g.ratio *
                                         1.001f);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) bound = fmaxf(bound, __shfl_xor_sync(0xffffffffu, bound, o));
    if (lane == 0) s_red[w] = bound;
    __syncthreads();
    float S = 0.f;
#pragma unroll
    for (int i = 0; i < kColThreads / 32; i++) S = fmaxf(S, s_red[i]);
    if (!(S > 0.f) || !(S < 3e38f)) return;   /* nothing to splat (or non-finite input) */
    const int sh = fix_shift(S);
    const float fscale = ldexpf(1.0f, sh);
    const float finv = ldexpf(1.0f, -sh);
    const float wsc = __fmul_rn(g.vs, g.ratio);

    const size_t NdNd = (size_t)Nd * Nd;
    float *outc = a.out + (size_t)cond * g.V * NdNd;
    for (int jj = 0; jj < nv; jj++) {
        const ViewFrame &f = fr[jj];
        const int4 bb4 = bbox[jj];
        int *T = smem + (jj & 1) * 2 * kColTileCap;   /* hi words, lo words after */
        float *P = outc + (size_t)f.view * NdNd;
        const bool use_tile = (bb4.z > 0) && (bb4.z * bb4.w <= kColTileCap);
        if (bb4.z > 0 && col_ok) {
            /* rayCastingFiber's per-column part: the g terms of its three-term
             * dot products are exact zeros */
            const float oa = __fsub_rn(__fsub_rn(ba, f.off[A]), f.t[A]);
            const float ob = __fsub_rn(__fsub_rn(bb, f.off[B]), f.t[B]);
            const float da = __fsub_rn(oa, f.src[A]), db = __fsub_rn(ob, f.src[B]);
            const float sd = __fadd_rn(__fmul_rn(f.src[A], da), __fmul_rn(f.src[B], db));
            const float coeff = __fdiv_rn(-f.ss, sd);
            const float pa = __fadd_rn(f.src[A], __fmul_rn(coeff, da));
            const float pb = __fadd_rn(f.src[B], __fmul_rn(coeff, db));
            const float u = __fadd_rn(
                fdiv_det(__fmul_rn(__fadd_rn(__fmul_rn(pa, f.eu[A]), __fmul_rn(pb, f.eu[B])), g.mag), g), g.half);
            if (0.55f < u && u < g.lim) {
                const float ut = __fsub_rn(u, 0.5f);
                const float fiu = floorf(ut);
                const int iu = (int)fiu;
                const float fu = __fsub_rn(ut, fiu), gu = __fsub_rn(1.0f, fu);
                const int lu = iu - bb4.x;
                const bool col_tile = use_tile && lu >= 0 && lu + 1 < bb4.z;
                const int W = bb4.z;
                const float da2 = __fmul_rn(da, da), db2 = __fmul_rn(db, db);
                const float dab2 = __fadd_rn(da2, db2);
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    if (!okv[q]) continue;
                    const float v = __fadd_rn(fdiv_det(__fmul_rn(__fmul_rn(coeff, dg[q]), msig), g), g.half);
                    if (!(0.55f < v && v < g.lim)) continue;
                    const float vt = __fsub_rn(v, 0.5f);
                    const float fiv = floorf(vt);
                    const int iv = (int)fiv;
                    const float fv = __fsub_rn(vt, fiv), gv = __fsub_rn(1.0f, fv);
                    /* |d|^2 in the reference's x, y, z order */
                    const float l2 = (G == 0) ? __fadd_rn(__fadd_rn(dg2[q], da2), db2)
                                              : (G == 1 ? __fadd_rn(__fadd_rn(da2, dg2[q]), db2)
                                                        : __fadd_rn(dab2, dg2[q]));
                    const float rl = l2 > 1e-16f ? rsqrtf(l2) : 0.f;
                    const float ps = fmaf(fmaf(db, ta[q], -da * tb[q]), rl, m3[q]);
                    const float c1 = __fmul_rn(gu, fv), c2 = __fmul_rn(fu, fv);
                    const float c3 = __fmul_rn(fu, gv), c4 = __fmul_rn(gu, gv);
                    const int lv = iv - bb4.y;
                    if (col_tile && lv >= 0 && lv + 1 < bb4.w) {
                        /* the taps as two packed FP32x2 pairs (rows iv + 1 and iv) */
                        const float pw = fabsf(ps) * wsc * fscale;
                        int *t0 = T + lu + W * lv;
                        const float2 up = make_float2(gu * pw, fu * pw);
                        int2 h, l;
                        fix_split2(make_float2(up.x * fv, up.y * fv), h, l);
                        atomicAdd(t0 + W, h.x);
                        atomicAdd(t0 + W + kColTileCap, l.x);
                        atomicAdd(t0 + W + 1, h.y);
                        atomicAdd(t0 + W + 1 + kColTileCap, l.y);
                        fix_split2(make_float2(up.x * gv, up.y * gv), h, l);
                        atomicAdd(t0, h.x);
                        atomicAdd(t0 + kColTileCap, l.x);
                        atomicAdd(t0 + 1, h.y);
                        atomicAdd(t0 + 1 + kColTileCap, l.y);
                    } else {
                        const float pw = fabsf(ps) * wsc;
                        float *p0 = P + iu + (size_t)Nd * iv;
                        atomicAdd(p0 + Nd, c1 * pw);
                        atomicAdd(p0 + Nd + 1, c2 * pw);
                        atomicAdd(p0 + 1, c3 * pw);
                        atomicAdd(p0, c4 * pw);
                    }
                }
            }
        }
        __syncthreads();
        if (use_tile) {   /* one warp per tile row; the tile is cleared behind */
            for (int r = w; r < bb4.w; r += kColThreads / 32) {
                for (int cc = lane; cc < bb4.z; cc += 32) {
                    float t;
                    if (fix_take(T + cc + bb4.z * r, kColTileCap, finv, t))
                        atomicAdd(P + (bb4.x + cc) + (size_t)Nd * (bb4.y + r), t);
                }
            }
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Back-projection by bricks, fused with the update of channel 0.            */
/* A CTA owns an 8 x 8 x 8 brick; per axis its 128 threads map to 64 voxel    */
/* columns x 2 segments of 4 voxels along that axis's column axis g (any      */
/* mapping for a general axis), carry each voxel's running (tmp, fac) through */
/* shared memory from axis to axis, and add the axis's views in order: every  */
/* voxel's sums run in the reference's (axis, view) order, bit for bit.       */
/* Column-aligned axes (G = s e_g): coeff, u and the (a, b) components of the */
/* ray are per column and view; per voxel v, |d| and the weight               */
/*     w_0 = |(B x G)_0| = |d_b / |d||  (g = y or z),                         */
/* while for g = x the weight (B x G)_0 = B_y*0 - B_z*0 is exactly zero and   */
/* the axis adds (0 * c) * r = 0 to tmp and 0 to fac: the axis is skipped,    */
/* unless a ratio image of the session holds an infinity or a NaN (then       */
/* 0 * r is a NaN, and the axis runs as the reference's loop does).           */
/* ------------------------------------------------------------------------ */
constexpr int kBackColThreads = 128;
constexpr int kBackChunk = 32;   /* frames staged per pass */

struct FiberBackColArgs {
    GeomConst g;
    const ViewFrame *frames;   /* [C][V] */
    const int *view_list;
    int n_views, n_cond;
    const int *axis_g;         /* per axis: column axis, -1 general */
    const float *magsig;       /* per axis: sign(ev[g]) * mag       */
    const float *proj;         /* ratio images, C blocks            */
    float *vol;                /* channel 0 updated in place        */
    const int *nonfinite;      /* set: some ratio image held an inf or a NaN */
    int art;
    float alpha;
    int nb;                    /* bricks per dimension */
    cudaTextureObject_t rtex;  /* non-zero: the ratio images as a 2D-layered array, layer = axis * n_views + position */
};

/* One view of a column-aligned axis for a thread's segment of 4 voxels (the
 * 4 taps loaded, or with rtex gathered from layer `layer` in one texture
 * instruction: the same values in the same order). */
template <int G>
__device__ __forceinline__ void fiber_back_col_view(const ViewFrame &f, const GeomConst &g, const float *Pc, float ba,
                                                    float bb, float msig, const float dg[4], const float dg2[4],
                                                    const bool okv[4], float tmp[4], float fac[4],
                                                    cudaTextureObject_t rtex, int layer) {
    constexpr int A = FAx<G>::A, B = FAx<G>::B;
    const float oa = __fsub_rn(__fsub_rn(ba, f.off[A]), f.t[A]);
    const float ob = __fsub_rn(__fsub_rn(bb, f.off[B]), f.t[B]);
    const float da = __fsub_rn(oa, f.src[A]), db = __fsub_rn(ob, f.src[B]);
    const float sd = __fadd_rn(__fmul_rn(f.src[A], da), __fmul_rn(f.src[B], db));
    const float coeff = __fdiv_rn(-f.ss, sd);
    const float pa = __fadd_rn(f.src[A], __fmul_rn(coeff, da));
    const float pb = __fadd_rn(f.src[B], __fmul_rn(coeff, db));
    const float u = __fadd_rn(
        fdiv_det(__fmul_rn(__fadd_rn(__fmul_rn(pa, f.eu[A]), __fmul_rn(pb, f.eu[B])), g.mag), g), g.half);
    if (!(0.55f < u && u < g.lim)) return;
    const float ut = __fsub_rn(u, 0.5f);
    const float fiu = floorf(ut);
    const int iu = (int)fiu;
    const float fu = __fsub_rn(ut, fiu), gu = __fsub_rn(1.0f, fu);
    const float da2 = __fmul_rn(da, da), db2 = __fmul_rn(db, db);
    const float dab2 = __fadd_rn(da2, db2);
    const float *P = Pc + (size_t)f.view * g.Nd * g.Nd + iu;
    const float xu = __int2float_rn(iu + 1);
#pragma unroll
    for (int q = 0; q < 4; q++) {
        if (!okv[q]) continue;
        const float v = __fadd_rn(fdiv_det(__fmul_rn(__fmul_rn(coeff, dg[q]), msig), g), g.half);
        if (!(0.55f < v && v < g.lim)) continue;
        const float vt = __fsub_rn(v, 0.5f);
        const float fiv = floorf(vt);
        const int iv = (int)fiv;
        const float fv = __fsub_rn(vt, fiv), gv = __fsub_rn(1.0f, fv);
        float w0 = 0.f;
        if (G != 0) {
            const float l2 = (G == 1) ? __fadd_rn(__fadd_rn(da2, dg2[q]), db2) : __fadd_rn(dab2, dg2[q]);
            const float len = __fsqrt_rn(l2);
            w0 = len > 1e-8f ? fabsf(__fdiv_rn(db, len)) : 0.f;
        }
        float r0, r1, r2, r3;   /* P[iv+1][iu], P[iv+1][iu+1], P[iv][iu+1], P[iv][iu] */
        if (rtex) {
            const float4 t = gather_a2d(rtex, layer, xu, __fadd_rn(fiv, 1.0f));
            r0 = t.x;
            r1 = t.y;
            r2 = t.z;
            r3 = t.w;
        } else {
            const float *Pq = P + (size_t)g.Nd * iv;
            r0 = __ldg(Pq + g.Nd);
            r1 = __ldg(Pq + g.Nd + 1);
            r2 = __ldg(Pq + 1);
            r3 = __ldg(Pq);
        }
        float nb = __fmul_rn(__fmul_rn(w0, __fmul_rn(gu, fv)), r0);
        nb = __fadd_rn(nb, __fmul_rn(__fmul_rn(w0, __fmul_rn(fu, fv)), r1));
        nb = __fadd_rn(nb, __fmul_rn(__fmul_rn(w0, __fmul_rn(fu, gv)), r2));
        nb = __fadd_rn(nb, __fmul_rn(__fmul_rn(w0, __fmul_rn(gu, gv)), r3));
        tmp[q] = __fadd_rn(tmp[q], nb);
        fac[q] = __fadd_rn(fac[q], w0);
    }
}

/* The views of axis cond for the thread's 4 voxels (column axis G, or the
 * general ray casting when G < 0). */
template <int G>
__device__ __forceinline__ void fiber_back_axis(const FiberBackColArgs &a, ViewFrame *sfr, int cond, int x0,
                                                int y0, int z0, float tmp[4], float fac[4], const bool okv[4]) {
    const GeomConst &g = a.g;
    constexpr int GG = G < 0 ? 2 : G;
    constexpr int A = FAx<GG>::A, B = FAx<GG>::B;
    const int tid = threadIdx.x;
    int c0[3];
    c0[0] = x0; c0[1] = y0; c0[2] = z0;
    const int ia = c0[A] + (tid & 7), ib = c0[B] + ((tid >> 3) & 7), igb = c0[GG] + (tid >> 6) * 4;
    const float ba = fiber_base(ia, g.N, g.vs), bb = fiber_base(ib, g.N, g.vs);
    const float *Pc = a.proj + (size_t)cond * g.V * g.Nd * g.Nd;
    float dg[4], dg2[4], msig = 0.f;
    if (G >= 0) {
        msig = -a.magsig[cond];
        const ViewFrame &f0 = a.frames[(size_t)cond * g.V];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            dg[q] = __fsub_rn(__fsub_rn(fiber_base(igb + q, g.N, g.vs), f0.off[GG]), f0.t[GG]);
            dg2[q] = __fmul_rn(dg[q], dg[q]);
        }
    }
    for (int j0 = 0; j0 < a.n_views; j0 += kBackChunk) {
        const int nv = min(kBackChunk, a.n_views - j0);
        __syncthreads();   /* the previous chunk's frames are no longer read */
        for (int i = tid; i < nv * 5; i += kBackColThreads) {
            const int jj = i / 5, q = i % 5;
            reinterpret_cast<float4 *>(&sfr[jj])[q] =
                reinterpret_cast<const float4 *>(&a.frames[(size_t)cond * g.V + a.view_list[j0 + jj]])[q];
        }
        __syncthreads();
        for (int jj = 0; jj < nv; jj++) {
            const ViewFrame &f = sfr[jj];
            if (G >= 0) {
                fiber_back_col_view<GG>(f, g, Pc, ba, bb, msig, dg, dg2, okv, tmp, fac, a.rtex,
                                        cond * a.n_views + j0 + jj);
            } else {
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    if (!okv[q]) continue;
                    int cc[3];
                    cc[A] = ia; cc[B] = ib; cc[GG] = igb + q;
                    float u, v, Bv[3], w[4];
                    int iu, iv;
                    fiber_ray(f, g, cc[0], cc[1], cc[2], u, v, Bv);
                    if (!fiber_taps(g, u, v, iu, iv, w)) continue;
                    const float w0 = fabsf(__fsub_rn(__fmul_rn(Bv[1], f.ev[2]), __fmul_rn(Bv[2], f.ev[1])));
                    const float *P = Pc + (size_t)f.view * g.Nd * g.Nd + iu + (size_t)g.Nd * iv;
                    float nb = __fmul_rn(__fmul_rn(w0, w[0]), __ldg(P + g.Nd));
                    nb = __fadd_rn(nb, __fmul_rn(__fmul_rn(w0, w[1]), __ldg(P + g.Nd + 1)));
                    nb = __fadd_rn(nb, __fmul_rn(__fmul_rn(w0, w[2]), __ldg(P + 1)));
                    nb = __fadd_rn(nb, __fmul_rn(__fmul_rn(w0, w[3]), __ldg(P)));
                    tmp[q] = __fadd_rn(tmp[q], nb);
                    fac[q] = __fadd_rn(fac[q], w0);
                }
            }
        }
    }
}

/* local index in the 8^3 brick of the thread's voxel q for column axis GG */
template <int GG>
__device__ __forceinline__ int fiber_local(int q) {
    constexpr int A = FAx<GG>::A, B = FAx<GG>::B;
    const int tid = threadIdx.x;
    int c[3];
    c[A] = tid & 7;
    c[B] = (tid >> 3) & 7;
    c[GG] = (tid >> 6) * 4 + q;
    return c[0] + 8 * c[1] + 64 * c[2];
}

template <int G>
__device__ __forceinline__ void fiber_back_axis_shared(const FiberBackColArgs &a, ViewFrame *sfr, int cond,
                                                       int x0, int y0, int z0, float *s_tmp, float *s_fac) {
    constexpr int GG = G < 0 ? 2 : G;
    const int N = a.g.N;
    float tmp[4], fac[4];
    bool okv[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int l = fiber_local<GG>(q);
        tmp[q] = s_tmp[l];
        fac[q] = s_fac[l];
        okv[q] = x0 + (l & 7) < N && y0 + ((l >> 3) & 7) < N && z0 + (l >> 6) < N;
    }
    fiber_back_axis<G>(a, sfr, cond, x0, y0, z0, tmp, fac, okv);
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int l = fiber_local<GG>(q);
        s_tmp[l] = tmp[q];
        s_fac[l] = fac[q];
    }
}

__global__ void __launch_bounds__(kBackColThreads, 8) k_fiber_back_col(FiberBackColArgs a) {
    __shared__ float s_tmp[512], s_fac[512];
    __shared__ __align__(16) ViewFrame sfr[kBackChunk];
    const int nb = a.nb;
    const int x0 = (blockIdx.x % nb) * 8, y0 = ((blockIdx.x / nb) % nb) * 8, z0 = (blockIdx.x / (nb * nb)) * 8;
    const int tid = threadIdx.x;
    for (int i = tid; i < 512; i += kBackColThreads) {
        s_tmp[i] = 0.f;
        s_fac[i] = 0.f;
    }
    const bool zero_skip = *a.nonfinite == 0;
    for (int c = 0; c < a.n_cond; c++) {
        const int G = a.axis_g[c];
        if (G == 0 && zero_skip) continue;   /* adds exactly 0 to tmp and fac */
        __syncthreads();                     /* the previous axis's sums are in shared memory */
        if (G == 0) fiber_back_axis_shared<0>(a, sfr, c, x0, y0, z0, s_tmp, s_fac);
        else if (G == 1) fiber_back_axis_shared<1>(a, sfr, c, x0, y0, z0, s_tmp, s_fac);
        else if (G == 2) fiber_back_axis_shared<2>(a, sfr, c, x0, y0, z0, s_tmp, s_fac);
        else fiber_back_axis_shared<-1>(a, sfr, c, x0, y0, z0, s_tmp, s_fac);
    }
    __syncthreads();
    const int N = a.g.N;
    const size_t NN = (size_t)N * N;
    for (int l = tid; l < 512; l += kBackColThreads) {   /* x fastest: coalesced rows of 8 */
        const int x = x0 + (l & 7), y = y0 + ((l >> 3) & 7), z = z0 + (l >> 6);
        if (x >= N || y >= N || z >= N) continue;
        const size_t i = (size_t)x + (size_t)N * y + NN * z;
        const float mu0 = a.vol[i], tmp = s_tmp[l], fac = s_fac[l];
        if (a.art) a.vol[i] = __fadd_rn(mu0, __fmul_rn(a.alpha, tmp));
        else a.vol[i] = (fac == 0.0f) ? 0.0f : __fdiv_rn(__fmul_rn(mu0, tmp), fac);
    }
}

/* Sets *flag when a listed ratio image of the listed axes holds an infinity or a NaN. */
__global__ void k_fiber_nonfinite(GeomConst g, const int *view_list, int n_views, const float *proj, int *flag) {
    const size_t NdNd = (size_t)g.Nd * g.Nd;
    const int cond = blockIdx.y / n_views, j = blockIdx.y % n_views;
    const float *p = proj + ((size_t)cond * g.V + view_list[j]) * NdNd;
    bool bad = false;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < NdNd; i += (size_t)gridDim.x * blockDim.x)
        bad |= !isfinite(p[i]);
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}


}  // namespace

/* views per CTA: the whole list unless that leaves fewer than 2048 CTAs */
static int fiber_vpc(long ctas, int n_views) {
    const long chunks = ctas >= 2048 ? 1 : (2048 + ctas - 1) / ctas;
    int vpc = (int)((n_views + chunks - 1) / chunks);
    return vpc < 1 ? 1 : (vpc > 64 ? 64 : vpc);
}

cudaError_t launch_fiber_forward(const GeomConst &g, const ViewFrame *frames, const int *view_list, int n_views,
                                 const int *d_conds, int n_cond, const float *vol, float *out, cudaStream_t s) {
    if (n_views <= 0 || n_cond <= 0) return cudaSuccess;
    FiberFwdArgs a{};
    a.g = g;
    a.frames = frames;
    a.view_list = view_list;
    a.n_views = n_views;
    a.conds = d_conds;
    a.vol = vol;
    a.out = out;
    a.nbx = (g.N + kBX - 1) / kBX;
    a.nby = (g.N + kBY - 1) / kBY;
    const int nbz = (g.N + kBZ - 1) / kBZ;
    const long bricks = (long)a.nbx * a.nby * nbz;
    const int vpc = fiber_vpc(bricks * n_cond, n_views);
    a.vpc = vpc;
    const dim3 grid((unsigned)bricks, (unsigned)n_cond, (unsigned)((n_views + vpc - 1) / vpc));
    const size_t smem = 4 * kTileCap * sizeof(int) + (size_t)vpc * (sizeof(int4) + sizeof(ViewFrame));
    cudaError_t e = cudaFuncSetAttribute(k_fiber_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_fiber_forward<<<grid, kFwdThreads, smem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_fiber_forward_col(const GeomConst &g, const ViewFrame *frames, const int *view_list, int n_views,
                                     const int *d_conds, int n_cond, int G, const float *d_magsig, const float *vol,
                                     float *out, cudaStream_t s) {
    if (n_views <= 0 || n_cond <= 0) return cudaSuccess;
    FiberFwdArgs a{};
    a.g = g;
    a.frames = frames;
    a.view_list = view_list;
    a.n_views = n_views;
    a.conds = d_conds;
    a.magsig = d_magsig;
    a.vol = vol;
    a.out = out;
    a.nbx = (g.N + 15) / 16;   /* along g */
    a.nby = (g.N + 15) / 16;   /* along a */
    const long bricks = (long)a.nbx * a.nby * ((g.N + 7) / 8);
    const int vpc = fiber_vpc(bricks * n_cond, n_views);
    a.vpc = vpc;
    const dim3 grid((unsigned)bricks, (unsigned)n_cond, (unsigned)((n_views + vpc - 1) / vpc));
    const size_t smem = 4 * kColTileCap * sizeof(int) + (size_t)vpc * (sizeof(int4) + sizeof(ViewFrame));
#define XR_FIBER_COL(GG)                                                                                          \
    do {                                                                                                          \
        cudaError_t e = cudaFuncSetAttribute(k_fiber_fwd_col<GG>, cudaFuncAttributeMaxDynamicSharedMemorySize,    \
                                             (int)smem);                                                          \
        if (e != cudaSuccess) return e;                                                                           \
        k_fiber_fwd_col<GG><<<grid, kColThreads, smem, s>>>(a);                                                   \
    } while (0)
    if (G == 0) XR_FIBER_COL(0);
    else if (G == 1) XR_FIBER_COL(1);
    else XR_FIBER_COL(2);
#undef XR_FIBER_COL
    return cudaGetLastError();
}

cudaError_t launch_fiber_back(const GeomConst &g, const ViewFrame *frames, const int *view_list, int n_views,
                              int n_cond, const int *d_axis_g, const float *d_magsig, const float *proj, float *vol,
                              int art, float alpha, int *d_nonfinite, cudaStream_t s, cudaTextureObject_t rtex) {
    if (n_views <= 0 || n_cond <= 0) return cudaSuccess;
    {   /* the ratio images the back-projection reads: any inf or NaN? */
        const dim3 grid((unsigned)((g.Nd * g.Nd + 255) / 256 < 8 ? (g.Nd * g.Nd + 255) / 256 : 8),
                        (unsigned)(n_cond * n_views));
        k_fiber_nonfinite<<<grid, 256, 0, s>>>(g, view_list, n_views, proj, d_nonfinite);
    }
    FiberBackColArgs a{};
    a.g = g;
    a.frames = frames;
    a.view_list = view_list;
    a.n_views = n_views;
    a.n_cond = n_cond;
    a.axis_g = d_axis_g;
    a.magsig = d_magsig;
    a.proj = proj;
    a.vol = vol;
    a.nonfinite = d_nonfinite;
    a.rtex = rtex;
    a.art = art;
    a.alpha = alpha;
    a.nb = (g.N + 7) / 8;
    k_fiber_back_col<<<(unsigned)((long)a.nb * a.nb * a.nb), kBackColThreads, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace xr
