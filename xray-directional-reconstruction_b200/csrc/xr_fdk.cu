/*
 * FDK on the GPU (FDK::reconstruct, reconstruct.cu:1651-1724).
 *
 * The reference launches calcWeight once, then per view one projConv over the
 * detector followed by N filteredBackProj launches (one per y slab).  Here:
 *   k_fdk_weight  cosine weight sdd / sqrt(sdd^2 + u^2 + v^2) (fdk.cu:13-26)
 *   k_fdk_conv    every view's rows in one launch; a CTA stages one detector
 *                 row of the projection and of the weight in shared memory
 *                 and each thread sums filt[|u-j|] * src[j] * w[j] over j in
 *                 the reference's order (fdk.cu:28-43) for 4 outputs at once
 *   k_fdk_bp      one thread per voxel loops over all views, gathering the
 *                 bilinear taps and adding (sod/(sod+o_y))^2 * (2 pi/V) * tap
 *                 sum in the reference's view order (fdk.cu:62-170), one store
 *                 per voxel; k_fdk_bp_col is the same for axes that rotate
 *                 about a grid axis, with the ray set-up once per voxel column.
 * FP32 operations on the per-voxel path are explicitly rounded (no FMA
 * contraction), matching the reference's arithmetic.
 */
#include <cuda_runtime.h>

#include "xr_internal.h"
#include "xr_tex.cuh"

namespace xr {
namespace {

constexpr int kBpThreads = 256;
constexpr int kFrameChunk = 128;

__device__ __forceinline__ float dot_rn(float a0, float a1, float a2, float b0, float b1, float b2) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a0, b0), __fmul_rn(a1, b1)), __fmul_rn(a2, b2));
}

/* ((2i - N + 1) * 0.5) * vs: FDK's centred voxel grid (fdk.cu:132-135). */
__device__ __forceinline__ float vox_base_fdk(int i, int N, float vs) {
    const float a = __fadd_rn(__fsub_rn(__fmul_rn(2.0f, (float)i), (float)N), 1.0f);
    return __fmul_rn(__fmul_rn(a, 0.5f), vs);
}

__global__ void k_fdk_weight(GeomConst g, float *w) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int v = blockIdx.y * blockDim.y + threadIdx.y;
    if (u >= g.Nd || v >= g.Nd) return;
    const float hn = __fdiv_rn((float)g.Nd, 2.0f);
    const float ur = __fmul_rn(__fsub_rn(__fadd_rn((float)u, 0.5f), hn), g.det);
    const float vr = __fmul_rn(__fsub_rn(__fadd_rn((float)v, 0.5f), hn), g.det);
    const float r2 = __fadd_rn(__fadd_rn(__fmul_rn(g.sdd, g.sdd), __fmul_rn(ur, ur)), __fmul_rn(vr, vr));
    w[u + g.Nd * v] = __fdiv_rn(g.sdd, __fsqrt_rn(r2));
}

/* grid (row v, view, axis); dst row = sum_j filt[|u-j|] src[j] w[j], each
 * output's terms added in j order ((filt * src) * w, fdk.cu:28-43).  A thread
 * owns 4 consecutive outputs u0..u0+3: per j it reads src[j] and w[j] once
 * and the filter as a window sliding over the mirrored table
 * fs[Nd - 1 + k] = filt[|k|], so each j costs one new filter value. */
constexpr int kConvOut = 4;

/* surf (non-zero): the filtered rows also go to layer (axis * V + view) of
 * that 2D-layered surface, which k_fdk_bp_col gathers from. */
__global__ void k_fdk_conv(GeomConst g, const float *sino, float *dst, const float *filt, const float *w,
                           cudaSurfaceObject_t surf) {
    extern __shared__ float sm[];
    const int Nd = g.Nd;
    float *srow = sm, *wrow = sm + Nd, *fs = sm + 2 * Nd;   /* fs: 2 Nd - 1 entries */
    const int v = blockIdx.x, view = blockIdx.y, cond = blockIdx.z;
    const size_t off = ((size_t)cond * g.V + view) * (size_t)Nd * Nd + (size_t)Nd * v;
    for (int j = threadIdx.x; j < Nd; j += blockDim.x) {
        srow[j] = sino[off + j];
        wrow[j] = w[(size_t)Nd * v + j];
    }
    for (int k = threadIdx.x; k < 2 * Nd - 1; k += blockDim.x) fs[k] = filt[k >= Nd - 1 ? k - (Nd - 1) : (Nd - 1) - k];
    __syncthreads();
    for (int u0 = threadIdx.x * kConvOut; u0 < Nd; u0 += blockDim.x * kConvOut) {
        /* window f[r] = filt[|u0 + r - j|] = fs[Nd - 1 + u0 + r - j]; indices
         * beyond the table occur only for outputs u0 + r >= Nd (not stored) */
        const int base = Nd - 1 + u0;
        float acc[kConvOut] = {0.f, 0.f, 0.f, 0.f};
        float f[kConvOut];
#pragma unroll
        for (int r = 0; r < kConvOut; r++) f[r] = (base + r < 2 * Nd - 1) ? fs[base + r] : 0.f;
#pragma unroll 4
        for (int j = 0; j < Nd; j++) {
            const float sj = srow[j], wj = wrow[j];
#pragma unroll
            for (int r = 0; r < kConvOut; r++) acc[r] = __fadd_rn(acc[r], __fmul_rn(__fmul_rn(f[r], sj), wj));
            /* slide: f[r] <- fs[base + r - (j + 1)] */
#pragma unroll
            for (int r = kConvOut - 1; r > 0; r--) f[r] = f[r - 1];
            f[0] = (base - j - 1 >= 0) ? fs[base - j - 1] : 0.f;
        }
#pragma unroll
        for (int r = 0; r < kConvOut; r++) {
            if (u0 + r >= Nd) continue;
            dst[off + u0 + r] = acc[r];
            if (surf)
                surf2DLayeredwrite(acc[r], surf, (u0 + r) * (int)sizeof(float), v, cond * g.V + view,
                                   cudaBoundaryModeZero);
        }
    }
}

struct BpArgs {
    GeomConst g;
    const ViewFrame *frames;   /* FDK frames [C][V] (source at -sod)          */
    const float *filt_sino;    /* C blocks of filtered projections            */
    float *vol;                /* C channels of N^3                           */
    int cond, src_block;
    cudaTextureObject_t ftex;  /* k_fdk_bp_col<G, true>: the filtered projections, layer = block * V + view */
};

__global__ void __launch_bounds__(kBpThreads) k_fdk_bp(BpArgs a) {
    __shared__ ViewFrame fr[kFrameChunk];
    const GeomConst &g = a.g;
    const int N = g.N, Nd = g.Nd;
    const int nbx = (N + 7) / 8, nby = (N + 3) / 4;
    const int b = blockIdx.x;
    const int x = (b % nbx) * 8 + (threadIdx.x & 7);
    const int y = ((b / nbx) % nby) * 4 + ((threadIdx.x >> 3) & 3);
    const int z = (b / (nbx * nby)) * 8 + (threadIdx.x >> 5);
    const bool ok = x < N && y < N && z < N;
    const float bx = vox_base_fdk(x, N, g.vs), by = vox_base_fdk(y, N, g.vs), bz = vox_base_fdk(z, N, g.vs);
    const size_t NdNd = (size_t)Nd * Nd;
    const float *P = a.filt_sino + (size_t)a.src_block * g.V * NdNd;
    const float Cw = __fdiv_rn(__fmul_rn(2.0f, (float)M_PI), (float)g.V);
    float acc = 0.0f;
    for (int c0 = 0; c0 < g.V; c0 += kFrameChunk) {
        const int nc = min(kFrameChunk, g.V - c0);
        __syncthreads();
        for (int i = threadIdx.x; i < nc * 5; i += kBpThreads) {
            const int jj = i / 5, q = i % 5;
            reinterpret_cast<float4 *>(&fr[jj])[q] =
                reinterpret_cast<const float4 *>(&a.frames[(size_t)a.cond * g.V + c0 + jj])[q];
        }
        __syncthreads();
        if (!ok) continue;
        for (int jj = 0; jj < nc; jj++) {
            const ViewFrame &f = fr[jj];
            const float ox = __fsub_rn(__fsub_rn(bx, f.off[0]), f.t[0]);
            const float oy = __fsub_rn(__fsub_rn(by, f.off[1]), f.t[1]);
            const float oz = __fsub_rn(__fsub_rn(bz, f.off[2]), f.t[2]);
            const float d0 = __fsub_rn(ox, f.src[0]), d1 = __fsub_rn(oy, f.src[1]), d2 = __fsub_rn(oz, f.src[2]);
            const float coeff = __fdiv_rn(-f.ss, dot_rn(f.src[0], f.src[1], f.src[2], d0, d1, d2));
            const float p0 = __fadd_rn(f.src[0], __fmul_rn(coeff, d0));
            const float p1 = __fadd_rn(f.src[1], __fmul_rn(coeff, d1));
            const float p2 = __fadd_rn(f.src[2], __fmul_rn(coeff, d2));
            const float u = __fadd_rn(__fdiv_rn(__fmul_rn(dot_rn(p0, p1, p2, f.eu[0], f.eu[1], f.eu[2]), g.mag), g.det),
                                      g.half);
            const float v = __fadd_rn(__fdiv_rn(__fmul_rn(dot_rn(p0, p1, p2, f.ev[0], f.ev[1], f.ev[2]), g.mag), g.det),
                                      g.half);
            if (!(0.55f < u && u < g.lim && 0.55f < v && v < g.lim)) continue;
            const float ut = __fsub_rn(u, 0.5f), vt = __fsub_rn(v, 0.5f);
            const float fiu = floorf(ut), fiv = floorf(vt);
            const int iu = (int)fiu, iv = (int)fiv;
            const float fu = __fsub_rn(ut, fiu), fv = __fsub_rn(vt, fiv);
            const float gu = __fsub_rn(1.0f, fu), gv = __fsub_rn(1.0f, fv);
            const float c1 = __fmul_rn(gu, fv), c2 = __fmul_rn(fu, fv), c3 = __fmul_rn(fu, gv), c4 = __fmul_rn(gu, gv);
            const float U = __fdiv_rn(g.sod, __fadd_rn(g.sod, oy));
            const float *pp = P + (size_t)f.view * NdNd + iu + (size_t)Nd * iv;
            const float p4 = __ldg(pp), p3 = __ldg(pp + 1), p1v = __ldg(pp + Nd), p2v = __ldg(pp + Nd + 1);
            const float nb = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(c1, p1v), __fmul_rn(c2, p2v)), __fmul_rn(c3, p3)),
                                       __fmul_rn(c4, p4));
            acc = __fadd_rn(acc, __fmul_rn(__fmul_rn(__fmul_rn(U, U), Cw), nb));
        }
    }
    if (ok) a.vol[(size_t)a.cond * N * N * N + (size_t)x + (size_t)N * y + (size_t)N * N * z] = acc;
}

/* a / det, correctly rounded (one Markstein correction step with
 * rdet = RN(1/det), checked bit for bit against IEEE division on this device
 * when g.exact_rdet is set; else IEEE division). */
__device__ __forceinline__ float fdk_div_det(float a, const GeomConst &g) {
    if (!g.exact_rdet) return __fdiv_rn(a, g.det);
    const float q = __fmul_rn(a, g.rdet);
    const float r = __fmaf_rn(-q, g.det, a);
    return __fmaf_rn(r, g.rdet, q);
}

template <int G>
struct FdkAx {
    static constexpr int A = (G == 0) ? 1 : 0;   /* the two other axes, ascending */
    static constexpr int B = (G == 2) ? 1 : 2;
};

struct BpColArgs {
    BpArgs b;
    float magsig;              /* ev[G] * mag (ev = +-e_G for every view) */
    int nbg, nba;              /* bricks of 16 along G and of 8 along A  */
};

/* The same back-projection for an axis whose every view has ev = +-e_G,
 * src_G = eu_G = 0 and the same off_G and t_G (checked on the host): along
 * a voxel column parallel to G the ray set-up (coeff, u and, unless G is y,
 * the weight (sod / (sod + o_y))^2 * 2 pi / V) is the same bit for bit (the
 * dropped terms of the three-term dot products are exact zeros), so a thread
 * computes it once per view for its 4 voxels along G and per voxel only
 * v = ((coeff * o_G) * ev_G mag) / det + Nd/2, the taps and the gather.  Each
 * voxel still adds its views in order: the result equals k_fdk_bp's.
 * Brick: 16 along G x 8 x 8, 256 threads = 64 columns x 4 segments. */
template <int G, bool TEX>
__global__ void __launch_bounds__(kBpThreads, 4) k_fdk_bp_col(BpColArgs c) {
    __shared__ ViewFrame fr[kFrameChunk];
    constexpr int A = FdkAx<G>::A, B = FdkAx<G>::B;
    const BpArgs &a = c.b;
    const GeomConst &g = a.g;
    const int N = g.N, Nd = g.Nd;
    const int b = blockIdx.x;
    const int g0 = (b % c.nbg) * 16, a0 = ((b / c.nbg) % c.nba) * 8, b0 = (b / (c.nbg * c.nba)) * 8;
    const int tid = threadIdx.x;
    const int ia = a0 + (tid & 7), ib = b0 + ((tid >> 3) & 7), igb = g0 + (tid >> 6) * 4;
    const bool col_ok = ia < N && ib < N;
    const float ba = vox_base_fdk(ia, N, g.vs), bb = vox_base_fdk(ib, N, g.vs);
    const size_t NdNd = (size_t)Nd * Nd;
    const float *P = a.filt_sino + (size_t)a.src_block * g.V * NdNd;
    const float Cw = __fdiv_rn(__fmul_rn(2.0f, (float)M_PI), (float)g.V);
    float dg[4], acc[4] = {0.f, 0.f, 0.f, 0.f};
    bool okv[4];
    {
        const ViewFrame &f0 = a.frames[(size_t)a.cond * g.V];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            okv[q] = col_ok && igb + q < N;
            dg[q] = __fsub_rn(__fsub_rn(vox_base_fdk(igb + q, N, g.vs), f0.off[G]), f0.t[G]);
        }
    }
    for (int c0 = 0; c0 < g.V; c0 += kFrameChunk) {
        const int nc = min(kFrameChunk, g.V - c0);
        __syncthreads();
        for (int i = tid; i < nc * 5; i += kBpThreads) {
            const int jj = i / 5, q = i % 5;
            reinterpret_cast<float4 *>(&fr[jj])[q] =
                reinterpret_cast<const float4 *>(&a.frames[(size_t)a.cond * g.V + c0 + jj])[q];
        }
        __syncthreads();
        if (!col_ok) continue;
        for (int jj = 0; jj < nc; jj++) {
            const ViewFrame &f = fr[jj];
            const float oa = __fsub_rn(__fsub_rn(ba, f.off[A]), f.t[A]);
            const float ob = __fsub_rn(__fsub_rn(bb, f.off[B]), f.t[B]);
            const float da = __fsub_rn(oa, f.src[A]), db = __fsub_rn(ob, f.src[B]);
            const float coeff = __fdiv_rn(-f.ss, __fadd_rn(__fmul_rn(f.src[A], da), __fmul_rn(f.src[B], db)));
            const float pa = __fadd_rn(f.src[A], __fmul_rn(coeff, da));
            const float pb = __fadd_rn(f.src[B], __fmul_rn(coeff, db));
            const float u = __fadd_rn(
                fdk_div_det(__fmul_rn(__fadd_rn(__fmul_rn(pa, f.eu[A]), __fmul_rn(pb, f.eu[B])), g.mag), g), g.half);
            if (!(0.55f < u && u < g.lim)) continue;
            const float ut = __fsub_rn(u, 0.5f);
            const float fiu = floorf(ut);
            const int iu = (int)fiu;
            const float fu = __fsub_rn(ut, fiu), gu = __fsub_rn(1.0f, fu);
            /* (sod / (sod + o_y))^2 * 2 pi / V: per column unless y is the column axis */
            float w = 0.f;
            if (G != 1) {
                const float U = __fdiv_rn(g.sod, __fadd_rn(g.sod, A == 1 ? oa : ob));
                w = __fmul_rn(__fmul_rn(U, U), Cw);
            }
            const float *Pc = P + (size_t)f.view * NdNd + iu;
            const float xu = __int2float_rn(iu + 1);   /* TEX: texels iu, iu + 1 */
            const int layer = a.src_block * g.V + f.view;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                if (!okv[q]) continue;
                const float v = __fadd_rn(fdk_div_det(__fmul_rn(__fmul_rn(coeff, dg[q]), c.magsig), g), g.half);
                if (!(0.55f < v && v < g.lim)) continue;
                const float vt = __fsub_rn(v, 0.5f);
                const float fiv = floorf(vt);
                const int iv = (int)fiv;
                const float fv = __fsub_rn(vt, fiv), gv = __fsub_rn(1.0f, fv);
                const float c1 = __fmul_rn(gu, fv), c2 = __fmul_rn(fu, fv), c3 = __fmul_rn(fu, gv),
                            c4 = __fmul_rn(gu, gv);
                float p4, p3, p1v, p2v;
                if (TEX) {   /* one gather: the same four values, numBack's order */
                    const float4 t = gather_a2d(a.ftex, layer, xu, __fadd_rn(fiv, 1.0f));
                    p1v = t.x;
                    p2v = t.y;
                    p3 = t.z;
                    p4 = t.w;
                } else {
                    const float *pp = Pc + (size_t)Nd * iv;
                    p4 = __ldg(pp);
                    p3 = __ldg(pp + 1);
                    p1v = __ldg(pp + Nd);
                    p2v = __ldg(pp + Nd + 1);
                }
                const float nb = __fadd_rn(
                    __fadd_rn(__fadd_rn(__fmul_rn(c1, p1v), __fmul_rn(c2, p2v)), __fmul_rn(c3, p3)), __fmul_rn(c4, p4));
                float wq = w;
                if (G == 1) {   /* o_y = o_G: per voxel */
                    const float U = __fdiv_rn(g.sod, __fadd_rn(g.sod, dg[q]));
                    wq = __fmul_rn(__fmul_rn(U, U), Cw);
                }
                acc[q] = __fadd_rn(acc[q], __fmul_rn(wq, nb));
            }
        }
    }
    if (!col_ok) return;
    const size_t NN = (size_t)N * N;
    float *out = a.vol + (size_t)a.cond * NN * N;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        if (!okv[q]) continue;
        int cc[3];
        cc[A] = ia;
        cc[B] = ib;
        cc[G] = igb + q;
        out[(size_t)cc[0] + (size_t)N * cc[1] + NN * cc[2]] = acc[q];
    }
}

}  // namespace

cudaError_t launch_fdk(const GeomConst &g, const ViewFrame *fdk_frames, int n_cond, const float *sino,
                       float *sino_filt, float *vol, const float *filt, float *weight, int axis_blocks,
                       cudaStream_t s, const int *h_axis_g, const float *h_magsig, cudaSurfaceObject_t fsurf,
                       cudaTextureObject_t ftex) {
    {
        const dim3 blk(32, 8), grid((g.Nd + 31) / 32, (g.Nd + 7) / 8);
        k_fdk_weight<<<grid, blk, 0, s>>>(g, weight);
    }
    {
        const dim3 grid((unsigned)g.Nd, (unsigned)g.V, (unsigned)n_cond);
        const size_t smem = 4 * (size_t)g.Nd * sizeof(float);
        if (smem > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(k_fdk_conv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
        }
        int thr = ((g.Nd + kConvOut - 1) / kConvOut + 31) / 32 * 32;   /* one group of outputs per thread */
        thr = thr > 256 ? 256 : thr;
        k_fdk_conv<<<grid, thr, smem, s>>>(g, sino, sino_filt, filt, weight, ftex ? fsurf : 0);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const long nb = (long)((g.N + 7) / 8) * ((g.N + 3) / 4) * ((g.N + 7) / 8);
    for (int c = 0; c < n_cond; c++) {
        BpArgs a;
        a.g = g;
        a.frames = fdk_frames;
        a.filt_sino = sino_filt;
        a.vol = vol;
        a.cond = c;
        a.src_block = axis_blocks ? c : 0;
        a.ftex = ftex;
        const int G = h_axis_g ? h_axis_g[c] : -1;
        if (G < 0) {
            k_fdk_bp<<<(unsigned)nb, kBpThreads, 0, s>>>(a);
            continue;
        }
        BpColArgs cb;
        cb.b = a;
        cb.magsig = h_magsig[c];
        cb.nbg = (g.N + 15) / 16;
        cb.nba = (g.N + 7) / 8;
        const unsigned nbc = (unsigned)((long)cb.nbg * cb.nba * ((g.N + 7) / 8));
        if (ftex) {
            if (G == 0) k_fdk_bp_col<0, true><<<nbc, kBpThreads, 0, s>>>(cb);
            else if (G == 1) k_fdk_bp_col<1, true><<<nbc, kBpThreads, 0, s>>>(cb);
            else k_fdk_bp_col<2, true><<<nbc, kBpThreads, 0, s>>>(cb);
        } else {
            if (G == 0) k_fdk_bp_col<0, false><<<nbc, kBpThreads, 0, s>>>(cb);
            else if (G == 1) k_fdk_bp_col<1, false><<<nbc, kBpThreads, 0, s>>>(cb);
            else k_fdk_bp_col<2, false><<<nbc, kBpThreads, 0, s>>>(cb);
        }
    }
    return cudaGetLastError();
}

}  // namespace xr
