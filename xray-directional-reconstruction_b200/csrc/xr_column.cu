/*
 * Column-structured projector kernels for rotation axes whose grating
 * direction G = elemR_c e_z is a grid axis g (G = +-e_g).
 *
 * For such an axis every view's detector v axis is +-e_g and its source and
 * detector u axis have a zero g component, so along a voxel column parallel
 * to g the reference's rayCasting (ir.cu:1881-1897) produces the SAME u,
 * coeff and source-to-voxel (a, b) components — bit for bit, the dropped
 * terms being exact zeros — and v differs only through o_g:
 *     v = ((+-(coeff * o_g)) * mag) / det + Nd/2.
 * A thread owns a segment of 4 voxels along g: the ray set-up is paid once per
 * column and view, each voxel then costs ~8 operations for its v.  The
 * sample-rotation axes of the three-axis XTT scans (elemR = I and the two
 * 90-degree tilts) are of this kind; other axes take the general kernels in
 * xr_kernels.cu.
 *
 * Division by the detector pitch: a / det = q + r * rdet with q = a * rdet,
 * r = fma(-q, det, a) and rdet = RN(1/det) — one Markstein correction step
 * (P. Markstein, "Computation of elementary functions on the IBM RISC
 * System/6000 processor", IBM J. Res. Dev. 34(1), 1990).  Every context
 * checks it bit for bit against IEEE division over all the magnitudes a
 * projector meets before using it (k_check_div); otherwise __fdiv_rn is used.
 */
#include <cuda_runtime.h>

#include "xr_internal.h"
#include "xr_storage.cuh"
#include "xr_tile.cuh"
#include "xr_orth.cuh"
#include "xr_tex.cuh"

namespace xr {
namespace {

constexpr int kTileCap = 64 * 64;
constexpr int kFwdThreads = 512;               /* forward: 16 (g) x 16 x 8 brick, 4 voxels/thread */
constexpr int kBackThreads = 128;              /* back: 8 x 8 x 8 brick, 4 voxels/thread          */
constexpr int kFrameChunk = 48;                /* back: frames staged per pass (3.8 KB), 6 CTAs/SM */

__device__ __forceinline__ float vox_base(int i, int N, float vs) {
    const float a = __fsub_rn(__fsub_rn(__fmul_rn(2.0f, (float)i), (float)N), 1.0f);
    return __fmul_rn(__fmul_rn(a, 0.5f), vs);
}

/* a / det, correctly rounded. */
__device__ __forceinline__ float div_det(float a, const GeomConst &g) {
    if (!g.exact_rdet) return __fdiv_rn(a, g.det);
    const float q = __fmul_rn(a, g.rdet);
    const float r = __fmaf_rn(-q, g.det, a);
    return __fmaf_rn(r, g.rdet, q);
}

/* A pair with both lanes equal: the broadcast operand of packed FP32x2 ops. */
__device__ __forceinline__ float2 bc2(float x) { return make_float2(x, x); }

template <int G>
struct Ax {
    static constexpr int A = (G == 0) ? 1 : 0;   /* the two other axes, ascending */
    static constexpr int B = (G == 2) ? 1 : 2;
};

/* Per-column part of rayCasting for column axis G: u, coeff and the (a, b)
 * components of the source-to-voxel vector.  The reference's three-term dot
 * products lose their g terms (exact zeros). */
template <int G>
__device__ __forceinline__ void col_ray(const ViewFrame &f, const GeomConst &g, float ba, float bb, float &u,
                                        float &coeff, float &da, float &db) {
    constexpr int A = Ax<G>::A, B = Ax<G>::B;
    const float oa = __fsub_rn(__fsub_rn(ba, f.off[A]), f.t[A]);
    const float ob = __fsub_rn(__fsub_rn(bb, f.off[B]), f.t[B]);
    da = __fsub_rn(oa, f.src[A]);
    db = __fsub_rn(ob, f.src[B]);
    const float sd = __fadd_rn(__fmul_rn(f.src[A], da), __fmul_rn(f.src[B], db));
    coeff = __fdiv_rn(-f.ss, sd);
    const float pa = __fadd_rn(f.src[A], __fmul_rn(coeff, da));
    const float pb = __fadd_rn(f.src[B], __fmul_rn(coeff, db));
    const float pu = __fadd_rn(__fmul_rn(pa, f.eu[A]), __fmul_rn(pb, f.eu[B]));
    u = __fadd_rn(div_det(__fmul_rn(pu, g.mag), g), g.half);
}

/* Per-voxel v; dg receives o_g (= the g component of source-to-voxel). */
template <int G>
__device__ __forceinline__ float col_v(const ViewFrame &f, const GeomConst &g, float bg, float coeff, float magsig,
                                       float &dg) {
    dg = __fsub_rn(__fsub_rn(bg, f.off[G]), f.t[G]);
    return __fadd_rn(div_det(__fmul_rn(__fmul_rn(coeff, dg), magsig), g), g.half);
}

/* One axis of the bilinear taps: window test and weights, as ir.cu:1501-1509
 * (the reference's combined u-and-v test splits exactly into the two). */
__device__ __forceinline__ bool tap1(const GeomConst &g, float u, int &i, float &f, float &gm) {
    if (!(0.55f < u && u < g.lim)) return false;
    const float ut = __fsub_rn(u, 0.5f);
    const float fi = floorf(ut);
    i = (int)fi;
    f = __fsub_rn(ut, fi);
    gm = __fsub_rn(1.0f, f);
    return true;
}

template <int G>
__device__ __forceinline__ void xyz_of(int ia, int ib, int ig, int &x, int &y, int &z) {
    constexpr int A = Ax<G>::A, B = Ax<G>::B;
    int c[3];
    c[A] = ia;
    c[B] = ib;
    c[G] = ig;
    x = c[0];
    y = c[1];
    z = c[2];
}

/* ------------------------------------------------------------------------ */
/* Forward splat, column form.  Brick: 16 along g, 16 along a, 8 along b.    */
/* Warp = 4 segments x 4 (a) x 2 (b) columns; 16 warps tile 16 x 8 columns.  */
/* ------------------------------------------------------------------------ */
struct FwdColArgs {
    GeomConst g;
    const ViewFrame *frames;
    const int *view_list;
    int n_views, vpc;
    const int *conds;         /* n_cond axis indices (k_fwd_col: all with column axis G) */
    const float *magsig;      /* per axis: sign(ev[g]) * mag                 */
    const void *vol;          /* storage type T                              */
    float *out;
    const BasisConst *basis;
    const float *coef;        /* mode 3: per-voxel rotation planes           */
    int coef_kind;            /* 0: (phi, cos theta); 1: main direction      */
    int nbg, nba;             /* bricks along g and a                        */
    int zlo, zhi;             /* only bricks whose first z lies in [zlo, zhi) */
    const int *axis_g;        /* k_fwd_col_axes: per axis its column axis    */
};

/* One CTA's work: brick blockIdx.x, views chunk blockIdx.z of axis cond. */
template <int MODE, int G, typename T>
__device__ __forceinline__ void fwd_col_brick(const FwdColArgs &a, const int cond) {
    const T *vol = reinterpret_cast<const T *>(a.vol);
    constexpr int A = Ax<G>::A, B = Ax<G>::B;
    /* Two detector tiles (double-buffered over views) in two-word fixed
     * point, xr_tile.cuh: native 32-bit shared atomics, per-CTA sums exact
     * to 2^-39 of the brick's largest contribution. */
    extern __shared__ int smem[];
    __shared__ float s_red[kFwdThreads / 32];
    int4 *bbox = reinterpret_cast<int4 *>(smem + 4 * kTileCap);
    ViewFrame *fr = reinterpret_cast<ViewFrame *>(bbox + a.vpc);

    const GeomConst &g = a.g;
    const int N = g.N, Nd = g.Nd;
    const float magsig = a.magsig[cond];
    const int j0 = blockIdx.z * a.vpc;
    const int nv = min(a.vpc, a.n_views - j0);
    if (nv <= 0) return;

    const int brick = blockIdx.x;
    const int g0 = (brick % a.nbg) * 16, a0 = ((brick / a.nbg) % a.nba) * 16, b0 = (brick / (a.nbg * a.nba)) * 8;
    const int g1 = min(g0 + 16, N) - 1, a1 = min(a0 + 16, N) - 1, b1 = min(b0 + 8, N) - 1;
    {   /* z of the brick's first voxel: g for column axis z, b otherwise */
        const int z0 = (G == 2) ? g0 : b0;
        if (z0 < a.zlo || z0 >= a.zhi) return;
    }

    const int tid = threadIdx.x;
    for (int i = tid; i < 4 * kTileCap; i += kFwdThreads) smem[i] = 0;
    for (int i = tid; i < nv * 5; i += kFwdThreads) {
        const int jj = i / 5, q = i % 5;
        reinterpret_cast<float4 *>(&fr[jj])[q] =
            reinterpret_cast<const float4 *>(&a.frames[(size_t)cond * g.V + a.view_list[j0 + jj]])[q];
    }
    __syncthreads();
    /* footprint bounding box per view from the 8 brick corners */
    for (int i = tid; i < nv; i += kFwdThreads) {
        const ViewFrame &f = fr[i];
        float umin = 1e30f, umax = -1e30f, vmin = 1e30f, vmax = -1e30f;
        bool ok = true;
        for (int c = 0; c < 8; c++) {
            const float ba = vox_base((c & 1) ? a1 : a0, N, g.vs);
            const float bb = vox_base((c & 2) ? b1 : b0, N, g.vs);
            const float bg = vox_base((c & 4) ? g1 : g0, N, g.vs);
            float u, coeff, da, db, dg;
            col_ray<G>(f, g, ba, bb, u, coeff, da, db);
            const float v = col_v<G>(f, g, bg, coeff, magsig, dg);
            if (!(fabsf(u) < 1e7f && fabsf(v) < 1e7f)) ok = false;
            umin = fminf(umin, u); umax = fmaxf(umax, u);
            vmin = fminf(vmin, v); vmax = fmaxf(vmax, v);
        }
        int iu0 = (int)floorf(umin - 0.5f) - 1, iu1 = (int)floorf(umax - 0.5f) + 2;
        int iv0 = (int)floorf(vmin - 0.5f) - 1, iv1 = (int)floorf(vmax - 0.5f) + 2;
        iu0 = max(iu0, 0); iv0 = max(iv0, 0);
        iu1 = min(iu1, Nd - 1); iv1 = min(iv1, Nd - 1);
        int W = iu1 - iu0 + 1, H = iv1 - iv0 + 1;
        if (!ok) { W = 1 << 20; H = 1; }
        {   /* row stride = 6 mod 8: four rows apart (the thread segments of a warp)
             * lie 24 banks apart, spreading the warp's atomics over the banks */
            const int Wp = W + (((6 - W) % 8) + 8) % 8;
            if (Wp * H <= kTileCap) W = Wp;
        }
        if (iu1 < iu0 || iv1 < iv0) { W = 0; H = 0; }
        bbox[i] = make_int4(iu0, iv0, W, H);
    }

    const int lane = tid & 31, w = tid >> 5;
    const int seg = lane & 3;
    /* A warp's 8 columns are spread over the brick, 4 apart in a and in b:
     * columns that project onto the same detector pixel in one atomic
     * instruction serialise, and two columns d apart coincide in u only in
     * views within about 1/(d B) radians of their alignment with the ray. */
    const int ia = a0 + (w & 3) + 4 * ((lane >> 2) & 3);
    const int ib = b0 + (w >> 2) + 4 * (lane >> 4);
    const int igb = g0 + seg * 4;
    const bool col_ok = ia < N && ib < N;
    const float ba = vox_base(ia, N, g.vs), bb = vox_base(ib, N, g.vs);
    /* o_g = (p_g - off_g) - t_g of each voxel (rayCasting's g component of
     * the source-to-voxel vector): off_g and t_g are the same for every view
     * of a column-aligned axis (checked on the host), so this is per voxel */
    float2 dgp[2];
    /* the thread's voxels q < nqv lie in the volume (a count, not a mask:
     * four predicates held over the view loop cost the XTT form spills) */
    const int nqv = col_ok ? max(0, min(4, g1 - igb + 1)) : 0;
    {
        const float offg = fr[0].off[G], tg = fr[0].t[G];
        float dgq[4];
#pragma unroll
        for (int q = 0; q < 4; q++) dgq[q] = __fsub_rn(__fsub_rn(vox_base(igb + q, N, g.vs), offg), tg);
        dgp[0] = make_float2(dgq[0], dgq[1]);
        dgp[1] = make_float2(dgq[2], dgq[3]);
    }

    /* per-voxel value: plain mu; XTT a0 and M of this axis; kept as pairs
     * of voxels (q = 2p, 2p + 1) for the packed FP32x2 arithmetic below */
    float2 valp[2], mp[2][6];
    const size_t NN = (size_t)N * N, N3 = NN * N;
    {
        float val[4], m[4][6];
        /* the thread's voxels are consecutive along g: index idx0 + q * stride_g */
        const size_t sgs = (G == 0) ? 1 : (G == 1 ? (size_t)N : NN);
        size_t idx0;
        {
            int x, y, z;
            xyz_of<G>(ia, ib, igb, x, y, z);
            idx0 = (size_t)x + (size_t)N * y + NN * z;
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            val[q] = 0.f;
#pragma unroll
            for (int e = 0; e < 6; e++) m[q][e] = 0.f;
            if (q >= nqv) continue;
            const size_t iq = idx0 + (size_t)q * sgs;
            if (MODE == 0) {
                val[q] = ldgf<T>(vol + iq);
            } else if (MODE == 2) {
                val[q] = 1.0f;
            } else if (MODE == 3) {   /* XTT with the voxel's rotated basis (forwardOrth, ir.cu:294-364) */
                orth_moments<T>(a.basis, cond, g.K, a.coef_kind ? 1.0f : __fmul_rn(g.vs, g.ratio), vol, a.coef,
                                a.coef_kind, iq, N3, val[q], m[q]);
            }
        }
        if (MODE == 1) {
            /* a0 = sum_k g_kc |S_k|^2 mu_k and M = sum_k g_kc mu_k S_k S_k^T (scaled by
             * vs * ratio), channel by channel for the thread's 4 voxels at once */
            const BasisConst *Bc = a.basis;
            const float sc = __fmul_rn(g.vs, g.ratio);
            for (int k = 0; k < g.K; k++) {
                const float gk = Bc->g[cond * g.K + k] * sc;
                if (gk == 0.f) continue;
                const float s0 = Bc->S[3 * k], s1 = Bc->S[3 * k + 1], s2 = Bc->S[3 * k + 2], s2k = Bc->S2[k];
                const float e0 = s0 * s0, e1 = s1 * s1, e2 = s2 * s2;
                const float e3 = 2.f * s0 * s1, e4 = 2.f * s0 * s2, e5 = 2.f * s1 * s2;
                float mu[4];
#pragma unroll
                const T *vk = vol + (size_t)k * N3 + idx0;
#pragma unroll
                for (int q = 0; q < 4; q++) mu[q] = q < nqv ? ldgf<T>(vk + (size_t)q * sgs) * gk : 0.f;
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    val[q] = fmaf(s2k, mu[q], val[q]);
                    m[q][0] = fmaf(mu[q], e0, m[q][0]);
                    m[q][1] = fmaf(mu[q], e1, m[q][1]);
                    m[q][2] = fmaf(mu[q], e2, m[q][2]);
                    m[q][3] = fmaf(mu[q], e3, m[q][3]);
                    m[q][4] = fmaf(mu[q], e4, m[q][4]);
                    m[q][5] = fmaf(mu[q], e5, m[q][5]);
                }
            }
        }
        /* bound on |contribution| over the CTA's voxels (weights c <= 1) */
        float bound = 0.f;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            if (q >= nqv) continue;
            float bq = (MODE == 0) ? fabsf(val[q]) * g.ratio : (MODE == 2 ? 1.0f : fabsf(val[q]));
            if (MODE == 1 || MODE == 3)
#pragma unroll
                for (int e = 0; e < 6; e++) bq += fabsf(m[q][e]);
            bound = fmaxf(bound, bq * 1.001f);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) bound = fmaxf(bound, __shfl_xor_sync(0xffffffffu, bound, o));
        if ((tid & 31) == 0) s_red[tid >> 5] = bound;
        /* M in the column frame: (aa, bb, ab, ag, bg, gg), so that per view
         * d^T M d = aa da^2 + bb db^2 + ab da db + dg (ag da + bg db + gg dg) with
         * (da, db) fixed per column and view and dg fixed per voxel */
        constexpr int AB = 3 + A + B - 1, AG = 3 + A + G - 1, BG = 3 + B + G - 1;
        constexpr int perm[6] = {A, B, AB, AG, BG, G};
#pragma unroll
        for (int p = 0; p < 2; p++) {
            valp[p] = make_float2(val[2 * p], val[2 * p + 1]);
#pragma unroll
            for (int e = 0; e < 6; e++) mp[p][e] = make_float2(m[2 * p][perm[e]], m[2 * p + 1][perm[e]]);
            /* d_g does not depend on the view: fold it into (ag, bg, gg) once, so
             * per view d^T M d = aa da^2 + bb db^2 + ab da db + ag' da + bg' db + gg' */
            mp[p][3] = __fmul2_rn(mp[p][3], dgp[p]);
            mp[p][4] = __fmul2_rn(mp[p][4], dgp[p]);
            mp[p][5] = __fmul2_rn(mp[p][5], __fmul2_rn(dgp[p], dgp[p]));
        }
    }
    __syncthreads();
    float S = 0.f;
#pragma unroll
    for (int i = 0; i < kFwdThreads / 32; i++) S = fmaxf(S, s_red[i]);
    if (!(S > 0.f) || !(S < 3e38f)) return;      /* nothing to splat (or non-finite input) */
    const int sh = fix_shift(S);
    const float fscale = ldexpf(1.0f, sh);
    const float finv = ldexpf(1.0f, -sh);
    const size_t NdNd = (size_t)Nd * Nd;
    float *outc = a.out + (size_t)cond * g.V * NdNd;
    for (int jj = 0; jj < nv; jj++) {
        const ViewFrame &f = fr[jj];
        const int4 bb4 = bbox[jj];
        int *T = smem + (jj & 1) * 2 * kTileCap;   /* hi words, lo words after */
        float *P = outc + (size_t)f.view * NdNd;
        const bool use_tile = (bb4.z > 0) && (bb4.z * bb4.w <= kTileCap);
        float u, coeff, da, db;
        int iu;
        float fu, gu;
        if (bb4.z > 0 && col_ok) {
            col_ray<G>(f, g, ba, bb, u, coeff, da, db);
            if (tap1(g, u, iu, fu, gu)) {
                const int lu = iu - bb4.x;
                const bool col_tile = use_tile && lu >= 0 && lu + 1 < bb4.z;
                const int W = bb4.z;
                int *tcol = T + lu;
                float *pcol = P + iu;
                const float2 dab2 = bc2(fmaf(da, da, db * db));
                const float2 daa = bc2(da * da), dbb = bc2(db * db), dab = bc2(da * db);
                const float2 da2 = bc2(da), db2 = bc2(db);
                /* v of the 4 voxels in two packed pairs, each lane rounded as div_det */
                float2 vp[2];
#pragma unroll
                for (int p = 0; p < 2; p++) {
                    const float2 av = __fmul2_rn(__fmul2_rn(bc2(coeff), dgp[p]), bc2(magsig));
                    if (g.exact_rdet) {
                        const float2 qd = __fmul2_rn(av, bc2(g.rdet));
                        const float2 rd = __ffma2_rn(qd, bc2(-g.det), av);
                        vp[p] = __fadd2_rn(__ffma2_rn(rd, bc2(g.rdet), qd), bc2(g.half));
                    } else {
                        vp[p] = make_float2(__fadd_rn(__fdiv_rn(av.x, g.det), g.half),
                                            __fadd_rn(__fdiv_rn(av.y, g.det), g.half));
                    }
                }
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    if (q >= nqv) continue;
                    const float dgs = (q & 1) ? dgp[q >> 1].y : dgp[q >> 1].x;
                    const float v = (q & 1) ? vp[q >> 1].y : vp[q >> 1].x;
                    int iv;
                    float fv, gv;
                    if (!tap1(g, v, iv, fv, gv)) continue;
                    float pvs;
                    if (MODE == 0) {
                        pvs = (q & 1) ? valp[q >> 1].y : valp[q >> 1].x;
                    } else if (MODE == 2) {
                        pvs = fscale;
                    } else {
                        float m[6];
#pragma unroll
                        for (int e = 0; e < 6; e++) m[e] = (q & 1) ? mp[q >> 1][e].y : mp[q >> 1][e].x;
                        const float dd = fmaf(dgs, dgs, dab2.x);
                        const float q2 =
                            fmaf(m[3], da, fmaf(m[4], db, fmaf(m[0], daa.x, fmaf(m[1], dbb.x, fmaf(m[2], dab.x, m[5])))));
                        const float vq = (q & 1) ? valp[q >> 1].y : valp[q >> 1].x;
                        pvs = fmaf(q2, __fdividef(-1.0f, dd), vq) * fscale;
                    }
                    const float c1 = __fmul_rn(gu, fv), c2 = __fmul_rn(fu, fv);
                    const float c3 = __fmul_rn(fu, gv), c4 = __fmul_rn(gu, gv);
                    const int lv = iv - bb4.y;
                    if (col_tile && lv >= 0 && lv + 1 < bb4.w) {
                        /* the four taps as two packed pairs, row iv + 1 (times f_v) and
                         * row iv (times g_v), split in FP32x2.  XTT: (g_u, f_u) pvs times
                         * f_v / g_v; plain and weights: each lane rounded as the scalar
                         * tap ((c ratio) pvs) fscale / c pvs with c = g_u f_v etc. */
                        int *t0 = tcol + W * lv;
                        const float2 guf = make_float2(gu, fu);
                        const float2 up = (MODE == 1 || MODE == 3) ? __fmul2_rn(guf, bc2(pvs)) : guf;
                        auto xs2 = [&](float w) {
                            if (MODE == 1 || MODE == 3) return __fmul2_rn(up, bc2(w));
                            const float2 c = __fmul2_rn(guf, bc2(w));
                            if (MODE == 0)
                                return __fmul2_rn(__fmul2_rn(__fmul2_rn(c, bc2(g.ratio)), bc2(pvs)), bc2(fscale));
                            return __fmul2_rn(c, bc2(pvs));
                        };
                        int2 h, l;
                        fix_split2(xs2(fv), h, l);
                        atomicAdd(t0 + W, h.x);
                        atomicAdd(t0 + W + kTileCap, l.x);
                        atomicAdd(t0 + W + 1, h.y);
                        atomicAdd(t0 + W + 1 + kTileCap, l.y);
                        fix_split2(xs2(gv), h, l);
                        atomicAdd(t0, h.x);
                        atomicAdd(t0 + kTileCap, l.x);
                        atomicAdd(t0 + 1, h.y);
                        atomicAdd(t0 + 1 + kTileCap, l.y);
                    } else {
                        float *p0 = pcol + (size_t)Nd * iv;
                        auto tapg = [&](float c, float *adr) {
                            float xs;
                            if (MODE == 0) xs = __fmul_rn(__fmul_rn(c, g.ratio), pvs);
                            else xs = c * pvs * finv;
                            atomicAdd(adr, xs);
                        };
                        tapg(c1, p0 + Nd); tapg(c2, p0 + Nd + 1); tapg(c3, p0 + 1); tapg(c4, p0);
                    }
                }
            }
        }
        __syncthreads();
        if (use_tile) {   /* one warp per tile row: coalesced flush, tile cleared behind */
            for (int r = tid >> 5; r < bb4.w; r += kFwdThreads / 32) {
                for (int c = tid & 31; c < bb4.z; c += 32) {
                    float t;
                    if (fix_take(T + c + bb4.z * r, kTileCap, finv, t)) {
                        atomicAdd(P + (bb4.x + c) + (size_t)Nd * (bb4.y + r), t);
                    }
                }
            }
        }
    }
}

/* Axes of one column axis G (blockIdx.y indexes a.conds). */
template <int MODE, int G, typename T>
__global__ void __launch_bounds__(kFwdThreads, 2) k_fwd_col(FwdColArgs a) {
    fwd_col_brick<MODE, G, T>(a, a.conds[blockIdx.y]);
}

/* Every listed axis in one launch, whatever its column axis: the CTA's axis
 * picks the instance (uniform over the CTA). */
template <int MODE, typename T>
__global__ void __launch_bounds__(kFwdThreads, 2) k_fwd_col_axes(FwdColArgs a) {
    const int cond = a.conds[blockIdx.y];
    const int G = a.axis_g[cond];
    if (G == 0) fwd_col_brick<MODE, 0, T>(a, cond);
    else if (G == 1) fwd_col_brick<MODE, 1, T>(a, cond);
    else fwd_col_brick<MODE, 2, T>(a, cond);
}

/* ------------------------------------------------------------------------ */
/* Back-projection, column form, fused with the update.                      */
/* Brick 8 x 8 x 8 voxels, 128 threads.  For each axis the threads map to     */
/* 64 columns x 2 segments of 4 voxels along that axis's g.                  */
/*   PLAIN: one axis (IR), tmp/factor in registers, voxelProduct/voxelPlus.   */
/*   XTT:   every axis; per axis the moments sum(r), sum(r d d^T / d.d) of    */
/*          4 voxels fold into shared tmp_k; factor_k is the per-subset       */
/*          sensitivity precomputed by SENS.                                  */
/*   SENS:  moments sum(1), sum(d d^T / d.d) folded into factor_k, written    */
/*          to global (geometry only; once per subset).                       */
/* ------------------------------------------------------------------------ */
/* B_XTT_TEX / B_PLAIN_TEX: B_XTT / B_PLAIN with the 4 taps of each
 * voxel-view gathered in one texture instruction from the subset's ratio
 * images in a 2D-layered array. */
enum { B_PLAIN = 0, B_XTT = 1, B_SENS = 2, B_XTT_TEX = 3, B_PLAIN_TEX = 4 };
__host__ __device__ constexpr bool b_plain(int m) { return m == B_PLAIN || m == B_PLAIN_TEX; }
__host__ __device__ constexpr bool b_tex(int m) { return m == B_XTT_TEX || m == B_PLAIN_TEX; }

struct BackColArgs {
    GeomConst g;
    const ViewFrame *frames;
    const int *view_list;
    int n_views, n_cond;
    const int *conds;         /* n_cond axes (PLAIN: 1)                      */
    const int *axis_g;        /* per axis: column axis 0/1/2                 */
    const float *magsig;      /* per axis: sign * mag                        */
    const float *proj;        /* ratio images, C blocks                      */
    void *vol;                /* PLAIN: the axis's N^3; XTT: K*N^3 (type T)  */
    const float *fac_in;      /* XTT: K*N^3 sensitivity of this subset       */
    float *fac_out;           /* SENS: K*N^3                                 */
    const BasisConst *basis;
    int art;
    float alpha;
    int sr;                   /* 16-bit volumes: stochastic rounding of updates */
    const float *coef;        /* non-null: per-voxel rotated basis (backwardOrth) */
    int coef_kind;            /* 0: (phi, cos theta); 1: main direction            */
    cudaTextureObject_t rtex; /* *_TEX: the ratio images, layer = (index in conds) * n_views + position */
    int brick0;               /* first brick of the launch (z-slab launches)  */
};

/* Shared-memory slot of brick voxel lv (x + 8y + 64z) in the per-voxel
 * accumulators: lv with bits 5-7 folded into bits 0-2 and bits 6-7 into bits
 * 3-4, so that for every column axis the 32 lanes of a warp (8 x 4 columns)
 * and the brick-linear final pass all hit 32 different banks. */
__device__ __forceinline__ int sacc_slot(int lv) { return lv ^ ((lv >> 5) & 7) ^ (((lv >> 6) & 3) << 3); }

/* One view of one axis for a thread's column segment of 4 voxels (two pairs
 * in packed FP32x2 arithmetic, each lane rounded as the scalar form): the
 * ray set-up once, then per voxel v, the taps and the 4-tap gather from the
 * (L2-resident) ratio image, accumulated into the moments of the pair.
 * dg: o_g of the voxels (per axis, view-independent); okq: voxel in range. */
template <int MODE, int G>
__device__ __forceinline__ void back_view(const GeomConst &g, const ViewFrame &f, float magsig, float ba, float bb,
                                          const float2 dg[2], const bool okq[4], const float *Pv, float2 acc[2][7],
                                          cudaTextureObject_t rtex, int layer) {
    constexpr int A = Ax<G>::A, B = Ax<G>::B;
    const int Nd = g.Nd;
    float u, coeff, da, db;
    col_ray<G>(f, g, ba, bb, u, coeff, da, db);
    int iu;
    float fu, gu;
    if (!tap1(g, u, iu, fu, gu)) return;
    const float2 dab2 = bc2(fmaf(da, da, db * db));
    const float *Pc = Pv + iu;
    /* the products of d = (d_A, d_B, d_G) that do not involve d_G */
    const float2 daa = bc2(da * da), dbb = bc2(db * db), dab = bc2(da * db), da2 = bc2(da), db2 = bc2(db);
    const float xu = __int2float_rn(iu + 1);   /* gathers texels iu, iu + 1 */
    /* Two phases: first both pairs' taps and their 16 gathers (a voxel off
     * the detector reads row 0 and is dropped), then the accumulation. */
    float2 fv[2], gv[2], p0[2], p1[2], p2[2], p3[2];
    bool ok[4];
#pragma unroll
    for (int p = 0; p < 2; p++) {
        const float2 av = __fmul2_rn(__fmul2_rn(bc2(coeff), dg[p]), bc2(magsig));
        float2 v;
        if (g.exact_rdet) {
            const float2 qd = __fmul2_rn(av, bc2(g.rdet));
            const float2 rd = __ffma2_rn(qd, bc2(-g.det), av);
            v = __fadd2_rn(__ffma2_rn(rd, bc2(g.rdet), qd), bc2(g.half));
        } else {
            v = __fadd2_rn(make_float2(__fdiv_rn(av.x, g.det), __fdiv_rn(av.y, g.det)), bc2(g.half));
        }
        ok[2 * p] = okq[2 * p] && 0.55f < v.x && v.x < g.lim;
        ok[2 * p + 1] = okq[2 * p + 1] && 0.55f < v.y && v.y < g.lim;
        const float2 ut = __fadd2_rn(v, bc2(-0.5f));
        const float2 fi = make_float2(floorf(ut.x), floorf(ut.y));
        fv[p] = __ffma2_rn(fi, bc2(-1.0f), ut);
        gv[p] = __ffma2_rn(fv[p], bc2(-1.0f), bc2(1.0f));
        if (b_tex(MODE)) {
            const float4 t0 = gather_a2d(rtex, layer, xu, fi.x + 1.0f);
            const float4 t1 = gather_a2d(rtex, layer, xu, fi.y + 1.0f);
            p0[p] = make_float2(t0.w, t1.w);
            p1[p] = make_float2(t0.z, t1.z);
            p2[p] = make_float2(t0.x, t1.x);
            p3[p] = make_float2(t0.y, t1.y);
        } else if (MODE != B_SENS) {
            const float *q0 = Pc + Nd * (ok[2 * p] ? (int)fi.x : 0);
            const float *q1 = Pc + Nd * (ok[2 * p + 1] ? (int)fi.y : 0);
            p0[p] = make_float2(__ldg(q0), __ldg(q1));
            p1[p] = make_float2(__ldg(q0 + 1), __ldg(q1 + 1));
            p2[p] = make_float2(__ldg(q0 + Nd), __ldg(q1 + Nd));
            p3[p] = make_float2(__ldg(q0 + Nd + 1), __ldg(q1 + Nd + 1));
        }
    }
#pragma unroll
    for (int p = 0; p < 2; p++) {
        if (!(ok[2 * p] || ok[2 * p + 1])) continue;
        /* a voxel off the detector contributes nothing: its lane is zeroed */
        const float2 m = make_float2(ok[2 * p] ? 1.0f : 0.0f, ok[2 * p + 1] ? 1.0f : 0.0f);
        float2 nb = bc2(0.0f);
        if (MODE != B_SENS) {
            /* numBack in the reference's order (ir.cu:1744-1750) */
            const float2 c1 = __fmul2_rn(bc2(gu), fv[p]), c2 = __fmul2_rn(bc2(fu), fv[p]);
            const float2 c3 = __fmul2_rn(bc2(fu), gv[p]), c4 = __fmul2_rn(bc2(gu), gv[p]);
            nb = __fadd2_rn(__fadd2_rn(__fadd2_rn(__fmul2_rn(c1, p2[p]), __fmul2_rn(c2, p3[p])),
                                       __fmul2_rn(c3, p1[p])),
                            __fmul2_rn(c4, p0[p]));
            nb = __fmul2_rn(nb, m);
        }
        if (b_plain(MODE)) {
            acc[p][0] = __fadd2_rn(acc[p][0], nb);   /* tmp    (ir.cu:1750) */
            acc[p][1] = __fadd2_rn(acc[p][1], m);    /* factor (ir.cu:1749) */
        } else {
            const float2 dd = __ffma2_rn(dg[p], dg[p], dab2);
            const float2 inv = make_float2(__fdividef(1.0f, dd.x), __fdividef(1.0f, dd.y));  /* ~2 ulp */
            float2 wgt;
            if (MODE == B_XTT || MODE == B_XTT_TEX) {
                acc[p][6] = __fadd2_rn(acc[p][6], nb);
                wgt = __fmul2_rn(nb, inv);
            } else {
                acc[p][6] = __fadd2_rn(acc[p][6], m);
                wgt = __fmul2_rn(inv, m);
            }
            /* sum wgt d d^T in the column frame: d_G = dg does not depend on
             * the view, so its products need only sum wgt, sum wgt da and
             * sum wgt db (turned into xyz moments after the view loop) */
            acc[p][0] = __ffma2_rn(wgt, daa, acc[p][0]);
            acc[p][1] = __ffma2_rn(wgt, dbb, acc[p][1]);
            acc[p][2] = __ffma2_rn(wgt, dab, acc[p][2]);
            acc[p][3] = __ffma2_rn(wgt, da2, acc[p][3]);
            acc[p][4] = __ffma2_rn(wgt, db2, acc[p][4]);
            acc[p][5] = __fadd2_rn(acc[p][5], wgt);
        }
    }
}

/* One axis of the back kernel: threads map to 64 columns x 2 segments along
 * this axis's column axis G; moments accumulate over all listed views; then
 * PLAIN updates the voxels in place, XTT/SENS fold into the shared per-voxel
 * channel accumulators. */
template <int MODE, int G, typename T>
__device__ __forceinline__ void axis_pass(const BackColArgs &a, ViewFrame *fr, float *sacc, int ci, int cond,
                                          int bx0, int by0, int bz0) {
    constexpr int A = Ax<G>::A, B = Ax<G>::B;
    const GeomConst &g = a.g;
    const int N = g.N, K = g.K, Nd = g.Nd;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int ca = lane & 7, cb = ((lane >> 3) & 3) + (w & 1) * 4, sg = w >> 1;
    const int o[3] = {bx0, by0, bz0};
    const int ia = o[A] + ca, ib = o[B] + cb, igb = o[G] + sg * 4;
    const bool col_ok = ia < N && ib < N;
    const int nq = col_ok ? max(0, min(4, N - igb)) : 0;
    const float magsig = a.magsig[cond];
    const float *P = a.proj + (size_t)cond * g.V * (size_t)Nd * Nd;
    const size_t NN = (size_t)N * N, NdNd = (size_t)Nd * Nd;
    const float ba = vox_base(ia, N, g.vs), bb = vox_base(ib, N, g.vs);
    /* o_g of the 4 voxels: off_g and t_g are the same for every view of a
     * column-aligned axis (checked on the host) */
    float2 dg[2];
    bool okq[4];
    {
        const ViewFrame &f0 = a.frames[(size_t)cond * g.V];
        const float offg = f0.off[G], tg = f0.t[G];
        float d[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            d[q] = __fsub_rn(__fsub_rn(vox_base(igb + q, N, g.vs), offg), tg);
            okq[q] = q < nq;
        }
        dg[0] = make_float2(d[0], d[1]);
        dg[1] = make_float2(d[2], d[3]);
    }
    float2 acc[2][7];
#pragma unroll
    for (int p = 0; p < 2; p++)
#pragma unroll
        for (int e = 0; e < 7; e++) acc[p][e] = bc2(0.f);
    for (int c0 = 0; c0 < a.n_views; c0 += kFrameChunk) {
        const int nc = min(kFrameChunk, a.n_views - c0);
        __syncthreads();
        for (int i = tid; i < nc * 5; i += kBackThreads) {
            const int jj = i / 5, q = i % 5;
            reinterpret_cast<float4 *>(&fr[jj])[q] =
                reinterpret_cast<const float4 *>(&a.frames[(size_t)cond * g.V + a.view_list[c0 + jj]])[q];
        }
        __syncthreads();
        if (nq > 0)
            for (int jj = 0; jj < nc; jj++)
                back_view<MODE, G>(g, fr[jj], magsig, ba, bb, dg, okq, P + (size_t)fr[jj].view * NdNd, acc, a.rtex,
                                   ci * a.n_views + c0 + jj);
    }
    if (!col_ok) return;
    if (!b_plain(MODE)) {
        /* column-frame sums (wgt da^2, wgt db^2, wgt da db, wgt da, wgt db, wgt)
         * -> xyz moments (xx, yy, zz, xy, xz, yz) with d_A = da, d_B = db, d_G = dg */
        constexpr int AB = 3 + A + B - 1, AG = 3 + A + G - 1, BG = 3 + B + G - 1;
#pragma unroll
        for (int p = 0; p < 2; p++) {
            const float2 c[6] = {acc[p][0], acc[p][1], acc[p][2], acc[p][3], acc[p][4], acc[p][5]};
            acc[p][A] = c[0];
            acc[p][B] = c[1];
            acc[p][G] = __fmul2_rn(__fmul2_rn(dg[p], dg[p]), c[5]);
            acc[p][AB] = c[2];
            acc[p][AG] = __fmul2_rn(dg[p], c[3]);
            acc[p][BG] = __fmul2_rn(dg[p], c[4]);
        }
    }
    if (!b_plain(MODE) && !a.coef) {
        /* fold the basis-independent moments into the channels:
         * tmp_k += g_kc (|S_k|^2 sum r - S_k^T (sum r d d^T / d.d) S_k), channel by
         * channel for the thread's 4 voxels at once */
        const BasisConst *Bc = a.basis;
        int lvq[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            int lx, ly, lz;
            xyz_of<G>(ca, cb, sg * 4 + q, lx, ly, lz);
            lvq[q] = sacc_slot(lx + 8 * ly + 64 * lz);
        }
        for (int k = 0; k < K; k++) {
            const float gk = Bc->g[cond * K + k];
            if (gk == 0.f) continue;
            const float s0 = Bc->S[3 * k], s1 = Bc->S[3 * k + 1], s2 = Bc->S[3 * k + 2], s2k = Bc->S2[k];
            const float e0 = s0 * s0, e1 = s1 * s1, e2 = s2 * s2;
            const float e3 = 2.f * s0 * s1, e4 = 2.f * s0 * s2, e5 = 2.f * s1 * s2;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                if (q >= nq) continue;
                const float2 *ap = acc[q >> 1];
#define XR_AQ(e) ((q & 1) ? ap[e].y : ap[e].x)
                const float sAs = e0 * XR_AQ(0) + e1 * XR_AQ(1) + e2 * XR_AQ(2) + e3 * XR_AQ(3) + e4 * XR_AQ(4) +
                                  e5 * XR_AQ(5);
                sacc[k * 512 + lvq[q]] += gk * fmaf(s2k, XR_AQ(6), -sAs);
#undef XR_AQ
            }
        }
        return;
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
        if (q >= nq) continue;
        float aq[7];
#pragma unroll
        for (int e = 0; e < 7; e++) aq[e] = (q & 1) ? acc[q >> 1][e].y : acc[q >> 1][e].x;
        if (b_plain(MODE)) {
            /* voxelProduct (ir.cu:1637-1654) / voxelPlus (ir.cu:1682-1693) */
            int x, y, z;
            xyz_of<G>(ia, ib, igb + q, x, y, z);
            T *vp = reinterpret_cast<T *>(a.vol) + (size_t)x + (size_t)N * y + NN * z;
            const float tmp = aq[0], fac = aq[1], mu = ldf<T>(vp);
            const uint32_t key = (uint32_t)((size_t)x + (size_t)N * y + NN * z);
            if (a.art) stu<T>(vp, __fadd_rn(mu, __fmul_rn(a.alpha, tmp)), key, a.sr);
            else stu<T>(vp, (fac == 0.0f) ? 0.0f : __fdiv_rn(__fmul_rn(mu, tmp), fac), key, a.sr);
        } else {   /* backwardOrth(ByMD) (ir.cu:366-423, :233-292): the voxel's rotated basis */
            int lx, ly, lz;
            xyz_of<G>(ca, cb, sg * 4 + q, lx, ly, lz);
            const int lv = sacc_slot(lx + 8 * ly + 64 * lz);
            const BasisConst *Bc = a.basis;
            int x, y, z;
            xyz_of<G>(ia, ib, igb + q, x, y, z);
            float R[9];
            src_rotation(a.coef, a.coef_kind, NN * N, (size_t)x + (size_t)N * y + NN * z, R);
            const float G0 = Bc->G[3 * cond], G1 = Bc->G[3 * cond + 1], G2 = Bc->G[3 * cond + 2];
            for (int k = 0; k < K; k++) {
                float S[3];
                orth_basis(Bc, k, R, S);
                const float h = S[0] * G0 + S[1] * G1 + S[2] * G2;
                const float sAs = S[0] * S[0] * aq[0] + S[1] * S[1] * aq[1] + S[2] * S[2] * aq[2] +
                                  2.f * (S[0] * S[1] * aq[3] + S[0] * S[2] * aq[4] + S[1] * S[2] * aq[5]);
                sacc[k * 512 + lv] += (h * h) * fmaf(S[0] * S[0] + S[1] * S[1] + S[2] * S[2], aq[6], -sAs);
            }
        }
    }
}

template <int MODE, typename T>
__global__ void __launch_bounds__(kBackThreads, 6) k_back_col(BackColArgs a) {
    __shared__ ViewFrame fr[kFrameChunk];
    extern __shared__ float sacc[];   /* XTT / SENS: K x 512 per-voxel accumulators */
    const GeomConst &g = a.g;
    const int N = g.N;
    const int nb8 = (N + 7) / 8;
    const int b = blockIdx.x + a.brick0;
    const int bx0 = (b % nb8) * 8, by0 = ((b / nb8) % nb8) * 8, bz0 = (b / (nb8 * nb8)) * 8;
    const int tid = threadIdx.x;
    const int K = g.K;
    const size_t NN = (size_t)N * N, N3 = NN * N;
    if (!b_plain(MODE)) {
        for (int i = tid; i < K * 512; i += kBackThreads) sacc[i] = 0.0f;
    }
    for (int ci = 0; ci < a.n_cond; ci++) {
        const int cond = a.conds[ci];
        const int G = a.axis_g[cond];   /* uniform over the CTA */
        if (G == 0) axis_pass<MODE, 0, T>(a, fr, sacc, ci, cond, bx0, by0, bz0);
        else if (G == 1) axis_pass<MODE, 1, T>(a, fr, sacc, ci, cond, bx0, by0, bz0);
        else axis_pass<MODE, 2, T>(a, fr, sacc, ci, cond, bx0, by0, bz0);
        __syncthreads();
    }
    if (b_plain(MODE)) return;
    if (MODE != B_SENS && (N & 1) == 0) {
        /* even N: voxel pairs along x (x even, so both in range and the pair
         * aligned), one 2-element access per channel; the same arithmetic,
         * keys and results as the loop below */
        for (int lp = tid; lp < 256; lp += kBackThreads) {
            const int lv = 2 * lp;
            const int x = bx0 + (lv & 7), y = by0 + ((lv >> 3) & 7), z = bz0 + (lv >> 6);
            if (x >= N || y >= N || z >= N) continue;
            const size_t idx = (size_t)x + (size_t)N * y + NN * z;
            const int s0 = sacc_slot(lv), s1 = sacc_slot(lv + 1);
            for (int k0 = 0; k0 < K; k0 += 8) {
                float2 mu[8], f[8];
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    const int k = k0 + j;
                    if (k < K) {
                        mu[j] = ld2<T>(reinterpret_cast<T *>(a.vol) + idx + (size_t)k * N3);
                        f[j] = a.art ? make_float2(0.f, 0.f)
                                     : __ldg(reinterpret_cast<const float2 *>(a.fac_in + idx + (size_t)k * N3));
                    }
                }
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    const int k = k0 + j;
                    if (k >= K) break;
                    const float t0 = sacc[k * 512 + s0], t1 = sacc[k * 512 + s1];
                    T *vp = reinterpret_cast<T *>(a.vol) + idx + (size_t)k * N3;
                    const uint32_t key = (uint32_t)(idx + (size_t)k * N3);
                    float v0, v1;
                    if (a.art) {
                        v0 = __fadd_rn(mu[j].x, __fmul_rn(a.alpha, t0));
                        v1 = __fadd_rn(mu[j].y, __fmul_rn(a.alpha, t1));
                    } else {
                        v0 = (f[j].x == 0.0f) ? 0.0f : __fdiv_rn(__fmul_rn(mu[j].x, t0), f[j].x);
                        v1 = (f[j].y == 0.0f) ? 0.0f : __fdiv_rn(__fmul_rn(mu[j].y, t1), f[j].y);
                    }
                    stu2<T>(vp, v0, v1, key, key + 1u, a.sr);
                }
            }
        }
        return;
    }
    /* home layout: brick-linear voxel order */
    for (int lv = tid; lv < 512; lv += kBackThreads) {
        const int x = bx0 + (lv & 7), y = by0 + ((lv >> 3) & 7), z = bz0 + (lv >> 6);
        if (x >= N || y >= N || z >= N) continue;
        const size_t idx = (size_t)x + (size_t)N * y + NN * z;
        if (MODE == B_SENS) {
            for (int k = 0; k < K; k++) a.fac_out[idx + (size_t)k * N3] = sacc[k * 512 + sacc_slot(lv)];
            continue;
        }
        /* eight channels at a time: their loads are all in flight before the
         * first store (a load-update-store chain per channel would wait for
         * each load in turn) */
        for (int k0 = 0; k0 < K; k0 += 8) {
            float mu[8], f[8];
#pragma unroll
            for (int j = 0; j < 8; j++) {
                const int k = k0 + j;
                if (k < K) {
                    mu[j] = ldf<T>(reinterpret_cast<T *>(a.vol) + idx + (size_t)k * N3);
                    f[j] = a.art ? 0.f : __ldg(a.fac_in + idx + (size_t)k * N3);
                }
            }
#pragma unroll
            for (int j = 0; j < 8; j++) {
                const int k = k0 + j;
                if (k >= K) break;
                const float t = sacc[k * 512 + sacc_slot(lv)];
                T *vp = reinterpret_cast<T *>(a.vol) + idx + (size_t)k * N3;
                const uint32_t key = (uint32_t)(idx + (size_t)k * N3);
                if (a.art) stu<T>(vp, __fadd_rn(mu[j], __fmul_rn(a.alpha, t)), key, a.sr);
                else stu<T>(vp, (f[j] == 0.0f) ? 0.0f : __fdiv_rn(__fmul_rn(mu[j], t), f[j]), key, a.sr);
            }
        }
    }
}

/* Bit-for-bit check of div_det against IEEE division over every float
 * a in [2^-24, 2^24) * det (both signs give the same result by symmetry). */
__global__ void k_check_div(float det, float rdet, unsigned lo_bits, unsigned count, unsigned *mismatch) {
    unsigned bad = 0;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const float a = __uint_as_float(lo_bits + i);
        const float q = __fmul_rn(a, rdet);
        const float r = __fmaf_rn(-q, det, a);
        const float m = __fmaf_rn(r, rdet, q);
        if (__float_as_uint(m) != __float_as_uint(__fdiv_rn(a, det))) bad++;
    }
    if (bad) atomicAdd(mismatch, bad);
}

}  // namespace

cudaError_t check_exact_rdet(float det, float rdet, unsigned *d_flag, unsigned *h_result, cudaStream_t s) {
    const float lo = det * 5.9604645e-08f, hi = det * 16777216.0f;   /* det * 2^-24, det * 2^24 */
    const unsigned lo_bits = __builtin_bit_cast(unsigned, lo), hi_bits = __builtin_bit_cast(unsigned, hi);
    cudaMemsetAsync(d_flag, 0, sizeof(unsigned), s);
    k_check_div<<<148 * 8, 256, 0, s>>>(det, rdet, lo_bits, hi_bits - lo_bits, d_flag);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(h_result, d_flag, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(s);
}

cudaError_t launch_forward_col(const GeomConst &g, const BasisConst *d_basis, const ViewFrame *frames,
                               const int *view_list, int n_views, const int *d_conds, int n_cond, int G,
                               const float *d_magsig, const void *vol, float *out, int mode, int views_per_cta,
                               int storage, cudaStream_t s, const float *coef, int coef_kind, int zlo, int zhi,
                               const int *d_axis_g) {
    if (n_views <= 0 || n_cond <= 0) return cudaSuccess;
    if (coef && mode == 1) mode = 3;
    FwdColArgs a;
    a.zlo = zlo;
    a.zhi = zhi;
    a.coef_kind = coef_kind;
    a.axis_g = d_axis_g;
    if (G < 0 && (!d_axis_g || mode == 0)) return cudaErrorInvalidValue;
    a.g = g;
    a.frames = frames;
    a.view_list = view_list;
    a.n_views = n_views;
    a.conds = d_conds;
    a.magsig = d_magsig;
    a.vol = vol;
    a.out = out;
    a.basis = d_basis;
    a.coef = coef;
    a.nbg = (g.N + 15) / 16;
    a.nba = (g.N + 15) / 16;
    const int nbb = (g.N + 7) / 8;
    const long bricks = (long)a.nbg * a.nba * nbb;
    int vpc = views_per_cta;
    if (vpc <= 0) {
        const long ctas = bricks * n_cond;
        const long chunks = ctas >= 2048 ? 1 : (2048 + ctas - 1) / ctas;
        vpc = (int)((n_views + chunks - 1) / chunks);
    }
    vpc = vpc < 1 ? 1 : (vpc > 64 ? 64 : vpc);
    vpc = vpc > n_views ? n_views : vpc;
    a.vpc = vpc;
    const dim3 grid((unsigned)bricks, (unsigned)n_cond, (unsigned)((n_views + vpc - 1) / vpc));
    const size_t smem = 4 * kTileCap * sizeof(int) + vpc * (sizeof(int4) + sizeof(ViewFrame));
#define XR_FWD_COL(M, GG, TT)                                                                                     \
    do {                                                                                                          \
        cudaError_t e = cudaFuncSetAttribute(k_fwd_col<M, GG, TT>, cudaFuncAttributeMaxDynamicSharedMemorySize,   \
                                             (int)smem);                                                          \
        if (e != cudaSuccess) return e;                                                                           \
        k_fwd_col<M, GG, TT><<<grid, kFwdThreads, smem, s>>>(a);                                                  \
    } while (0)
#define XR_FWD_AXES(M, TT)                                                                                        \
    do {                                                                                                          \
        cudaError_t e = cudaFuncSetAttribute(k_fwd_col_axes<M, TT>, cudaFuncAttributeMaxDynamicSharedMemorySize,  \
                                             (int)smem);                                                          \
        if (e != cudaSuccess) return e;                                                                           \
        k_fwd_col_axes<M, TT><<<grid, kFwdThreads, smem, s>>>(a);                                                 \
    } while (0)
#define XR_FWD_COL_G(M, TT)                                                                                       \
    do {                                                                                                          \
        if (G < 0 && M != 0) XR_FWD_AXES(M == 0 ? 1 : M, TT);                                                     \
        else if (G == 0) XR_FWD_COL(M, 0, TT); else if (G == 1) XR_FWD_COL(M, 1, TT); else XR_FWD_COL(M, 2, TT); \
    } while (0)
    if (mode == 2) {
        XR_FWD_COL_G(2, float);
    } else if (storage == kBF16) {
        if (mode == 0) XR_FWD_COL_G(0, __nv_bfloat16);
        else if (mode == 3) XR_FWD_COL_G(3, __nv_bfloat16);
        else XR_FWD_COL_G(1, __nv_bfloat16);
    } else if (storage == kF16) {
        if (mode == 0) XR_FWD_COL_G(0, __half);
        else if (mode == 3) XR_FWD_COL_G(3, __half);
        else XR_FWD_COL_G(1, __half);
    } else {
        if (mode == 0) XR_FWD_COL_G(0, float);
        else if (mode == 3) XR_FWD_COL_G(3, float);
        else XR_FWD_COL_G(1, float);
    }
#undef XR_FWD_COL_G
#undef XR_FWD_AXES
#undef XR_FWD_COL
    return cudaGetLastError();
}

cudaError_t launch_back_col(const GeomConst &g, const BasisConst *d_basis, const ViewFrame *frames,
                            const int *view_list, int n_views, const int *d_conds, int n_cond, const int *d_axis_g,
                            const float *d_magsig, const float *proj, void *vol, const float *fac_in, float *fac_out,
                            int mode, int art, float alpha, int storage, cudaStream_t s, const float *coef,
                            int coef_kind, cudaTextureObject_t rtex, int zb0, int zb1) {
    BackColArgs a;
    a.rtex = rtex;
    if (rtex && mode == B_XTT) mode = B_XTT_TEX;
    if (rtex && mode == B_PLAIN) mode = B_PLAIN_TEX;
    a.coef = coef;
    a.coef_kind = coef_kind;
    a.sr = (storage & kStoreStochastic) != 0;
    storage &= ~kStoreStochastic;
    a.g = g;
    a.frames = frames;
    a.view_list = view_list;
    a.n_views = n_views;
    a.n_cond = n_cond;
    a.conds = d_conds;
    a.axis_g = d_axis_g;
    a.magsig = d_magsig;
    a.proj = proj;
    a.vol = vol;
    a.fac_in = fac_in;
    a.fac_out = fac_out;
    a.basis = d_basis;
    a.art = art;
    a.alpha = alpha;
    const int nb8 = (g.N + 7) / 8;
    if (zb1 < 0 || zb1 > nb8) zb1 = nb8;
    if (zb0 < 0) zb0 = 0;
    if (zb0 >= zb1) return cudaSuccess;
    a.brick0 = zb0 * nb8 * nb8;
    const unsigned blocks = (unsigned)((long)nb8 * nb8 * (zb1 - zb0));
    const size_t smem = b_plain(mode) ? 0 : (size_t)g.K * 512 * sizeof(float);
#define XR_BACK_COL(M, TT)                                                                                        \
    do {                                                                                                          \
        cudaError_t e = cudaFuncSetAttribute(k_back_col<M, TT>, cudaFuncAttributeMaxDynamicSharedMemorySize,       \
                                             (int)smem);                                                          \
        if (e != cudaSuccess) return e;                                                                           \
        k_back_col<M, TT><<<blocks, kBackThreads, smem, s>>>(a);                                                  \
    } while (0)
    if (mode == B_SENS) {
        XR_BACK_COL(B_SENS, float);
    } else if (storage == kBF16) {
        if (mode == B_PLAIN) XR_BACK_COL(B_PLAIN, __nv_bfloat16);
        else if (mode == B_PLAIN_TEX) XR_BACK_COL(B_PLAIN_TEX, __nv_bfloat16);
        else if (mode == B_XTT_TEX) XR_BACK_COL(B_XTT_TEX, __nv_bfloat16);
        else XR_BACK_COL(B_XTT, __nv_bfloat16);
    } else if (storage == kF16) {
        if (mode == B_PLAIN) XR_BACK_COL(B_PLAIN, __half);
        else if (mode == B_PLAIN_TEX) XR_BACK_COL(B_PLAIN_TEX, __half);
        else if (mode == B_XTT_TEX) XR_BACK_COL(B_XTT_TEX, __half);
        else XR_BACK_COL(B_XTT, __half);
    } else {
        if (mode == B_PLAIN) XR_BACK_COL(B_PLAIN, float);
        else if (mode == B_PLAIN_TEX) XR_BACK_COL(B_PLAIN_TEX, float);
        else if (mode == B_XTT_TEX) XR_BACK_COL(B_XTT_TEX, float);
        else XR_BACK_COL(B_XTT, float);
    }
#undef XR_BACK_COL
    return cudaGetLastError();
}

}  // namespace xr
