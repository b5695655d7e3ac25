/*
 * Projector kernels for B200 (sm_100a): forward splat, chord-length
 * normaliser, ratio/subtract with FP64 loss, back-projection fused with the
 * MLEM/ART update, residual and sqrt.
 *
 * Parity rule.  The reference computes each voxel's detector coordinate
 * (u, v) and bilinear weights with plain FP32 operations (rayCasting,
 * ir.cu:1852-1902).  Every such operation here is an explicitly rounded
 * intrinsic (__fmul_rn, __fadd_rn, __fdiv_rn ...) so the compiler cannot
 * contract it into an FMA: the taps and weights are bit-identical to the
 * reference's host-compiled arithmetic.  Only sums differ in order.
 *
 * Design (the reference launches one (x,z)-slab per view, each followed by a
 * device sync, and splats with 8 global float atomics per voxel-view):
 *   forward   a CTA owns a 16x8x8 voxel brick and a chunk of views; per view
 *             it splats into a shared-memory detector tile covering the brick's
 *             footprint (two tiles, one __syncthreads per view), then flushes
 *             the tile with one global atomic per touched pixel.  The weight
 *             image the reference re-splats every view (devProjFactor) is
 *             geometry only, so it is splatted once per session (mode 2) and
 *             turned into the normaliser L/(sum c + 1e-5) by k_chord.
 *   back      one thread per voxel loops over every (axis, view) of the
 *             subset, gathering the 4 taps from L1/L2-resident ratio images,
 *             and applies the MLEM/ART update in registers: the reference's
 *             per-slab tmp/factor buffers and their read-modify-writes vanish.
 *   XTT       the dark-field weight (|B x S_k| |S_k . G|)^2 is rewritten as
 *             g_kc (|S_k|^2 - (B . S_k)^2) with g_kc = (S_k . G_c)^2 fixed per
 *             axis (G_c = elemR_c e_z for every view).  The forward then needs
 *             a0 - B^T M B with a 3x3 M per voxel and axis, and the back only
 *             the 7 moments sum(r), sum(r B B^T) (and sum 1, sum B B^T for the
 *             normaliser) per axis: ~15 FLOP per voxel-view instead of ~20 per
 *             channel.
 */
#include <cuda_runtime.h>

#include "xr_internal.h"
#include "xr_storage.cuh"
#include "xr_tile.cuh"
#include "xr_orth.cuh"

namespace xr {
namespace {

constexpr int kFwdThreads = 256;
constexpr int kBX = 16, kBY = 8, kBZ = 8;     /* forward brick                 */
constexpr int kTileCap = 48 * 48;             /* pixels per shared tile        */
constexpr int kBackThreads = 256;             /* 8 x 4 x 8 brick per CTA       */
constexpr int kFrameChunk = 128;              /* frames staged in smem at once */

/* ((2i - N - 1) * 0.5) * vs, the reference's voxel centre (ir.cu:1882-1884). */
__device__ __forceinline__ float vox_base(int i, int N, float vs) {
    const float a = __fsub_rn(__fsub_rn(__fmul_rn(2.0f, (float)i), (float)N), 1.0f);
    return __fmul_rn(__fmul_rn(a, 0.5f), vs);
}

__device__ __forceinline__ float dot_rn(float a0, float a1, float a2, float b0, float b1, float b2) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a0, b0), __fmul_rn(a1, b1)), __fmul_rn(a2, b2));
}

/* a / det, correctly rounded: a Markstein-corrected product when the context
 * verified it on this device (xr_column.cu), else IEEE division. */
__device__ __forceinline__ float div_det(float a, const GeomConst &g) {
    if (!g.exact_rdet) return __fdiv_rn(a, g.det);
    const float q = __fmul_rn(a, g.rdet);
    const float r = __fmaf_rn(-q, g.det, a);
    return __fmaf_rn(r, g.rdet, q);
}

/* Per-voxel half of rayCasting (ir.cu:1881-1897): returns u, v and the
 * source-to-voxel vector d (unnormalised B). */
__device__ __forceinline__ void ray_uv(const ViewFrame &f, const GeomConst &g, float bx, float by, float bz,
                                       float &u, float &v, float &d0, float &d1, float &d2) {
    const float ox = __fsub_rn(__fsub_rn(bx, f.off[0]), f.t[0]);
    const float oy = __fsub_rn(__fsub_rn(by, f.off[1]), f.t[1]);
    const float oz = __fsub_rn(__fsub_rn(bz, f.off[2]), f.t[2]);
    d0 = __fsub_rn(ox, f.src[0]);
    d1 = __fsub_rn(oy, f.src[1]);
    d2 = __fsub_rn(oz, f.src[2]);
    const float coeff = __fdiv_rn(-f.ss, dot_rn(f.src[0], f.src[1], f.src[2], d0, d1, d2));
    const float p0 = __fadd_rn(f.src[0], __fmul_rn(coeff, d0));
    const float p1 = __fadd_rn(f.src[1], __fmul_rn(coeff, d1));
    const float p2 = __fadd_rn(f.src[2], __fmul_rn(coeff, d2));
    u = __fadd_rn(div_det(__fmul_rn(dot_rn(p0, p1, p2, f.eu[0], f.eu[1], f.eu[2]), g.mag), g), g.half);
    v = __fadd_rn(div_det(__fmul_rn(dot_rn(p0, p1, p2, f.ev[0], f.ev[1], f.ev[2]), g.mag), g), g.half);
}

/* Detector window and bilinear taps (ir.cu:1501-1509).  Weights in the
 * reference's tap order: c1 (iu, iv+1), c2 (iu+1, iv+1), c3 (iu+1, iv),
 * c4 (iu, iv). */
__device__ __forceinline__ bool taps(const GeomConst &g, float u, float v, int &iu, int &iv, float &c1, float &c2,
                                     float &c3, float &c4) {
    if (!(0.55f < u && u < g.lim && 0.55f < v && v < g.lim)) return false;
    const float ut = __fsub_rn(u, 0.5f), vt = __fsub_rn(v, 0.5f);
    const float fiu = floorf(ut), fiv = floorf(vt);
    iu = (int)fiu;
    iv = (int)fiv;
    const float fu = __fsub_rn(ut, fiu), fv = __fsub_rn(vt, fiv);
    const float gu = __fsub_rn(1.0f, fu), gv = __fsub_rn(1.0f, fv);
    c1 = __fmul_rn(gu, fv);
    c2 = __fmul_rn(fu, fv);
    c3 = __fmul_rn(fu, gv);
    c4 = __fmul_rn(gu, gv);
    return true;
}

/* ------------------------------------------------------------------------ */
/* Forward splat.                                                            */
/* ------------------------------------------------------------------------ */

struct FwdArgs {
    GeomConst g;
    const ViewFrame *frames;  /* [C][V]                      */
    const int *view_list;     /* n_views view indices        */
    int n_views, vpc, cond0;
    const void *vol;          /* mode 0: N^3; mode 1: K*N^3 (type T) */
    float *out;               /* C blocks of V*Nd*Nd         */
    const BasisConst *basis;  /* device                      */
    const float *coef;        /* mode 3: rotation planes     */
    int coef_kind;            /* 0: (phi, cos); 1: md        */
    int nbx, nby;             /* bricks along x, y           */
};

template <int MODE, typename T>
__global__ void __launch_bounds__(kFwdThreads, 3) k_forward(FwdArgs a) {
    const T *vol = reinterpret_cast<const T *>(a.vol);
    /* Detector tiles in two-word fixed point (xr_tile.cuh). */
    extern __shared__ int smem[];
    __shared__ float s_red[kFwdThreads / 32];
    int4 *bbox = reinterpret_cast<int4 *>(smem + 4 * kTileCap);  /* vpc entries */
    ViewFrame *fr = reinterpret_cast<ViewFrame *>(bbox + a.vpc);

    const GeomConst &g = a.g;
    const int N = g.N, Nd = g.Nd;
    const int cond = a.cond0 + blockIdx.y;
    const int j0 = blockIdx.z * a.vpc;
    const int nv = min(a.vpc, a.n_views - j0);
    if (nv <= 0) return;

    const int brick = blockIdx.x;
    const int bxi = brick % a.nbx, byi = (brick / a.nbx) % a.nby, bzi = brick / (a.nbx * a.nby);
    const int x0 = bxi * kBX, y0 = byi * kBY, z0 = bzi * kBZ;
    const int x1 = min(x0 + kBX, N) - 1, y1 = min(y0 + kBY, N) - 1, z1 = min(z0 + kBZ, N) - 1;

    const int tid = threadIdx.x;
    for (int i = tid; i < 4 * kTileCap; i += kFwdThreads) smem[i] = 0;
    for (int i = tid; i < nv * 5; i += kFwdThreads) {
        const int jj = i / 5, q = i % 5;
        const float4 *s4 = reinterpret_cast<const float4 *>(&a.frames[(size_t)cond * g.V + a.view_list[j0 + jj]]);
        reinterpret_cast<float4 *>(&fr[jj])[q] = s4[q];
    }
    __syncthreads();

    /* Footprint bounding box of the brick for each view: project the 8
     * corner voxel centres (the box's image is the hull of its corners),
     * widen by one pixel for rounding and clamp to the detector. */
    for (int i = tid; i < nv; i += kFwdThreads) {
        const ViewFrame &f = fr[i];
        float umin = 1e30f, umax = -1e30f, vmin = 1e30f, vmax = -1e30f;
        bool ok = true;
        for (int c = 0; c < 8; c++) {
            const float bx = vox_base((c & 1) ? x1 : x0, N, g.vs);
            const float by = vox_base((c & 2) ? y1 : y0, N, g.vs);
            const float bz = vox_base((c & 4) ? z1 : z0, N, g.vs);
            float u, v, d0, d1, d2;
            ray_uv(f, g, bx, by, bz, u, v, d0, d1, d2);
            if (!(fabsf(u) < 1e7f && fabsf(v) < 1e7f)) ok = false;
            umin = fminf(umin, u); umax = fmaxf(umax, u);
            vmin = fminf(vmin, v); vmax = fmaxf(vmax, v);
        }
        int iu0 = (int)floorf(umin - 0.5f) - 1, iu1 = (int)floorf(umax - 0.5f) + 2;
        int iv0 = (int)floorf(vmin - 0.5f) - 1, iv1 = (int)floorf(vmax - 0.5f) + 2;
        iu0 = max(iu0, 0); iv0 = max(iv0, 0);
        iu1 = min(iu1, Nd - 1); iv1 = min(iv1, Nd - 1);
        int W = iu1 - iu0 + 1, H = iv1 - iv0 + 1;
        if (!ok) { W = 1 << 20; H = 1; }              /* global path       */
        if (iu1 < iu0 || iv1 < iv0) { W = 0; H = 0; } /* off the detector  */
        bbox[i] = make_int4(iu0, iv0, W, H);
    }

    /* This thread's 4 voxels: a warp is a 4(x) x 4(z) x 2(y) block so its
     * projections spread over >= 4x2 pixels in any view. */
    const int lane = tid & 31, w = tid >> 5;
    const int x = x0 + (w & 3) * 4 + (lane & 3);
    const int z = z0 + ((w >> 2) & 1) * 4 + ((lane >> 2) & 3);
    const int yb = y0 + (lane >> 4);
    const bool xz_ok = (x < N) && (z < N);
    const float bx = vox_base(x, N, g.vs), bz = vox_base(z, N, g.vs);
    float by[4];
    bool okv[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        by[q] = vox_base(yb + 2 * q, N, g.vs);
        okv[q] = xz_ok && (yb + 2 * q < N) && (yb + 2 * q <= y1);
    }

    /* Per-voxel value (mode 0: ratio*mu; mode 2: 1) or XTT moments of this axis:
     * val = a0 - d^T M d / (d.d), with a0 = vs*ratio*sum_k g_k |S_k|^2 mu_k and
     * M = vs*ratio*sum_k g_k mu_k S_k S_k^T. */
    float val[4], m[4][6];
    const size_t NN = (size_t)N * N, N3 = NN * N;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        val[q] = 0.f;
#pragma unroll
        for (int e = 0; e < 6; e++) m[q][e] = 0.f;
        if (!okv[q]) continue;
        const size_t idx = (size_t)x + (size_t)N * (yb + 2 * q) + NN * z;
        if (MODE == 0) {
            val[q] = ldgf<T>(vol + idx);
        } else if (MODE == 2) {
            val[q] = 1.0f;
        } else if (MODE == 3) {   /* forwardOrth (ir.cu:294-364) */
            orth_moments<T>(a.basis, cond, g.K, a.coef_kind ? 1.0f : __fmul_rn(g.vs, g.ratio), vol, a.coef,
                            a.coef_kind, idx, N3, val[q], m[q]);
        } else {
            const BasisConst *B = a.basis;
            const float sc = __fmul_rn(g.vs, g.ratio);
            float a0 = 0.f, mm[6] = {0, 0, 0, 0, 0, 0};
            for (int k = 0; k < g.K; k++) {
                const float gk = B->g[cond * g.K + k] * sc;
                if (gk == 0.f) continue;
                const float mu = ldgf<T>(vol + idx + (size_t)k * N3) * gk;
                const float s0 = B->S[3 * k], s1 = B->S[3 * k + 1], s2 = B->S[3 * k + 2];
                a0 = fmaf(B->S2[k], mu, a0);
                mm[0] = fmaf(mu * s0, s0, mm[0]);
                mm[1] = fmaf(mu * s1, s1, mm[1]);
                mm[2] = fmaf(mu * s2, s2, mm[2]);
                mm[3] = fmaf(2.f * mu * s0, s1, mm[3]);
                mm[4] = fmaf(2.f * mu * s0, s2, mm[4]);
                mm[5] = fmaf(2.f * mu * s1, s2, mm[5]);
            }
            val[q] = a0;
#pragma unroll
            for (int e = 0; e < 6; e++) m[q][e] = mm[e];
        }
    }
    float bound = 0.f;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        if (!okv[q]) continue;
        float bq = (MODE == 0) ? fabsf(val[q]) * g.ratio : (MODE == 2 ? 1.0f : fabsf(val[q]));
        if (MODE == 1 || MODE == 3)
#pragma unroll
            for (int e = 0; e < 6; e++) bq += fabsf(m[q][e]);
        bound = fmaxf(bound, bq * 1.001f);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) bound = fmaxf(bound, __shfl_xor_sync(0xffffffffu, bound, o));
    if ((tid & 31) == 0) s_red[tid >> 5] = bound;
    __syncthreads();
    float S = 0.f;
#pragma unroll
    for (int i = 0; i < kFwdThreads / 32; i++) S = fmaxf(S, s_red[i]);
    if (!(S > 0.f) || !(S < 3e38f)) return;
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
                float u, v, d0, d1, d2;
                ray_uv(f, g, bx, by[q], bz, u, v, d0, d1, d2);
                int iu, iv;
                float c1, c2, c3, c4;
                if (!taps(g, u, v, iu, iv, c1, c2, c3, c4)) continue;
                float pv;
                if (MODE == 1 || MODE == 3) {
                    const float dd = fmaf(d0, d0, fmaf(d1, d1, d2 * d2));
                    const float q2 = m[q][0] * d0 * d0 + m[q][1] * d1 * d1 + m[q][2] * d2 * d2 +
                                     m[q][3] * d0 * d1 + m[q][4] * d0 * d2 + m[q][5] * d1 * d2;
                    pv = val[q] - __fdividef(q2, dd);
                } else if (MODE == 0) {
                    pv = val[q];
                } else {
                    pv = 1.0f;
                }
                float w1, w2, w3, w4;
                if (MODE == 0) { /* (c * ratio) * mu, ir.cu:1518-1525 */
                    w1 = __fmul_rn(__fmul_rn(c1, g.ratio), pv);
                    w2 = __fmul_rn(__fmul_rn(c2, g.ratio), pv);
                    w3 = __fmul_rn(__fmul_rn(c3, g.ratio), pv);
                    w4 = __fmul_rn(__fmul_rn(c4, g.ratio), pv);
                } else if (MODE == 2) {
                    w1 = c1; w2 = c2; w3 = c3; w4 = c4;
                } else {
                    w1 = __fmul_rn(c1, pv); w2 = __fmul_rn(c2, pv);
                    w3 = __fmul_rn(c3, pv); w4 = __fmul_rn(c4, pv);
                }
                const int lu = iu - bb.x, lv = iv - bb.y;
                if (use_tile && lu >= 0 && lu + 1 < bb.z && lv >= 0 && lv + 1 < bb.w) {
                    int *t0 = T + lu + bb.z * lv;
                    fix_add(t0 + bb.z, kTileCap, w1 * fscale);
                    fix_add(t0 + bb.z + 1, kTileCap, w2 * fscale);
                    fix_add(t0 + 1, kTileCap, w3 * fscale);
                    fix_add(t0, kTileCap, w4 * fscale);
                } else {
                    float *p0 = P + iu + (size_t)Nd * iv;
                    atomicAdd(p0 + Nd, w1);
                    atomicAdd(p0 + Nd + 1, w2);
                    atomicAdd(p0 + 1, w3);
                    atomicAdd(p0, w4);
                }
            }
        }
        __syncthreads();
        if (use_tile) {
            for (int r = tid >> 5; r < bb.w; r += kFwdThreads / 32) {
                for (int c = tid & 31; c < bb.z; c += 32) {
                    float t;
                    if (fix_take(T + c + bb.z * r, kTileCap, finv, t)) {
                        atomicAdd(P + (bb.x + c) + (size_t)Nd * (bb.y + r), t);
                    }
                }
            }
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Chord length through the shifted volume box (correlationProjByLength,    */
/* ir.cu:1533-1603), turned into the normaliser L / (sum c + 1e-5).          */
/* ------------------------------------------------------------------------ */
__global__ void k_chord(GeomConst g, const ViewFrame *frames, float *norm, int n_cond) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int v = blockIdx.y * blockDim.y + threadIdx.y;
    const int cv = blockIdx.z;  /* cond * V + view */
    if (u >= g.Nd || v >= g.Nd || cv >= n_cond * g.V) return;
    const ViewFrame f = frames[cv];
    const float Ndf = (float)g.Nd;
    /* origin2pix = Rotate * ((u - (Nd-1)/2) det, -(sdd - sod), (v - (Nd-1)/2) det) */
    const float hp = __fmul_rn(__fsub_rn(Ndf, 1.0f), 0.5f);
    const float px = __fmul_rn(__fsub_rn((float)u, hp), g.det);
    const float py = -__fsub_rn(g.sdd, g.sod);
    const float pz = __fmul_rn(__fsub_rn((float)v, hp), g.det);
    const float e0[3] = {f.eu[0], f.eu[1], f.eu[2]};
    const float e1[3] = {f.e1x, f.e1y, f.e1z};
    const float e2[3] = {f.ev[0], f.ev[1], f.ev[2]};
    float s2p[3], o2s[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        /* Matrix3X * Vector3X: ((0 + R_i0 px) + R_i1 py) + R_i2 pz */
        const float o2p = __fadd_rn(__fadd_rn(__fadd_rn(0.0f, __fmul_rn(e0[i], px)), __fmul_rn(e1[i], py)),
                                    __fmul_rn(e2[i], pz));
        o2s[i] = f.src[i];
        s2p[i] = __fsub_rn(o2s[i], o2p);
    }
    const float hb = __fdiv_rn((float)(g.N + 1), 2.0f);
    float plane[6];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        plane[2 * a] = __fsub_rn(__fsub_rn(__fmul_rn(-hb, g.vs), f.off[a]), f.t[a]);
        plane[2 * a + 1] = __fsub_rn(__fsub_rn(__fmul_rn(hb, g.vs), f.off[a]), f.t[a]);
    }
    int cnt = 0;
    float cd[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int p = 0; p < 3; p++) {
#pragma unroll
        for (int sg = 0; sg < 2; sg++) {
            const float tt = __fdiv_rn(__fsub_rn(plane[2 * p + sg], o2s[p]), s2p[p]);
            float pl[3];
#pragma unroll
            for (int i = 0; i < 3; i++) pl[i] = __fadd_rn(__fmul_rn(tt, s2p[i]), o2s[i]);
            const int p1 = (p + 1) % 3, p2 = (p + 2) % 3;
            if (plane[2 * p1] < pl[p1] && pl[p1] < plane[2 * p1 + 1] && plane[2 * p2] < pl[p2] &&
                pl[p2] < plane[2 * p2 + 1]) {
                if (cnt == 0) { cd[0] = pl[0]; cd[1] = pl[1]; cd[2] = pl[2]; }
                else if (cnt == 1) { cd[3] = pl[0]; cd[4] = pl[1]; cd[5] = pl[2]; }
                cnt++;
            }
        }
    }
    const float a0 = __fsub_rn(cd[0], cd[3]), a1 = __fsub_rn(cd[1], cd[4]), a2 = __fsub_rn(cd[2], cd[5]);
    const float L = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(a0, a0), __fmul_rn(a1, a1)), __fmul_rn(a2, a2)));
    const size_t idx = (size_t)cv * g.Nd * g.Nd + (size_t)v * g.Nd + u;
    norm[idx] = __fdiv_rn(L, __fadd_rn(norm[idx], 1e-5f));
}

/* ------------------------------------------------------------------------ */
/* Normalise + ratio / subtract with an FP64 loss (projRatio ir.cu:1616-1635, */
/* projSubtract ir.cu:1656-1666).                                            */
/* ------------------------------------------------------------------------ */
__device__ __forceinline__ double block_sum(double x) {
    __shared__ double red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[w] = x;
    __syncthreads();
    double s = 0.0;
    if (w == 0) {
        s = (lane < (int)(blockDim.x >> 5)) ? red[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    }
    return s;
}

/* surf (non-zero): each ratio value is also written to layer blockIdx.y
 * (axis * n_views + list position) of a 2D-layered array, which the XTT back
 * kernel gathers from; out-of-range writes are dropped (boundary mode zero). */
template <typename T>
__global__ void k_ratio(GeomConst g, const int *view_list, int n_views, float *proj, const float *norm,
                        const T *sino, int art, double *loss, cudaSurfaceObject_t surf) {
    const size_t NdNd = (size_t)g.Nd * g.Nd;
    const int cond = blockIdx.y / n_views, j = blockIdx.y % n_views;
    const size_t base = ((size_t)cond * g.V + view_list[j]) * NdNd;
    double acc = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < NdNd; i += (size_t)gridDim.x * blockDim.x) {
        const size_t idx = base + i;
        float p = norm ? __fmul_rn(proj[idx], norm[idx]) : proj[idx];
        const float b = ldgf<T>(sino + idx);
        acc += (double)fabsf(__fsub_rn(b, p));
        if (art) {
            p = __fsub_rn(b, p);
        } else {
            if (p != 0.0f) p = __fdiv_rn(b, p);
            if (p > 2.0f) p = 2.0f;
        }
        proj[idx] = p;
        if (surf) {
            const int iy = (int)(i / (unsigned)g.Nd), ix = (int)(i - (size_t)iy * g.Nd);
            surf2DLayeredwrite(p, surf, ix * (int)sizeof(float), iy, (int)blockIdx.y, cudaBoundaryModeZero);
        }
    }
    const double s = block_sum(acc);
    if (threadIdx.x == 0 && loss) atomicAdd(loss, s);
}

__global__ void k_normalize(size_t n, float *proj, const float *norm) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        proj[i] = __fmul_rn(proj[i], norm[i]);
}

/* ------------------------------------------------------------------------ */
/* Back-projection fused with the update.                                    */
/* Plain (ir.cu:1720-1751 then voxelProduct :1637-1654 / voxelPlus           */
/* :1682-1693): tmp and factor accumulate in the reference's order (axis,    */
/* then subset position), so the update is bit-identical to the reference's. */
/* XTT (ir.cu:1807-1850): per axis the moments sum(r), sum(r B B^T), sum(1), */
/* sum(B B^T), folded into tmp_k and factor_k with g_kc and S_k.             */
/* ------------------------------------------------------------------------ */
struct BackArgs {
    GeomConst g;
    const ViewFrame *frames;
    const int *view_list;
    int n_views, cond0, n_cond;
    const float *proj;
    void *vol;                /* type T */
    const BasisConst *basis;
    int art;
    float alpha;
    int sr;                   /* 16-bit volumes: stochastic rounding of updates */
    const float *coef;        /* non-null: per-voxel rotated basis (backwardOrth) */
    int coef_kind;            /* 0: (phi, cos theta); 1: main direction            */
};

template <bool XTT, typename T>
__global__ void __launch_bounds__(kBackThreads) k_back_update(BackArgs a) {
    __shared__ ViewFrame fr[kFrameChunk];
    const GeomConst &g = a.g;
    const int N = g.N, Nd = g.Nd;
    const int nbx = (N + 7) / 8, nby = (N + 3) / 4;
    const int b = blockIdx.x;
    const int x = (b % nbx) * 8 + (threadIdx.x & 7);
    const int y = ((b / nbx) % nby) * 4 + ((threadIdx.x >> 3) & 3);
    const int z = (b / (nbx * nby)) * 8 + (threadIdx.x >> 5);
    const bool ok = x < N && y < N && z < N;
    const float bx = vox_base(x, N, g.vs), by = vox_base(y, N, g.vs), bz = vox_base(z, N, g.vs);
    const size_t NdNd = (size_t)Nd * Nd;

    constexpr int KMAX = XTT ? kMaxBasis : 1;
    float tmpk[XTT ? 16 : 1], fack[XTT ? 16 : 1];
    /* K <= 16 in registers; larger K spill to local memory (rare). */
    float tmp = 0.f, fac = 0.f;
    if (XTT) {
#pragma unroll
        for (int k = 0; k < 16; k++) { tmpk[k] = 0.f; fack[k] = 0.f; }
    }
    (void)KMAX;

    for (int ci = 0; ci < a.n_cond; ci++) {
        const int cond = a.cond0 + ci;
        const float *P = a.proj + (size_t)cond * g.V * NdNd;
        float A0 = 0.f, F0 = 0.f, A[6] = {0, 0, 0, 0, 0, 0}, F[6] = {0, 0, 0, 0, 0, 0};
        for (int c0 = 0; c0 < a.n_views; c0 += kFrameChunk) {
            const int nc = min(kFrameChunk, a.n_views - c0);
            __syncthreads();
            for (int i = threadIdx.x; i < nc * 5; i += kBackThreads) {
                const int jj = i / 5, q = i % 5;
                const float4 *s4 =
                    reinterpret_cast<const float4 *>(&a.frames[(size_t)cond * g.V + a.view_list[c0 + jj]]);
                reinterpret_cast<float4 *>(&fr[jj])[q] = s4[q];
            }
            __syncthreads();
            if (!ok) continue;
            for (int jj = 0; jj < nc; jj++) {
                const ViewFrame &f = fr[jj];
                float u, v, d0, d1, d2;
                ray_uv(f, g, bx, by, bz, u, v, d0, d1, d2);
                int iu, iv;
                float c1, c2, c3, c4;
                if (!taps(g, u, v, iu, iv, c1, c2, c3, c4)) continue;
                const float *pp = P + (size_t)f.view * NdNd + iu + (size_t)Nd * iv;
                const float p4 = __ldg(pp), p3 = __ldg(pp + 1), p1 = __ldg(pp + Nd), p2 = __ldg(pp + Nd + 1);
                const float nb = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(c1, p1), __fmul_rn(c2, p2)),
                                                     __fmul_rn(c3, p3)), __fmul_rn(c4, p4));
                if (!XTT) {
                    fac = __fadd_rn(fac, 1.0f);
                    tmp = __fadd_rn(tmp, nb);
                } else {
                    const float inv = __frcp_rn(fmaf(d0, d0, fmaf(d1, d1, d2 * d2)));
                    const float q00 = d0 * d0 * inv, q11 = d1 * d1 * inv, q22 = d2 * d2 * inv;
                    const float q01 = d0 * d1 * inv, q02 = d0 * d2 * inv, q12 = d1 * d2 * inv;
                    A0 += nb; F0 += 1.0f;
                    A[0] = fmaf(nb, q00, A[0]); A[1] = fmaf(nb, q11, A[1]); A[2] = fmaf(nb, q22, A[2]);
                    A[3] = fmaf(nb, q01, A[3]); A[4] = fmaf(nb, q02, A[4]); A[5] = fmaf(nb, q12, A[5]);
                    F[0] += q00; F[1] += q11; F[2] += q22; F[3] += q01; F[4] += q02; F[5] += q12;
                }
            }
        }
        if (XTT && ok && a.coef) {   /* backwardOrth(ByMD) (ir.cu:366-423, :233-292): the voxel's rotated basis */
            const BasisConst *B = a.basis;
            float R[9];
            src_rotation(a.coef, a.coef_kind, (size_t)N * N * N, (size_t)x + (size_t)N * y + (size_t)N * N * z, R);
            const float G0 = B->G[3 * cond], G1 = B->G[3 * cond + 1], G2 = B->G[3 * cond + 2];
#pragma unroll
            for (int k = 0; k < 16; k++) {
                if (k >= g.K) break;
                float S[3];
                orth_basis(B, k, R, S);
                const float h = S[0] * G0 + S[1] * G1 + S[2] * G2, gk = h * h;
                const float s2 = S[0] * S[0] + S[1] * S[1] + S[2] * S[2];
                const float sAs = S[0] * S[0] * A[0] + S[1] * S[1] * A[1] + S[2] * S[2] * A[2] +
                                  2.f * (S[0] * S[1] * A[3] + S[0] * S[2] * A[4] + S[1] * S[2] * A[5]);
                const float sFs = S[0] * S[0] * F[0] + S[1] * S[1] * F[1] + S[2] * S[2] * F[2] +
                                  2.f * (S[0] * S[1] * F[3] + S[0] * S[2] * F[4] + S[1] * S[2] * F[5]);
                tmpk[k] = fmaf(gk, fmaf(s2, A0, -sAs), tmpk[k]);
                fack[k] = fmaf(gk, fmaf(s2, F0, -sFs), fack[k]);
            }
        } else if (XTT && ok) {
            const BasisConst *B = a.basis;
#pragma unroll
            for (int k = 0; k < 16; k++) {
                if (k >= g.K) break;
                const float gk = B->g[cond * g.K + k];
                const float s0 = B->S[3 * k], s1 = B->S[3 * k + 1], s2 = B->S[3 * k + 2];
                const float sAs = s0 * s0 * A[0] + s1 * s1 * A[1] + s2 * s2 * A[2] +
                                  2.f * (s0 * s1 * A[3] + s0 * s2 * A[4] + s1 * s2 * A[5]);
                const float sFs = s0 * s0 * F[0] + s1 * s1 * F[1] + s2 * s2 * F[2] +
                                  2.f * (s0 * s1 * F[3] + s0 * s2 * F[4] + s1 * s2 * F[5]);
                tmpk[k] = fmaf(gk, fmaf(B->S2[k], A0, -sAs), tmpk[k]);
                fack[k] = fmaf(gk, fmaf(B->S2[k], F0, -sFs), fack[k]);
            }
        }
    }
    if (!ok) return;
    const size_t NN = (size_t)N * N, N3 = NN * N;
    const size_t idx = (size_t)x + (size_t)N * y + NN * z;
    if (!XTT) {
        T *vp = reinterpret_cast<T *>(a.vol) + idx;
        const float mu = ldf<T>(vp);
        if (a.art) stu<T>(vp, __fadd_rn(mu, __fmul_rn(a.alpha, tmp)), (uint32_t)idx, a.sr);
        else stu<T>(vp, (fac == 0.0f) ? 0.0f : __fdiv_rn(__fmul_rn(mu, tmp), fac), (uint32_t)idx, a.sr);
    } else {
        /* four channels' loads in flight before their first store */
#pragma unroll
        for (int k0 = 0; k0 < 16; k0 += 4) {
            if (k0 >= g.K) break;
            float mu[4];
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (k0 + j < g.K) mu[j] = ldf<T>(reinterpret_cast<T *>(a.vol) + idx + (size_t)(k0 + j) * N3);
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int k = k0 + j;
                if (k >= g.K) break;
                T *vp = reinterpret_cast<T *>(a.vol) + idx + (size_t)k * N3;
                const uint32_t key = (uint32_t)(idx + (size_t)k * N3);
                if (a.art) stu<T>(vp, __fadd_rn(mu[j], __fmul_rn(a.alpha, tmpk[k])), key, a.sr);
                else stu<T>(vp, (fack[k] == 0.0f) ? 0.0f : __fdiv_rn(__fmul_rn(mu[j], tmpk[k]), fack[k]), key, a.sr);
            }
        }
    }
}

/* ------------------------------------------------------------------------ */
template <typename T>
__global__ void k_residual(size_t n, const float *p, const T *b, double *out) {
    double s2 = 0, b2 = 0, s1 = 0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double bi = (double)ldgf<T>(b + i);
        const double d = (double)p[i] - bi;
        s2 += d * d;
        b2 += bi * bi;
        s1 += fabs(d);
    }
    s2 = block_sum(s2);
    b2 = block_sum(b2);
    s1 = block_sum(s1);
    if (threadIdx.x == 0) {
        atomicAdd(out, s2);
        atomicAdd(out + 1, b2);
        atomicAdd(out + 2, s1);
    }
}

/* voxelSqrt, ir.cu:1707-1717. */
template <typename T>
__global__ void k_sqrt_abs(size_t n, T *mu) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float m = ldf<T>(mu + i);
        stf<T>(mu + i, (m < 0.0f) ? __fsqrt_rn(-m) : __fsqrt_rn(m));
    }
}

/* storage conversions (round to nearest even) */
template <typename S, typename D>
__global__ void k_convert(size_t n, const S *src, D *dst) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        stf<D>(dst + i, ldgf<S>(src + i));
}

int grid_for(size_t n, int threads) {
    size_t b = (n + threads - 1) / threads;
    if (b > 148 * 16) b = 148 * 16;
    if (b < 1) b = 1;
    return (int)b;
}

}  // namespace

cudaError_t launch_forward(const GeomConst &g, const BasisConst *d_basis, const ViewFrame *frames,
                           const int *view_list, int n_views, int cond0, int n_cond, const void *vol, float *out,
                           int mode, int views_per_cta, int storage, cudaStream_t s, const float *coef,
                           int coef_kind) {
    if (n_views <= 0 || n_cond <= 0) return cudaSuccess;
    if (coef && mode == 1) mode = 3;
    FwdArgs a;
    a.coef = coef;
    a.coef_kind = coef_kind;
    a.g = g;
    a.frames = frames;
    a.view_list = view_list;
    a.n_views = n_views;
    a.cond0 = cond0;
    a.vol = vol;
    a.out = out;
    a.basis = d_basis;
    a.nbx = (g.N + kBX - 1) / kBX;
    a.nby = (g.N + kBY - 1) / kBY;
    const int nbz = (g.N + kBZ - 1) / kBZ;
    const long bricks = (long)a.nbx * a.nby * nbz;
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
    cudaError_t e = cudaSuccess;
#define XR_FWD(M, TT)                                                                                             \
    do {                                                                                                          \
        e = cudaFuncSetAttribute(k_forward<M, TT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);       \
        if (e == cudaSuccess) k_forward<M, TT><<<grid, kFwdThreads, smem, s>>>(a);                                \
    } while (0)
    if (mode == 2) XR_FWD(2, float);
    else if (storage == kBF16) {
        if (mode == 0) XR_FWD(0, __nv_bfloat16); else if (mode == 3) XR_FWD(3, __nv_bfloat16); else XR_FWD(1, __nv_bfloat16);
    } else if (storage == kF16) {
        if (mode == 0) XR_FWD(0, __half); else if (mode == 3) XR_FWD(3, __half); else XR_FWD(1, __half);
    } else {
        if (mode == 0) XR_FWD(0, float); else if (mode == 3) XR_FWD(3, float); else XR_FWD(1, float);
    }
#undef XR_FWD
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

cudaError_t launch_chord(const GeomConst &g, const ViewFrame *frames, float *norm, int n_cond, cudaStream_t s) {
    const dim3 blk(32, 8);
    const dim3 grid((g.Nd + 31) / 32, (g.Nd + 7) / 8, (unsigned)(n_cond * g.V));
    k_chord<<<grid, blk, 0, s>>>(g, frames, norm, n_cond);
    return cudaGetLastError();
}

cudaError_t launch_ratio(const GeomConst &g, const int *view_list, int n_views, int n_cond, float *proj,
                         const float *norm, const void *sino, int art, double *loss, int storage, cudaStream_t s,
                         cudaSurfaceObject_t surf) {
    if (n_views <= 0) return cudaSuccess;
    const size_t NdNd = (size_t)g.Nd * g.Nd;
    int bx = (int)((NdNd + 255) / 256);
    if (bx > 64) bx = 64;
    const dim3 grid(bx, (unsigned)(n_views * n_cond));
    if (storage == kBF16)
        k_ratio<<<grid, 256, 0, s>>>(g, view_list, n_views, proj, norm, (const __nv_bfloat16 *)sino, art, loss, surf);
    else if (storage == kF16)
        k_ratio<<<grid, 256, 0, s>>>(g, view_list, n_views, proj, norm, (const __half *)sino, art, loss, surf);
    else
        k_ratio<<<grid, 256, 0, s>>>(g, view_list, n_views, proj, norm, (const float *)sino, art, loss, surf);
    return cudaGetLastError();
}

cudaError_t launch_normalize(const GeomConst &g, int n_cond, float *proj, const float *norm, cudaStream_t s) {
    const size_t n = (size_t)n_cond * g.V * g.Nd * g.Nd;
    k_normalize<<<grid_for(n, 256), 256, 0, s>>>(n, proj, norm);
    return cudaGetLastError();
}

cudaError_t launch_back_update(const GeomConst &g, const BasisConst *d_basis, const ViewFrame *frames,
                               const int *view_list, int n_views, int cond0, int n_cond, const float *proj,
                               void *vol, int xtt, int art, float alpha, int storage, cudaStream_t s,
                               const float *coef, int coef_kind) {
    BackArgs a;
    a.coef = coef;
    a.coef_kind = coef_kind;
    a.sr = (storage & kStoreStochastic) != 0;
    storage &= ~kStoreStochastic;
    a.g = g;
    a.frames = frames;
    a.view_list = view_list;
    a.n_views = n_views;
    a.cond0 = cond0;
    a.n_cond = n_cond;
    a.proj = proj;
    a.vol = vol;
    a.basis = d_basis;
    a.art = art;
    a.alpha = alpha;
    const long nb = (long)((g.N + 7) / 8) * ((g.N + 3) / 4) * ((g.N + 7) / 8);
#define XR_BACK(X, TT) k_back_update<X, TT><<<(unsigned)nb, kBackThreads, 0, s>>>(a)
    if (storage == kBF16) { if (xtt) XR_BACK(true, __nv_bfloat16); else XR_BACK(false, __nv_bfloat16); }
    else if (storage == kF16) { if (xtt) XR_BACK(true, __half); else XR_BACK(false, __half); }
    else { if (xtt) XR_BACK(true, float); else XR_BACK(false, float); }
#undef XR_BACK
    return cudaGetLastError();
}

cudaError_t launch_residual(long n, const float *p, const void *b, double *out, int storage, cudaStream_t s) {
    const int gr = grid_for((size_t)n, 256);
    if (storage == kBF16) k_residual<<<gr, 256, 0, s>>>((size_t)n, p, (const __nv_bfloat16 *)b, out);
    else if (storage == kF16) k_residual<<<gr, 256, 0, s>>>((size_t)n, p, (const __half *)b, out);
    else k_residual<<<gr, 256, 0, s>>>((size_t)n, p, (const float *)b, out);
    return cudaGetLastError();
}

cudaError_t launch_sqrt_abs(long n, void *mu, int storage, cudaStream_t s) {
    const int gr = grid_for((size_t)n, 256);
    if (storage == kBF16) k_sqrt_abs<<<gr, 256, 0, s>>>((size_t)n, (__nv_bfloat16 *)mu);
    else if (storage == kF16) k_sqrt_abs<<<gr, 256, 0, s>>>((size_t)n, (__half *)mu);
    else k_sqrt_abs<<<gr, 256, 0, s>>>((size_t)n, (float *)mu);
    return cudaGetLastError();
}

cudaError_t launch_convert(long n, const void *src, int src_storage, void *dst, int dst_storage, cudaStream_t s) {
    const int gr = grid_for((size_t)n, 256);
    const size_t m = (size_t)n;
    if (src_storage == kF32 && dst_storage == kBF16)
        k_convert<<<gr, 256, 0, s>>>(m, (const float *)src, (__nv_bfloat16 *)dst);
    else if (src_storage == kF32 && dst_storage == kF16)
        k_convert<<<gr, 256, 0, s>>>(m, (const float *)src, (__half *)dst);
    else if (src_storage == kBF16 && dst_storage == kF32)
        k_convert<<<gr, 256, 0, s>>>(m, (const __nv_bfloat16 *)src, (float *)dst);
    else if (src_storage == kF16 && dst_storage == kF32)
        k_convert<<<gr, 256, 0, s>>>(m, (const __half *)src, (float *)dst);
    else if (src_storage == dst_storage)
        return cudaMemcpyAsync(dst, src, m * storage_bytes(src_storage), cudaMemcpyDeviceToDevice, s);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

}  // namespace xr
