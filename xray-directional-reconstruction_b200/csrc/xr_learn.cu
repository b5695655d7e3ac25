/*
 * Learned warm start on sm_100a tensor cores: 3x3x3 convolutions as implicit
 * GEMMs on tcgen05.mma (BF16 operands in shared memory, FP32 accumulators in
 * tensor memory), the network's forward / backward passes, the MSE loss, Adam.
 * The network is defined in include/xr_learn.h; it is an extension with no
 * counterpart in the reference.
 *
 * Activations are channels-last BF16, element [v][c] with v the flattened
 * voxel index (x fastest) and c padded to 16 or 32 channels, so one voxel's
 * channels are 32 or 64 contiguous bytes: exactly the 16-byte rows the tensor
 * core's shared-memory operands are built of.
 *
 *  k_conv_halo (fprop and dgrad): M = 128 voxels (an 8 x 16 patch of one
 *    z-slice), N = output channels, K = 27 taps x input channels.  A CTA keeps
 *    all 27 taps of the weights in shared memory (K-major core matrices) and
 *    a ring of halo slices; every tap's operand is a shifted window of the
 *    halo, addressed by the descriptor alone, so a slice costs one load of
 *    its halo and 27 x K/16 back-to-back MMAs.  dgrad is the same operator on
 *    the output gradient with the weights transposed and the taps mirrored;
 *    its epilogue multiplies by the ReLU derivative (forward activation > 0).
 *  k_conv_wgrad: M = 128 (tap, input channel) rows, N = output channels,
 *    K = voxels in chunks of 64; both operands MN-major, so the 16-byte rows
 *    come straight from the channels-last tensors.  CTAs split the voxels
 *    and add their FP32 partial sums into the weight gradient.
 *
 * Every mbarrier wait is bounded (about two seconds); on timeout the CTA sets
 * the error flag, waits (bounded) for its MMAs in flight, frees its tensor
 * memory and leaves.
 */
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../include/xr_learn.h"
#include "xr_storage.cuh"
#include "xr_tc.cuh"

namespace xr {
namespace {

constexpr int kConvThreads = 128;
constexpr long long kWaitCycles = 4000000000LL;   /* ~2 s at 1.9 GHz */
constexpr int kTmemCols = 32;

typedef __nv_bfloat16 bf16;

__device__ __forceinline__ uint32_t pack2(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t *>(&h);
}

__device__ __forceinline__ float bf_lo(uint32_t u) { return __uint_as_float(u << 16); }
__device__ __forceinline__ float bf_hi(uint32_t u) { return __uint_as_float(u & 0xFFFF0000u); }

struct ConvArgs {
    const bf16 *x;      /* [nvox][KP]                                   */
    const bf16 *w;      /* [27][NP][KP]                                 */
    const float *bias;  /* [NP] or null                                 */
    const bf16 *mask;   /* [nvox][NP], epilogue 2                       */
    bf16 *y;            /* [nvox][NP], epilogues 0-2                    */
    const void *res;    /* epilogue 3: planar [nout][nvox] of `storage` */
    void *out;          /* epilogue 3: planar [nout][nvox] of `storage` */
    int storage, nout;
    float inv_scale, floor_value;
    int nx, ny, nz;
    int *err;
};

enum { EPI_BIAS = 0, EPI_RELU = 1, EPI_MASK = 2, EPI_RESID = 3 };

/* (x, y, z) of voxel v and whether its neighbour at tap t lies inside. */
__device__ __forceinline__ bool tap_src(int t, long v, int x, int y, int z, int nx, int ny, int nz, long &src) {
    const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
    const int xx = x + dx, yy = y + dy, zz = z + dz;
    src = v + dx + (long)nx * (dy + (long)ny * dz);
    return xx >= 0 && xx < nx && yy >= 0 && yy < ny && zz >= 0 && zz < nz;
}

template <int KP>
__device__ __forceinline__ void load_row(const bf16 *x, long v, bool ok, uint4 *r) {
    const uint4 *p = reinterpret_cast<const uint4 *>(x + (size_t)v * KP);
#pragma unroll
    for (int j = 0; j < KP / 8; j++) r[j] = ok ? __ldg(p + j) : make_uint4(0u, 0u, 0u, 0u);
}

__device__ __forceinline__ uint8_t *align1k(uint8_t *p) {
    const uint32_t s = tc::smem_u32(p);
    return p + (((s + 1023u) & ~1023u) - s);
}

/* Output of one voxel's NP accumulators (row of the M = 128 tile). */
template <int NP, int EPI>
__device__ __forceinline__ void conv_epilogue(const ConvArgs &a, long v, long nvox, const float *acc) {
    if (EPI == EPI_RESID) {
#pragma unroll
        for (int n = 0; n < NP; n++) {
            if (n >= a.nout) break;
            const size_t i = (size_t)n * nvox + v;
            float val = acc[n] + (a.bias ? a.bias[n] : 0.f);
            if (a.storage == kBF16) {
                val = fmaxf(ldf(reinterpret_cast<const __nv_bfloat16 *>(a.res) + i) + val * a.inv_scale,
                            a.floor_value);
                stf(reinterpret_cast<__nv_bfloat16 *>(a.out) + i, val);
            } else if (a.storage == kF16) {
                val = fmaxf(ldf(reinterpret_cast<const __half *>(a.res) + i) + val * a.inv_scale, a.floor_value);
                stf(reinterpret_cast<__half *>(a.out) + i, val);
            } else {
                val = fmaxf(ldf(reinterpret_cast<const float *>(a.res) + i) + val * a.inv_scale, a.floor_value);
                stf(reinterpret_cast<float *>(a.out) + i, val);
            }
        }
    } else {
        uint4 *yo = reinterpret_cast<uint4 *>(a.y + (size_t)v * NP);
        const uint4 *mk = reinterpret_cast<const uint4 *>(a.mask + (size_t)v * NP);
#pragma unroll
        for (int j = 0; j < NP / 8; j++) {
            float o[8];
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int n = 8 * j + i;
                o[i] = acc[n];
                if (EPI != EPI_MASK && a.bias) o[i] += a.bias[n];
                if (EPI == EPI_RELU) o[i] = fmaxf(o[i], 0.f);
            }
            if (EPI == EPI_MASK) {
                const uint4 m = mk[j];
                const uint32_t mw[4] = {m.x, m.y, m.z, m.w};
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    if (!(bf_lo(mw[i]) > 0.f)) o[2 * i] = 0.f;
                    if (!(bf_hi(mw[i]) > 0.f)) o[2 * i + 1] = 0.f;
                }
            }
            yo[j] = make_uint4(pack2(o[0], o[1]), pack2(o[2], o[3]), pack2(o[4], o[5]), pack2(o[6], o[7]));
        }
    }
}

/* ---------------------------------------------------------------------- */
/* Spatial-tile convolution (fprop / dgrad).                               */
/* An output tile is 8 (x) x 16 (y) voxels of one z-slice: M = 128 rows,   */
/* row r = (x = r % 8, y = r / 8).  The input around it is a halo slice of */
/* 10 x 18 voxels, stored as KP/8 planes of 16-byte rows (plane j holds    */
/* channels 8j..8j+7 of every halo voxel, x fastest).  For tap (dz,dy,dx)  */
/* the A operand is then a window of the halo: 8 consecutive 16-byte rows  */
/* are the 8 x-voxels of one y-row (a core matrix), y-rows are 160 bytes   */
/* apart (SBO), planes PLANE bytes apart (LBO) - the descriptor's start    */
/* address moves by (dy * 10 + dx) * 16 bytes and by one slice for dz.     */
/* No per-tap loads or barriers: each input slice is loaded once (zero     */
/* outside the volume) into a 4-slot ring and serves three output slices;  */
/* the 27 x KP/16 MMAs of a slice are issued back to back into one of two  */
/* tensor-memory accumulators while the previous slice's epilogue runs.    */
/* ---------------------------------------------------------------------- */
constexpr int kHX = 10, kHY = 18, kHV = kHX * kHY;   /* halo slice: 180 voxels */
constexpr int kRing = 4;

template <int KP, int NP>
struct HaloSmem {
    static constexpr int BT = NP * KP * 2;
    static constexpr int BB = ((27 * BT + 1023) / 1024) * 1024;
    static constexpr int PLANE = kHV * 16;                       /* 2880 bytes */
    static constexpr int SLOT = (KP / 8) * PLANE;
    static constexpr int bytes = 1024 + BB + kRing * SLOT + 2 * 8 + 16;
    static constexpr int LOADS = (kHV * KP / 8 + kConvThreads - 1) / kConvThreads;   /* 16-byte loads per thread */
};

template <int KP, int NP, int EPI>
__global__ void __launch_bounds__(kConvThreads) k_conv_halo(ConvArgs a, int zchunk) {
    using L = HaloSmem<KP, NP>;
    constexpr uint32_t SBO_B = (KP / 8) * 128;
    constexpr uint32_t IDESC = tc::idesc_bf16(128, NP, 0, 0);
    extern __shared__ uint8_t smem_raw[];
    uint8_t *sm = align1k(smem_raw);
    uint8_t *sB = sm, *ring = sm + L::BB;
    uint64_t *bar = reinterpret_cast<uint64_t *>(ring + kRing * L::SLOT);   /* one per accumulator */
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 2);
    __shared__ int s_abort;

    const int tid = threadIdx.x, warp = tid >> 5;
    if (tid == 0) {
        tc::mbar_init(&bar[0], 1);
        tc::mbar_init(&bar[1], 1);
        tc::fence_mbar_init();
        s_abort = 0;
    }
    if (warp == 0) tc::tmem_alloc(tslot, 2 * kTmemCols);
    for (int c = tid; c < 27 * NP * KP / 8; c += kConvThreads) {
        const int j = c % (KP / 8), n = (c / (KP / 8)) % NP, t = c / (NP * KP / 8);
        *reinterpret_cast<uint4 *>(sB + t * L::BT + (n >> 3) * SBO_B + j * 128 + (n & 7) * 16) =
            __ldg(reinterpret_cast<const uint4 *>(a.w) + c);
    }
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot;

    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const long nvox = (long)nx * ny * nz;
    const int ntx = (nx + 7) / 8, nty = (ny + 15) / 16, ntz = (nz + zchunk - 1) / zchunk;
    const long items = (long)ntx * nty * ntz;
    uint32_t uses0 = 0, uses1 = 0;        /* completions waited for, per accumulator   */
    uint32_t commits0 = 0, commits1 = 0;  /* commits issued (by thread 0; tracked by all) */
    bool aborted = false;

    /* 16-byte halo loads of input slice zin into registers */
    auto fetch = [&](int x0, int y0, int zin, uint4 *r) {
#pragma unroll
        for (int u = 0; u < L::LOADS; u++) {
            const int e = tid + u * kConvThreads;
            r[u] = make_uint4(0u, 0u, 0u, 0u);
            if (e < kHV * KP / 8 && zin >= 0 && zin < nz) {
                const int j = e % (KP / 8), hv = e / (KP / 8);
                const int gx = x0 - 1 + hv % kHX, gy = y0 - 1 + hv / kHX;
                if (gx >= 0 && gx < nx && gy >= 0 && gy < ny)
                    r[u] = __ldg(reinterpret_cast<const uint4 *>(
                                     a.x + ((size_t)gx + (size_t)nx * (gy + (size_t)ny * zin)) * KP) + j);
            }
        }
    };
    auto stash = [&](uint8_t *slot, const uint4 *r) {
#pragma unroll
        for (int u = 0; u < L::LOADS; u++) {
            const int e = tid + u * kConvThreads;
            if (e < kHV * KP / 8) {
                const int j = e % (KP / 8), hv = e / (KP / 8);
                *reinterpret_cast<uint4 *>(slot + j * L::PLANE + hv * 16) = r[u];
            }
        }
    };

    for (long item = blockIdx.x; item < items && !aborted; item += gridDim.x) {
        const int tx = (int)(item % ntx), ty = (int)((item / ntx) % nty), tz = (int)(item / ((long)ntx * nty));
        const int x0 = tx * 8, y0 = ty * 16, z0 = tz * zchunk;
        const int nzs = min(zchunk, nz - z0);      /* output slices of this item */
        const int ox = x0 + (tid & 7), oy = y0 + (tid >> 3);
        /* input slice k (z = z0 - 1 + k) lives in ring slot k % 4; prologue: k = 0, 1 */
        uint4 r[L::LOADS];
        fetch(x0, y0, z0 - 1, r);
        stash(ring + 0 * L::SLOT, r);
        fetch(x0, y0, z0, r);
        stash(ring + 1 * L::SLOT, r);
        fetch(x0, y0, z0 + 1, r);                 /* slice k = 2, stored in iteration 0 */
        for (int i = 0; i <= nzs; i++) {
            if (i < nzs) {
                /* slot (i+2) % 4 held slice i-2, whose last reader (output i-1... i-2)
                 * completed: output i-2's epilogue waited for its MMAs, and output
                 * i-1 reads slices i-1..i+1 only */
                stash(ring + ((i + 2) % kRing) * L::SLOT, r);
                if (i + 1 < nzs) fetch(x0, y0, z0 + i + 2, r);
                tc::fence_async_smem();
                tc::fence_before_sync();
                __syncthreads();
                if (s_abort) { aborted = true; break; }
                if (tid == 0) {
                    tc::fence_after_sync();
                    const int buf = i & 1;
                    const uint32_t d = tmem + buf * kTmemCols;
                    /* descriptors: a base per input slice (dz), the tap's (dy, dx)
                     * window and the K step added to the start-address field
                     * (16-byte units; no carry: shared addresses < 256 KB) */
                    uint64_t aS[3];
#pragma unroll
                    for (int dz = 0; dz < 3; dz++)
                        aS[dz] = tc::sdesc(tc::smem_u32(ring + ((i + dz) % kRing) * L::SLOT), L::PLANE, kHX * 16);
                    const uint64_t bS = tc::sdesc(tc::smem_u32(sB), 128, SBO_B);
#pragma unroll
                    for (int t = 0; t < 27; t++) {
                        const int dz = t / 9, dy = (t / 3) % 3, dx = t % 3;
                        const uint64_t at = aS[dz] + (uint64_t)(dy * kHX + dx);
                        const uint64_t bt = bS + (uint64_t)(t * (L::BT >> 4));
#pragma unroll
                        for (int kk = 0; kk < KP / 16; kk++)
                            tc::mma_bf16(d, at + (uint64_t)(kk * (2 * L::PLANE >> 4)), bt + (uint64_t)(kk * 16), IDESC,
                                         (t | kk) != 0);
                    }
                    tc::mma_commit(&bar[buf]);
                }
                if (i & 1) commits1++;
                else commits0++;
            }
            if (i >= 1) {   /* epilogue of output slice i - 1 */
                const int buf = (i - 1) & 1;
                const uint32_t k_use = buf ? uses1++ : uses0++;
                /* a wait that runs out is seen by every thread at the next barrier */
                if (!tc::mbar_wait(&bar[buf], k_use & 1, kWaitCycles)) {
                    s_abort = 1;
                } else {
                    tc::fence_after_sync();
                    float acc[NP];
                    const uint32_t taddr = tmem + buf * kTmemCols + ((uint32_t)(warp * 32) << 16);
                    if (NP == 16) tc::tmem_ld16(taddr, acc);
                    else tc::tmem_ld32(taddr, acc);
                    tc::fence_before_sync();
                    const int oz = z0 + i - 1;
                    if (ox < nx && oy < ny)
                        conv_epilogue<NP, EPI>(a, (long)ox + (long)nx * (oy + (long)ny * oz), nvox, acc);
                }
            }
            if (aborted) break;
        }
        if (aborted) break;
    }
    tc::fence_before_sync();
    __syncthreads();
    if (s_abort) aborted = true;
    /* a wait that ran out leaves MMAs possibly in flight: wait (bounded) for
     * each accumulator's last commit */
    if (aborted) {
        if (commits0 > 0) tc::mbar_wait(&bar[0], (commits0 - 1) & 1, kWaitCycles);
        if (commits1 > 0) tc::mbar_wait(&bar[1], (commits1 - 1) & 1, kWaitCycles);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, 2 * kTmemCols);
    }
    if (aborted && tid == 0) atomicExch(a.err, 1);
}

struct WgradArgs {
    const bf16 *x;    /* [nvox][KP] */
    const bf16 *dy;   /* [nvox][NP] */
    float *dw;        /* [27][NP][KP], accumulated */
    int nx, ny, nz;
    long chunks_per_cta;
    int *err;
};

template <int KP, int NP>
struct WgSmem {
    static constexpr int VC = 64;                       /* voxels (K) per stage */
    static constexpr int AB = 128 * VC * 2;
    static constexpr int BBy = NP * VC * 2;
    static constexpr int SB = AB + BBy;
    static constexpr int S = 3;
    static constexpr int bytes = 1024 + S * SB + S * 8 + 16;
};

template <int KP, int NP>
__global__ void __launch_bounds__(kConvThreads) k_conv_wgrad(WgradArgs a) {
    using L = WgSmem<KP, NP>;
    constexpr int VC = L::VC, S = L::S;
    constexpr int TPB = 128 / KP;                        /* taps per block of 128 rows */
    constexpr uint32_t SBO = (VC / 8) * 128;             /* next 8 rows (M or N)       */
    constexpr uint32_t IDESC = tc::idesc_bf16(128, NP, 1, 1);
    constexpr int A_PER = 128 * VC / 8 / kConvThreads;   /* 16-byte chunks per thread  */
    constexpr int B_PER = NP * VC / 8 / kConvThreads;
    extern __shared__ uint8_t smem_raw[];
    uint8_t *sm = align1k(smem_raw);
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + S * L::SB);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + S);
    __shared__ int s_abort;

    const int tid = threadIdx.x, warp = tid >> 5;
    const int tb = blockIdx.x;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const long nvox = (long)nx * ny * nz;
    const long nchunks = (nvox + VC - 1) / VC;
    const long c0 = (long)blockIdx.y * a.chunks_per_cta;
    const long c1 = min(nchunks, c0 + a.chunks_per_cta);
    if (c0 >= c1) return;   /* uniform over the CTA, before any allocation */

    if (tid == 0) {
        for (int s = 0; s < S; s++) tc::mbar_init(&bar[s], 1);
        tc::fence_mbar_init();
        s_abort = 0;
    }
    if (warp == 0) tc::tmem_alloc(tslot, kTmemCols);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot;

    uint4 ra[A_PER], rb[B_PER];
    auto load = [&](long c) {
#pragma unroll
        for (int i = 0; i < A_PER; i++) {
            const int ch = tid + i * kConvThreads;
            const int j = ch % (KP / 8), k = (ch / (KP / 8)) % VC, tl = ch / (VC * KP / 8);
            const int t = tb * TPB + tl;
            const long v = c * VC + k;
            bool ok = (t < 27) && (v < nvox);
            long src = 0;
            if (ok) {
                const int x = (int)(v % nx);
                const long q = v / nx;
                ok = tap_src(t, v, x, (int)(q % ny), (int)(q / ny), nx, ny, nz, src);
            }
            ra[i] = ok ? __ldg(reinterpret_cast<const uint4 *>(a.x + (size_t)src * KP) + j) : make_uint4(0u, 0u, 0u, 0u);
        }
#pragma unroll
        for (int i = 0; i < B_PER; i++) {
            const int ch = tid + i * kConvThreads;
            const int jn = ch % (NP / 8), k = ch / (NP / 8);
            const long v = c * VC + k;
            rb[i] = (v < nvox) ? __ldg(reinterpret_cast<const uint4 *>(a.dy + (size_t)v * NP) + jn)
                               : make_uint4(0u, 0u, 0u, 0u);
        }
    };
    auto store = [&](uint8_t *sa, uint8_t *sb) {
#pragma unroll
        for (int i = 0; i < A_PER; i++) {
            const int ch = tid + i * kConvThreads;
            const int j = ch % (KP / 8), k = (ch / (KP / 8)) % VC, tl = ch / (VC * KP / 8);
            const int g = tl * (KP / 8) + j;
            *reinterpret_cast<uint4 *>(sa + g * SBO + (k >> 3) * 128 + (k & 7) * 16) = ra[i];
        }
#pragma unroll
        for (int i = 0; i < B_PER; i++) {
            const int ch = tid + i * kConvThreads;
            const int jn = ch % (NP / 8), k = ch / (NP / 8);
            *reinterpret_cast<uint4 *>(sb + jn * SBO + (k >> 3) * 128 + (k & 7) * 16) = rb[i];
        }
    };

    uint32_t use = 0;
    bool aborted = false;
    load(c0);
    for (long c = c0; c < c1; c++) {
        const int s = use % S;
        const uint32_t k_use = use / S;
        if (k_use > 0 && !tc::mbar_wait(&bar[s], (k_use - 1) & 1, kWaitCycles)) s_abort = 1;
        uint8_t *sa = sm + s * L::SB, *sb = sa + L::AB;
        store(sa, sb);
        if (c + 1 < c1) load(c + 1);
        tc::fence_async_smem();
        __syncthreads();
        if (s_abort) { aborted = true; break; }
        if (tid == 0) {
            tc::fence_after_sync();
            const uint32_t a0 = tc::smem_u32(sa), b0 = tc::smem_u32(sb);
#pragma unroll
            for (int kk = 0; kk < VC / 16; kk++)
                tc::mma_bf16(tmem, tc::sdesc(a0 + kk * 256, 128, SBO), tc::sdesc(b0 + kk * 256, 128, SBO), IDESC,
                             (c != c0 || kk != 0));
            tc::mma_commit(&bar[s]);
        }
        use++;
    }
    if (!aborted) {
        const uint32_t last = use - 1;
        if (!tc::mbar_wait(&bar[last % S], (last / S) & 1, kWaitCycles)) s_abort = 1;
        __syncthreads();
        if (s_abort) aborted = true;
    } else if (use > 0) {
        const uint32_t last = use - 1;
        tc::mbar_wait(&bar[last % S], (last / S) & 1, kWaitCycles);
    }
    if (!aborted) {
        tc::fence_after_sync();
        float acc[NP];
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
        if (NP == 16) tc::tmem_ld16(taddr, acc);
        else tc::tmem_ld32(taddr, acc);
        const int t = tb * TPB + tid / KP, k = tid % KP;
        if (t < 27)
#pragma unroll
            for (int n = 0; n < NP; n++) atomicAdd(a.dw + ((size_t)t * NP + n) * KP + k, acc[n]);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, kTmemCols);
    }
    if (aborted && tid == 0) atomicExch(a.err, 1);
}

/* ---------------------------------------------------------------------- */
/* Element-wise kernels                                                    */
/* ---------------------------------------------------------------------- */

/* planar K x nvox (storage T) -> channels-last BF16 [nvox][16], scaled, zero-padded */
template <typename T>
__global__ void k_pack_in(const T *x, int K, long nvox, float scale, bf16 *out) {
    for (long v = (long)blockIdx.x * blockDim.x + threadIdx.x; v < nvox; v += (long)gridDim.x * blockDim.x) {
        float f[16];
#pragma unroll
        for (int c = 0; c < 16; c++) f[c] = (c < K) ? ldgf<T>(x + (size_t)c * nvox + v) * scale : 0.f;
        uint4 *o = reinterpret_cast<uint4 *>(out + (size_t)v * 16);
        o[0] = make_uint4(pack2(f[0], f[1]), pack2(f[2], f[3]), pack2(f[4], f[5]), pack2(f[6], f[7]));
        o[1] = make_uint4(pack2(f[8], f[9]), pack2(f[10], f[11]), pack2(f[12], f[13]), pack2(f[14], f[15]));
    }
}

/* g[v][c] = bf16(gscale * (pred - target)) (zero for c >= K); loss += sum (pred - target)^2 */
__global__ void k_loss_grad(const float *pred, const float *target, int K, long nvox, float gscale, bf16 *g,
                            double *loss) {
    double s = 0.0;
    for (long v = (long)blockIdx.x * blockDim.x + threadIdx.x; v < nvox; v += (long)gridDim.x * blockDim.x) {
        float f[16];
#pragma unroll
        for (int c = 0; c < 16; c++) {
            f[c] = 0.f;
            if (c < K) {
                const float d = pred[(size_t)c * nvox + v] - target[(size_t)c * nvox + v];
                s += (double)d * d;
                f[c] = gscale * d;
            }
        }
        uint4 *o = reinterpret_cast<uint4 *>(g + (size_t)v * 16);
        o[0] = make_uint4(pack2(f[0], f[1]), pack2(f[2], f[3]), pack2(f[4], f[5]), pack2(f[6], f[7]));
        o[1] = make_uint4(pack2(f[8], f[9]), pack2(f[10], f[11]), pack2(f[12], f[13]), pack2(f[14], f[15]));
    }
    __shared__ double red[256];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(loss, red[0]);
}

/* db[c] += sum_v g[v][c] for c < C (g channels-last, NP channels) */
template <int NP>
__global__ void k_bias_grad(const bf16 *g, long nvox, int C, float *db) {
    float s[NP];
#pragma unroll
    for (int c = 0; c < NP; c++) s[c] = 0.f;
    for (long v = (long)blockIdx.x * blockDim.x + threadIdx.x; v < nvox; v += (long)gridDim.x * blockDim.x) {
        const uint4 *p = reinterpret_cast<const uint4 *>(g + (size_t)v * NP);
#pragma unroll
        for (int j = 0; j < NP / 8; j++) {
            const uint4 q = p[j];
            const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
            for (int i = 0; i < 4; i++) {
                s[8 * j + 2 * i] += bf_lo(w[i]);
                s[8 * j + 2 * i + 1] += bf_hi(w[i]);
            }
        }
    }
#pragma unroll
    for (int c = 0; c < NP; c++) {
        float t = s[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if ((threadIdx.x & 31) == 0 && c < C) atomicAdd(db + c, t);
    }
}

/* master W[tap][cout][cin] (FP32) -> wk[tap][NP][KP] and mirrored transposed wd[26-tap][KP][NP] (BF16) */
__global__ void k_pack_w(const float *W, int cin, int cout, int KP, int NP, bf16 *wk, bf16 *wd) {
    const int n_el = 27 * NP * KP;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_el; i += gridDim.x * blockDim.x) {
        const int k = i % KP, n = (i / KP) % NP, t = i / (KP * NP);
        const float w = (n < cout && k < cin) ? W[((size_t)t * cout + n) * cin + k] : 0.f;
        const bf16 h = __float2bfloat16_rn(w);
        wk[i] = h;
        wd[((size_t)(26 - t) * KP + k) * NP + n] = h;
    }
}

/* padded dw[tap][NP][KP] -> master gradient slot [tap][cout][cin] */
__global__ void k_unpack_dw(const float *dw, int cin, int cout, int KP, int NP, float *G) {
    const int n_el = 27 * cout * cin;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_el; i += gridDim.x * blockDim.x) {
        const int k = i % cin, n = (i / cin) % cout, t = i / (cin * cout);
        G[i] = dw[((size_t)t * NP + n) * KP + k];
    }
}

__global__ void k_adam(float *p, const float *g, float *m, float *v, long n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    }
}

/* Synthetic fiber phantom: straight cylinders (unit direction f, a point p0,
 * radius r); inside a fiber channel k holds eta_k = |S_k x f|^2, outside 0;
 * a later fiber overwrites an earlier one.  Voxel centres at i - (N-1)/2,
 * FP64 geometry. */
constexpr int kMaxFibers = 32;
struct PhantomArgs {
    int N, K, n_fib;
    float fib[kMaxFibers][7];     /* f (3), p0 (3), r */
    float eta[kMaxFibers][16];
};

__global__ void k_fiber_phantom(PhantomArgs a, float *out) {
    const long N = a.N, n3 = N * N * N;
    const double h = 0.5 * (double)(N - 1);
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += (long)gridDim.x * blockDim.x) {
        const double x = (double)(i % N) - h, y = (double)((i / N) % N) - h, z = (double)(i / (N * N)) - h;
        int hit = -1;
        for (int f = 0; f < a.n_fib; f++) {
            const double dx = x - a.fib[f][3], dy = y - a.fib[f][4], dz = z - a.fib[f][5];
            const double t = dx * a.fib[f][0] + dy * a.fib[f][1] + dz * a.fib[f][2];
            const double d2 = dx * dx + dy * dy + dz * dz - t * t;
            const double r = a.fib[f][6];
            if (d2 <= r * r) hit = f;
        }
        for (int k = 0; k < a.K; k++) out[(size_t)k * n3 + i] = hit >= 0 ? a.eta[hit][k] : 0.f;
    }
}

/* ---------------------------------------------------------------------- */
/* Launchers                                                               */
/* ---------------------------------------------------------------------- */

int g_sms = 0;

int sm_count() {
    if (g_sms == 0) {
        int d = 0;
        cudaGetDevice(&d);
        cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, d);
        if (g_sms <= 0) g_sms = 148;
    }
    return g_sms;
}

template <int KP, int NP, int EPI>
cudaError_t launch_halo_t(const ConvArgs &a, cudaStream_t s) {
    const int bytes = HaloSmem<KP, NP>::bytes;
    cudaError_t e = cudaFuncSetAttribute(k_conv_halo<KP, NP, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_conv_halo<KP, NP, EPI>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    /* CTAs per SM from shared memory (228 KB per SM, 1 KB reserved per CTA),
     * at most 4 (tensor memory: 4 x 64 of 512 columns) */
    int occ = 233472 / (bytes + 1024);
    occ = occ < 1 ? 1 : (occ > 4 ? 4 : occ);
    const long grid0 = (long)sm_count() * occ;
    const long xy = (long)((a.nx + 7) / 8) * ((a.ny + 15) / 16);
    /* z-chunk: long enough to amortise the two halo slices, short enough
     * for two work items per CTA */
    const long zc = std::max<long>(1, std::min<long>(64, ((long)a.nz * xy) / (2 * grid0)));
    const long items = xy * ((a.nz + zc - 1) / zc);
    const long grid = std::min<long>(items, grid0);
    k_conv_halo<KP, NP, EPI><<<(int)grid, kConvThreads, bytes, s>>>(a, (int)zc);
    return cudaGetLastError();
}

cudaError_t launch_fwd(int KP, int NP, int epi, const ConvArgs &a, cudaStream_t s) {
#define XR_FWD(kp, np)                                                       \
    if (KP == kp && NP == np) {                                              \
        switch (epi) {                                                       \
            case EPI_BIAS: return launch_halo_t<kp, np, EPI_BIAS>(a, s);     \
            case EPI_RELU: return launch_halo_t<kp, np, EPI_RELU>(a, s);     \
            case EPI_MASK: return launch_halo_t<kp, np, EPI_MASK>(a, s);     \
            default: break;                                                  \
        }                                                                    \
    }
    XR_FWD(16, 16)
    XR_FWD(16, 32)
    XR_FWD(32, 16)
    XR_FWD(32, 32)
#undef XR_FWD
    if (epi == EPI_RESID && NP == 16) {
        if (KP == 16) return launch_halo_t<16, 16, EPI_RESID>(a, s);
        if (KP == 32) return launch_halo_t<32, 16, EPI_RESID>(a, s);
    }
    return cudaErrorInvalidValue;
}

template <int KP, int NP>
cudaError_t launch_wgrad_t(WgradArgs a, cudaStream_t s) {
    const int bytes = WgSmem<KP, NP>::bytes;
    cudaError_t e = cudaFuncSetAttribute(k_conv_wgrad<KP, NP>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_conv_wgrad<KP, NP>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    int occ = 233472 / (bytes + 1024);
    occ = occ < 1 ? 1 : (occ > 4 ? 4 : occ);
    const int tbs = (27 + 128 / KP - 1) / (128 / KP);
    const long nvox = (long)a.nx * a.ny * a.nz;
    const long nchunks = (nvox + WgSmem<KP, NP>::VC - 1) / WgSmem<KP, NP>::VC;
    long splits = ((long)sm_count() * occ + tbs - 1) / tbs;
    splits = std::max<long>(1, std::min<long>(splits, nchunks));
    a.chunks_per_cta = (nchunks + splits - 1) / splits;
    splits = (nchunks + a.chunks_per_cta - 1) / a.chunks_per_cta;
    k_conv_wgrad<KP, NP><<<dim3(tbs, (unsigned)splits), kConvThreads, bytes, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_wgrad(int KP, int NP, const WgradArgs &a, cudaStream_t s) {
    if (KP == 16 && NP == 16) return launch_wgrad_t<16, 16>(a, s);
    if (KP == 16 && NP == 32) return launch_wgrad_t<16, 32>(a, s);
    if (KP == 32 && NP == 16) return launch_wgrad_t<32, 16>(a, s);
    if (KP == 32 && NP == 32) return launch_wgrad_t<32, 32>(a, s);
    return cudaErrorInvalidValue;
}

int grid1d(long n, int threads) {
    long b = (n + threads - 1) / threads;
    const long cap = (long)sm_count() * 8;
    if (b > cap) b = cap;
    return (int)(b < 1 ? 1 : b);
}

bool device_ok(int dev) {
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, dev) != cudaSuccess) return false;
    return p.major == 10;
}

}  // namespace
}  // namespace xr

using namespace xr;

/* ---------------------------------------------------------------------- */
/* Network                                                                 */
/* ---------------------------------------------------------------------- */

struct XrLayer {
    int cin, cout, KP, NP;
    size_t w_off, b_off;    /* offsets into the flat parameter vector */
    bf16 *wk = nullptr, *wd = nullptr;
};

struct xr_net {
    int device = 0;
    cudaStream_t stream = nullptr;
    int K = 0, width = 0, depth = 0;
    std::vector<XrLayer> layers;
    size_t n_params = 0;
    float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;   /* device FP32 */
    float *dwpad = nullptr;                                          /* 27*32*32    */
    int adam_t = 0;
    bool packed = false;
    long cap = 0;                       /* voxels the buffers hold */
    bf16 *in0 = nullptr;                /* [cap][16]               */
    std::vector<bf16 *> act;            /* depth-1 x [cap][NP]     */
    std::vector<bf16 *> grd;            /* depth x [cap][NP]       */
    float *pred = nullptr;              /* [K][cap] FP32           */
    double *loss = nullptr;
    int *err = nullptr;
    std::string msg;
};

namespace {

xr_status net_fail(xr_net *n, xr_status st, const std::string &m) {
    if (n) n->msg = m;
    return st;
}

xr_status net_cuda(xr_net *n, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return XR_OK;
    return net_fail(n, e == cudaErrorMemoryAllocation ? XR_ERR_OOM : XR_ERR_CUDA,
                    std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename T>
cudaError_t dalloc(T **p, size_t count) {
    return cudaMalloc((void **)p, count * sizeof(T));
}

void free_buffers(xr_net *n) {
    cudaFree(n->in0);
    n->in0 = nullptr;
    for (auto *a : n->act) cudaFree(a);
    for (auto *a : n->grd) cudaFree(a);
    n->act.clear();
    n->grd.clear();
    cudaFree(n->pred);
    n->pred = nullptr;
    n->cap = 0;
}

xr_status ensure_buffers(xr_net *n, long nvox, bool training) {
    const bool need_grad = training && n->grd.empty();
    if (nvox <= n->cap && !need_grad) return XR_OK;
    cudaStreamSynchronize(n->stream);
    const bool had_grad = !n->grd.empty();
    free_buffers(n);
    const long cap = nvox;
    xr_status st;
    if ((st = net_cuda(n, dalloc(&n->in0, (size_t)cap * 16), "alloc"))) return st;
    for (int l = 0; l + 1 < n->depth; l++) {
        bf16 *a = nullptr;
        if ((st = net_cuda(n, dalloc(&a, (size_t)cap * n->layers[l].NP), "alloc"))) return st;
        n->act.push_back(a);
    }
    if (training || had_grad) {
        for (int l = 0; l < n->depth; l++) {
            bf16 *a = nullptr;
            if ((st = net_cuda(n, dalloc(&a, (size_t)cap * n->layers[l].NP), "alloc"))) return st;
            n->grd.push_back(a);
        }
        if ((st = net_cuda(n, dalloc(&n->pred, (size_t)cap * n->K), "alloc"))) return st;
    }
    n->cap = cap;
    return XR_OK;
}

xr_status pack_weights(xr_net *n) {
    if (n->packed) return XR_OK;
    for (auto &L : n->layers) {
        k_pack_w<<<grid1d(27 * L.NP * L.KP, 256), 256, 0, n->stream>>>(n->p + L.w_off, L.cin, L.cout, L.KP, L.NP,
                                                                       L.wk, L.wd);
        xr_status st = net_cuda(n, cudaGetLastError(), "pack weights");
        if (st) return st;
    }
    n->packed = true;
    return XR_OK;
}

xr_status check_err(xr_net *n) {
    int e = 0;
    xr_status st = net_cuda(n, cudaMemcpyAsync(&e, n->err, sizeof(int), cudaMemcpyDeviceToHost, n->stream), "flag");
    if (st) return st;
    if ((st = net_cuda(n, cudaStreamSynchronize(n->stream), "sync"))) return st;
    if (e) {
        cudaMemsetAsync(n->err, 0, sizeof(int), n->stream);
        return net_fail(n, XR_ERR_TIMEOUT, "tensor-core pipeline wait timed out");
    }
    return XR_OK;
}

/* hidden layers on in0 (already packed); the last layer's epilogue writes
 * res + net/s into `out` (planar) */
xr_status run_forward(xr_net *n, long nvox, int nx, int ny, int nz, const void *res, void *out, int storage,
                      float in_scale, float floor_value) {
    xr_status st;
    const bf16 *cur = n->in0;
    for (int l = 0; l < n->depth; l++) {
        const XrLayer &L = n->layers[l];
        ConvArgs a{};
        a.x = cur;
        a.w = L.wk;
        a.bias = n->p + L.b_off;
        a.nx = nx; a.ny = ny; a.nz = nz;
        a.err = n->err;
        int epi;
        if (l + 1 < n->depth) {
            a.y = n->act[l];
            epi = EPI_RELU;
        } else {
            a.res = res;
            a.out = out;
            a.storage = storage;
            a.nout = n->K;
            a.inv_scale = 1.0f / in_scale;
            a.floor_value = floor_value;
            epi = EPI_RESID;
        }
        if ((st = net_cuda(n, launch_fwd(L.KP, L.NP, epi, a, n->stream), "conv fprop"))) return st;
        if (l + 1 < n->depth) cur = n->act[l];
    }
    (void)nvox;
    return XR_OK;
}

}  // namespace

extern "C" {

xr_status xr_net_create(int device, int channels, int width, int depth, unsigned long long seed, xr_net **out) {
    if (!out) return XR_ERR_ARG;
    *out = nullptr;
    if (channels < 1 || channels > 16 || (width != 16 && width != 32) || depth < 2 || depth > 16) return XR_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev || !device_ok(device))
        return XR_ERR_NODEV;
    cudaSetDevice(device);
    xr_net *n = new xr_net();
    n->device = device;
    n->K = channels;
    n->width = width;
    n->depth = depth;
    size_t off = 0;
    for (int l = 0; l < depth; l++) {
        XrLayer L;
        L.cin = (l == 0) ? channels : width;
        L.cout = (l + 1 == depth) ? channels : width;
        L.KP = (l == 0) ? 16 : width;
        L.NP = (l + 1 == depth) ? 16 : width;
        L.w_off = off;
        off += (size_t)27 * L.cin * L.cout;
        L.b_off = off;
        off += L.cout;
        n->layers.push_back(L);
    }
    n->n_params = off;
    std::vector<float> h(off, 0.f);
    std::mt19937_64 rng(seed);
    for (int l = 0; l < depth; l++) {
        const XrLayer &L = n->layers[l];
        std::normal_distribution<float> nd(0.f, std::sqrt(2.0f / (27.0f * L.cin)) * (l + 1 == depth ? 0.1f : 1.0f));
        for (size_t i = 0; i < (size_t)27 * L.cin * L.cout; i++) h[L.w_off + i] = nd(rng);
    }
    xr_status st = XR_OK;
    if (!st) st = net_cuda(n, dalloc(&n->p, off), "alloc");
    if (!st) st = net_cuda(n, dalloc(&n->g, off), "alloc");
    if (!st) st = net_cuda(n, dalloc(&n->m, off), "alloc");
    if (!st) st = net_cuda(n, dalloc(&n->v, off), "alloc");
    if (!st) st = net_cuda(n, dalloc(&n->dwpad, (size_t)27 * 32 * 32), "alloc");
    if (!st) st = net_cuda(n, dalloc(&n->loss, 1), "alloc");
    if (!st) st = net_cuda(n, dalloc(&n->err, 1), "alloc");
    for (auto &L : n->layers) {
        if (!st) st = net_cuda(n, dalloc(&L.wk, (size_t)27 * L.NP * L.KP), "alloc");
        if (!st) st = net_cuda(n, dalloc(&L.wd, (size_t)27 * L.NP * L.KP), "alloc");
    }
    if (!st) st = net_cuda(n, cudaMemcpy(n->p, h.data(), off * sizeof(float), cudaMemcpyHostToDevice), "upload");
    if (!st) st = net_cuda(n, cudaMemset(n->m, 0, off * sizeof(float)), "memset");
    if (!st) st = net_cuda(n, cudaMemset(n->v, 0, off * sizeof(float)), "memset");
    if (!st) st = net_cuda(n, cudaMemset(n->err, 0, sizeof(int)), "memset");
    if (st) {
        xr_net_destroy(n);
        return st;
    }
    *out = n;
    return XR_OK;
}

void xr_net_destroy(xr_net *n) {
    if (!n) return;
    cudaSetDevice(n->device);
    if (n->stream) cudaStreamSynchronize(n->stream);
    else cudaDeviceSynchronize();
    free_buffers(n);
    for (auto &L : n->layers) {
        cudaFree(L.wk);
        cudaFree(L.wd);
    }
    cudaFree(n->p);
    cudaFree(n->g);
    cudaFree(n->m);
    cudaFree(n->v);
    cudaFree(n->dwpad);
    cudaFree(n->loss);
    cudaFree(n->err);
    delete n;
}

const char *xr_net_last_error(const xr_net *n) { return n ? n->msg.c_str() : "null network"; }

xr_status xr_net_set_stream(xr_net *n, void *stream) {
    if (!n) return XR_ERR_ARG;
    n->stream = (cudaStream_t)stream;
    return XR_OK;
}

size_t xr_net_num_params(const xr_net *n) { return n ? n->n_params : 0; }

xr_status xr_net_get_params(xr_net *n, float *host, size_t count) {
    if (!n || !host || count != n->n_params) return n ? net_fail(n, XR_ERR_ARG, "parameter count") : XR_ERR_ARG;
    cudaSetDevice(n->device);
    xr_status st = net_cuda(n, cudaMemcpyAsync(host, n->p, count * sizeof(float), cudaMemcpyDeviceToHost, n->stream),
                            "download");
    if (st) return st;
    return net_cuda(n, cudaStreamSynchronize(n->stream), "sync");
}

xr_status xr_net_set_params(xr_net *n, const float *host, size_t count) {
    if (!n || !host || count != n->n_params) return n ? net_fail(n, XR_ERR_ARG, "parameter count") : XR_ERR_ARG;
    cudaSetDevice(n->device);
    xr_status st = net_cuda(n, cudaMemcpyAsync(n->p, host, count * sizeof(float), cudaMemcpyHostToDevice, n->stream),
                            "upload");
    if (st) return st;
    n->packed = false;
    return net_cuda(n, cudaStreamSynchronize(n->stream), "sync");
}

xr_status xr_net_save(xr_net *n, const char *path) {
    if (!n || !path) return XR_ERR_ARG;
    std::vector<float> h(n->n_params);
    xr_status st = xr_net_get_params(n, h.data(), h.size());
    if (st) return st;
    FILE *f = std::fopen(path, "wb");
    if (!f) return net_fail(n, XR_ERR_IO, std::string("cannot write ") + path);
    const char magic[8] = {'X', 'R', 'N', 'E', 'T', '1', 0, 0};
    const int32_t hdr[3] = {n->K, n->width, n->depth};
    bool ok = std::fwrite(magic, 1, 8, f) == 8 && std::fwrite(hdr, 4, 3, f) == 3 &&
              std::fwrite(h.data(), 4, h.size(), f) == h.size();
    ok = (std::fclose(f) == 0) && ok;
    return ok ? XR_OK : net_fail(n, XR_ERR_IO, std::string("short write ") + path);
}

xr_status xr_net_load(xr_net *n, const char *path) {
    if (!n || !path) return XR_ERR_ARG;
    FILE *f = std::fopen(path, "rb");
    if (!f) return net_fail(n, XR_ERR_IO, std::string("cannot read ") + path);
    char magic[8];
    int32_t hdr[3];
    std::vector<float> h(n->n_params);
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "XRNET1", 6) == 0 &&
              std::fread(hdr, 4, 3, f) == 3;
    if (ok && (hdr[0] != n->K || hdr[1] != n->width || hdr[2] != n->depth)) {
        std::fclose(f);
        return net_fail(n, XR_ERR_CONFIG, "network shape in file differs");
    }
    ok = ok && std::fread(h.data(), 4, h.size(), f) == h.size();
    std::fclose(f);
    if (!ok) return net_fail(n, XR_ERR_IO, std::string("bad network file ") + path);
    return xr_net_set_params(n, h.data(), h.size());
}

xr_status xr_net_infer(xr_net *n, const void *d_in, void *d_out, int storage, int nx, int ny, int nz, float in_scale,
                       float floor_value) {
    if (!n) return XR_ERR_ARG;
    if (!d_in || !d_out || nx < 1 || ny < 1 || nz < 1 || storage < 0 || storage > 2 || !(in_scale > 0.f))
        return net_fail(n, XR_ERR_ARG, "bad arguments");
    cudaSetDevice(n->device);
    const long nvox = (long)nx * ny * nz;
    xr_status st;
    if ((st = ensure_buffers(n, nvox, false))) return st;
    if ((st = pack_weights(n))) return st;
    if (storage == kBF16)
        k_pack_in<<<grid1d(nvox, 256), 256, 0, n->stream>>>((const __nv_bfloat16 *)d_in, n->K, nvox, in_scale, n->in0);
    else if (storage == kF16)
        k_pack_in<<<grid1d(nvox, 256), 256, 0, n->stream>>>((const __half *)d_in, n->K, nvox, in_scale, n->in0);
    else
        k_pack_in<<<grid1d(nvox, 256), 256, 0, n->stream>>>((const float *)d_in, n->K, nvox, in_scale, n->in0);
    if ((st = net_cuda(n, cudaGetLastError(), "pack"))) return st;
    if ((st = run_forward(n, nvox, nx, ny, nz, d_in, d_out, storage, in_scale, floor_value))) return st;
    return check_err(n);
}

xr_status xr_net_loss_grad(xr_net *n, const float *d_in, const float *d_target, int nx, int ny, int nz, float in_scale,
                           double *loss, float *host_grad) {
    if (!n) return XR_ERR_ARG;
    if (!d_in || !d_target || nx < 1 || ny < 1 || nz < 1 || !(in_scale > 0.f))
        return net_fail(n, XR_ERR_ARG, "bad arguments");
    cudaSetDevice(n->device);
    const long nvox = (long)nx * ny * nz;
    xr_status st;
    if ((st = ensure_buffers(n, nvox, true))) return st;
    if ((st = pack_weights(n))) return st;
    cudaStream_t s = n->stream;
    k_pack_in<<<grid1d(nvox, 256), 256, 0, s>>>(d_in, n->K, nvox, in_scale, n->in0);
    if ((st = net_cuda(n, cudaGetLastError(), "pack"))) return st;
    if ((st = run_forward(n, nvox, nx, ny, nz, d_in, n->pred, kF32, in_scale, -INFINITY))) return st;
    cudaMemsetAsync(n->loss, 0, sizeof(double), s);
    cudaMemsetAsync(n->g, 0, n->n_params * sizeof(float), s);
    const int D = n->depth;
    /* dL/d(last conv) = 2 (y - t) / (K nvox) / s */
    k_loss_grad<<<grid1d(nvox, 256), 256, 0, s>>>(n->pred, d_target, n->K, nvox,
                                                  2.0f / ((float)n->K * (float)nvox) / in_scale, n->grd[D - 1], n->loss);
    if ((st = net_cuda(n, cudaGetLastError(), "loss"))) return st;
    for (int l = D - 1; l >= 0; l--) {
        const XrLayer &L = n->layers[l];
        const bf16 *xin = (l == 0) ? n->in0 : n->act[l - 1];
        cudaMemsetAsync(n->dwpad, 0, (size_t)27 * 32 * 32 * sizeof(float), s);
        WgradArgs w{};
        w.x = xin;
        w.dy = n->grd[l];
        w.dw = n->dwpad;
        w.nx = nx; w.ny = ny; w.nz = nz;
        w.err = n->err;
        if ((st = net_cuda(n, launch_wgrad(L.KP, L.NP, w, s), "conv wgrad"))) return st;
        k_unpack_dw<<<grid1d(27 * L.cin * L.cout, 256), 256, 0, s>>>(n->dwpad, L.cin, L.cout, L.KP, L.NP,
                                                                     n->g + L.w_off);
        if (L.NP == 16) k_bias_grad<16><<<grid1d(nvox, 256), 256, 0, s>>>(n->grd[l], nvox, L.cout, n->g + L.b_off);
        else k_bias_grad<32><<<grid1d(nvox, 256), 256, 0, s>>>(n->grd[l], nvox, L.cout, n->g + L.b_off);
        if ((st = net_cuda(n, cudaGetLastError(), "bias grad"))) return st;
        if (l > 0) {   /* dgrad into the previous activation, masked by its ReLU */
            ConvArgs a{};
            a.x = n->grd[l];
            a.w = L.wd;
            a.mask = n->act[l - 1];
            a.y = n->grd[l - 1];
            a.nx = nx; a.ny = ny; a.nz = nz;
            a.err = n->err;
            if ((st = net_cuda(n, launch_fwd(L.NP, L.KP, EPI_MASK, a, s), "conv dgrad"))) return st;
        }
    }
    double h_loss = 0.0;
    if ((st = net_cuda(n, cudaMemcpyAsync(&h_loss, n->loss, sizeof(double), cudaMemcpyDeviceToHost, s), "loss"))) return st;
    if (host_grad &&
        (st = net_cuda(n, cudaMemcpyAsync(host_grad, n->g, n->n_params * sizeof(float), cudaMemcpyDeviceToHost, s),
                       "grad")))
        return st;
    if ((st = check_err(n))) return st;
    if (loss) *loss = h_loss / ((double)n->K * (double)nvox);
    return XR_OK;
}

xr_status xr_net_adam_step(xr_net *n, float lr, float beta1, float beta2, float eps) {
    if (!n) return XR_ERR_ARG;
    cudaSetDevice(n->device);
    n->adam_t++;
    const float c1 = 1.0f / (1.0f - std::pow(beta1, (float)n->adam_t));
    const float c2 = 1.0f / (1.0f - std::pow(beta2, (float)n->adam_t));
    k_adam<<<grid1d((long)n->n_params, 256), 256, 0, n->stream>>>(n->p, n->g, n->m, n->v, (long)n->n_params, lr, beta1,
                                                                  beta2, eps, c1, c2);
    n->packed = false;
    return net_cuda(n, cudaGetLastError(), "adam");
}

static xr_status conv_shape_ok(int c) { return (c == 16 || c == 32) ? XR_OK : XR_ERR_ARG; }

xr_status xr_conv3d_fprop(void *stream, const uint16_t *x, int cin, const uint16_t *w, const float *bias,
                          const uint16_t *mask, uint16_t *y, int cout, int nx, int ny, int nz, int epilogue) {
    if (conv_shape_ok(cin) || conv_shape_ok(cout) || !x || !w || !y || nx < 1 || ny < 1 || nz < 1 || epilogue < 0 ||
        epilogue > 2 || (epilogue == EPI_MASK && !mask))
        return XR_ERR_ARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || !device_ok(dev)) return XR_ERR_NODEV;
    int *err = nullptr;
    if (cudaMalloc(&err, sizeof(int)) != cudaSuccess) return XR_ERR_OOM;
    cudaStream_t s = (cudaStream_t)stream;
    cudaMemsetAsync(err, 0, sizeof(int), s);
    ConvArgs a{};
    a.x = (const bf16 *)x;
    a.w = (const bf16 *)w;
    a.bias = bias;
    a.mask = (const bf16 *)mask;
    a.y = (bf16 *)y;
    a.nx = nx; a.ny = ny; a.nz = nz;
    a.err = err;
    cudaError_t e = launch_fwd(cin, cout, epilogue, a, s);
    int h = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(err);
    if (e != cudaSuccess) return XR_ERR_CUDA;
    return h ? XR_ERR_TIMEOUT : XR_OK;
}

xr_status xr_dev_fiber_phantom(void *stream, int N, int K, const float *basis, int n_fib, const float *fibers,
                               float *d_out) {
    if (N < 1 || K < 1 || K > 16 || n_fib < 0 || n_fib > kMaxFibers || !basis || (n_fib && !fibers) || !d_out)
        return XR_ERR_ARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || !device_ok(dev)) return XR_ERR_NODEV;
    PhantomArgs a{};
    a.N = N;
    a.K = K;
    a.n_fib = n_fib;
    for (int f = 0; f < n_fib; f++) {
        for (int j = 0; j < 7; j++) a.fib[f][j] = fibers[7 * f + j];
        const double fx = fibers[7 * f], fy = fibers[7 * f + 1], fz = fibers[7 * f + 2];
        for (int k = 0; k < K; k++) {
            const double sx = basis[3 * k], sy = basis[3 * k + 1], sz = basis[3 * k + 2];
            const double cx = sy * fz - sz * fy, cy = sz * fx - sx * fz, cz = sx * fy - sy * fx;
            a.eta[f][k] = (float)(cx * cx + cy * cy + cz * cz);
        }
    }
    const long n3 = (long)N * N * N;
    k_fiber_phantom<<<grid1d(n3, 256), 256, 0, (cudaStream_t)stream>>>(a, d_out);
    return cudaGetLastError() == cudaSuccess ? XR_OK : XR_ERR_CUDA;
}

xr_status xr_conv3d_wgrad(void *stream, const uint16_t *x, int cin, const uint16_t *dy, int cout, float *dw, int nx,
                          int ny, int nz) {
    if (conv_shape_ok(cin) || conv_shape_ok(cout) || !x || !dy || !dw || nx < 1 || ny < 1 || nz < 1) return XR_ERR_ARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || !device_ok(dev)) return XR_ERR_NODEV;
    int *err = nullptr;
    if (cudaMalloc(&err, sizeof(int)) != cudaSuccess) return XR_ERR_OOM;
    cudaStream_t s = (cudaStream_t)stream;
    cudaMemsetAsync(err, 0, sizeof(int), s);
    WgradArgs a{};
    a.x = (const bf16 *)x;
    a.dy = (const bf16 *)dy;
    a.dw = dw;
    a.nx = nx; a.ny = ny; a.nz = nz;
    a.err = err;
    cudaError_t e = launch_wgrad(cin, cout, a, s);
    int h = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(err);
    if (e != cudaSuccess) return XR_ERR_CUDA;
    return h ? XR_ERR_TIMEOUT : XR_OK;
}

}  // extern "C"
