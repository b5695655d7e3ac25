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
 *  k_conv_ws (fprop and dgrad): M = 128 voxels (an 8 x 16 patch of one
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
#include <cuda.h>
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

/* What the epilogue of one voxel reads from global memory, fetched before
 * its accumulators are ready: the residual input (EPI_RESID; it may be the
 * output itself, each element read by the thread that then writes it) or
 * the ReLU mask (EPI_MASK). */
template <int NP, int EPI>
struct EpiIn {
    float r[EPI == EPI_RESID ? NP : 1];
    uint4 m[EPI == EPI_MASK ? NP / 8 : 1];
};

template <int NP, int EPI>
__device__ __forceinline__ void epi_fetch(const ConvArgs &a, long v, long nvox, EpiIn<NP, EPI> &in) {
    if (EPI == EPI_RESID) {
#pragma unroll
        for (int n = 0; n < NP; n++) {
            const size_t i = (size_t)n * nvox + v;
            float r = 0.f;
            if (n < a.nout) {
                if (a.storage == kBF16) r = ldf(reinterpret_cast<const __nv_bfloat16 *>(a.res) + i);
                else if (a.storage == kF16) r = ldf(reinterpret_cast<const __half *>(a.res) + i);
                else r = ldf(reinterpret_cast<const float *>(a.res) + i);
            }
            in.r[n] = r;
        }
    } else if (EPI == EPI_MASK) {
        const uint4 *mk = reinterpret_cast<const uint4 *>(a.mask + (size_t)v * NP);
#pragma unroll
        for (int j = 0; j < NP / 8; j++) in.m[j] = __ldg(mk + j);
    }
}

/* Output of one voxel's NP accumulators (row of the M = 128 tile); `bias`
 * holds NP values (zeros when the layer has none). */
template <int NP, int EPI>
__device__ __forceinline__ void conv_epilogue(const ConvArgs &a, const float *bias, long v, long nvox,
                                              const float *acc, const EpiIn<NP, EPI> &in) {
    if (EPI == EPI_RESID) {
#pragma unroll
        for (int n = 0; n < NP; n++) {
            if (n >= a.nout) break;
            const size_t i = (size_t)n * nvox + v;
            const float val = fmaxf(in.r[n] + (acc[n] + bias[n]) * a.inv_scale, a.floor_value);
            if (a.storage == kBF16) stf(reinterpret_cast<__nv_bfloat16 *>(a.out) + i, val);
            else if (a.storage == kF16) stf(reinterpret_cast<__half *>(a.out) + i, val);
            else stf(reinterpret_cast<float *>(a.out) + i, val);
        }
    } else {
        uint4 *yo = reinterpret_cast<uint4 *>(a.y + (size_t)v * NP);
#pragma unroll
        for (int j = 0; j < NP / 8; j++) {
            float o[8];
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int n = 8 * j + i;
                o[i] = acc[n];
                if (EPI != EPI_MASK) o[i] += bias[n];
                if (EPI == EPI_RELU) o[i] = fmaxf(o[i], 0.f);
            }
            if (EPI == EPI_MASK) {
                const uint32_t mw[4] = {in.m[j].x, in.m[j].y, in.m[j].z, in.m[j].w};
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
/* apart (SBO), planes kPlane bytes apart (LBO) - the descriptor's start   */
/* address moves by (dy * 10 + dx) * 16 bytes.                             */
/*                                                                         */
/* Each input slice is read once and feeds three output slices: the three  */
/* dz taps of one (dy, dx) are stacked along N (the weights of tap         */
/* (dz, dy, dx) sit at block dz of group dy * 3 + dx), so one MMA with     */
/* N = 3 x NP multiplies the window by all three and adds into the         */
/* accumulators of output slices z + 1, z and z - 1 at once.  Those live   */
/* in a ring of tensor-memory blocks of NP columns whose position falls as */
/* the output index rises (block CR - 1 - o % CR), so the three are        */
/* adjacent columns in the order of the stacked weights; at the ring's     */
/* wrap the MMA is split per block.  An input slice costs 9 x KP/16 MMAs   */
/* and its window bytes are read from shared memory once instead of three  */
/* times.  A slice's first MMA overwrites (accumulate = 0) the blocks of   */
/* the output slices it starts.                                            */
/*                                                                         */
/* The CTA is warp-specialised, with no CTA-wide barrier in the loop:      */
/* warp 5 (one thread) loads halo slices with tensor-map copies (zero fill */
/* outside the volume) into a ring of R slots, warp 4 (one thread) issues  */
/* the MMAs, warps 0-3 read the accumulators out and run the epilogue.     */
/* They hand off through mbarriers:                                        */
/*   full[s]   slot s holds its slice    (copy transaction bytes)          */
/*   empty[s]  slot s may be refilled    (MMA commit)                      */
/*   acc[p]    ring block p complete     (MMA commit)                      */
/*   free[p]   ring block p read out     (128 epilogue arrivals)           */
/* Every CTA walks the same static item sequence (an xy tile and a range   */
/* of z); slice and output counters run on across items, which fixes each  */
/* barrier's phase.  Input slices outside the volume are not loaded and    */
/* issue no MMAs.                                                          */
/* ---------------------------------------------------------------------- */
constexpr int kHX = 10, kHY = 18, kHV = kHX * kHY;   /* halo slice: 180 voxels   */
constexpr int kPlane = 2944;                         /* 2880 bytes, 128-aligned */
constexpr int kConvWsThreads = 192;
constexpr int kConvSmemBudget = 115712;              /* two CTAs per SM          */
constexpr int kConvTmemCols = 256;

template <int KP, int NP>
struct ConvSmem {
    static constexpr int BT = NP * KP * 2;                        /* one tap's weights  */
    static constexpr int BB = ((27 * BT + 1023) / 1024) * 1024;
    static constexpr int SLOT = (KP / 8) * kPlane;
    static constexpr int CR = kConvTmemCols / NP;                 /* accumulator ring   */
    static constexpr int RR = (kConvSmemBudget - 1024 - BB - 8 * (2 * CR + 1) - 16) / (SLOT + 16);
    static constexpr int R = RR > 16 ? 16 : RR;                   /* halo-slice ring    */
    static constexpr int NBAR = 2 * R + 2 * CR + 1;               /* full, empty, acc, free, drain */
    static constexpr int bytes = 1024 + BB + R * SLOT + NBAR * 8 + 16;
    static constexpr uint32_t TX = (KP / 8) * kHV * 16;           /* bytes per slice    */
    static_assert(R >= 3, "halo ring too shallow");
    static_assert(bytes <= kConvSmemBudget, "shared memory over budget");
    static_assert(3 * (bytes + 1024) > 233472, "a third CTA per SM would exceed tensor memory");
};

template <int KP, int NP, int EPI>
__global__ void __launch_bounds__(kConvWsThreads) k_conv_ws(const __grid_constant__ CUtensorMap xmap, ConvArgs a,
                                                            int zchunk) {
    using L = ConvSmem<KP, NP>;
    constexpr int R = L::R, CR = L::CR;
    constexpr uint32_t SBO_B = (KP / 8) * 128;
    extern __shared__ uint8_t smem_raw[];
    uint8_t *sm = align1k(smem_raw);
    uint8_t *sB = sm, *ring = sm + L::BB;
    uint64_t *full = reinterpret_cast<uint64_t *>(ring + R * L::SLOT);
    uint64_t *empty = full + R, *accb = empty + R, *freeb = accb + CR, *drain = freeb + CR;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(drain + 1);
    __shared__ volatile int s_abort;
    __shared__ float s_bias[NP];

    const int tid = threadIdx.x, warp = tid >> 5;
    if (tid == 0) {
        for (int i = 0; i < R; i++) {
            tc::mbar_init(&full[i], 1);
            tc::mbar_init(&empty[i], 1);
        }
        for (int i = 0; i < CR; i++) {
            tc::mbar_init(&accb[i], 1);
            tc::mbar_init(&freeb[i], 128);
        }
        tc::mbar_init(drain, 1);
        tc::fence_mbar_init();
        s_abort = 0;
    }
    if (tid < NP) s_bias[tid] = (EPI != EPI_MASK && a.bias && (EPI != EPI_RESID || tid < a.nout)) ? a.bias[tid] : 0.f;
    if (warp == 0) tc::tmem_alloc(tslot, kConvTmemCols);
    /* weights of tap t = (dz, dy, dx) at block dz of group dy * 3 + dx */
    for (int c = tid; c < 27 * NP * KP / 8; c += kConvWsThreads) {
        const int j = c % (KP / 8), n = (c / (KP / 8)) % NP, t = c / (NP * KP / 8);
        const int pos = (t % 9) * 3 + t / 9;
        *reinterpret_cast<uint4 *>(sB + pos * L::BT + (n >> 3) * SBO_B + j * 128 + (n & 7) * 16) =
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

    if (warp == 5) {
        /* ---------------- halo loads (one thread) ---------------- */
        if ((tid & 31) == 0) {
            uint32_t gs = 0;
            bool ok = true;
            for (long item = blockIdx.x; item < items && ok; item += gridDim.x) {
                const int tx = (int)(item % ntx), ty = (int)((item / ntx) % nty), tz = (int)(item / ((long)ntx * nty));
                const int z0 = tz * zchunk, nzs = min(zchunk, nz - z0);
                for (int li = -1; li <= nzs && ok; li++, gs++) {
                    const int slot = gs % R;
                    if (gs >= (uint32_t)R &&
                        (s_abort || !tc::mbar_wait(&empty[slot], ((gs / R) - 1) & 1, kWaitCycles))) {
                        ok = false;
                        break;
                    }
                    const int z = z0 + li;
                    if (z >= 0 && z < nz) {
                        tc::mbar_arrive_tx(&full[slot], L::TX);
                        uint8_t *dst = ring + slot * L::SLOT;
#pragma unroll
                        for (int j = 0; j < KP / 8; j++)
                            tc::tma_load_4d(dst + j * kPlane, &xmap, &full[slot], 8 * j, tx * 8 - 1, ty * 16 - 1, z);
                    } else {
                        tc::mbar_arrive(&full[slot]);
                    }
                }
            }
            /* no copy may still be writing when the CTA leaves */
            for (uint32_t g = gs > (uint32_t)R ? gs - R : 0; g < gs; g++)
                if (!tc::mbar_wait(&full[g % R], (g / R) & 1, kWaitCycles)) ok = false;
            if (!ok) s_abort = 1;
        }
    } else if (warp == 4) {
        /* ---------------- MMA issue (one thread) ---------------- */
        if ((tid & 31) == 0) {
            uint32_t gs = 0, ob = 0;   /* slices and outputs so far */
            bool ok = true;
            const uint64_t bS = tc::sdesc(tc::smem_u32(sB), 128, SBO_B);
            for (long item = blockIdx.x; item < items && ok; item += gridDim.x) {
                const int tz = (int)(item / ((long)ntx * nty));
                const int z0 = tz * zchunk, nzs = min(zchunk, nz - z0);
                for (int li = -1; li <= nzs && ok; li++, gs++) {
                    const int slot = gs % R, z = z0 + li;
                    if (s_abort || !tc::mbar_wait(&full[slot], (gs / R) & 1, kWaitCycles)) {
                        ok = false;
                        break;
                    }
                    if (z >= 0 && z < nz) {
                        /* outputs olo..ohi (item-local) take blocks j = li + 1 - o; the ones this
                         * slice starts (no earlier slice inside the volume) are the top nf */
                        const int olo = max(0, li - 1), ohi = min(nzs - 1, li + 1);
                        const int nf = (li + 1 <= nzs - 1) + (li >= 0 && li <= nzs - 1 && z == 0);
                        for (int f = 0; f < nf && ok; f++) {
                            const uint32_t O = ob + (uint32_t)(ohi - f);
                            if (O >= (uint32_t)CR &&
                                (s_abort || !tc::mbar_wait(&freeb[CR - 1 - O % CR], ((O / CR) - 1) & 1, kWaitCycles)))
                                ok = false;
                        }
                        if (!ok) break;
                        tc::fence_after_sync();
                        const uint64_t aS = tc::sdesc(tc::smem_u32(ring + slot * L::SLOT), kPlane, kHX * 16);
                        const int jlo = li + 1 - ohi, jhi = li + 1 - olo;
                        const uint32_t Otop = ob + (uint32_t)ohi;   /* output of block jlo */
                        /* the rest: blocks jlo..jw in one MMA, and jw+1..jhi in a second where the
                         * ring wraps between them */
                        const int jw = min(jhi, jlo + (int)(Otop % CR));
                        const uint32_t dA = tmem + (CR - 1 - Otop % CR) * NP, dB = tmem;
                        const uint64_t bA = bS + (uint64_t)(jlo * (L::BT >> 4)), bB = bS + (uint64_t)((jw + 1) * (L::BT >> 4));
                        const uint32_t iA = tc::idesc_bf16(128, NP * (jw - jlo + 1), 0, 0);
                        const uint32_t iB = tc::idesc_bf16(128, NP * max(1, jhi - jw), 0, 0);
                        /* first MMA of the slice: it overwrites (accumulate = 0) the blocks of the
                         * outputs it starts, the top nf; in one or two MMAs where the blocks are
                         * adjacent, else one per block */
                        if (jw == jhi) {
                            const int nb = jhi - jlo + 1;
                            if (nf > 0) tc::mma_bf16(dA, aS, bA, tc::idesc_bf16(128, NP * nf, 0, 0), 0u);
                            if (nf < nb)
                                tc::mma_bf16(dA + nf * NP, aS, bA + (uint64_t)(nf * (L::BT >> 4)),
                                             tc::idesc_bf16(128, NP * (nb - nf), 0, 0), 1u);
                        } else {
                            for (int j = jlo; j <= jhi; j++) {
                                const uint32_t O = Otop - (uint32_t)(j - jlo);
                                tc::mma_bf16(tmem + (CR - 1 - O % CR) * NP, aS, bS + (uint64_t)(j * (L::BT >> 4)),
                                             tc::idesc_bf16(128, NP, 0, 0), j < jlo + nf ? 0u : 1u);
                            }
                        }
                        if (jw == jhi) {
#pragma unroll
                            for (int m = 1; m < 9 * (KP / 16); m++) {
                                const int g = m / (KP / 16), kk = m % (KP / 16);
                                const uint64_t ao = (uint64_t)((g / 3) * kHX + g % 3 + kk * (2 * kPlane >> 4));
                                const uint64_t bo = (uint64_t)(g * 3 * (L::BT >> 4) + kk * 16);
                                tc::mma_bf16(dA, aS + ao, bA + bo, iA, 1u);
                            }
                        } else {
#pragma unroll
                            for (int m = 1; m < 9 * (KP / 16); m++) {
                                const int g = m / (KP / 16), kk = m % (KP / 16);
                                const uint64_t ao = (uint64_t)((g / 3) * kHX + g % 3 + kk * (2 * kPlane >> 4));
                                const uint64_t bo = (uint64_t)(g * 3 * (L::BT >> 4) + kk * 16);
                                tc::mma_bf16(dA, aS + ao, bA + bo, iA, 1u);
                                tc::mma_bf16(dB, aS + ao, bB + bo, iB, 1u);
                            }
                        }
                        tc::mma_commit(&empty[slot]);
                    } else {
                        tc::mbar_arrive(&empty[slot]);   /* nothing was loaded or read */
                    }
                    if (li >= 1) tc::mma_commit(&accb[CR - 1 - (ob + li - 1) % CR]);   /* output li - 1 complete */
                }
                ob += (uint32_t)nzs;
            }
            if (!ok) s_abort = 1;
            tc::mma_commit(drain);   /* arrives once every MMA issued here has completed */
        }
    } else {
        /* ---------------- epilogue (warps 0-3) ---------------- */
        uint32_t O = 0;
        bool ok = true;
        for (long item = blockIdx.x; item < items && ok; item += gridDim.x) {
            const int tx = (int)(item % ntx), ty = (int)((item / ntx) % nty), tz = (int)(item / ((long)ntx * nty));
            const int z0 = tz * zchunk, nzs = min(zchunk, nz - z0);
            const int ox = tx * 8 + (tid & 7), oy = ty * 16 + (tid >> 3);
            const bool in_tile = ox < nx && oy < ny;
            for (int o = 0; o < nzs; o++, O++) {
                const int p = CR - 1 - (int)(O % CR);
                const long v = (long)ox + (long)nx * (oy + (long)ny * (z0 + o));
                EpiIn<NP, EPI> in;
                if (in_tile) epi_fetch<NP, EPI>(a, v, nvox, in);
                if (s_abort || !tc::mbar_wait(&accb[p], (O / CR) & 1, kWaitCycles)) {
                    ok = false;
                    break;
                }
                tc::fence_after_sync();
                float acc[NP];
                const uint32_t taddr = tmem + p * NP + ((uint32_t)(warp * 32) << 16);
                if (NP == 16) tc::tmem_ld16(taddr, acc);
                else tc::tmem_ld32(taddr, acc);
                tc::fence_before_sync();
                tc::mbar_arrive(&freeb[p]);
                if (in_tile) conv_epilogue<NP, EPI>(a, s_bias, v, nvox, acc, in);
            }
        }
        if (!ok) s_abort = 1;
    }
    /* every MMA complete before the tensor memory is freed */
    if (tid == 0) {
        if (!tc::mbar_wait(drain, 0, kWaitCycles)) s_abort = 1;
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, kConvTmemCols);
    }
    if (s_abort && tid == 0) atomicExch(a.err, 1);
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

/* Orientation term of the training loss.  A voxel's main direction is the
 * smallest-eigenvalue eigenvector of T(mu) = (1/K) sum_k mu_k S_k S_k^T
 * (calcEigenVector on sqrt|mu|, whose squares are mu for mu >= 0), a linear
 * map of the channels: the term weight * ||T(pred) - T(target)||_F^2 (without
 * the 1/K) adds sum_j w_j (sum_k d_k E_kj)^2 per voxel, E_k = (xx, yy, zz, xy,
 * xz, yz) of S_k S_k^T and w = (1, 1, 1, 2, 2, 2) (the off-diagonal pairs). */
struct TensorLoss {
    float weight;        /* 0: plain MSE */
    float E[16][6];
};

/* g[v][c] = bf16(gscale * dL/dpred_c / 2) (zero for c >= K), with d = pred -
 * target and L = sum_c d_c^2 + weight * sum_j w_j dT_j^2, dT_j = sum_c d_c E_cj;
 * loss += L */
__global__ void k_loss_grad(const float *pred, const float *target, int K, long nvox, float gscale, bf16 *g,
                            double *loss, const TensorLoss tl) {
    constexpr float wj[6] = {1.f, 1.f, 1.f, 2.f, 2.f, 2.f};
    double s = 0.0;
    for (long v = (long)blockIdx.x * blockDim.x + threadIdx.x; v < nvox; v += (long)gridDim.x * blockDim.x) {
        float d[16];
#pragma unroll
        for (int c = 0; c < 16; c++) d[c] = (c < K) ? pred[(size_t)c * nvox + v] - target[(size_t)c * nvox + v] : 0.f;
        float f[16];
#pragma unroll
        for (int c = 0; c < 16; c++) {
            s += (double)d[c] * d[c];
            f[c] = d[c];
        }
        if (tl.weight > 0.f) {
#pragma unroll
            for (int j = 0; j < 6; j++) {
                float dt = 0.f;
#pragma unroll
                for (int c = 0; c < 16; c++) dt = fmaf(d[c], tl.E[c][j], dt);
                s += (double)(tl.weight * wj[j]) * dt * dt;
                const float a = tl.weight * wj[j] * dt;
#pragma unroll
                for (int c = 0; c < 16; c++) f[c] = fmaf(a, tl.E[c][j], f[c]);
            }
        }
#pragma unroll
        for (int c = 0; c < 16; c++) f[c] = (c < K) ? gscale * f[c] : 0.f;
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

/* cuTensorMapEncodeTiled through the runtime's driver entry point (no
 * link-time dependency on the driver library). */
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
    static const EncodeTiledFn fn = []() -> EncodeTiledFn {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return nullptr;
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    return fn;
}

/* Tensor map of a channels-last BF16 activation [nz][ny][nx][KP]: boxes of
 * 8 channels x 10 x 18 voxels x 1 slice, i.e. one plane of a halo slice. */
cudaError_t halo_map(const bf16 *x, int KP, int nx, int ny, int nz, CUtensorMap *m) {
    const EncodeTiledFn enc = encode_tiled();
    if (!enc || (reinterpret_cast<uintptr_t>(x) & 15u)) return cudaErrorInvalidValue;
    const cuuint64_t dims[4] = {(cuuint64_t)KP, (cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
    const cuuint64_t strides[3] = {(cuuint64_t)KP * 2, (cuuint64_t)KP * 2 * nx, (cuuint64_t)KP * 2 * nx * ny};
    const cuuint32_t box[4] = {8, kHX, kHY, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16 *>(x), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

/* z-chunk of the work items: the fewest slices on the busiest CTA, counting
 * one slice of overhead per item for its two halo slices. */
long conv_zchunk(long xy, int nz, long grid0) {
    long best = nz, best_cost = -1;
    for (long ntz = 1; ntz <= nz; ntz++) {
        const long zc = (nz + ntz - 1) / ntz;
        if (zc > 64) continue;
        const long items = xy * ((nz + zc - 1) / zc);
        const long cost = ((items + grid0 - 1) / grid0) * (zc + 1);
        if (best_cost < 0 || cost < best_cost) {
            best_cost = cost;
            best = zc;
        }
    }
    return best;
}

template <int KP, int NP, int EPI>
cudaError_t launch_halo_t(const ConvArgs &a, cudaStream_t s) {
    using L = ConvSmem<KP, NP>;
    CUtensorMap map;
    cudaError_t e = halo_map(a.x, KP, a.nx, a.ny, a.nz, &map);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_conv_ws<KP, NP, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, L::bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_conv_ws<KP, NP, EPI>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    /* two CTAs per SM: shared memory and the 2 x 256 tensor-memory columns */
    const long grid0 = (long)sm_count() * 2;
    const long xy = (long)((a.nx + 7) / 8) * ((a.ny + 15) / 16);
    const long zc = conv_zchunk(xy, a.nz, grid0);
    const long items = xy * ((a.nz + zc - 1) / zc);
    const long grid = std::min<long>(items, grid0);
    k_conv_ws<KP, NP, EPI><<<(int)grid, kConvWsThreads, L::bytes, s>>>(map, a, (int)zc);
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
    TensorLoss tloss{};                 /* orientation term of the training loss */
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

xr_status xr_net_set_tensor_loss(xr_net *n, const float *basis, float weight) {
    if (!n) return XR_ERR_ARG;
    if (!(weight >= 0.f) || !std::isfinite(weight)) return net_fail(n, XR_ERR_ARG, "tensor loss weight must be >= 0");
    if (weight > 0.f && !basis) return net_fail(n, XR_ERR_ARG, "tensor loss needs the K basis vectors");
    TensorLoss t{};
    t.weight = weight;
    if (weight > 0.f)
        for (int k = 0; k < n->K; k++) {
            const float x = basis[3 * k], y = basis[3 * k + 1], z = basis[3 * k + 2];
            if (!std::isfinite(x) || !std::isfinite(y) || !std::isfinite(z))
                return net_fail(n, XR_ERR_ARG, "non-finite basis vector");
            const float e[6] = {x * x, y * y, z * z, x * y, x * z, y * z};
            for (int j = 0; j < 6; j++) t.E[k][j] = e[j];
        }
    n->tloss = t;
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
                                                  2.0f / ((float)n->K * (float)nvox) / in_scale, n->grd[D - 1], n->loss,
                                                  n->tloss);
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
