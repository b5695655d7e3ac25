/*
 * Two-word fixed-point detector tiles for the forward splats.
 *
 * A 32-bit integer atomicAdd on shared memory is a native instruction, a
 * float (or 64-bit) one runs as a compare-and-swap loop.  Each contribution
 * x, scaled by the CTA's power of two (xs = x * 2^sh, |xs| < 2^19), is split
 * into an integer part h = rint(xs) and a remainder r = xs - h (exact, Sterbenz)
 * kept to 2^-20 in a second word: two native atomics per tap, each term of a
 * per-CTA sum exact to 2^-39 of the CTA's largest contribution, i.e. below the
 * FP32 rounding of every pixel the reference itself accumulates.  With at most
 * 2048 contributions per pixel (one tap per voxel of a brick) both words stay
 * below 2^30.  A pixel's relative precision matters: the normalised projection
 * divides by the weight image, so footprint-edge pixels with small sums are
 * amplified to the scale of the largest ones.
 */
#ifndef XR_TILE_CUH
#define XR_TILE_CUH

namespace xr {

constexpr float kFixLoScale = 1048576.0f;           /* 2^20  */
constexpr float kFixLoInvF = 9.5367431640625e-07f;  /* 2^-20 */

/* Rounding to the nearest integer (ties to even) without the conversion
 * unit: for |x| < 2^22, t = x + 1.5 * 2^23 lies in [2^23, 2^24), where the
 * float spacing is 1, so the addition itself rounds x, and t's bit pattern
 * minus that of 1.5 * 2^23 is the integer (the magic-number method). */
constexpr float kRoundMagic = 12582912.0f;          /* 1.5 * 2^23 */
constexpr int kRoundMagicBits = 0x4B400000;

/* The two words of one contribution |xs| < 2^19: h = rint(xs) and
 * l = rint((xs - h) * 2^20), as integers. */
__device__ __forceinline__ void fix_split(float xs, int &h, int &l) {
    const float t = __fadd_rn(xs, kRoundMagic);
    const float hf = __fsub_rn(t, kRoundMagic);
    h = __float_as_int(t) - kRoundMagicBits;
    /* (xs - hf) is exact and so is its product with 2^20: one rounding */
    l = __float_as_int(__fmaf_rn(__fsub_rn(xs, hf), kFixLoScale, kRoundMagic)) - kRoundMagicBits;
}

/* fix_split of two contributions at once (packed FP32x2 arithmetic on
 * sm_100, each lane rounded exactly as the scalar form). */
__device__ __forceinline__ void fix_split2(float2 xs, int2 &h, int2 &l) {
    const float2 t = __fadd2_rn(xs, make_float2(kRoundMagic, kRoundMagic));
    const float2 hf = __fadd2_rn(t, make_float2(-kRoundMagic, -kRoundMagic));
    h = make_int2(__float_as_int(t.x) - kRoundMagicBits, __float_as_int(t.y) - kRoundMagicBits);
    /* xs - hf (exact) as fma(hf, -1, xs), then one rounding of its 2^20 multiple */
    const float2 r = __ffma2_rn(hf, make_float2(-1.0f, -1.0f), xs);
    const float2 lt = __ffma2_rn(r, make_float2(kFixLoScale, kFixLoScale), make_float2(kRoundMagic, kRoundMagic));
    l = make_int2(__float_as_int(lt.x) - kRoundMagicBits, __float_as_int(lt.y) - kRoundMagicBits);
}

/* tile word layout per buffer: [hi: cap ints][lo: cap ints] */
__device__ __forceinline__ void fix_add(int *hi, int cap, float xs) {
    int h, l;
    fix_split(xs, h, l);
    atomicAdd(hi, h);
    atomicAdd(hi + cap, l);
}

/* Reads and clears one pixel's two words; returns the sum unscaled by 2^-sh. */
__device__ __forceinline__ bool fix_take(int *hi, int cap, float finv, float &out) {
    const int h = *hi, l = hi[cap];
    if ((h | l) == 0) return false;
    *hi = 0;
    hi[cap] = 0;
    out = __fmul_rn(__fmaf_rn((float)l, kFixLoInvF, (float)h), finv);
    return true;
}

/* Power-of-two scale for a CTA whose contributions are bounded by S > 0. */
__device__ __forceinline__ int fix_shift(float S) {
    int ex;
    frexpf(S, &ex);          /* S < 2^ex */
    return max(-126, min(126, 19 - ex));
}

}  // namespace xr

#endif
