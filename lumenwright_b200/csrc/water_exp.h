/*
 * The exponential of the water's Beer-Lambert transmittance, exp(-sigma * t) (`V3::exp` as
 * `transmittance` uses it, crates/lumenwright-kernel/src/math.rs:300), written once for the CUDA
 * kernels and the CPU oracle so both round it to the same f32, bit for bit.
 *
 * The reference's CPU path calls the platform `expf` (Rust's f32::exp) and its PTX build calls the
 * `libm` crate's expf; CUDA's expf is a third implementation, and a last-place difference between
 * them can flip a later Russian-roulette draw. This function is the project's own, in f32
 * arithmetic with fused multiply-adds (an evaluation in double costs the shading kernel 12 % on a
 * B200, a table-driven one in pairs of floats 9 %; this one under 1 %):
 *
 *   1. Cody and Waite's additive argument reduction (W. J. Cody and W. Waite, "Software Manual for
 *      the Elementary Functions", 1980): x = k ln2 + r with k the integer nearest x / ln2 and
 *      |r| <= ln2 / 2 (plus a rounding), r = (x - k C1) - k C2 with ln 2 = C1 + C2 split into its
 *      nearest float and the nearest float to the rest, each step one fused multiply-add;
 *   2. e^r by its Taylor series to degree 8 with Horner's rule, one fused multiply-add a step (the
 *      next term is below 2^-32 of the result);
 *   3. the scaling by 2^k, in two steps at the ends of the range; exact while the result is normal.
 * Measured over every float of [-87.3365, 0] (the transmittance's arguments with a normal
 * result), it is within one unit in the last place of exp(x) rounded to the nearest float, and
 * equal to it on all but about 0.45 % of them.
 *
 * Every operation is an IEEE f32 add, multiply or fused multiply-add written out as such (the
 * library is built with --fmad=false, the oracle with -ffp-contract=off, so nothing else is fused,
 * and neither compiler reorders floating-point operations), so the host and the device give the
 * same bits.
 */
#ifndef LW_WATER_EXP_H
#define LW_WATER_EXP_H

#include <stdint.h>
#include <string.h>

#ifdef __CUDACC__
#define LW_WEXP_FN __host__ __device__ static inline
#else
#define LW_WEXP_FN static inline
#include <math.h>
#endif

#ifdef __CUDA_ARCH__
#define LW_WEXP_FMA(a, b, c) __fmaf_rn(a, b, c)
#else
#define LW_WEXP_FMA(a, b, c) fmaf(a, b, c)
#endif

LW_WEXP_FN float lw_f32_of_bits(uint32_t u) {
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float f;
    memcpy(&f, &u, sizeof f);
    return f;
#endif
}

/* 2^e for -126 <= e <= 127. */
LW_WEXP_FN float lw_pow2f(int e) { return lw_f32_of_bits((uint32_t)(e + 127) << 23); }

/* exp(x) in f32 (see above). NaN gives NaN, anything below -104 (-inf included) 0, and anything
 * above 88.72283 (+inf included) +inf, as the rounded e^x is there. */
LW_WEXP_FN float lw_water_expf(float x) {
    if (x != x) return x;
    if (x > 88.72283172607421875f) return lw_f32_of_bits(0x7F800000u);
    if (x < -104.0f) return 0.0f;
    const float INV_LN2 = 0x1.715476p+0f;  /* 1 / ln 2, rounded */
    const float C1 = 0x1.62e43p-1f;        /* ln 2, rounded */
    const float C2 = -0x1.05c61p-29f;      /* ln 2 - C1, rounded */
    const float MAGIC = 12582912.0f;       /* 1.5 * 2^23: adding and subtracting it rounds to an integer */
    const float kf = (x * INV_LN2 + MAGIC) - MAGIC;
    float r = LW_WEXP_FMA(-kf, C1, x);
    r = LW_WEXP_FMA(-kf, C2, r);
    /* e^r = sum r^n / n!, n = 0..8 */
    float p = 1.0f / 40320.0f;
    p = LW_WEXP_FMA(r, p, 1.0f / 5040.0f);
    p = LW_WEXP_FMA(r, p, 1.0f / 720.0f);
    p = LW_WEXP_FMA(r, p, 1.0f / 120.0f);
    p = LW_WEXP_FMA(r, p, 1.0f / 24.0f);
    p = LW_WEXP_FMA(r, p, 1.0f / 6.0f);
    p = LW_WEXP_FMA(r, p, 0.5f);
    p = LW_WEXP_FMA(r, p, 1.0f);
    p = LW_WEXP_FMA(r, p, 1.0f);
    const int k = (int)kf; /* -150 .. 128 */
    if (k > 126) return (p * lw_pow2f(k - 1)) * 2.0f;
    if (k >= -126) return p * lw_pow2f(k);
    return (p * lw_pow2f(k + 64)) * lw_pow2f(-64);
}

#endif
