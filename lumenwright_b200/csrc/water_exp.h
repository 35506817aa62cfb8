/*
 * The exponential of the water's Beer-Lambert transmittance, exp(-sigma * t) (`V3::exp` as
 * `transmittance` uses it, crates/lumenwright-kernel/src/math.rs:300), written once for the CUDA
 * kernels and the CPU oracle so both round it to the same f32, bit for bit.
 *
 * The reference's CPU path calls the platform `expf` (Rust's f32::exp) and its PTX build calls the
 * `libm` crate's expf; CUDA's expf is a third implementation, and a last-place difference between
 * them can flip a later Russian-roulette draw. This function is the project's own: it returns
 * exp(x) rounded to the nearest f32, which is what a correctly rounded expf returns, computed as
 *
 *   1. Cody and Waite's additive argument reduction (W. J. Cody and W. Waite, "Software Manual for
 *      the Elementary Functions", 1980): x = k ln2 + r with k = round(x / ln2), |r| <= ln2 / 2
 *      (plus a rounding), ln2 split into a high part with 32 significant bits, so k * ln2_hi and
 *      x - k * ln2_hi are exact for the k that occur here, and a low part;
 *   2. the Taylor series of e^r to degree 13 by Horner's rule (remainder below 2^-57 relative);
 *   3. the scaling by 2^k, exact;
 * all in IEEE double, with one rounding to f32 at the end. The double result is within a few
 * units of 2^-53 relative of e^x, so the f32 result is the correctly rounded one except where e^x
 * lies that close to the midpoint between two floats.
 *
 * Every operation is an IEEE double add, multiply or floor, with no fused multiply-add (the
 * library is built with --fmad=false, the oracle with -ffp-contract=off), so the host and the
 * device give the same bits.
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

/* 2^k as a double, for -1022 <= k <= 1023. */
LW_WEXP_FN double lw_pow2i(int k) {
    uint64_t bits = (uint64_t)(int64_t)(k + 1023) << 52;
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)bits);
#else
    double d;
    memcpy(&d, &bits, sizeof d);
    return d;
#endif
}

/* exp(x) rounded to f32. NaN gives NaN, -inf 0, +inf +inf; below -150 the result is 0 and above
 * 100 +inf, as the rounded e^x is there. */
LW_WEXP_FN float lw_water_expf(float x) {
    if (x != x) return x;
    double xd = (double)x;
    xd = xd < -150.0 ? -150.0 : (xd > 100.0 ? 100.0 : xd);
    const double LN2_HI = 6.93147180369123816490e-01; /* ln 2 to 32 significant bits */
    const double LN2_LO = 1.90821492927058770002e-10; /* ln 2 - LN2_HI */
    const double INV_LN2 = 1.44269504088896338700e+00;
    double kd = floor(xd * INV_LN2 + 0.5);
    int k = (int)kd;
    double r = (xd - kd * LN2_HI) - kd * LN2_LO;
    /* e^r = sum r^n / n!, n = 0..13, by Horner's rule. */
    double p = 1.0 / 6227020800.0;                /* 1/13! */
    p = 1.0 / 479001600.0 + r * p;                /* 1/12! */
    p = 1.0 / 39916800.0 + r * p;                 /* 1/11! */
    p = 1.0 / 3628800.0 + r * p;                  /* 1/10! */
    p = 1.0 / 362880.0 + r * p;                   /* 1/9!  */
    p = 1.0 / 40320.0 + r * p;                    /* 1/8!  */
    p = 1.0 / 5040.0 + r * p;                     /* 1/7!  */
    p = 1.0 / 720.0 + r * p;                      /* 1/6!  */
    p = 1.0 / 120.0 + r * p;                      /* 1/5!  */
    p = 1.0 / 24.0 + r * p;                       /* 1/4!  */
    p = 1.0 / 6.0 + r * p;                        /* 1/3!  */
    p = 0.5 + r * p;                              /* 1/2!  */
    p = 1.0 + r * p;                              /* 1/1!  */
    p = 1.0 + r * p;                              /* 1/0!  */
    return (float)(p * lw_pow2i(k));
}

#endif
