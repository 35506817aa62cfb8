// Device arithmetic of the hq path tracer: the reference kernel's f32 functions
// (crates/lumenwright-kernel/src/math.rs, rng.rs), operation for operation. The library is built
// with --fmad=false and IEEE division and square root, so each expression rounds as the
// reference's f32 code does; the comparisons below keep the reference's NaN behaviour.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "water_exp.h"

namespace lw {

#define LW_DI __device__ __forceinline__
#define LW_HDI __host__ __device__ __forceinline__
// Rarely taken paths (sky lookups, the sun texture, water interfaces, see-through quads) are kept
// out of line so the hot loop stays small in the instruction cache.
#ifndef LW_NOINLINE_COLD
#define LW_NOINLINE_COLD 0
#endif
#if LW_NOINLINE_COLD
#define LW_COLD static __device__ __noinline__
#else
#define LW_COLD __device__ __forceinline__
#endif

constexpr float kPI = 3.14159265358979323846f;
constexpr float kFRAC_PI_2 = 1.57079632679489661923f;
constexpr float kINF = __builtin_huge_valf();

struct V3 {
    float x, y, z;
};
LW_HDI V3 v3(float x, float y, float z) { return V3{x, y, z}; }
LW_HDI V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
LW_HDI V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
LW_HDI V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
LW_HDI V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
LW_HDI V3 vmul(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
LW_HDI float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
LW_HDI V3 cross(V3 a, V3 o) { return v3(a.y * o.z - a.z * o.y, a.z * o.x - a.x * o.z, a.x * o.y - a.y * o.x); }
// min/max/abs/clamp of math.rs:149-169: `b` when either is NaN.
LW_HDI float fmin_r(float a, float b) { return a < b ? a : b; }
LW_HDI float fmax_r(float a, float b) { return a > b ? a : b; }
LW_HDI float fabs_r(float x) { return x < 0.0f ? -x : x; }
LW_HDI float clamp_r(float x, float lo, float hi) { return fmin_r(fmax_r(x, lo), hi); }
LW_HDI int clamp_i(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
LW_DI float vlength(V3 a) { return __fsqrt_rn(dot(a, a)); }
// V3::normalize (math.rs:275-278): times the reciprocal of the length.
LW_DI V3 normalize(V3 a) {
    float l = vlength(a);
    return l > 0.0f ? a * __fdiv_rn(1.0f, l) : a;
}
LW_DI V3 vdiv(V3 a, float s) { return a * __fdiv_rn(1.0f, s); }
LW_HDI float max_elem(V3 a) { return fmax_r(a.x, fmax_r(a.y, a.z)); }
LW_HDI float vget(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
LW_HDI V3 lerp(V3 a, V3 o, float t) { return a + (o - a) * t; }
// Beer-Lambert through water (math.rs:300, `(-a * t).exp()`), with the project's exponential
// (water_exp.h), which the CPU oracle calls too.
LW_DI V3 transmittance(V3 a, float t) {
    return v3(lw_water_expf(-a.x * t), lw_water_expf(-a.y * t), lw_water_expf(-a.z * t));
}
LW_HDI V3 f4v(float4 a) { return v3(a.x, a.y, a.z); }

// Rust's saturating `as i32` / `as u32` (NaN gives 0): the PTX cvt.rzi.sat conversions.
LW_DI int to_i32(float x) { return __float2int_rz(x); }
LW_DI uint32_t to_u32(float x) { return __float2uint_rz(x); }

// rng.rs:5-34.
LW_HDI uint32_t pcg_hash(uint32_t v) {
    uint32_t state = v * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28) + 4u)) ^ state) * 277803737u;
    return (word >> 22) ^ word;
}
LW_HDI uint32_t rng_new(uint32_t pixel, uint32_t sample, uint32_t seed) {
    return pcg_hash(pixel ^ pcg_hash(sample + pcg_hash(seed)));
}
LW_DI float rng_next(uint32_t &st) {
    st = pcg_hash(st);
    return __uint2float_rn(st >> 8) * (1.0f / 16777216.0f);
}

// sin_cos_turns (math.rs:45-64).
LW_DI void sin_cos_turns(float u, float &so, float &co) {
    const float ROUND = 12582912.0f;
    float t = u * 4.0f;
    float q = __fsub_rn(__fadd_rn(t, ROUND), ROUND);
    float x = (t - q) * kFRAC_PI_2;
    float x2 = x * x;
    float s = x * (1.0f + x2 * (-1.0f / 6.0f + x2 * (1.0f / 120.0f + x2 * (-1.0f / 5040.0f + x2 * (1.0f / 362880.0f)))));
    float c = 1.0f + x2 * (-0.5f + x2 * (1.0f / 24.0f + x2 * (-1.0f / 720.0f + x2 * (1.0f / 40320.0f + x2 * (-1.0f / 3628800.0f)))));
    int k = to_i32(q) & 3;
    bool odd = (k & 1) != 0;
    float s2 = odd ? c : s;
    float c2 = odd ? -s : c;
    if (k & 2) {
        s2 = -s2;
        c2 = -c2;
    }
    so = s2;
    co = c2;
}

// acos (math.rs:87-103), Abramowitz and Stegun 4.4.46.
LW_DI float acos_r(float x) {
    float a = clamp_r(fabs_r(x), 0.0f, 1.0f);
    float p = 1.5707963f +
              a * (-0.2145988f +
                   a * (0.08897899f +
                        a * (-0.0501743f + a * (0.03089188f + a * (-0.017088126f + a * (0.00667009f + a * -0.0012624911f))))));
    float r = __fsqrt_rn(1.0f - a) * p;
    return x < 0.0f ? kPI - r : r;
}

// atan2 (math.rs:114-142), Abramowitz and Stegun 4.4.49.
LW_DI float atan2_r(float y, float x) {
    float ax = fabs_r(x), ay = fabs_r(y);
    float lo = fmin_r(ax, ay), hi = fmax_r(ax, ay);
    if (hi == 0.0f) return 0.0f;
    float t = __fdiv_rn(lo, hi);
    float t2 = t * t;
    float p = t * (1.0f + t2 * (-0.33333145f +
                               t2 * (0.19993551f +
                                     t2 * (-0.142089f +
                                           t2 * (0.10656264f +
                                                 t2 * (-0.07528964f + t2 * (0.042909614f + t2 * (-0.016165737f + t2 * 0.0028662257f))))))));
    float r = ay > ax ? kFRAC_PI_2 - p : p;
    r = x < 0.0f ? kPI - r : r;
    return y < 0.0f ? -r : r;
}

// Duff et al. 2017 basis (math.rs:348-356).
LW_DI void onb(V3 n, V3 &t, V3 &b) {
    float sign = n.z >= 0.0f ? 1.0f : -1.0f;
    float a = __fdiv_rn(-1.0f, sign + n.z);
    float bb = n.x * n.y * a;
    t = v3(1.0f + sign * n.x * n.x * a, sign * bb, -sign * n.x);
    b = v3(bb, sign + n.y * n.y * a, -n.y);
}

}  // namespace lw
