/*
 * FP32 oracle: the reference kernel's own f32 arithmetic (see lw_oracle.h).
 * Test infrastructure only. Compile with -ffp-contract=off (oracle/Makefile).
 */
#include <math.h>
#include <omp.h>
#include <stdlib.h>

#define REAL float
#define K(x) x##f
#define R_SQRT sqrtf
#define R_FLOOR floorf
#define R_EXP expf
/* The water transmittance's exponential: the function the CUDA kernels call (water_exp.h, the
 * project's correctly rounded f32 exp), where the reference's CPU build calls the platform expf;
 * tests/test_water_exp.py holds it against both the platform expf and f64 exp. */
#define R_TEXP lw_water_expf
#define R_FMOD fmodf
#define R_ACOS k_acos
#define R_ATAN2 k_atan2
#define R_GAMMA k_gamma_to_linear
#define R_SINCOS_TURNS k_sin_cos_turns

static inline float k_ln(float x);
static inline float k_acos(float x);
static inline float k_atan2(float y, float x);
static inline float k_gamma_to_linear(float c);
static inline void k_sin_cos_turns(float u, float *s, float *c);

#include "water_exp.h"
#include "kernel_impl.h"

uint64_t lwo_bounds_error_count;
__thread lwo_counters *lwo_cnt;

/* sin_cos_turns (crates/lumenwright-kernel/src/math.rs:45-64): the quarter-turn reduction
 * by adding and subtracting 1.5 * 2^23, Taylor series to x^9 and x^10, quadrant selects. */
static inline void k_sin_cos_turns(float u, float *ps, float *pc) {
    const float ROUND = 12582912.0f;
    float t = u * 4.0f;
    float q = (t + ROUND) - ROUND;
    float x = (t - q) * 1.57079632679489661923f;
    float x2 = x * x;
    float s = x * (1.0f + x2 * (-1.0f / 6.0f + x2 * (1.0f / 120.0f + x2 * (-1.0f / 5040.0f + x2 * (1.0f / 362880.0f)))));
    float c = 1.0f + x2 * (-0.5f + x2 * (1.0f / 24.0f + x2 * (-1.0f / 720.0f + x2 * (1.0f / 40320.0f + x2 * (-1.0f / 3628800.0f)))));
    int32_t k = to_i32(q) & 3;
    int odd = (k & 1) != 0;
    float s2 = odd ? c : s;
    float c2 = odd ? -s : c;
    if (k & 2) { s2 = -s2; c2 = -c2; }
    *ps = s2;
    *pc = c2;
}

/* acos (math.rs:87-103): Abramowitz and Stegun 4.4.46. */
static inline float k_acos(float x) {
    float a = rclamp(rabs(x), 0.0f, 1.0f);
    float p = 1.5707963f +
              a * (-0.2145988f +
                   a * (0.08897899f +
                        a * (-0.0501743f + a * (0.03089188f + a * (-0.017088126f + a * (0.00667009f + a * -0.0012624911f))))));
    float r = sqrtf(1.0f - a) * p;
    return x < 0.0f ? 3.14159265358979323846f - r : r;
}

/* atan2 (math.rs:114-142): Abramowitz and Stegun 4.4.49. */
static inline float k_atan2(float y, float x) {
    float ax = rabs(x), ay = rabs(y);
    float lo = rmin(ax, ay), hi = rmax(ax, ay);
    if (hi == 0.0f) return 0.0f;
    float t = lo / hi;
    float t2 = t * t;
    float p = t * (1.0f + t2 * (-0.33333145f +
                               t2 * (0.19993551f +
                                     t2 * (-0.142089f +
                                           t2 * (0.10656264f +
                                                 t2 * (-0.07528964f + t2 * (0.042909614f + t2 * (-0.016165737f + t2 * 0.0028662257f))))))));
    float r = ay > ax ? 1.57079632679489661923f - p : p;
    r = x < 0.0f ? 3.14159265358979323846f - r : r;
    return y < 0.0f ? -r : r;
}

/* ln (math.rs:183-203): m * 2^e with m in [sqrt(1/2), sqrt(2)], 2 atanh series to s^9. */
static inline float k_ln(float x) {
    if (x <= 0.0f) return x == 0.0f ? -INFINITY : NAN;
    uint32_t bits = bits_of(x);
    int32_t e = (int32_t)((bits >> 23) & 0xFFu) - 127;
    float m = f32_of((bits & 0x007FFFFFu) | 0x3F800000u);
    if (m > 1.41421356237309504880f) {
        m *= 0.5f;
        e += 1;
    }
    float s = (m - 1.0f) / (m + 1.0f);
    float s2 = s * s;
    float series = 2.0f * s * (1.0f + s2 * (1.0f / 3.0f + s2 * (1.0f / 5.0f + s2 * (1.0f / 7.0f + s2 * (1.0f / 9.0f)))));
    return (float)e * 0.693147180559945309417f + series;
}

/* gamma_to_linear (math.rs:214-216): exp(2.2 * ln c). */
static inline float k_gamma_to_linear(float c) { return c <= 0.0f ? 0.0f : expf(2.2f * k_ln(c)); }

/* ---- exported API ------------------------------------------------------------------- */
static inline V3 v3a(const float a[3]) { return v3(a[0], a[1], a[2]); }
static inline void v3o(V3 v, float o[3]) { o[0] = v.x; o[1] = v.y; o[2] = v.z; }
static lwo_hit to_pub(Hit h) {
    lwo_hit r = {h.t, h.quad, h.texel, h.s, h.tt, h.quad != NO_QUAD};
    return r;
}
static Cam params_cam(const lwo_params *p) {
    Cam c = {v3f4(p->cam_pos), v3f4(p->cam_fwd), v3f4(p->cam_right), v3f4(p->cam_up), p->cam_pos[3], p->cam_fwd[3],
             p->see_through[2], p->see_through[3]};
    return c;
}

uint64_t lwo_bounds_errors(void) { return __atomic_load_n(&lwo_bounds_error_count, __ATOMIC_RELAXED); }
void lwo_reset_bounds_errors(void) { __atomic_store_n(&lwo_bounds_error_count, 0, __ATOMIC_RELAXED); }

uint32_t lwo32_pcg_hash(uint32_t v) { return pcg_hash(v); }
uint32_t lwo32_rng_new(uint32_t pixel, uint32_t sample, uint32_t seed) { return rng_new(pixel, sample, seed); }
float lwo32_rng_next(uint32_t *state) { return rng_next(state); }
void lwo32_sin_cos_turns(float u, float *s, float *c) { k_sin_cos_turns(u, s, c); }
float lwo32_acos(float x) { return k_acos(x); }
float lwo32_atan2(float y, float x) { return k_atan2(y, x); }
float lwo32_ln(float x) { return k_ln(x); }
float lwo32_gamma_to_linear(float c) { return k_gamma_to_linear(c); }
uint32_t lwo32_voxel(const lwo_scene *s, int32_t x, int32_t y, int32_t z) { return voxel(s, x, y, z); }
lwo_hit lwo32_trace(const lwo_scene *s, const float o[3], const float d[3], float tmin, float tmax) {
    return to_pub(trace(s, v3a(o), v3a(d), tmin, tmax));
}
lwo_hit lwo32_see_through_hit(const lwo_scene *s, const float o[3], const float d[3], float tmin) {
    return to_pub(see_through_hit(s, v3a(o), v3a(d), tmin));
}
void lwo32_render_sample(const lwo_scene *s, uint32_t px, uint32_t py, uint32_t sample, float out[3]) {
    Cam c = params_cam(s->params);
    v3o(render_sample(s, &c, px, py, sample), out);
}
void lwo32_sample_emitters(const lwo_scene *s, const float pos[3], const float origin[3], const float n[3],
                           uint32_t *rng_state, float out[3]) {
    v3o(sample_emitters(s, v3a(pos), v3a(origin), v3a(n), rng_state), out);
}
void lwo32_rebase(float x[3], uint32_t *word) {
    frame_unpack(*word, lwo_fa);
    v3o(rebase(v3a(x)), x);
    *word = ((uint32_t)(lwo_fa[0] >> 4) & 0x7FFu) | (((uint32_t)(lwo_fa[1] >> 4) & 0x3FFu) << 11) |
            (((uint32_t)(lwo_fa[2] >> 4) & 0x7FFu) << 21);
    lwo_fa[0] = lwo_fa[1] = lwo_fa[2] = 0;
}
void lwo32_emitter_cell(const lwo_scene *s, const float p[3], uint32_t *start, uint32_t *count) {
    emitter_cell(s, v3a(p), start, count);
}
void lwo32_preetham_radiance(const lwo_scene *s, const float d[3], float out[3]) { v3o(preetham_radiance(s, v3a(d)), out); }
void lwo32_build_sky_cache(const lwo_scene *s, uint32_t n, float *out) { build_sky_cache(s, n, out); }
void lwo32_sky_radiance(const lwo_scene *s, const float d[3], float out[3]) { v3o(sky_radiance(s, v3a(d)), out); }
void lwo32_sky_lens(const lwo_scene *s, const float d[3], float out[3]) { v3o(sky_lens(s, v3a(d)), out); }
void lwo32_sky_light(const lwo_scene *s, const float d[3], float out[3]) { v3o(sky_light(s, v3a(d)), out); }
void lwo32_sun_texture(const lwo_scene *s, const float d[3], float out[3]) { v3o(sun_texture(s, v3a(d)), out); }

/* The transmittance's exponential (water_exp.h) and the platform expf over n arguments. */
void lwo32_water_exp(uint64_t n, const float *x, float *out) {
    for (uint64_t i = 0; i < n; i++) out[i] = lw_water_expf(x[i]);
}
void lwo_platform_expf(uint64_t n, const float *x, float *out) {
    for (uint64_t i = 0; i < n; i++) out[i] = expf(x[i]);
}

/* Every `stride`-th float x with bits in [lo_bits, hi_bits] (as unsigned words): counts where
 * lw_water_expf(x) differs from the platform expf(x) and from exp((double)x) rounded to f32, and
 * the largest difference from each in units of the last place of the f32 result. */
void lwo32_water_exp_sweep(uint32_t lo_bits, uint32_t hi_bits, uint32_t stride, uint64_t out[5]) {
    uint64_t n = 0, diff_platform = 0, diff_f64 = 0, ulp_platform = 0, ulp_f64 = 0;
    if (stride == 0) stride = 1;
    int64_t steps = ((int64_t)hi_bits - (int64_t)lo_bits) / (int64_t)stride + 1;
#pragma omp parallel for schedule(static) reduction(+ : n, diff_platform, diff_f64) reduction(max : ulp_platform, ulp_f64)
    for (int64_t i = 0; i < steps; i++) {
        float x = f32_of(lo_bits + (uint32_t)(i * (int64_t)stride));
        float a = lw_water_expf(x), b = expf(x), c = (float)exp((double)x);
        uint32_t ab = bits_of(a), bb = bits_of(b), cb = bits_of(c);
        uint64_t db = ab > bb ? ab - bb : bb - ab, dc = ab > cb ? ab - cb : cb - ab;
        n++;
        if (db) diff_platform++;
        if (dc) diff_f64++;
        if (db > ulp_platform) ulp_platform = db;
        if (dc > ulp_f64) ulp_f64 = dc;
    }
    out[0] = n;
    out[1] = diff_platform;
    out[2] = ulp_platform;
    out[3] = diff_f64;
    out[4] = ulp_f64;
}

void lwo32_sky_radiance_many(const lwo_scene *s, uint64_t n, const float *d, float *out) {
#pragma omp parallel for schedule(static)
    for (uint64_t i = 0; i < n; i++) v3o(sky_radiance(s, v3a(d + 3 * i)), out + 3 * i);
}

void lwo32_render_samples(const lwo_scene *s, uint32_t x0, uint32_t y0, uint32_t w, uint32_t h,
                          uint32_t sample_start, uint32_t count, float *out, int threads) {
    Cam c = params_cam(s->params);
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
    for (uint32_t py = 0; py < h; py++)
        for (uint32_t px = 0; px < w; px++)
            for (uint32_t k = 0; k < count; k++) {
                V3 r = render_sample(s, &c, x0 + px, y0 + py, sample_start + k);
                v3o(r, out + ((uint64_t)(py * w + px) * count + k) * 3u);
            }
}

/* CpuBackend::render_hq's per-pixel loop (crates/lumenwright/src/render/cpu/mod.rs:61-80):
 * f64 sums of the finite samples, divided by spp. */
void lwo32_render_mean(const lwo_scene *s, uint32_t x0, uint32_t y0, uint32_t w, uint32_t h, uint32_t spp,
                       float *out, int threads) {
    Cam c = params_cam(s->params);
    if (spp < 1) spp = 1;
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
    for (uint32_t py = 0; py < h; py++)
        for (uint32_t px = 0; px < w; px++) {
            double acc[3] = {0, 0, 0};
            for (uint32_t k = 0; k < spp; k++) {
                V3 r = render_sample(s, &c, x0 + px, y0 + py, k);
                if (isfinite(r.x) && isfinite(r.y) && isfinite(r.z)) {
                    acc[0] += (double)r.x;
                    acc[1] += (double)r.y;
                    acc[2] += (double)r.z;
                }
            }
            float *o = out + (uint64_t)(py * w + px) * 3u;
            o[0] = (float)(acc[0] / (double)spp);
            o[1] = (float)(acc[1] / (double)spp);
            o[2] = (float)(acc[2] / (double)spp);
        }
}

void lwo32_count_work(const lwo_scene *s, uint32_t x0, uint32_t y0, uint32_t w, uint32_t h, uint32_t spp,
                      lwo_counters *out) {
    Cam c = params_cam(s->params);
    memset(out, 0, sizeof *out);
#pragma omp parallel
    {
        lwo_counters mine;
        memset(&mine, 0, sizeof mine);
        lwo_cnt = &mine;
#pragma omp for schedule(dynamic, 1)
        for (uint32_t py = 0; py < h; py++)
            for (uint32_t px = 0; px < w; px++)
                for (uint32_t k = 0; k < spp; k++) (void)render_sample(s, &c, x0 + px, y0 + py, k);
        lwo_cnt = NULL;
#pragma omp critical
        {
            uint64_t *a = (uint64_t *)out, *b = (uint64_t *)&mine;
            for (size_t i = 0; i < sizeof mine / sizeof(uint64_t); i++) a[i] += b[i];
        }
    }
}
