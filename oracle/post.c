/*
 * The reference's display pass restated in C: `post::tonemap` and `post::tonemap_mix`
 * (crates/lumenwright/src/render/post.rs:152-217) with the Hable curve of `HableCurve`
 * (:29-138): Chunky's FILMIC_WORLDS preset, its white scale in f32, `h` with the parameter
 * products in f32 and the rest in f64, and the game's curve (the preset brightened by the gain
 * that holds mid-grey). The display gamma is the platform's `powf`, as Rust's `f32::powf` on the
 * host build. Test infrastructure only (see lw_oracle.h). Compile with -ffp-contract=off.
 */
#include <math.h>
#include <stdint.h>

#include "lw_oracle.h"

typedef struct { float a, b, c, d, e, f, w; } Hable;

static const Hable FILMIC_WORLDS = {0.15f, 0.5f, 0.1f, 0.2f, 0.02f, 0.3f, 11.2f}; /* post.rs:57-65 */

static float white_scale(Hable k) { /* post.rs:74-88 */
    float num = k.w * (k.a * k.w + k.c * k.b) + k.d * k.e;
    float den = k.w * (k.a * k.w + k.b) + k.d * k.f;
    return 1.0f / (num / den - k.e / k.f);
}

static double h(Hable k, double y) { /* post.rs:91-104 */
    double a = k.a, b = k.b, cb = (double)(k.c * k.b), de = (double)(k.d * k.e), df = (double)(k.d * k.f),
           ef = (double)(k.e / k.f);
    return (y * (a * y + cb) + de) / (y * (a * y + b) + df) - ef;
}

static double mid_grey_gain(Hable k, double m) { /* post.rs:125-137 */
    double a = k.a, b = k.b, cb = (double)(k.c * k.b), de = (double)(k.d * k.e), df = (double)(k.d * k.f),
           ef = (double)(k.e / k.f);
    double q = m / (double)white_scale(k) + ef;
    double qa = a * (1.0 - q), qb = cb - q * b, qc = de - q * df;
    double y = (-qb + sqrt(qb * qb - 4.0 * qa * qc)) / (2.0 * qa);
    return y / (2.0 * m);
}

static Hable brightened(Hable k, double g) { /* post.rs:113-120 */
    Hable r = k;
    r.a = (float)((double)k.a * g * g);
    r.b = (float)((double)k.b * g);
    r.w = (float)((double)k.w / g);
    return r;
}

static Hable game_tone_curve(void) { return brightened(FILMIC_WORLDS, mid_grey_gain(FILMIC_WORLDS, 0.18)); }

static float clamp_rs(float x, float lo, float hi) { return x < lo ? lo : (x > hi ? hi : x); }
static float max_rs(float x, float y) { return x != x ? y : (x > y ? x : y); }

static float aces(float x) { /* post.rs:23-26 */
    float a = 2.51f, b = 0.03f, c = 2.43f, d = 0.59f, e = 0.14f;
    return clamp_rs((x * (a * x + b)) / (x * (c * x + d) + e), 0.0f, 1.0f);
}

static float encode(float v) { return powf(clamp_rs(v, 0.0f, 1.0f), 1.0f / 2.2f); } /* post.rs:146-149 */

static float shown(uint32_t op, float exposure, float v) {
    Hable k = op == 3u ? game_tone_curve() : FILMIC_WORLDS;
    v = max_rs(v * exposure, 0.0f);
    if (op == 1u) v = aces(v);
    else if (op == 2u || op == 3u) v = (float)(h(k, 2.0 * (double)v) * (double)white_scale(k));
    return encode(v);
}

static uint32_t byte_of(float d) { /* `(d * 255.0 + 0.5) as u32`, saturating, NaN to 0 */
    float x = d * 255.0f + 0.5f;
    if (x != x || x <= 0.0f) return 0u;
    if (x >= 4294967295.0f) return 0xFFFFFFFFu;
    return (uint32_t)x;
}

void lwo_tonemap(const float *hdr, uint64_t n, float exposure, uint32_t op, uint32_t mix, uint32_t op_b, float weight,
                 uint32_t *out) {
    for (uint64_t i = 0; i < n; i++) {
        uint32_t px = 0xFF000000u;
        for (int c = 0; c < 3; c++) {
            float v = hdr[3 * i + c], d;
            if (!mix || weight >= 1.0f) d = shown(op, exposure, v);
            else if (weight <= 0.0f) d = shown(op_b, exposure, v);
            else d = weight * shown(op, exposure, v) + (1.0f - weight) * shown(op_b, exposure, v);
            px |= byte_of(d) << (8 * c);
        }
        out[i] = px;
    }
}

void lwo_game_tone_curve(float out[7]) {
    Hable g = game_tone_curve();
    out[0] = g.a, out[1] = g.b, out[2] = g.c, out[3] = g.d, out[4] = g.e, out[5] = g.f, out[6] = g.w;
}

double lwo_mid_grey_gain(void) { return mid_grey_gain(FILMIC_WORLDS, 0.18); }

double lwo_game_before_gamma(double x) { /* post.rs:107-109 for the game curve */
    Hable g = game_tone_curve();
    return h(g, 2.0 * x) * (double)white_scale(g);
}
