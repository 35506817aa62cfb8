/*
 * The game's sky drawn into an equirectangular map: `QuickSky::background` (crates/lumenwright/
 * src/render/sky.rs:509-530, with `disc` :395-424, `fan_alpha` :427-461, `body` :464-486,
 * `star_hits` :489-505, `star_bin` :138-150, `linear_fog` :295-304) for the direction of every texel
 * (`map_direction`, :853-858), decoded to linear with powf(c, 2.2) (`draw_map`, :861-878). f32
 * arithmetic in the reference's order with the platform's f32 atan2f, asinf, sinf, cosf, floorf
 * and powf, as the reference's f32 methods call them.
 *
 * TEST INFRASTRUCTURE (see lw_oracle.h): the checker of the library's device pass.
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <string.h>

#include "lw_oracle.h"

typedef struct {
    float x, y, z;
} G3;
static G3 g3(float x, float y, float z) {
    G3 r = {x, y, z};
    return r;
}
static G3 gadd(G3 a, G3 b) { return g3(a.x + b.x, a.y + b.y, a.z + b.z); }
static G3 gsub(G3 a, G3 b) { return g3(a.x - b.x, a.y - b.y, a.z - b.z); }
static G3 gmul(G3 a, float s) { return g3(a.x * s, a.y * s, a.z * s); }
static float gdot(G3 a, G3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static G3 gcross(G3 a, G3 o) { return g3(a.y * o.z - o.y * a.z, a.z * o.x - o.z * a.x, a.x * o.y - o.x * a.y); }
static G3 g4(const float v[4]) { return g3(v[0], v[1], v[2]); }
/* Vec3::lerp of glam 0.34.1 (not in this tree), restated as a + (b - a) * t; its other published
 * form, a * (1 - t) + b * t, differs from it by at most an ulp. */
static G3 glerp(G3 a, G3 b, float t) { return gadd(a, gmul(gsub(b, a), t)); }
static float gminf(float a, float b) { return a < b ? a : b; }
static float gmaxf(float a, float b) { return a > b ? a : b; }
static G3 gmin1(G3 a) { return g3(gminf(a.x, 1.0f), gminf(a.y, 1.0f), gminf(a.z, 1.0f)); }
static float f32_bits(uint32_t u) {
    float f;
    memcpy(&f, &u, 4);
    return f;
}

#define PI_F 3.14159265358979323846f
#define TAU_F 6.28318530717958647692f
#define FRAC_PI_2_F 1.57079632679489661923f
#define FRAC_PI_4_F 0.78539816339744830962f
#define RIM_SPHERICAL 512.24994f
#define STAR_BINS_AZ 128
#define STAR_BINS_EL 64
#define STAR_WORDS 9

static float linear_fog(float v, float start, float end) {
    if (v <= start) return 0.0f;
    if (v >= end) return 1.0f;
    return (v - start) / (end - start);
}

/* The sky disc's colour along d; 0 past its rim or below the horizon. */
static int disc(const lwo_quick_sky *q, G3 d, G3 *out) {
    if (d.y <= 0.0f) return 0;
    G3 p = gmul(d, 16.0f / d.y);
    const float step = FRAC_PI_4_F;
    float phi = atan2f(p.z, p.x);
    float k = floorf((phi + PI_F) / step);
    k = k < 0.0f ? 0.0f : (k > 7.0f ? 7.0f : k); /* f32::clamp */
    float th0 = -PI_F + k * step;
    float s0 = sinf(th0), c0 = cosf(th0);
    float s1 = sinf(th0 + step), c1 = cosf(th0 + step);
    float r0x = 512.0f * c0, r0z = 512.0f * s0, r1x = 512.0f * c1, r1z = 512.0f * s1;
    float det = r0x * r1z - r1x * r0z;
    float b1 = (p.x * r1z - r1x * p.z) / det;
    float b2 = (r0x * p.z - p.x * r0z) / det;
    float s = b1 + b2;
    if (s > 1.0f) return 0;
    float end = q->sky_color[3];
    float sph = 16.0f * (1.0f - s) + RIM_SPHERICAL * s;
    float cyl = 16.0f * (1.0f - s) + 512.0f * s;
    float f = gmaxf(linear_fog(sph, 0.0f, end), linear_fog(cyl, end, end));
    *out = glerp(g4(q->sky_color), g4(q->fog_color), f);
    return 1;
}

static float fan_alpha(const lwo_quick_sky *q, G3 d) {
    G3 c = g4(q->fan[0]);
    float best_t = INFINITY, alpha = 0.0f;
    for (int k = 0; k < 16; k++) {
        G3 v1 = g4(q->fan[k + 1]), v2 = g4(q->fan[k + 2]);
        G3 e1 = gsub(v1, c), e2 = gsub(v2, c);
        G3 pv = gcross(d, e2);
        float det = gdot(e1, pv);
        if (fabsf(det) < 1e-6f) continue;
        float inv = 1.0f / det;
        G3 tv = gmul(c, -1.0f);
        float u = gdot(tv, pv) * inv;
        if (!(u >= 0.0f && u <= 1.0f)) continue;
        G3 qv = gcross(tv, e1);
        float v = gdot(d, qv) * inv;
        if (v < 0.0f || u + v > 1.0f) continue;
        float t = gdot(e2, qv) * inv;
        if (t > 0.0f && t < best_t) {
            best_t = t;
            alpha = (1.0f - u - v) * q->fan[0][3];
        }
    }
    return alpha;
}

static void body(const float b[4][4], G3 d, const uint32_t *atlas, uint32_t atlas_w, float out[4]) {
    out[0] = out[1] = out[2] = out[3] = 0.0f;
    if (b[0][3] == 0.0f || b[3][2] <= 0.0f) return;
    G3 c = g4(b[0]);
    float dn = gdot(d, c);
    if (dn <= 0.0f) return;
    G3 qv = gsub(gmul(d, gdot(c, c) / dn), c);
    float lx = gdot(qv, g4(b[1])), lz = gdot(qv, g4(b[2]));
    if (fabsf(lx) >= 1.0f || fabsf(lz) >= 1.0f) return;
    float u = b[3][0] + (lx * 0.5f + 0.5f) * b[3][2];
    float v = b[3][1] + (lz * 0.5f + 0.5f) * b[3][3];
    uint32_t t = atlas[(uint32_t)floorf(v) * atlas_w + (uint32_t)floorf(u)];
    out[0] = (float)(t & 0xFFu) / 255.0f;
    out[1] = (float)((t >> 8) & 0xFFu) / 255.0f;
    out[2] = (float)((t >> 16) & 0xFFu) / 255.0f;
    out[3] = (float)(t >> 24) / 255.0f;
}

static uint32_t star_hits(const lwo_quick_sky *q, G3 d, const uint32_t *table) {
    G3 qd = g3(gdot(g4(q->star_rot[0]), d), gdot(g4(q->star_rot[1]), d), gdot(g4(q->star_rot[2]), d));
    float az = atan2f(qd.z, qd.x);
    float y = qd.y < -1.0f ? -1.0f : (qd.y > 1.0f ? 1.0f : qd.y);
    float el = asinf(y);
    int ia = (int)floorf(((az + PI_F) / TAU_F) * (float)STAR_BINS_AZ);
    int ie = (int)floorf(((el + FRAC_PI_2_F) / PI_F) * (float)STAR_BINS_EL);
    ia = ia < 0 ? 0 : (ia > STAR_BINS_AZ - 1 ? STAR_BINS_AZ - 1 : ia);
    ie = ie < 0 ? 0 : (ie > STAR_BINS_EL - 1 ? STAR_BINS_EL - 1 : ie);
    uint32_t b = (uint32_t)(ie * STAR_BINS_AZ + ia);
    const uint32_t base = STAR_BINS_AZ * STAR_BINS_EL + 1;
    uint32_t n = 0;
    for (uint32_t e = table[b]; e < table[b + 1]; e++) {
        const uint32_t o = base + e * STAR_WORDS;
        G3 c = g3(f32_bits(table[o]), f32_bits(table[o + 1]), f32_bits(table[o + 2]));
        G3 a1 = g3(f32_bits(table[o + 3]), f32_bits(table[o + 4]), f32_bits(table[o + 5]));
        G3 a2 = g3(f32_bits(table[o + 6]), f32_bits(table[o + 7]), f32_bits(table[o + 8]));
        float dn = gdot(qd, c);
        if (dn <= 0.0f) continue;
        G3 p = gsub(gmul(qd, gdot(c, c) / dn), c);
        if (fabsf(gdot(p, a1)) < 1.0f && fabsf(gdot(p, a2)) < 1.0f) n++;
    }
    return n;
}

static G3 background(const lwo_quick_sky *q, G3 d, const uint32_t *atlas, uint32_t atlas_w, const uint32_t *stars) {
    G3 c = g4(q->fog_color), dc;
    if (q->flags[0] > 0.5f && disc(q, d, &dc)) c = dc;
    if (q->flags[1] > 0.5f) c = glerp(c, g4(q->sunrise), fan_alpha(q, d));
    float t[4];
    body(q->sun, d, atlas, atlas_w, t);
    c = gmin1(gadd(c, gmul(g3(t[0], t[1], t[2]), t[3])));
    body(q->moon, d, atlas, atlas_w, t);
    c = gmin1(gadd(c, gmul(g3(t[0], t[1], t[2]), t[3])));
    if (q->flags[2] > 0.5f) {
        uint32_t n = star_hits(q, d, stars);
        for (uint32_t k = 0; k < n; k++) c = gmin1(gadd(c, g3(q->fog_dist[3], q->fog_dist[3], q->fog_dist[3])));
    }
    /* Vec3::clamp(ZERO, ONE): max with the lower bound, then min with the upper */
    return g3(gminf(gmaxf(c.x, 0.0f), 1.0f), gminf(gmaxf(c.y, 0.0f), 1.0f), gminf(gmaxf(c.z, 0.0f), 1.0f));
}

static G3 map_direction(uint32_t i, uint32_t j, uint32_t w, uint32_t h) {
    float az = ((float)i + 0.5f) / (float)w * TAU_F;
    float el = ((float)j + 0.5f) / (float)h * PI_F - FRAC_PI_2_F;
    return g3(cosf(el) * cosf(az), sinf(el), cosf(el) * sinf(az));
}

void lwo_draw_sky_map(const lwo_quick_sky *q, const uint32_t *atlas, uint32_t atlas_w, const uint32_t *stars, uint32_t w,
                      uint32_t h, float *out, int threads) {
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(static) num_threads(threads)
    for (uint32_t j = 0; j < h; j++)
        for (uint32_t i = 0; i < w; i++) {
            G3 c = background(q, map_direction(i, j, w, h), atlas, atlas_w, stars);
            float *o = out + 3 * ((uint64_t)j * w + i);
            o[0] = powf(c.x, 2.2f);
            o[1] = powf(c.y, 2.2f);
            o[2] = powf(c.z, 2.2f);
        }
}
