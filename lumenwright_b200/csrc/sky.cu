// Sky precompute on the device: Chunky's sky cache (`build_sky_cache`,
// crates/lumenwright-kernel/src/integrator.rs:133-148, which the reference evaluates on the host
// per frame), the game sky's maps (`draw_map`, crates/lumenwright/src/render/sky.rs:861-878) and
// the blend of Chunky's sky into them (`blend_chunky_sky`, sky.rs:836-850). One thread per cache
// entry or map texel.
#include <cstring>

#include "device_integrator.cuh"
#include "internal.h"

namespace lw {

// preetham_radiance (integrator.rs:44-74). `expf` is CUDA's; the reference calls the platform's.
LW_DI V3 preetham_radiance(const DevParams &P, V3 d) {
    V3 sun = f4v(P.sky_sun);
    float cos_theta = fmax_r(d.y + P.sky_zenith.w, 0.0f);
    float cos_gamma = clamp_r(dot(d, sun), -1.0f, 1.0f);
    float gamma = acos_r(cos_gamma);
    float cos2_gamma = cos_gamma * cos_gamma;
    const float A[3] = {P.perez_a.x, P.perez_a.y, P.perez_a.z}, B[3] = {P.perez_b.x, P.perez_b.y, P.perez_b.z};
    const float Cc[3] = {P.perez_c.x, P.perez_c.y, P.perez_c.z}, D[3] = {P.perez_d.x, P.perez_d.y, P.perez_d.z};
    const float E[3] = {P.perez_e.x, P.perez_e.y, P.perez_e.z};
    float pz[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        float a = cos_theta > 0.0f ? A[k] * expf(__fdiv_rn(B[k], cos_theta)) : 0.0f;
        pz[k] = (1.0f + a) * (1.0f + Cc[k] * expf(D[k] * gamma) + E[k] * cos2_gamma);
    }
    float x = P.sky_zenith.x * pz[0];
    float y = P.sky_zenith.y * pz[1];
    float lum = P.sky_zenith.z * pz[2];
    if (y <= 5e-8f) return v3(0.0f, 0.0f, 0.0f);
    float f = __fdiv_rn(lum, y);
    float cx = x * f, cy = lum, cz = (1.0f - x - y) * f;
    return v3(2.3706743f * cx - 0.9000405f * cy - 0.4706338f * cz, -0.513885f * cx + 1.4253036f * cy + 0.0885814f * cz,
              0.0052982f * cx - 0.0146949f * cy + 1.0093968f * cz) *
           0.045f;
}

// rgb_to_hsl (integrator.rs:79-104).
LW_DI void rgb_to_hsl(V3 c, float &hue, float &sat, float &light) {
    float r = clamp_r(c.x, 0.0f, 1.0f), g = clamp_r(c.y, 0.0f, 1.0f), b = clamp_r(c.z, 0.0f, 1.0f);
    float cmax = fmax_r(fmax_r(r, g), b);
    float cmin = fmin_r(fmin_r(r, g), b);
    float delta = cmax - cmin;
    light = __fdiv_rn(cmax + cmin, 2.0f);
    if (delta == 0.0f) hue = 0.0f;
    else if (cmax == r) hue = __fdiv_rn(fmodf(__fdiv_rn(g - b, delta), 6.0f), 6.0f);
    else if (cmax == g) hue = __fdiv_rn(__fdiv_rn(b - r, delta) + 2.0f, 6.0f);
    else hue = __fdiv_rn(__fdiv_rn(r - g, delta) + 4.0f, 6.0f);
    sat = delta < 5e-8f ? 0.0f : __fdiv_rn(delta, 1.0f - fabs_r(2.0f * light - 1.0f));
}

__global__ void k_sky_cache(const DevParams P, uint32_t n, float *out) {
    uint32_t m = n + 1;
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m * m) return;
    uint32_t i = k / m, j = k - i * m;
    float sin_t, cos_t, sin_p, cos_p;
    sin_cos_turns(__fdiv_rn((float)i, (float)n), sin_t, cos_t);
    sin_cos_turns(__fdiv_rn((float)j, (float)(2 * n)) - 0.25f, sin_p, cos_p);
    float r = fabs_r(cos_p);
    float h, s, l;
    rgb_to_hsl(preetham_radiance(P, v3(cos_t * r, sin_p, sin_t * r)), h, s, l);
    out[3 * k] = h;
    out[3 * k + 1] = s;
    out[3 * k + 2] = l;
}

// map_direction (sky.rs:853-858) and the blend of sky_radiance into the map texel.
__global__ void k_blend_chunky(const DevScene S, const DevParams P, float *map, uint32_t w, uint32_t h, float weight) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= w * h) return;
    uint32_t i = k % w, j = k / w;
    float az = __fdiv_rn((float)i + 0.5f, (float)w) * (2.0f * kPI);
    float el = __fdiv_rn((float)j + 0.5f, (float)h) * kPI - kFRAC_PI_2;
    V3 d = v3(cosf(el) * cosf(az), sinf(el), cosf(el) * sinf(az));
    V3 c = sky_radiance(S, P, d);
    float *t = map + 3 * (size_t)k;
    t[0] = weight * c.x + (1.0f - weight) * t[0];
    t[1] = weight * c.y + (1.0f - weight) * t[1];
    t[2] = weight * c.z + (1.0f - weight) * t[2];
}

cudaError_t launch_sky_cache(const DevParams &P, uint32_t n, float *out, cudaStream_t st) {
    uint32_t cnt = (n + 1) * (n + 1);
    k_sky_cache<<<(cnt + 127) / 128, 128, 0, st>>>(P, n, out);
    return cudaGetLastError();
}

cudaError_t launch_blend_chunky(const DevScene &S, const DevParams &P, float *map, uint32_t w, uint32_t h, float weight,
                                cudaStream_t st) {
    k_blend_chunky<<<(w * h + 127) / 128, 128, 0, st>>>(S, P, map, w, h, weight);
    return cudaGetLastError();
}

}  // namespace lw

// ---- the game sky's maps ----------------------------------------------------------------------
// QuickSky::background (crates/lumenwright/src/render/sky.rs:509-530) for every texel of a map,
// decoded to linear (draw_map, :861-878): the same steps as the reference in f32, with CUDA's
// atan2f, asinf, sinf, cosf and powf where the reference calls the platform's.
namespace lw {
namespace {

struct __align__(16) QuickSkyDev {
    float4 sky_color, fog_color, fog_dist, sunrise, flags;
    float4 sun[4], moon[4], star_rot[3], fan[18];
    float4 cam[4];
};
static_assert(sizeof(QuickSkyDev) == 608, "QuickSky is 608 bytes");

constexpr int kStarBinsAz = 128, kStarBinsEl = 64, kStarWords = 9;
constexpr float kTau = 6.28318530717958647692f, kFracPi4 = 0.78539816339744830962f;

LW_DI float linear_fog(float v, float start, float end) {  // sky.rs:295-304
    if (v <= start) return 0.0f;
    if (v >= end) return 1.0f;
    return __fdiv_rn(v - start, end - start);
}
LW_DI V3 glerp(V3 a, V3 b, float t) { return a + (b - a) * t; }
LW_DI V3 min1(V3 a) { return v3(fmin_r(a.x, 1.0f), fmin_r(a.y, 1.0f), fmin_r(a.z, 1.0f)); }

LW_DI bool sky_disc(const QuickSkyDev &q, V3 d, V3 &out) {  // sky.rs:395-424
    if (d.y <= 0.0f) return false;
    V3 p = d * __fdiv_rn(16.0f, d.y);
    const float step = kFracPi4;
    float phi = atan2f(p.z, p.x);
    float k = floorf(__fdiv_rn(phi + kPI, step));
    k = k < 0.0f ? 0.0f : (k > 7.0f ? 7.0f : k);
    float th0 = -kPI + k * step;
    float s0 = sinf(th0), c0 = cosf(th0), s1 = sinf(th0 + step), c1 = cosf(th0 + step);
    float r0x = 512.0f * c0, r0z = 512.0f * s0, r1x = 512.0f * c1, r1z = 512.0f * s1;
    float det = r0x * r1z - r1x * r0z;
    float b1 = __fdiv_rn(p.x * r1z - r1x * p.z, det);
    float b2 = __fdiv_rn(r0x * p.z - p.x * r0z, det);
    float s = b1 + b2;
    if (s > 1.0f) return false;
    float end = q.sky_color.w;
    float sph = 16.0f * (1.0f - s) + 512.24994f * s;
    float cyl = 16.0f * (1.0f - s) + 512.0f * s;
    float f = fmax_r(linear_fog(sph, 0.0f, end), linear_fog(cyl, end, end));
    out = glerp(f4v(q.sky_color), f4v(q.fog_color), f);
    return true;
}

LW_DI float fan_alpha(const QuickSkyDev &q, V3 d) {  // sky.rs:427-461
    V3 c = f4v(q.fan[0]);
    float best_t = kINF, alpha = 0.0f;
    for (int k = 0; k < 16; k++) {
        V3 e1 = f4v(q.fan[k + 1]) - c, e2 = f4v(q.fan[k + 2]) - c;
        V3 pv = cross(d, e2);
        float det = dot(e1, pv);
        if (fabs_r(det) < 1e-6f) continue;
        float inv = __fdiv_rn(1.0f, det);
        V3 tv = -c;
        float u = dot(tv, pv) * inv;
        if (!(u >= 0.0f && u <= 1.0f)) continue;
        V3 qv = cross(tv, e1);
        float v = dot(d, qv) * inv;
        if (v < 0.0f || u + v > 1.0f) continue;
        float t = dot(e2, qv) * inv;
        if (t > 0.0f && t < best_t) {
            best_t = t;
            alpha = (1.0f - u - v) * q.fan[0].w;
        }
    }
    return alpha;
}

LW_DI float4 body(const float4 *b, V3 d, const uint32_t *atlas, uint32_t atlas_w) {  // sky.rs:464-486
    if (b[0].w == 0.0f || b[3].z <= 0.0f) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    V3 c = f4v(b[0]);
    float dn = dot(d, c);
    if (dn <= 0.0f) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    V3 qv = d * __fdiv_rn(dot(c, c), dn) - c;
    float lx = dot(qv, f4v(b[1])), lz = dot(qv, f4v(b[2]));
    if (fabs_r(lx) >= 1.0f || fabs_r(lz) >= 1.0f) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    float u = b[3].x + (lx * 0.5f + 0.5f) * b[3].z;
    float v = b[3].y + (lz * 0.5f + 0.5f) * b[3].w;
    uint32_t t = ldg(atlas + (to_u32(floorf(v)) * atlas_w + to_u32(floorf(u))));
    return make_float4(__fdiv_rn((float)(t & 0xFFu), 255.0f), __fdiv_rn((float)((t >> 8) & 0xFFu), 255.0f),
                       __fdiv_rn((float)((t >> 16) & 0xFFu), 255.0f), __fdiv_rn((float)(t >> 24), 255.0f));
}

LW_DI uint32_t star_hits(const QuickSkyDev &q, V3 d, const uint32_t *table) {  // sky.rs:489-505, :138-150
    V3 qd = v3(dot(f4v(q.star_rot[0]), d), dot(f4v(q.star_rot[1]), d), dot(f4v(q.star_rot[2]), d));
    float az = atan2f(qd.z, qd.x);
    float el = asinf(qd.y < -1.0f ? -1.0f : (qd.y > 1.0f ? 1.0f : qd.y));
    int ia = to_i32(floorf(__fdiv_rn(az + kPI, kTau) * (float)kStarBinsAz));
    int ie = to_i32(floorf(__fdiv_rn(el + kFRAC_PI_2, kPI) * (float)kStarBinsEl));
    ia = clamp_i(ia, 0, kStarBinsAz - 1);
    ie = clamp_i(ie, 0, kStarBinsEl - 1);
    const uint32_t b = (uint32_t)(ie * kStarBinsAz + ia), base = kStarBinsAz * kStarBinsEl + 1;
    uint32_t n = 0;
    for (uint32_t e = ldg(table + b), e_end = ldg(table + b + 1); e < e_end; e++) {
        const uint32_t *o = table + base + e * kStarWords;
        V3 c = v3(__uint_as_float(ldg(o)), __uint_as_float(ldg(o + 1)), __uint_as_float(ldg(o + 2)));
        V3 a1 = v3(__uint_as_float(ldg(o + 3)), __uint_as_float(ldg(o + 4)), __uint_as_float(ldg(o + 5)));
        V3 a2 = v3(__uint_as_float(ldg(o + 6)), __uint_as_float(ldg(o + 7)), __uint_as_float(ldg(o + 8)));
        float dn = dot(qd, c);
        if (dn <= 0.0f) continue;
        V3 p = qd * __fdiv_rn(dot(c, c), dn) - c;
        if (fabs_r(dot(p, a1)) < 1.0f && fabs_r(dot(p, a2)) < 1.0f) n++;
    }
    return n;
}

__global__ void k_sky_map(const QuickSkyDev q, const uint32_t *atlas, uint32_t atlas_w, const uint32_t *stars, uint32_t w,
                          uint32_t h, float *out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (i >= w || j >= h) return;
    float az = __fdiv_rn((float)i + 0.5f, (float)w) * kTau;  // map_direction (sky.rs:853-858)
    float el = __fdiv_rn((float)j + 0.5f, (float)h) * kPI - kFRAC_PI_2;
    V3 d = v3(cosf(el) * cosf(az), sinf(el), cosf(el) * sinf(az));
    V3 c = f4v(q.fog_color), dc;
    if (q.flags.x > 0.5f && sky_disc(q, d, dc)) c = dc;
    if (q.flags.y > 0.5f) c = glerp(c, f4v(q.sunrise), fan_alpha(q, d));
    float4 t = body(q.sun, d, atlas, atlas_w);
    c = min1(c + v3(t.x, t.y, t.z) * t.w);
    t = body(q.moon, d, atlas, atlas_w);
    c = min1(c + v3(t.x, t.y, t.z) * t.w);
    if (q.flags.z > 0.5f) {
        uint32_t n = star_hits(q, d, stars);
        for (uint32_t k = 0; k < n; k++) c = min1(c + v3(q.fog_dist.w, q.fog_dist.w, q.fog_dist.w));
    }
    c = v3(fmin_r(fmax_r(c.x, 0.0f), 1.0f), fmin_r(fmax_r(c.y, 0.0f), 1.0f), fmin_r(fmax_r(c.z, 0.0f), 1.0f));
    float *o = out + 3 * ((size_t)j * w + i);
    o[0] = powf(c.x, 2.2f);
    o[1] = powf(c.y, 2.2f);
    o[2] = powf(c.z, 2.2f);
}

}  // namespace

cudaError_t launch_sky_map(const void *quick_sky, const uint32_t *atlas, uint32_t atlas_w, const uint32_t *stars,
                           uint32_t w, uint32_t h, float *out, cudaStream_t st) {
    QuickSkyDev q;
    memcpy(&q, quick_sky, sizeof q);
    k_sky_map<<<dim3((w + 127) / 128, h), 128, 0, st>>>(q, atlas, atlas_w, stars, w, h, out);
    return cudaGetLastError();
}

}  // namespace lw
