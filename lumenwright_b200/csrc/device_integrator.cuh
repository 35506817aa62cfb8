// The reference integrator (crates/lumenwright-kernel/src/integrator.rs) as a per-lane state
// machine. `render_sample` traces a path ray, then, at a diffuse surface, up to eight sun shadow
// segments and one visibility ray per sampled emitter face, each from inside a branch that only
// some lanes of a warp take. Here every lane keeps its path in a `Path` record and each step of
// the kernel's loop traces exactly one ray per lane (path, shadow or emitter ray, whichever the
// lane needs next), then advances the lane's state machine to its next ray. The random draws, the
// order of the additions to the radiance and every comparison are the reference's, so a lane
// produces the reference's radiance for its (pixel, sample).
#pragma once

#include "device_scene.cuh"

namespace lw {

// ---- sky (integrator.rs:79-277) ---------------------------------------------------------------
LW_DI V3 rgb_from_hsl(float hue, float saturation, float lightness) {  // :108-127
    float c = fmin_r(1.0f, (1.0f - fabs_r(2.0f * lightness - 1.0f)) * saturation);
    float h = hue * 6.0f;
    float x = c * (1.0f - fabs_r(fmodf(h, 2.0f) - 1.0f));
    V3 rgb;
    if (h < 1.0f) rgb = v3(c, x, 0.0f);
    else if (h < 2.0f) rgb = v3(x, c, 0.0f);
    else if (h < 3.0f) rgb = v3(0.0f, c, x);
    else if (h < 4.0f) rgb = v3(0.0f, x, c);
    else if (h < 5.0f) rgb = v3(x, 0.0f, c);
    else rgb = v3(c, 0.0f, x);
    float m = fmax_r(0.0f, lightness - 0.5f * c);
    return rgb + v3(m, m, m);
}

LW_COLD V3 sky_radiance(const DevScene &S, const DevParams &P, V3 d) {  // :158-188
    float n = P.misc_f.z;
    if (n < 1.0f) return v3(0.0f, 0.0f, 0.0f);
    float theta = __fdiv_rn(atan2_r(d.z, d.x), 2.0f * kPI);
    theta = fmodf(fmodf(theta, 1.0f) + 1.0f, 1.0f);
    float phi = 1.0f - __fdiv_rn(acos_r(clamp_r(d.y, -1.0f, 1.0f)), kPI);
    float x = theta * n, y = phi * n;
    float fx = floorf(clamp_r(x, 0.0f, n - 1.0f));
    float fy = floorf(clamp_r(y, 0.0f, n - 1.0f));
    uint32_t m = to_u32(n) + 1u;
    uint32_t a00 = (to_u32(fx) * m + to_u32(fy)) * 3u;
    uint32_t a10 = (to_u32(fx + 1.0f) * m + to_u32(fy)) * 3u;
    uint32_t a01 = (to_u32(fx) * m + to_u32(fy + 1.0f)) * 3u;
    uint32_t a11 = (to_u32(fx + 1.0f) * m + to_u32(fy + 1.0f)) * 3u;
    float hsl[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        float s00 = ldg(S.sky + a00 + k), s10 = ldg(S.sky + a10 + k);
        float s01 = ldg(S.sky + a01 + k), s11 = ldg(S.sky + a11 + k);
        float y0 = s00 + (x - fx) * (s10 - s00);
        float y1 = s01 + (x - fx) * (s11 - s01);
        hsl[k] = y0 + (y - fy) * (y1 - y0);
    }
    return rgb_from_hsl(hsl[0], hsl[1], hsl[2]) * P.sky_sun.w;
}

LW_DI V3 sky_texel(const DevScene &S, uint32_t base, uint32_t w, float i, float j) {
    size_t k = (size_t)base + ((size_t)to_u32(j) * w + to_u32(i)) * 3u;
    return v3(ldg(S.sky + k), ldg(S.sky + k + 1), ldg(S.sky + k + 2));
}

LW_COLD V3 map_lookup(const DevScene &S, uint32_t base, float w, float h, V3 d) {  // :196-217
    float u = __fdiv_rn(atan2_r(d.z, d.x), 2.0f * kPI);
    u = fmodf(fmodf(u, 1.0f) + 1.0f, 1.0f);
    float v = 1.0f - __fdiv_rn(acos_r(clamp_r(d.y, -1.0f, 1.0f)), kPI);
    float x = u * w - 0.5f;
    float y = clamp_r(v * h - 0.5f, 0.0f, h - 1.0f);
    float fx = floorf(x), fy = floorf(y);
    float tx = x - fx, ty = y - fy;
    float i0 = fx < 0.0f ? w - 1.0f : fx;
    float i1 = fx + 1.0f >= w ? 0.0f : fx + 1.0f;
    float j1 = fmin_r(fy + 1.0f, h - 1.0f);
    uint32_t wu = to_u32(w);
    V3 top = sky_texel(S, base, wu, i0, fy) * (1.0f - tx) + sky_texel(S, base, wu, i1, fy) * tx;
    V3 bottom = sky_texel(S, base, wu, i0, j1) * (1.0f - tx) + sky_texel(S, base, wu, i1, j1) * tx;
    return top * (1.0f - ty) + bottom * ty;
}

// sky_lens (lens = true) or sky_light, with one inlined copy of each lookup.
LW_DI V3 sky_of(const DevScene &S, const DevParams &P, V3 d, bool lens) {
    if (P.sky_map.x < 1.0f) return sky_radiance(S, P, d);
    uint32_t base = lens ? 0u : to_u32(P.sky_map.x * P.sky_map.y) * 3u;
    return map_lookup(S, base, lens ? P.sky_map.x : P.sky_map.z, lens ? P.sky_map.y : P.sky_map.w, d);
}
LW_DI V3 sky_lens(const DevScene &S, const DevParams &P, V3 d) {  // :225-231
    if (P.sky_map.x < 1.0f) return sky_radiance(S, P, d);
    return map_lookup(S, 0u, P.sky_map.x, P.sky_map.y, d);
}
LW_DI V3 sky_light(const DevScene &S, const DevParams &P, V3 d) {  // :237-243
    if (P.sky_map.x < 1.0f) return sky_radiance(S, P, d);
    return map_lookup(S, to_u32(P.sky_map.x * P.sky_map.y) * 3u, P.sky_map.z, P.sky_map.w, d);
}

LW_COLD V3 sun_texture(const DevScene &S, const DevParams &P, V3 d) {  // :252-277
    float4 sprite = P.sun_sprite;
    if (sprite.z <= 0.0f || dot(d, f4v(P.sun_dir)) < 0.5f) return v3(0.0f, 0.0f, 0.0f);
    float width = P.sun_sv.w;
    float width2 = width * 2.0f;
    float a = 0.5f * kPI - acos_r(dot(d, f4v(P.sun_su))) + width;
    float b = 0.5f * kPI - acos_r(dot(d, f4v(P.sun_sv))) + width;
    if (a < 0.0f || a >= width2 || b < 0.0f || b >= width2) return v3(0.0f, 0.0f, 0.0f);
    float x = clamp_r(floorf(__fdiv_rn(a, width2) * sprite.z - 5e-8f), 0.0f, sprite.z - 1.0f);
    float y = clamp_r(floorf((1.0f - __fdiv_rn(b, width2)) * sprite.w - 5e-8f), 0.0f, sprite.w - 1.0f);
    return linear_rgb(S.gamma, texel(S, P, sprite.x + x + 0.5f, sprite.y + y + 0.5f)) * P.sun_su.w;
}

// ---- sampling (integrator.rs:280-302, 350-373) -------------------------------------------------
LW_DI V3 cosine_hemisphere(V3 n, uint32_t &rng) {
    float r1 = rng_next(rng);
    float r2 = rng_next(rng);
    float r = __fsqrt_rn(r1);
    float sin_phi, cos_phi;
    sin_cos_turns(r2, sin_phi, cos_phi);
    V3 t, b;
    onb(n, t, b);
    return normalize(t * (r * cos_phi) + b * (r * sin_phi) + n * __fsqrt_rn(fmax_r(1.0f - r1, 0.0f)));
}

LW_DI V3 sample_sun(const DevParams &P, uint32_t &rng) {
    V3 sun = f4v(P.sun_dir);
    float cos_max = P.sun_dir.w;
    float r1 = rng_next(rng);
    float r2 = rng_next(rng);
    float cos_t = 1.0f - r1 * (1.0f - cos_max);
    float sin_t = __fsqrt_rn(fmax_r(1.0f - cos_t * cos_t, 0.0f));
    float sin_phi, cos_phi;
    sin_cos_turns(r2, sin_phi, cos_phi);
    V3 t, b;
    onb(sun, t, b);
    return normalize(t * (sin_t * cos_phi) + b * (sin_t * sin_phi) + sun * cos_t);
}

LW_DI uint32_t pick(uint32_t n, float u) {
    uint32_t i = to_u32(u * (float)n);
    return i < n ? i : n - 1u;
}

// The cell of integer block coordinate b in cells of `cell` (an integer) blocks, floor(b / cell):
// exact in f32 for |b| < 2^24, which every block coordinate of a packable frame is: the quotient's
// rounding error, at most |b| / cell * 2^-24, is below 1 / cell, the least distance from a quotient
// that is not an integer to the integers.
LW_DI int cell_of_block(int b, float cell) { return to_i32(floorf(__fdiv_rn((float)b, cell))); }

// emitter_cell (integrator.rs:358-373). REB: p is in frame A, and the cell is found from p's
// block in the grid, floor(p) + A: for an integer cell size, floor((b + f) / size) =
// floor(b / size) for every fraction f in [0, 1), so this is the cell of the exact position.
template <bool REB = false>
LW_DI void emitter_cell(const DevScene &S, V3 p, uint32_t &start, uint32_t &count, const Frame &A = Frame{}) {
    const uint32_t *g = S.emitter_grid;
    float cell = (float)ldg(g);
    int sx = (int)ldg(g + 1), sy = (int)ldg(g + 2), sz = (int)ldg(g + 3);
    int cx, cy, cz;
    if (REB) {
        cx = cell_of_block(to_i32(floorf(p.x)) + A.x(), cell) - (int)ldg(g + 4);
        cy = cell_of_block(to_i32(floorf(p.y)) + A.y(), cell) - (int)ldg(g + 5);
        cz = cell_of_block(to_i32(floorf(p.z)) + A.z(), cell) - (int)ldg(g + 6);
    } else {
        cx = to_i32(floorf(__fdiv_rn(p.x, cell))) - (int)ldg(g + 4);
        cy = to_i32(floorf(__fdiv_rn(p.y, cell))) - (int)ldg(g + 5);
        cz = to_i32(floorf(__fdiv_rn(p.z, cell))) - (int)ldg(g + 6);
    }
    if (cx < 0 || cy < 0 || cz < 0 || cx >= sx || cy >= sy || cz >= sz) {
        start = 0u;
        count = 0u;
        return;
    }
    uint32_t i = (uint32_t)((cy * sz + cz) * sx + cx);
    start = ldg(g + EMITTER_GRID_HEADER + i * 2u);
    count = ldg(g + EMITTER_GRID_HEADER + i * 2u + 1u);
}

// ---- water (integrator.rs:477-534) ------------------------------------------------------------
LW_COLD bool water_interface(const DevParams &P, V3 pos, V3 d, V3 n, bool front, bool in_water, float eps,
                           uint32_t &rng, V3 &nd, V3 &no) {
    float ior = P.water_color.w;
    float eta = front ? __fdiv_rn(1.0f, ior) : ior;
    float cos_i = -dot(n, d);
    float sin2_t = eta * eta * fmax_r(1.0f - cos_i * cos_i, 0.0f);
    float r0 = __fdiv_rn(1.0f - ior, 1.0f + ior);
    r0 = r0 * r0;
    float m = 1.0f - cos_i;
    float fresnel = r0 + (1.0f - r0) * m * m * m * m * m;
    if (sin2_t >= 1.0f || rng_next(rng) < fresnel) {
        nd = normalize(d + n * (2.0f * cos_i));
        no = pos + n * eps;
        return in_water;
    }
    float cos_t = __fsqrt_rn(1.0f - sin2_t);
    nd = normalize(d * eta + n * (eta * cos_i - cos_t));
    no = pos - n * eps;
    return front;
}

// The water plane's height in frame A.
LW_DI float water_height(const DevParams &P, const Frame &A) { return P.water_plane.x - (float)A.y(); }

// water_plane (integrator.rs:511-526); o in frame A, where the grid's columns span [-A, size - A).
LW_DI bool water_plane(const DevParams &P, V3 o, V3 d, float &tp, const Frame &A = Frame{}) {
    if (P.water_plane.y == 0.0f || d.y == 0.0f) return false;
    float t = __fdiv_rn(water_height(P, A) - o.y, d.y);
    if (!(t > 0.0f && t < kINF)) return false;
    V3 at = o + d * t;
    float x0 = (float)(-A.x()), z0 = (float)(-A.z());
    float sx = (float)((int)(P.grid_dims.x * 16u) - A.x()), sz = (float)((int)(P.grid_dims.z * 16u) - A.z());
    if (at.x >= x0 && at.z >= z0 && at.x < sx && at.z < sz) return false;
    tp = t;
    return true;
}

LW_DI bool under_water_plane(const DevParams &P, V3 o, V3 d, const Frame &A = Frame{}) {
    return P.water_plane.y != 0.0f && o.y < water_height(P, A) && d.y <= 0.0f;
}

// ---- the per-lane path ----------------------------------------------------------------------
enum : uint32_t { K_EXTEND = 0, K_SHADOW = 1, K_EMIT = 2, K_IDLE = 3 };
// Emitter sampling modes of the state machine.
enum : uint32_t { E_SINGLE = 0, E_ALL = 1 };

struct Path {
    // the ray the lane traces next
    V3 o, d;
    float tmin, tmax;
    uint32_t kind;
    // the path (render_sample's locals, integrator.rs:558-569)
    V3 radiance, beta;
    uint32_t rng, bounces, events;
    bool specular, in_water;
    // next-event estimation at the current diffuse surface
    V3 n, origin;   // shading normal and offset origin
    V3 tr;          // sun transmittance so far
    float cos_l;
    uint32_t seg;   // shadow segments traced
    // emitter sampling (sample_emitters / sample_emitter / sample_emitter_face)
    V3 esum, fsum;  // the sum over the cell's emitters (ALL) and over an emitter's faces
    uint32_t list, count, k;   // the cell's index list, its length, the emitter being sampled
    uint32_t first, faces, f;  // that emitter's first quad, face count, face being sampled
    uint32_t emode, fmode;
    V3 eoff;
    float dist;
    // with chunk-origin rebasing, the frame (frame_word) that o and origin are held in
    uint32_t frame;
};

}  // namespace lw
