// A straight CUDA port of the reference's CUDA backend, the comparison point for the B200 kernels
// (the reference's own CUDA backend needs nightly Rust with the nvptx target, which this box does
// not have). It is a benchmark baseline, built as its own library (liblw_refport.so) apart from
// the product. It keeps the reference's structure on purpose:
//   * `pt_render` (crates/lumenwright-ptx/src/lib.rs:37-87): one thread per pixel in 16x16
//     blocks, `samples` path samples per launch summed into an f32 (r, g, b, n) accumulator;
//   * `render_sample` with its nested control flow: the shadow loop and the emitter sampling run
//     inside the branches of the event loop (crates/lumenwright-kernel/src/integrator.rs:539-709);
//   * `trace` on the reference's grid words: two top-level loads per step, the voxel id from the
//     packed brick word, n = eu x ev recomputed per quad test (trace.rs:37-290);
//   * the host side of CudaBackend::render_hq (crates/lumenwright/src/render/cuda.rs:77-184): the
//     seven buffers copied to the device for the call, batches of 1 to 64 spp doubling or halving
//     towards 150 ms a launch with a synchronize after each, the accumulator read back and
//     divided on the host, the buffers freed.
// The sky, sun-texture and emitter-cell helpers and the decoded-byte table are the product's
// (device_integrator.cuh): they are the reference's arithmetic and not where the time goes.
//
// The library also holds the benchmark's L2 read probe (lwr_l2_read_gbs), the peak the tracing
// kernel's scene reads are held against while the scene stays in L2.
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "device_integrator.cuh"
#include "refport.h"

namespace lw {
namespace refport {

struct RefScene {
    const uint32_t *grid;
    const uint4 *models;
    const float4 *quads;  // GpuQuad: 5 float4 each
    const uint32_t *atlas;
    const float4 *emitters;
    const uint32_t *emitter_grid;
    const float *sky;
    const float *gamma;
};

struct QuadRef {
    float4 p0, eu, ev, uv, uvt;
};
LW_DI QuadRef load_quad(const RefScene &S, uint32_t qi) {
    const float4 *q = S.quads + 5u * qi;
    return QuadRef{q[0], q[1], q[2], q[3], q[4]};
}

LW_DI uint32_t texel_ref(const RefScene &S, const DevParams &P, float u, float v) {
    int w = (int)P.off2.y, h = (int)P.off2.z;
    int x = clamp_i(to_i32(floorf(u)), 0, w - 1);
    int y = clamp_i(to_i32(floorf(v)), 0, h - 1);
    return S.atlas[(uint32_t)(y * w + x)];
}

// test_quad (trace.rs:81-109) with intersect_quad (:37-58), as written.
LW_DI void test_quad_ref(const RefScene &S, const DevParams &P, uint32_t qi, V3 o, V3 d, float tmin, Hit &best) {
    QuadRef q = load_quad(S, qi);
    float reach = (best.quad != NO_QUAD && qi > best.quad) ? best.t + COPLANAR : best.t;
    V3 eu = f4v(q.eu), ev = f4v(q.ev);
    V3 n = cross(eu, ev);
    float denom = dot(n, d);
    if (fabs_r(denom) < 1e-12f) return;
    V3 p0 = f4v(q.p0);
    float t = __fdiv_rn(dot(n, p0 - o), denom);
    if (!(t > tmin && t < reach)) return;
    V3 p = (o + d * t) - p0;
    float nn = dot(n, n);
    float s = __fdiv_rn(dot(cross(p, ev), n), nn);
    float tt = __fdiv_rn(dot(cross(eu, p), n), nn);
    if (s < 0.0f || s > 1.0f || tt < 0.0f || tt > 1.0f) return;
    uint32_t flags = __float_as_uint(q.p0.w);
    if ((flags & FLAG_FRONT_ONLY) && dot(cross(ev, eu), d) >= 0.0f) return;
    float sc = fmin_r(fmax_r(s, 0.0005f), 0.9995f);
    float tc = fmin_r(fmax_r(tt, 0.0005f), 0.9995f);
    uint32_t tx = texel_ref(S, P, q.uv.x + sc * q.uv.z + tc * q.uvt.x, q.uv.y + sc * q.uv.w + tc * q.uvt.y);
    uint32_t alpha = tx >> 24, mode = flags & FLAG_ALPHA_MASK;
    if ((mode == ALPHA_CUTOUT && alpha < 128u) || (mode == ALPHA_TRANSLUCENT && alpha == 0u)) return;
    best = Hit{t, qi, tx, s, tt};
}

// trace (trace.rs:137-290) on the reference grid.
LW_DI Hit trace_ref(const RefScene &S, const DevParams &P, V3 o, V3 d, float tmin, float tmax) {
    const uint32_t dx = P.grid_dims.x, dy = P.grid_dims.y, dz = P.grid_dims.z;
    V3 size = v3((float)(dx * 16u), (float)(dy * 16u), (float)(dz * 16u));
    V3 inv = v3(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z));
    V3 ta = vmul(v3(0.0f, 0.0f, 0.0f) - o, inv);
    V3 tb = vmul(size - o, inv);
    float t_enter = fmax_r(fmax_r(fmin_r(ta.x, tb.x), fmin_r(ta.y, tb.y)), fmin_r(ta.z, tb.z));
    float t_exit = fmin_r(fmin_r(fmax_r(ta.x, tb.x), fmax_r(ta.y, tb.y)), fmax_r(ta.z, tb.z));
    float t = fmax_r(t_enter, 0.0f);
    float t_end = fmin_r(t_exit, tmax);
    if (t > t_end) return no_hit();
    V3 start = o + d * (t + 1e-4f);
    int gs[3] = {(int)dx * 16, (int)dy * 16, (int)dz * 16};
    int cell[3] = {clamp_i(to_i32(floorf(start.x)), 0, gs[0] - 1), clamp_i(to_i32(floorf(start.y)), 0, gs[1] - 1),
                   clamp_i(to_i32(floorf(start.z)), 0, gs[2] - 1)};
    int step[3] = {sgn(d.x), sgn(d.y), sgn(d.z)};
    float next[3];
    for (int a = 0; a < 3; a++) next[a] = next_boundary(vget(o, a), vget(inv, a), cell[a], step[a]);
    float best_t = t_end + 1e-3f;
    for (uint32_t it = 0; it < MAX_STEPS; it++) {
        uint32_t bx = (uint32_t)(cell[0] >> 4), by = (uint32_t)(cell[1] >> 4), bz = (uint32_t)(cell[2] >> 4);
        uint32_t b = (by * dz + bz) * dx + bx;
        uint32_t entry = S.grid[P.off.x + b];
        uint32_t ov = S.grid[P.off.z + b];
        if (entry == EMPTY && ov == EMPTY) {
            int bc[3] = {(int)bx, (int)by, (int)bz};
            float t_out = kINF;
            int axis = 0;
            for (int a = 0; a < 3; a++) {
                if (step[a] != 0) {
                    int bound = step[a] > 0 ? (bc[a] + 1) * 16 : bc[a] * 16;
                    float tt = ((float)bound - vget(o, a)) * vget(inv, a);
                    if (tt < t_out) {
                        t_out = tt;
                        axis = a;
                    }
                }
            }
            if (t_out > t_end) break;
            V3 pos = o + d * t_out;
            for (int a = 0; a < 3; a++) {
                if (a == axis) cell[a] = step[a] > 0 ? (bc[a] + 1) * 16 : bc[a] * 16 - 1;
                else cell[a] = clamp_i(to_i32(floorf(vget(pos, a))), bc[a] * 16, bc[a] * 16 + 15);
            }
            if (cell[axis] < 0 || cell[axis] >= gs[axis]) break;
            for (int a = 0; a < 3; a++) next[a] = next_boundary(vget(o, a), vget(inv, a), cell[a], step[a]);
            t = t_out;
            continue;
        }
        float t_cell_exit = fmin_r(next[0], fmin_r(next[1], next[2]));
        float t_lo = fmax_r(t - 1e-4f, tmin);
        float t_hi = t_cell_exit + 1e-4f;
        uint32_t model;
        if (entry == EMPTY) model = 0;
        else if (entry & UNIFORM) model = entry & ~UNIFORM;
        else {
            uint32_t local = (uint32_t)((((cell[1] & 15) * 16 + (cell[2] & 15)) * 16) + (cell[0] & 15));
            uint32_t w = S.grid[P.off.y + entry * 2048u + (local >> 1)];
            model = (w >> ((local & 1u) * 16u)) & 0xFFFFu;
        }
        Hit cand = no_hit();
        cand.t = fmin_r(t_hi, best_t);
        if (model != 0) {
            uint4 m = S.models[model];
            V3 lo = o - v3((float)cell[0], (float)cell[1], (float)cell[2]);
            for (uint32_t i = 0; i < m.y; i++) test_quad_ref(S, P, m.x + i, lo, d, t_lo, cand);
        }
        if (ov != EMPTY) {
            uint32_t local = (uint32_t)((((cell[1] & 15) * 16 + (cell[2] & 15)) * 16) + (cell[0] & 15));
            uint32_t base = P.off.w + ov * OV_CELL_WORDS + local * 2u;
            uint32_t off = S.grid[base], count = S.grid[base + 1];
            for (uint32_t i = 0; i < count; i++) test_quad_ref(S, P, S.grid[P.off2.x + off + i], o, d, t_lo, cand);
        }
        if (cand.quad != NO_QUAD) return cand;
        int axis = next[0] < next[1] ? (next[0] < next[2] ? 0 : 2) : (next[1] < next[2] ? 1 : 2);
        t = next[axis];
        if (t > t_end) break;
        cell[axis] += step[axis];
        if (cell[axis] < 0 || cell[axis] >= gs[axis]) break;
        next[axis] = next_boundary(vget(o, axis), vget(inv, axis), cell[axis], step[axis]);
    }
    return no_hit();
}

LW_DI V3 shadow_ref(const RefScene &S, const DevParams &P, V3 o, V3 d, float tmax) {  // integrator.rs:319-346
    float eps = P.misc_f.y;
    V3 tr = v3(1.0f, 1.0f, 1.0f);
    for (int i = 0; i < 8; i++) {
        Hit h = trace_ref(S, P, o, d, eps, tmax);
        if (h.quad == NO_QUAD) return tr;
        QuadRef q = load_quad(S, h.quad);
        uint32_t flags = __float_as_uint(q.p0.w);
        if (flags & FLAG_WATER) {
            if (dot(cross(f4v(q.ev), f4v(q.eu)), d) > 0.0f) tr = vmul(tr, transmittance(f4v(P.water_color), h.t));
        } else if ((flags & FLAG_ALPHA_MASK) == ALPHA_TRANSLUCENT) {
            float a = __fdiv_rn((float)(h.texel >> 24), 255.0f);
            V3 col = vmul(linear_rgb(S.gamma, h.texel), linear_rgb(S.gamma, __float_as_uint(q.eu.w)));
            tr = vmul(tr, lerp(v3(1.0f, 1.0f, 1.0f), col, a));
        } else {
            return v3(0.0f, 0.0f, 0.0f);
        }
        o = o + d * (h.t + eps);
        tmax -= h.t + eps;
    }
    return tr;
}

LW_DI V3 face_ref(const RefScene &S, const DevParams &P, V3 origin, V3 n, float4 e0, uint32_t face, float scaler,
                  uint32_t &rng) {  // integrator.rs:381-414
    QuadRef q = load_quad(S, __float_as_uint(e0.w) + face);
    float s = rng_next(rng), t = rng_next(rng);
    V3 at = f4v(e0) + f4v(q.p0) + f4v(q.eu) * s + f4v(q.ev) * t;
    V3 to = at - origin;
    if (dot(to, n) <= 0.0f) return v3(0.0f, 0.0f, 0.0f);
    float dist = vlength(to);
    V3 l = vdiv(to, dist);
    float eps = P.misc_f.y;
    Hit h = trace_ref(S, P, origin, l, eps, dist + 2.0f * eps);
    if (h.quad == NO_QUAD || fabs_r(h.t - dist) >= 2.0f * eps) return v3(0.0f, 0.0f, 0.0f);
    V3 nq = cross(f4v(q.ev), f4v(q.eu));
    float area = vlength(nq);
    float cos_l = __fdiv_rn(fabs_r(dot(nq, l)), area);
    QuadRef hq = load_quad(S, h.quad);
    V3 c = vmul(linear_rgb(S.gamma, h.texel), linear_rgb(S.gamma, __float_as_uint(hq.eu.w)));
    return c * (__fdiv_rn(cos_l, fmax_r(dist * dist, 1.0f)) * area * q.ev.w * P.misc_f.x * scaler);
}

LW_DI V3 emitter_ref(const RefScene &S, const DevParams &P, V3 origin, V3 n, uint32_t i, uint32_t &rng) {
    float4 e0 = S.emitters[2u * i], e1 = S.emitters[2u * i + 1u];
    uint32_t faces = __float_as_uint(e1.x);
    if (faces == 0) return v3(0.0f, 0.0f, 0.0f);
    if (P.emitter.x == EMITTER_SAMPLING_ONE) return face_ref(S, P, origin, n, e0, pick(faces, rng_next(rng)), 1.0f, rng);
    V3 sum = v3(0.0f, 0.0f, 0.0f);
    for (uint32_t f = 0; f < faces; f++) sum = sum + face_ref(S, P, origin, n, e0, f, __fdiv_rn(1.0f, (float)faces), rng);
    return sum;
}

LW_DI V3 sample_emitters_ref(const RefScene &S, const DevParams &P, V3 pos, V3 origin, V3 n, uint32_t &rng) {
    DevScene D{};
    D.emitter_grid = S.emitter_grid;
    uint32_t start, count;
    emitter_cell(D, pos, start, count);
    if (count == 0) return v3(0.0f, 0.0f, 0.0f);
    const uint32_t *g = S.emitter_grid;
    uint32_t list = EMITTER_GRID_HEADER + g[1] * g[2] * g[3] * 2u + start;
    uint32_t st = P.emitter.x;
    if (st == EMITTER_SAMPLING_ONE || st == EMITTER_SAMPLING_ONE_BLOCK) {
        uint32_t i = g[list + pick(count, rng_next(rng))];
        return emitter_ref(S, P, origin, n, i, rng) * kPI;
    }
    if (st == EMITTER_SAMPLING_ALL) {
        V3 sum = v3(0.0f, 0.0f, 0.0f);
        for (uint32_t k = 0; k < count; k++) sum = sum + emitter_ref(S, P, origin, n, g[list + k], rng);
        return sum * __fdiv_rn(kPI, (float)count);
    }
    return v3(0.0f, 0.0f, 0.0f);
}

// render_sample (integrator.rs:539-709) as written, see-through quads included.
LW_DI V3 render_sample_ref(const RefScene &S, const DevParams &P, const DevScene &Sv, uint32_t px, uint32_t py,
                           uint32_t sample) {
    Path p;
    {
        uint32_t width = P.frame.x, height = P.frame.y;
        p.rng = rng_new(py * width + px, sample, P.misc_u.x);
        float jx = rng_next(p.rng), jy = rng_next(p.rng);
        float sx = (__fdiv_rn(2.0f * ((float)px + jx), (float)width) - 1.0f) * P.cam_fwd.w * P.cam_pos.w;
        float sy = (1.0f - __fdiv_rn(2.0f * ((float)py + jy), (float)height)) * P.cam_pos.w;
        p.d = normalize(f4v(P.cam_fwd) + f4v(P.cam_right) * sx + f4v(P.cam_up) * sy);
        p.o = f4v(P.cam_pos);
    }
    V3 radiance = v3(0.0f, 0.0f, 0.0f), beta = v3(1.0f, 1.0f, 1.0f);
    uint32_t bounces = 0;
    bool specular = true, in_water = false;
    uint32_t strategy = P.misc_u.w > 0u ? P.emitter.x : EMITTER_SAMPLING_NONE;
    float tmin = 0.0f, eps = P.misc_f.y;
    V3 sigma = f4v(P.water_color), o = p.o, d = p.d;
    for (uint32_t ev = 0; ev < MAX_EVENTS; ev++) {
        Hit h = trace_ref(S, P, o, d, tmin, kINF);
        bool found = h.quad != NO_QUAD, forced = false;
        if (bounces == 0 && P.see_through.y > 0u && found && !is_see_through(P, h.quad)) {
            Hit st = no_hit();
            for (uint32_t i = 0; i < P.see_through.y; i++) test_quad_ref(S, P, P.see_through.x + i, o, d, h.t, st);
            if (st.quad != NO_QUAD) {
                QuadRef sq = load_quad(S, st.quad);
                if ((__float_as_uint(sq.p0.w) & FLAG_ALPHA_MASK) == ALPHA_TRANSLUCENT) {
                    if (rng_next(p.rng) < __fdiv_rn((float)(st.texel >> 24), 255.0f)) {
                        h = st;
                        forced = true;
                    }
                } else {
                    h = st;
                }
            }
        }
        float tp;
        if (water_plane(P, o, d, tp) && (!found || tp < h.t)) {
            if (in_water) beta = vmul(beta, transmittance(sigma, tp));
            bool front = d.y < 0.0f;
            V3 nd, no;
            in_water = water_interface(P, o + d * tp, d, v3(0.0f, front ? 1.0f : -1.0f, 0.0f), front, in_water, eps, p.rng, nd, no);
            d = nd;
            o = no;
            specular = true;
            tmin = 0.0f;
            continue;
        }
        if (!found) {
            if (!in_water && !under_water_plane(P, o, d)) {
                radiance = radiance + vmul(beta, bounces == 0 ? sky_lens(Sv, P, d) : sky_light(Sv, P, d));
                if (specular && bounces == 0) radiance = radiance + vmul(beta, sun_texture(Sv, P, d));
            }
            break;
        }
        if (in_water) beta = vmul(beta, transmittance(sigma, h.t));
        QuadRef q = load_quad(S, h.quad);
        uint32_t flags = __float_as_uint(q.p0.w);
        V3 pos = o + d * h.t;
        float alpha = __fdiv_rn((float)(h.texel >> 24), 255.0f);
        V3 albedo = vmul(linear_rgb(S.gamma, h.texel), linear_rgb(S.gamma, __float_as_uint(q.eu.w)));
        V3 n = normalize(cross(f4v(q.ev), f4v(q.eu)));
        bool front = true;
        if (!(dot(n, d) < 0.0f)) {
            n = -n;
            front = false;
        }
        if (flags & FLAG_WATER) {
            V3 nd, no;
            in_water = water_interface(P, pos, d, n, front, in_water, eps, p.rng, nd, no);
            d = nd;
            o = no;
            specular = true;
            tmin = 0.0f;
            continue;
        }
        if (!forced && (flags & FLAG_ALPHA_MASK) == ALPHA_TRANSLUCENT && rng_next(p.rng) >= alpha) {
            beta = vmul(beta, lerp(v3(1.0f, 1.0f, 1.0f), albedo, alpha));
            o = pos + d * eps;
            tmin = 0.0f;
            continue;
        }
        if (bounces >= P.frame.w) break;
        float emittance = q.ev.w * P.misc_f.x;
        bool emits = emittance > 0.0f && (P.emitter.y == 0u || strategy == EMITTER_SAMPLING_NONE || bounces == 0u);
        if (emits) radiance = radiance + vmul(beta, vmul(albedo, albedo)) * emittance;
        bounces += 1;
        V3 origin = pos + n * eps;
        V3 sun = f4v(P.sun_dir);
        float sin_r = __fsqrt_rn(fmax_r(1.0f - P.sun_dir.w * P.sun_dir.w, 0.0f));
        bool lit = P.sun_color.x > 0.0f || P.sun_color.y > 0.0f || P.sun_color.z > 0.0f;
        if (lit && dot(n, sun) > -sin_r && P.sun_dir.y > -sin_r) {
            V3 l = sample_sun(P, p.rng);
            float cos_l = dot(n, l);
            if (cos_l > 0.0f && l.y >= 0.0f) {
                V3 tr = shadow_ref(S, P, origin, l, kINF);
                radiance = radiance + vmul(vmul(vmul(beta, albedo), f4v(P.sun_color)), tr) * cos_l;
            }
        }
        if (!emits && strategy != EMITTER_SAMPLING_NONE)
            radiance = radiance + vmul(vmul(beta, albedo), sample_emitters_ref(S, P, pos, origin, n, p.rng));
        beta = vmul(beta, albedo);
        if (bounces >= 3u) {
            float q_rr = clamp_r(max_elem(beta), 0.05f, 0.95f);
            if (rng_next(p.rng) > q_rr) break;
            beta = vdiv(beta, q_rr);
        }
        d = cosine_hemisphere(n, p.rng);
        o = origin;
        tmin = 0.0f;
        specular = false;
    }
    return radiance;
}

// pt_render (crates/lumenwright-ptx/src/lib.rs:37-87).
__global__ void pt_render_ref(const RefScene S, const DevParams P, const DevScene Sv, float4 *accum, uint32_t sample_start,
                              uint32_t samples) {
    uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= P.frame.x || y >= P.frame.y) return;
    uint32_t idx = y * P.frame.x + x;
    float4 acc = accum[idx];
    for (uint32_t s = 0; s < samples; s++) {
        V3 c = render_sample_ref(S, P, Sv, x, y, sample_start + s);
        if (isfinite(c.x) && isfinite(c.y) && isfinite(c.z)) {
            acc.x += c.x;
            acc.y += c.y;
            acc.z += c.z;
        }
        acc.w += 1.0f;
    }
    accum[idx] = acc;
}

__global__ void k_finalize_ref(const float4 *acc, uint32_t n, float *out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 a = acc[i];
    float cnt = fmax_r(a.w, 1.0f);
    out[3 * i] = __fdiv_rn(a.x, cnt);
    out[3 * i + 1] = __fdiv_rn(a.y, cnt);
    out[3 * i + 2] = __fdiv_rn(a.z, cnt);
}

}  // namespace refport

}  // namespace lw

namespace {

using namespace lw;

// gamma_to_linear (crates/lumenwright-kernel/src/math.rs:183-216) per byte value, with the
// reference's f32 `ln` and the platform expf, as the product's context builds its table.
float ref_ln(float x) {
    if (x <= 0.0f) return x == 0.0f ? -INFINITY : NAN;
    uint32_t bits;
    std::memcpy(&bits, &x, 4);
    int32_t e = (int32_t)((bits >> 23) & 0xFFu) - 127;
    uint32_t mb = (bits & 0x007FFFFFu) | 0x3F800000u;
    float m;
    std::memcpy(&m, &mb, 4);
    if (m > 1.41421356237309504880f) {
        m *= 0.5f;
        e += 1;
    }
    float sv = (m - 1.0f) / (m + 1.0f);
    float s2 = sv * sv;
    float series = 2.0f * sv * (1.0f + s2 * (1.0f / 3.0f + s2 * (1.0f / 5.0f + s2 * (1.0f / 7.0f + s2 * (1.0f / 9.0f)))));
    return (float)e * 0.693147180559945309417f + series;
}

float ref_gamma_to_linear(float c) { return c <= 0.0f ? 0.0f : expf(2.2f * ref_ln(c)); }

struct Bufs {
    std::vector<void *> ptrs;
    ~Bufs() {
        for (void *p : ptrs) cudaFree(p);
    }
    template <typename T>
    cudaError_t copy(T **dst, const void *src, size_t bytes, cudaStream_t st) {
        void *p = nullptr;
        cudaError_t e = cudaMalloc(&p, bytes ? bytes : 4);
        if (e != cudaSuccess) return e;
        ptrs.push_back(p);
        *dst = (T *)p;
        return bytes ? cudaMemcpyAsync(p, src, bytes, cudaMemcpyHostToDevice, st) : cudaSuccess;
    }
};

}  // namespace

namespace {

// Every thread reads 16-byte words of the buffer in a grid-stride loop, `passes` times over, and
// keeps an XOR of what it read so the loads are not dropped.
__global__ void k_l2_read(const uint4 *buf, uint64_t n, uint32_t passes, uint32_t *sink) {
    uint32_t x = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint32_t p = 0; p < passes; p++)
        for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
            uint4 v = __ldcg(buf + i);
            x ^= v.x ^ v.y ^ v.z ^ v.w;
        }
    if (x == 0x9E3779B9u) sink[0] = x;  // almost never taken; keeps x live
}

}  // namespace

extern "C" int lwr_l2_read_gbs(int device, uint64_t bytes, uint32_t passes, double *gbs) {
    if (!gbs || bytes < 16 || passes == 0) return 1;
    if (cudaSetDevice(device) != cudaSuccess) return 7;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    uint4 *buf = nullptr;
    uint32_t *sink = nullptr;
    const uint64_t n = bytes / 16;
    if (cudaMalloc(&buf, n * 16) != cudaSuccess) return 3;
    if (cudaMalloc(&sink, 4) != cudaSuccess) {
        cudaFree(buf);
        return 3;
    }
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaMemset(buf, 0x5A, n * 16);
    const int blocks = sms * 8, threads = 256;
    k_l2_read<<<blocks, threads>>>(buf, n, 2, sink);  // brings the buffer into L2
    cudaEventRecord(a);
    k_l2_read<<<blocks, threads>>>(buf, n, passes, sink);
    cudaEventRecord(b);
    cudaError_t e = cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    *gbs = e == cudaSuccess && ms > 0.f ? (double)n * 16.0 * passes / (ms * 1e-3) / 1e9 : 0.0;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(buf);
    cudaFree(sink);
    return e == cudaSuccess ? 0 : 5;
}

extern "C" int lwr_render_hq(int device, const lw_scene_desc *sc, const lw_params *params, const float *sky,
                             uint64_t sky_len, uint32_t spp, float *out_rgb, lwr_timing *timing) {
    if (!sc || !params || !out_rgb) return 1;
    auto t_start = std::chrono::steady_clock::now();
    if (cudaSetDevice(device) != cudaSuccess) return 7;
    if (spp < 1) spp = 1;
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return 5;
    cudaEvent_t a = nullptr, b = nullptr;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    DevParams P;
    std::memcpy(&P, params, sizeof P);
    const uint32_t w = params->frame[0], h = params->frame[1];
    float lut[256];
    for (int k = 0; k < 256; k++) lut[k] = ref_gamma_to_linear((float)k / 255.0f);
    int rc = 0;
    {
        Bufs B;
        refport::RefScene S{};
        const float *dsky = nullptr, *dgamma = nullptr;
        float4 *acc = nullptr;
        cudaError_t e = B.copy(&S.grid, sc->grid, sc->grid_len * 4, st);
        if (e == cudaSuccess) e = B.copy(&S.models, sc->models, sc->models_len * 16, st);
        if (e == cudaSuccess) e = B.copy(&S.quads, sc->quads, sc->quads_len * 80, st);
        if (e == cudaSuccess) e = B.copy(&S.atlas, sc->atlas, sc->atlas_len * 4, st);
        if (e == cudaSuccess) e = B.copy(&S.emitters, sc->emitters, sc->emitters_len * 32, st);
        if (e == cudaSuccess) e = B.copy(&S.emitter_grid, sc->emitter_grid, sc->emitter_grid_len * 4, st);
        if (e == cudaSuccess) e = B.copy(&dsky, sky, sky_len * 4, st);
        if (e == cudaSuccess) e = B.copy(&dgamma, lut, sizeof lut, st);
        if (e == cudaSuccess) {  // the accumulator, zeroed (cuda.rs:113)
            void *p = nullptr;
            e = cudaMalloc(&p, sizeof(float4) * (size_t)w * h);
            if (e == cudaSuccess) {
                B.ptrs.push_back(p);
                acc = (float4 *)p;
                e = cudaMemsetAsync(acc, 0, sizeof(float4) * (size_t)w * h, st);
            }
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        S.sky = dsky;
        S.gamma = dgamma;
        DevScene Sv{};
        Sv.atlas = S.atlas;
        Sv.emitters = S.emitters;
        Sv.emitter_grid = S.emitter_grid;
        Sv.sky = dsky;
        Sv.gamma = dgamma;
        auto t_up = std::chrono::steady_clock::now();
        double kernel_ms = 0.0;
        uint32_t launches = 0, done = 0, batch = 1;
        dim3 block(16, 16, 1), grd((w + 15) / 16, (h + 15) / 16, 1);
        while (e == cudaSuccess && done < spp) {
            uint32_t n = batch < spp - done ? batch : spp - done;
            auto t0 = std::chrono::steady_clock::now();
            e = cudaEventRecord(a, st);
            if (e == cudaSuccess) {
                refport::pt_render_ref<<<grd, block, 0, st>>>(S, P, Sv, acc, done, n);
                e = cudaGetLastError();
            }
            if (e == cudaSuccess) e = cudaEventRecord(b, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) break;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, a, b);
            kernel_ms += ms;
            launches++;
            double took = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            done += n;
            if (took < 75.0) batch = batch * 2 < 64 ? batch * 2 : 64;
            else if (took > 300.0 && batch > 1) batch /= 2;
        }
        if (e == cudaSuccess) {
            std::vector<float> host((size_t)4 * w * h);
            e = cudaMemcpy(host.data(), acc, host.size() * 4, cudaMemcpyDeviceToHost);
            for (size_t i = 0; e == cudaSuccess && i < (size_t)w * h; i++) {
                float cnt = host[4 * i + 3] > 1.0f ? host[4 * i + 3] : 1.0f;
                for (int c = 0; c < 3; c++) out_rgb[3 * i + c] = host[4 * i + c] / cnt;
            }
        }
        if (e != cudaSuccess) rc = e == cudaErrorMemoryAllocation ? 3 : 5;
        if (timing) {
            timing->kernel_ms = kernel_ms;
            timing->upload_ms = std::chrono::duration<double, std::milli>(t_up - t_start).count();
            timing->launches = launches;
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaStreamDestroy(st);
    if (timing) timing->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    return rc;
}
