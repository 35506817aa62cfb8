// The path-tracing kernels: the persistent render kernel with its per-lane path state machine
// (replacing `pt_render`, crates/lumenwright-ptx/src/lib.rs:37-87), the per-pixel reduction of
// its partial sums, and the parity kernels (trace, voxel lookup).
#include "device_integrator.cuh"
#include "internal.h"

namespace lw {

// Next step of a lane's state machine after a trace or between two of them.
enum Act : uint32_t {
    A_TRACE,            // the lane's next ray is set: trace it
    A_END,              // the path is over: `radiance` is the sample's value
    A_CONTINUE,         // trace the next path ray, unless the path has had MAX_EVENTS events
    A_SUN_DONE,         // add the sun's light (transmittance in `tr`)
    A_EMIT_START,       // sample the emitters of the surface's cell
    A_BEGIN_EMITTER,    // sample emitter `k` of the cell (or the one picked)
    A_START_FACE,       // sample face `f` of the current emitter
    A_FACE_DONE,        // a face gave `val`
    A_EMITTER_DONE,     // an emitter gave `val`
    A_EMIT_FINISH,      // the emitters gave `val`: add it
    A_FINISH_SURFACE,   // Russian roulette and the next direction
};

// The camera ray of sample `sample` at pixel (px, py) (integrator.rs:545-569).
LW_DI void begin_sample(Path &p, const DevParams &P, uint32_t px, uint32_t py, uint32_t sample) {
    uint32_t width = P.frame.x, height = P.frame.y;
    p.rng = rng_new(py * width + px, sample, P.misc_u.x);
    float tan_half = P.cam_pos.w, aspect = P.cam_fwd.w;
    float jx = rng_next(p.rng);
    float jy = rng_next(p.rng);
    float sx = (__fdiv_rn(2.0f * ((float)px + jx), (float)width) - 1.0f) * aspect * tan_half;
    float sy = (1.0f - __fdiv_rn(2.0f * ((float)py + jy), (float)height)) * tan_half;
    p.d = normalize(f4v(P.cam_fwd) + f4v(P.cam_right) * sx + f4v(P.cam_up) * sy);
    p.o = f4v(P.cam_pos);
    p.radiance = v3(0.0f, 0.0f, 0.0f);
    p.beta = v3(1.0f, 1.0f, 1.0f);
    p.bounces = 0;
    p.events = 0;
    p.specular = true;
    p.in_water = false;
    p.tmin = 0.0f;
    p.tmax = kINF;
    p.kind = K_EXTEND;
}

LW_DI uint32_t strategy_of(const DevParams &P) { return P.misc_u.w > 0u ? P.emitter.x : EMITTER_SAMPLING_NONE; }

// The result of a path ray (the body of render_sample's event loop, integrator.rs:571-706).
LW_DI Act on_extend(Path &p, const DevScene &S, const DevParams &P, Hit h) {
    const float eps = P.misc_f.y;
    p.events++;
    bool found = h.quad != NO_QUAD;
    bool forced = false;
    if (p.bounces == 0 && P.see_through.y > 0u && found && !is_see_through(P, h.quad)) {
        Hit st = see_through_hit(S, P, p.o, p.d, h.t);
        if (st.quad != NO_QUAD) {
            uint32_t sflags = __float_as_uint(ldg(&S.quads[st.quad].p0_flags).w);
            if ((sflags & FLAG_ALPHA_MASK) == ALPHA_TRANSLUCENT) {
                if (rng_next(p.rng) < __fdiv_rn((float)(st.texel >> 24), 255.0f)) {
                    h = st;
                    forced = true;
                }
            } else {
                h = st;
            }
        }
    }
    const V3 sigma = f4v(P.water_color);
    float tp;
    if (water_plane(P, p.o, p.d, tp) && (!found || tp < h.t)) {
        if (p.in_water) p.beta = vmul(p.beta, transmittance(sigma, tp));
        bool front = p.d.y < 0.0f;
        V3 n = v3(0.0f, front ? 1.0f : -1.0f, 0.0f);
        V3 nd, no;
        p.in_water = water_interface(P, p.o + p.d * tp, p.d, n, front, p.in_water, eps, p.rng, nd, no);
        p.d = nd;
        p.o = no;
        p.specular = true;
        p.tmin = 0.0f;
        return A_CONTINUE;
    }
    if (!found) {
        if (!p.in_water && !under_water_plane(P, p.o, p.d)) {
            if (p.bounces == 0) p.radiance = p.radiance + vmul(p.beta, sky_lens(S, P, p.d));
            else p.radiance = p.radiance + vmul(p.beta, sky_light(S, P, p.d));
            if (p.specular && p.bounces == 0) p.radiance = p.radiance + vmul(p.beta, sun_texture(S, P, p.d));
        }
        return A_END;
    }
    if (p.in_water) p.beta = vmul(p.beta, transmittance(sigma, h.t));
    const DevQuad *q = S.quads + h.quad;
    float4 qn = ldg(&q->n_nn);
    uint32_t flags = __float_as_uint(ldg(&q->p0_flags).w);
    uint32_t tint = __float_as_uint(ldg(&q->eu_tint).w);
    float qemit = ldg(&q->ev_em).w;
    V3 pos = p.o + p.d * h.t;
    float alpha = __fdiv_rn((float)(h.texel >> 24), 255.0f);
    V3 albedo = vmul(linear_rgb(S.gamma, h.texel), linear_rgb(S.gamma, tint));
    // shading_normal (integrator.rs:308-315): normal() = ev x eu = -(eu x ev), exactly.
    V3 n = normalize(-f4v(qn));
    bool front = true;
    if (!(dot(n, p.d) < 0.0f)) {
        n = -n;
        front = false;
    }
    if (flags & FLAG_WATER) {
        V3 nd, no;
        p.in_water = water_interface(P, pos, p.d, n, front, p.in_water, eps, p.rng, nd, no);
        p.d = nd;
        p.o = no;
        p.specular = true;
        p.tmin = 0.0f;
        return A_CONTINUE;
    }
    if (!forced && (flags & FLAG_ALPHA_MASK) == ALPHA_TRANSLUCENT && rng_next(p.rng) >= alpha) {
        p.beta = vmul(p.beta, lerp(v3(1.0f, 1.0f, 1.0f), albedo, alpha));
        p.o = pos + p.d * eps;
        p.tmin = 0.0f;
        return A_CONTINUE;
    }
    if (p.bounces >= P.frame.w) return A_END;
    const uint32_t strategy = strategy_of(P);
    float emittance = qemit * P.misc_f.x;
    bool emits = emittance > 0.0f && (P.emitter.y == 0u || strategy == EMITTER_SAMPLING_NONE || p.bounces == 0u);
    if (emits) p.radiance = p.radiance + vmul(p.beta, vmul(albedo, albedo)) * emittance;
    p.bounces += 1;

    p.n = n;
    p.origin = pos + n * eps;
    // beta.mul(albedo), the factor of the sun and emitter terms and the path's next beta.
    p.beta = vmul(p.beta, albedo);
    if (!emits && strategy != EMITTER_SAMPLING_NONE) {
        emitter_cell(S, pos, p.list, p.count);  // no draw: evaluated here, used after the sun
        p.emode = 1u;                           // emitters to sample
    } else {
        p.emode = 0u;
    }

    V3 sun = f4v(P.sun_dir);
    float sin_r = __fsqrt_rn(fmax_r(1.0f - P.sun_dir.w * P.sun_dir.w, 0.0f));
    bool lit = P.sun_color.x > 0.0f || P.sun_color.y > 0.0f || P.sun_color.z > 0.0f;
    if (lit && dot(n, sun) > -sin_r && P.sun_dir.y > -sin_r) {
        V3 l = sample_sun(P, p.rng);
        float cos_l = dot(n, l);
        if (cos_l > 0.0f && l.y >= 0.0f) {
            // shadow (integrator.rs:319-346): the first segment.
            p.cos_l = cos_l;
            p.tr = v3(1.0f, 1.0f, 1.0f);
            p.seg = 0;
            p.o = p.origin;
            p.d = l;
            p.tmin = eps;
            p.tmax = kINF;
            p.kind = K_SHADOW;
            return A_TRACE;
        }
    }
    return A_EMIT_START;
}

// A shadow segment's result (integrator.rs:322-345).
LW_DI Act on_shadow(Path &p, const DevScene &S, const DevParams &P, const Hit &h) {
    const float eps = P.misc_f.y;
    if (h.quad == NO_QUAD) return A_SUN_DONE;
    const DevQuad *q = S.quads + h.quad;
    uint32_t flags = __float_as_uint(ldg(&q->p0_flags).w);
    if (flags & FLAG_WATER) {
        V3 qn = f4v(ldg(&q->n_nn));
        if (-dot(qn, p.d) > 0.0f) p.tr = vmul(p.tr, transmittance(f4v(P.water_color), h.t));
    } else if ((flags & FLAG_ALPHA_MASK) == ALPHA_TRANSLUCENT) {
        float a = __fdiv_rn((float)(h.texel >> 24), 255.0f);
        uint32_t tint = __float_as_uint(ldg(&q->eu_tint).w);
        V3 col = vmul(linear_rgb(S.gamma, h.texel), linear_rgb(S.gamma, tint));
        p.tr = vmul(p.tr, lerp(v3(1.0f, 1.0f, 1.0f), col, a));
    } else {
        p.tr = v3(0.0f, 0.0f, 0.0f);
        return A_SUN_DONE;
    }
    p.o = p.o + p.d * (h.t + eps);
    p.tmax -= h.t + eps;
    p.seg++;
    if (p.seg < 8u) return A_TRACE;
    return A_SUN_DONE;
}

// An emitter visibility ray's result: the rest of sample_emitter_face (integrator.rs:402-413).
LW_DI Act on_emit(Path &p, const DevScene &S, const DevParams &P, const Hit &h, V3 &val) {
    const float eps = P.misc_f.y;
    val = v3(0.0f, 0.0f, 0.0f);
    if (h.quad == NO_QUAD) return A_FACE_DONE;
    if (fabs_r(h.t - p.dist) >= 2.0f * eps) return A_FACE_DONE;
    const DevQuad *q = S.quads + p.first + p.f;
    V3 nq = -f4v(ldg(&q->n_nn));
    float area = vlength(nq);
    float cos_l = __fdiv_rn(fabs_r(dot(nq, p.d)), area);
    const DevQuad *hq = S.quads + h.quad;
    uint32_t tint = __float_as_uint(ldg(&hq->eu_tint).w);
    V3 c = vmul(linear_rgb(S.gamma, h.texel), linear_rgb(S.gamma, tint));
    float scaler = p.fmode == E_SINGLE ? 1.0f : __fdiv_rn(1.0f, (float)p.faces);
    val = c * (__fdiv_rn(cos_l, fmax_r(p.dist * p.dist, 1.0f)) * area * ldg(&q->ev_em).w * P.misc_f.x * scaler);
    return A_FACE_DONE;
}

// Runs the state machine from `act` until the lane needs a trace or its path ends.
LW_DI Act advance(Path &p, const DevScene &S, const DevParams &P, Act act, V3 val) {
    const float eps = P.misc_f.y;
    for (;;) {
        switch (act) {
        case A_TRACE:
        case A_END:
            return act;
        case A_CONTINUE:
            if (p.events >= MAX_EVENTS) return A_END;
            p.kind = K_EXTEND;
            p.tmax = kINF;
            return A_TRACE;
        case A_SUN_DONE:
            p.radiance = p.radiance + vmul(vmul(p.beta, f4v(P.sun_color)), p.tr) * p.cos_l;
            act = A_EMIT_START;
            break;
        case A_EMIT_START: {
            // sample_emitters (integrator.rs:441-469).
            if (p.emode == 0u) {
                act = A_FINISH_SURFACE;
                break;
            }
            if (p.count == 0u) {
                val = v3(0.0f, 0.0f, 0.0f);
                act = A_EMIT_FINISH;
                break;
            }
            const uint32_t *g = S.emitter_grid;
            uint32_t start = p.list;
            p.list = EMITTER_GRID_HEADER + ldg(g + 1) * ldg(g + 2) * ldg(g + 3) * 2u + start;
            uint32_t strategy = strategy_of(P);
            if (strategy == EMITTER_SAMPLING_ONE || strategy == EMITTER_SAMPLING_ONE_BLOCK) {
                p.emode = E_SINGLE;
                p.k = pick(p.count, rng_next(p.rng));
                act = A_BEGIN_EMITTER;
            } else if (strategy == EMITTER_SAMPLING_ALL) {
                p.emode = E_ALL;
                p.esum = v3(0.0f, 0.0f, 0.0f);
                p.k = 0;
                act = A_BEGIN_EMITTER;
            } else {
                val = v3(0.0f, 0.0f, 0.0f);
                act = A_EMIT_FINISH;
            }
            break;
        }
        case A_BEGIN_EMITTER: {
            // sample_emitter (integrator.rs:419-433) for emitter list[k].
            uint32_t i = ldg(S.emitter_grid + p.list + p.k);
            float4 e0 = ldg(S.emitters + 2u * i);
            float4 e1 = ldg(S.emitters + 2u * i + 1u);
            p.eoff = f4v(e0);
            p.first = __float_as_uint(e0.w);
            p.faces = __float_as_uint(e1.x);
            if (p.faces == 0u) {
                val = v3(0.0f, 0.0f, 0.0f);
                act = A_EMITTER_DONE;
                break;
            }
            if (P.emitter.x == EMITTER_SAMPLING_ONE) {
                p.fmode = E_SINGLE;
                p.f = pick(p.faces, rng_next(p.rng));
            } else {
                p.fmode = E_ALL;
                p.fsum = v3(0.0f, 0.0f, 0.0f);
                p.f = 0;
            }
            act = A_START_FACE;
            break;
        }
        case A_START_FACE: {
            // sample_emitter_face (integrator.rs:381-401), up to its visibility trace.
            const DevQuad *q = S.quads + p.first + p.f;
            float s = rng_next(p.rng);
            float t = rng_next(p.rng);
            V3 at = p.eoff + f4v(ldg(&q->p0_flags)) + f4v(ldg(&q->eu_tint)) * s + f4v(ldg(&q->ev_em)) * t;
            V3 to = at - p.origin;
            if (dot(to, p.n) <= 0.0f) {
                val = v3(0.0f, 0.0f, 0.0f);
                act = A_FACE_DONE;
                break;
            }
            p.dist = vlength(to);
            p.o = p.origin;
            p.d = vdiv(to, p.dist);
            p.tmin = eps;
            p.tmax = p.dist + 2.0f * eps;
            p.kind = K_EMIT;
            return A_TRACE;
        }
        case A_FACE_DONE:
            if (p.fmode == E_SINGLE) {
                act = A_EMITTER_DONE;
            } else {
                p.fsum = p.fsum + val;
                p.f++;
                if (p.f < p.faces) {
                    act = A_START_FACE;
                } else {
                    val = p.fsum;
                    act = A_EMITTER_DONE;
                }
            }
            break;
        case A_EMITTER_DONE:
            if (p.emode == E_SINGLE) {
                val = val * kPI;
                act = A_EMIT_FINISH;
            } else {
                p.esum = p.esum + val;
                p.k++;
                if (p.k < p.count) {
                    act = A_BEGIN_EMITTER;
                } else {
                    val = p.esum * __fdiv_rn(kPI, (float)p.count);
                    act = A_EMIT_FINISH;
                }
            }
            break;
        case A_EMIT_FINISH:
            p.radiance = p.radiance + vmul(p.beta, val);
            act = A_FINISH_SURFACE;
            break;
        case A_FINISH_SURFACE:
            // integrator.rs:695-705.
            if (p.bounces >= 3u) {
                float q_rr = clamp_r(max_elem(p.beta), 0.05f, 0.95f);
                if (rng_next(p.rng) > q_rr) return A_END;
                p.beta = vdiv(p.beta, q_rr);
            }
            p.d = cosine_hemisphere(p.n, p.rng);
            p.o = p.origin;
            p.tmin = 0.0f;
            p.specular = false;
            act = A_CONTINUE;
            break;
        }
    }
}

LW_DI Act shade(Path &p, const DevScene &S, const DevParams &P, const Hit &h) {
    V3 val = v3(0.0f, 0.0f, 0.0f);
    Act a;
    if (p.kind == K_EXTEND) a = on_extend(p, S, P, h);
    else if (p.kind == K_SHADOW) a = on_shadow(p, S, P, h);
    else a = on_emit(p, S, P, h, val);
    return advance(p, S, P, a, val);
}

LW_DI void kahan_add(float &s, float &c, float x) {
    float y = x - c;
    float t = s + y;
    c = (t - s) - y;
    s = t;
}

LW_DI bool finite3(V3 v) { return isfinite(v.x) && isfinite(v.y) && isfinite(v.z); }

#ifndef LW_STATS
#define LW_STATS 0
#endif
#if LW_STATS
// Divergence counters of the instrumented build (not part of the product build):
// [0] loop iterations per warp, [1] lanes active in them, [2] lanes tracing, [3] lane DDA
// steps, [4] warp DDA steps (the slowest lane's), [5..7] lanes shading a path/shadow/emitter
// ray, [8] lanes ending a path, [9] iterations with a lane taking work
__device__ unsigned long long g_stats[16];
#endif
constexpr int kThreads = 128;
#ifndef LW_MIN_BLOCKS
#define LW_MIN_BLOCKS 4
#endif

// The persistent render kernel. Each lane takes an item (sub consecutive samples of one pixel),
// traces its samples one after another, and takes the next item as soon as it is done; each
// loop iteration traces one ray per active lane.
template <int MODE>
__global__ void __launch_bounds__(kThreads, LW_MIN_BLOCKS) k_render(const DevScene S, const DevParams P, const WorkDesc W) {
    const uint32_t lane = threadIdx.x & 31u;
    const unsigned FULL = 0xFFFFFFFFu;
    Path p;
    bool active = false, exhausted = false;
    uint32_t px = 0, py = 0, slot = 0, j = 0, sample = 0, s_end = 0;
    float s0 = 0.f, s1 = 0.f, s2 = 0.f, c0 = 0.f, c1 = 0.f, c2 = 0.f;
    for (;;) {
        // Lanes without an item take the next ones, one atomic per warp.
        bool need = !active && !exhausted;
        unsigned mask = __ballot_sync(FULL, need);
        if (mask) {
            uint32_t base = 0;
            int leader = __ffs(mask) - 1;
            if ((int)lane == leader) {
                uint32_t n = (uint32_t)__popc(mask);
                base = atomicAdd(W.counter, n);
                // The cancel word is polled once per 4096 items taken, not on every take.
                if ((base & 4095u) < n && *W.cancel) base = W.n_items;
            }
            base = __shfl_sync(FULL, base, leader);
            if (need) {
                uint32_t item = base + (uint32_t)__popc(mask & ((1u << lane) - 1u));
                if (item >= W.n_items) {
                    exhausted = true;
                } else {
                    j = item / W.n_slots;
                    slot = item - j * W.n_slots;
                    uint32_t tile = slot >> 5, in = slot & 31u;
                    uint32_t rx = (tile % W.tiles_x) * 8u + (in & 7u);
                    uint32_t ry = (tile / W.tiles_x) * 4u + (in >> 3);
                    if (rx < W.w && ry < W.h) {
                        px = W.x0 + rx;
                        py = W.y0 + ry;
                        sample = W.sample_start + j * W.sub;
                        s_end = min(sample + W.sub, W.sample_start + W.spp);
                        s0 = s1 = s2 = c0 = c1 = c2 = 0.0f;
                        begin_sample(p, P, px, py, sample);
                        active = true;
                    }
                }
            }
        }
        if (__all_sync(FULL, exhausted)) break;
#if LW_STATS
        {
            unsigned act = __ballot_sync(FULL, active);
            if (lane == 0) {
                atomicAdd(&g_stats[0], 1ull);
                atomicAdd(&g_stats[1], (unsigned long long)__popc(act));
                if (mask) atomicAdd(&g_stats[9], 1ull);
            }
        }
#endif
        if (!active) continue;

#if LW_STATS
        uint32_t steps = 0;
        Hit h = trace(S, P, p.o, p.d, p.tmin, p.tmax, steps);
        {
            unsigned am = __activemask();
            uint32_t lsum = __reduce_add_sync(am, steps), lmax = __reduce_max_sync(am, steps);
            uint32_t kind = p.kind;
            unsigned k0 = __ballot_sync(am, kind == K_EXTEND), k1 = __ballot_sync(am, kind == K_SHADOW);
            unsigned k2 = __ballot_sync(am, kind == K_EMIT);
            if ((int)lane == __ffs(am) - 1) {
                atomicAdd(&g_stats[2], (unsigned long long)__popc(am));
                atomicAdd(&g_stats[3], (unsigned long long)lsum);
                atomicAdd(&g_stats[4], (unsigned long long)lmax);
                atomicAdd(&g_stats[5], (unsigned long long)__popc(k0));
                atomicAdd(&g_stats[6], (unsigned long long)__popc(k1));
                atomicAdd(&g_stats[7], (unsigned long long)__popc(k2));
            }
        }
#else
        Hit h = trace(S, P, p.o, p.d, p.tmin, p.tmax);
#endif
        Act a = shade(p, S, P, h);
#if LW_STATS
        {
            unsigned am = __activemask();
            unsigned e = __ballot_sync(am, a == A_END);
            if ((int)lane == __ffs(am) - 1) atomicAdd(&g_stats[8], (unsigned long long)__popc(e));
        }
#endif
        if (a == A_END) {
            if (MODE == MODE_SAMPLES) {
                size_t at = ((size_t)((py - W.y0) * W.w + (px - W.x0)) * W.spp + (sample - W.sample_start)) * 3u;
                W.samples_out[at] = p.radiance.x;
                W.samples_out[at + 1] = p.radiance.y;
                W.samples_out[at + 2] = p.radiance.z;
            } else if (finite3(p.radiance)) {
                kahan_add(s0, c0, p.radiance.x);
                kahan_add(s1, c1, p.radiance.y);
                kahan_add(s2, c2, p.radiance.z);
            }
            sample++;
            if (sample < s_end) {
                begin_sample(p, P, px, py, sample);
            } else {
                if (MODE == MODE_ACCUM) W.partials[(size_t)j * W.n_slots + slot] = make_float4(s0 - c0, s1 - c1, s2 - c2, 0.0f);
                active = false;
            }
        }
    }
}

// Adds the launch's item sums into the per-pixel accumulator, in item order (Kahan).
__global__ void k_reduce(const WorkDesc W, Accum *acc, uint32_t frame_w) {
    uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= W.n_slots) return;
    uint32_t tile = slot >> 5, in = slot & 31u;
    uint32_t rx = (tile % W.tiles_x) * 8u + (in & 7u);
    uint32_t ry = (tile / W.tiles_x) * 4u + (in >> 3);
    if (rx >= W.w || ry >= W.h) return;
    Accum &a = acc[(size_t)(W.y0 + ry) * frame_w + (W.x0 + rx)];
    float4 s = a.sum, c = a.comp;
    for (uint32_t j = 0; j < W.n_sub; j++) {
        float4 v = W.partials[(size_t)j * W.n_slots + slot];
        kahan_add(s.x, c.x, v.x);
        kahan_add(s.y, c.y, v.y);
        kahan_add(s.z, c.z, v.z);
    }
    s.w += (float)W.spp;
    a.sum = s;
    a.comp = c;
}

// The mean radiance per pixel: (sum - compensation) / count (cuda.rs:175-183 divides by the count).
__global__ void k_finalize(const Accum *acc, uint32_t n, float *out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Accum a = acc[i];
    float cnt = fmax_r(a.sum.w, 1.0f);
    out[3 * i] = __fdiv_rn(a.sum.x - a.comp.x, cnt);
    out[3 * i + 1] = __fdiv_rn(a.sum.y - a.comp.y, cnt);
    out[3 * i + 2] = __fdiv_rn(a.sum.z - a.comp.z, cnt);
}

struct DevHit {
    float t;
    uint32_t quad, texel;
    float s, tt;
    int32_t found;
};

__global__ void k_trace_rays(const DevScene S, const DevParams P, uint32_t n, const float *o, const float *d, float tmin,
                             float tmax, DevHit *out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Hit h = trace(S, P, v3(o[3 * i], o[3 * i + 1], o[3 * i + 2]), v3(d[3 * i], d[3 * i + 1], d[3 * i + 2]), tmin, tmax);
    out[i] = DevHit{h.t, h.quad, h.texel, h.s, h.tt, h.quad != NO_QUAD};
}

__global__ void k_voxel_lookup(const DevScene S, const DevParams P, uint32_t n, const int32_t *xyz, uint32_t *out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = voxel(S, P, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
}

#if LW_STATS
extern "C" int lw_debug_counters(unsigned long long *out, int reset) {
    cudaDeviceSynchronize();
    if (cudaMemcpyFromSymbol(out, g_stats, sizeof(g_stats)) != cudaSuccess) return 1;
    if (reset) {
        unsigned long long z[16] = {};
        cudaMemcpyToSymbol(g_stats, z, sizeof(z));
    }
    return 0;
}
#endif

LaunchShape render_shape(int mode, int device) {
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (mode == MODE_SAMPLES) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_render<MODE_SAMPLES>, kThreads, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_render<MODE_ACCUM>, kThreads, 0);
    if (per_sm < 1) per_sm = 1;
    return LaunchShape{sms * per_sm, kThreads};
}

cudaError_t launch_render(int mode, const DevScene &S, const DevParams &P, const WorkDesc &W, LaunchShape shape,
                          cudaStream_t st) {
    if (mode == MODE_SAMPLES) k_render<MODE_SAMPLES><<<shape.blocks, shape.threads, 0, st>>>(S, P, W);
    else k_render<MODE_ACCUM><<<shape.blocks, shape.threads, 0, st>>>(S, P, W);
    return cudaGetLastError();
}

cudaError_t launch_reduce(const WorkDesc &W, Accum *acc, uint32_t frame_w, cudaStream_t st) {
    k_reduce<<<(W.n_slots + 255) / 256, 256, 0, st>>>(W, acc, frame_w);
    return cudaGetLastError();
}

cudaError_t launch_finalize(const Accum *acc, uint32_t n, float *out_rgb, cudaStream_t st) {
    k_finalize<<<(n + 255) / 256, 256, 0, st>>>(acc, n, out_rgb);
    return cudaGetLastError();
}

cudaError_t launch_trace_rays(const DevScene &S, const DevParams &P, uint32_t n, const float *o, const float *d,
                              float tmin, float tmax, void *out_hits, cudaStream_t st) {
    k_trace_rays<<<(n + 127) / 128, 128, 0, st>>>(S, P, n, o, d, tmin, tmax, (DevHit *)out_hits);
    return cudaGetLastError();
}

cudaError_t launch_voxel_lookup(const DevScene &S, const DevParams &P, uint32_t n, const int32_t *xyz, uint32_t *out,
                                cudaStream_t st) {
    k_voxel_lookup<<<(n + 255) / 256, 256, 0, st>>>(S, P, n, xyz, out);
    return cudaGetLastError();
}

}  // namespace lw
