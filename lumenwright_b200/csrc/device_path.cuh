// The per-lane path state machine shared by the render kernels: the camera ray of a sample, the
// handling of each ray's result (integrator.rs:571-706 split at every trace) and the Kahan sums.
#pragma once

#include "device_integrator.cuh"

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

// Whether the frame's Params ask for chunk-origin rebasing: the camera's position is then given
// relative to the chunk corner of word see_through.w.
LW_HDI bool rebased(const DevParams &P) { return P.see_through.z != 0u; }

// The camera ray of sample `sample` at pixel (px, py) (integrator.rs:545-569).
template <bool REB = false>
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
    if (REB) p.frame = P.see_through.w;
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
// REB (chunk-origin rebasing): the path's positions are in the frame of p.frame; each new origin
// (the offset origin of a surface, a water crossing, a translucent pass) moves the path to the
// frame of the chunk corner nearest it (rebase), after the last use of the old frame.
template <bool REB = false>
LW_DI Act on_extend(Path &p, const DevScene &S, const DevParams &P, Hit h) {
    const float eps = P.misc_f.y;
    const Frame A = REB ? frame_of(p.frame) : Frame{};
    p.events++;
    bool found = h.quad != NO_QUAD;
    bool forced = false;
    if (p.bounces == 0 && P.see_through.y > 0u && found && !is_see_through(P, h.quad)) {
        Hit st = see_through_hit<REB>(S, P, p.o, p.d, h.t, A);
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
    // Water (the plane outside the grid columns, or a water surface) refracts or reflects the ray;
    // both cases meet at one call of water_interface.
    V3 wpos, wn;
    bool wfront, water = false;
    float tp;
    uint32_t flags = 0u;
    V3 pos = v3(0.0f, 0.0f, 0.0f), albedo = pos, n = pos;
    float alpha = 0.0f, qemit = 0.0f;
    // One exit: a lane that is done (the sky, water, a translucent pass, the last bounce) falls
    // through the remaining steps.
    Act act = A_EMIT_START;
    bool done = false;
    if (water_plane(P, p.o, p.d, tp, A) && (!found || tp < h.t)) {
        if (p.in_water) p.beta = vmul(p.beta, transmittance(sigma, tp));
        wfront = p.d.y < 0.0f;
        wn = v3(0.0f, wfront ? 1.0f : -1.0f, 0.0f);
        wpos = p.o + p.d * tp;
        water = true;
    } else if (!found) {
        if (!p.in_water && !under_water_plane(P, p.o, p.d, A)) {
            p.radiance = p.radiance + vmul(p.beta, sky_of(S, P, p.d, p.bounces == 0));
            if (p.specular && p.bounces == 0) p.radiance = p.radiance + vmul(p.beta, sun_texture(S, P, p.d));
        }
        act = A_END;
        done = true;
    } else {
        if (p.in_water) p.beta = vmul(p.beta, transmittance(sigma, h.t));
        const DevQuad *q = S.quads + h.quad;
        float4 qn = ldg(&q->n_nn);
        flags = __float_as_uint(ldg(&q->p0_flags).w);
        uint32_t tint = __float_as_uint(ldg(&q->eu_tint).w);
        qemit = ldg(&q->ev_em).w;
        pos = p.o + p.d * h.t;
        alpha = __fdiv_rn((float)(h.texel >> 24), 255.0f);
        albedo = vmul(linear_rgb(S.gamma, h.texel), linear_rgb(S.gamma, tint));
        // shading_normal (integrator.rs:308-315): normal() = ev x eu = -(eu x ev), exactly.
        n = normalize(-f4v(qn));
        bool front = true;
        if (!(dot(n, p.d) < 0.0f)) {
            n = -n;
            front = false;
        }
        if (flags & FLAG_WATER) {
            wpos = pos;
            wn = n;
            wfront = front;
            water = true;
        }
    }
    if (water) {
        V3 nd, no;
        p.in_water = water_interface(P, wpos, p.d, wn, wfront, p.in_water, eps, p.rng, nd, no);
        p.d = nd;
        p.o = no;
        if (REB) rebase(p.o, p.frame);
        p.specular = true;
        p.tmin = 0.0f;
        act = A_CONTINUE;
        done = true;
    }
    if (!done && !forced && (flags & FLAG_ALPHA_MASK) == ALPHA_TRANSLUCENT && rng_next(p.rng) >= alpha) {
        p.beta = vmul(p.beta, lerp(v3(1.0f, 1.0f, 1.0f), albedo, alpha));
        p.o = pos + p.d * eps;
        if (REB) rebase(p.o, p.frame);
        p.tmin = 0.0f;
        act = A_CONTINUE;
        done = true;
    }
    if (!done && p.bounces >= P.frame.w) {
        act = A_END;
        done = true;
    }
    if (!done) {
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
            emitter_cell<REB>(S, pos, p.list, p.count, A);  // no draw: evaluated here, used after the sun
            p.emode = 1u;                                   // emitters to sample
        } else {
            p.emode = 0u;
        }
        if (REB) rebase(p.origin, p.frame);  // the rays from this surface start in the new frame

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
                act = A_TRACE;
            }
        }
    }
    return act;
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

// Runs the state machine from `act` until the lane needs a trace or its path ends. The steps are
// written in the order a lane meets them (the sun's light, the emitters, Russian roulette and the
// next direction), each at most once per pass, so the lanes of a warp that are at different steps
// run each step's code together as they fall through it; only the loop over emitters and faces
// goes back. A lane that is done (a ray to trace, or the path's end) falls through the remaining
// steps rather than leaving early: one exit keeps the steps' code and registers shared.
template <bool REB = false>
LW_DI Act advance(Path &p, const DevScene &S, const DevParams &P, Act act, V3 val) {
    const float eps = P.misc_f.y;
    bool done = act == A_TRACE || act == A_END;
    Act out = act;
    if (!done && act == A_SUN_DONE) {
        p.radiance = p.radiance + vmul(vmul(p.beta, f4v(P.sun_color)), p.tr) * p.cos_l;
        act = A_EMIT_START;
    }
    if (!done && act == A_EMIT_START) {
        // sample_emitters (integrator.rs:441-469).
        if (p.emode == 0u) {
            act = A_FINISH_SURFACE;
        } else if (p.count == 0u) {
            val = v3(0.0f, 0.0f, 0.0f);
            act = A_EMIT_FINISH;
        } else {
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
        }
    }
    for (;;) {
            if (!done && act == A_BEGIN_EMITTER) {
            // sample_emitter (integrator.rs:419-433) for emitter list[k].
            uint32_t i = ldg(S.emitter_grid + p.list + p.k);
            float4 e0 = ldg(S.emitters + 2u * i);
            float4 e1 = ldg(S.emitters + 2u * i + 1u);
            p.eoff = f4v(e0);
            if (REB) p.eoff = p.eoff - frame_origin(frame_of(p.frame));  // the block's corner in the frame: exact
            p.first = __float_as_uint(e0.w);
            p.faces = __float_as_uint(e1.x);
            if (p.faces == 0u) {
                val = v3(0.0f, 0.0f, 0.0f);
                act = A_EMITTER_DONE;
            } else {
                if (P.emitter.x == EMITTER_SAMPLING_ONE) {
                    p.fmode = E_SINGLE;
                    p.f = pick(p.faces, rng_next(p.rng));
                } else {
                    p.fmode = E_ALL;
                    p.fsum = v3(0.0f, 0.0f, 0.0f);
                    p.f = 0;
                }
                act = A_START_FACE;
            }
        }
            if (!done && act == A_START_FACE) {
            // sample_emitter_face (integrator.rs:381-401), up to its visibility trace.
            const DevQuad *q = S.quads + p.first + p.f;
            float s = rng_next(p.rng);
            float t = rng_next(p.rng);
            V3 at = p.eoff + f4v(ldg(&q->p0_flags)) + f4v(ldg(&q->eu_tint)) * s + f4v(ldg(&q->ev_em)) * t;
            V3 to = at - p.origin;
            if (dot(to, p.n) <= 0.0f) {
                val = v3(0.0f, 0.0f, 0.0f);
                act = A_FACE_DONE;
            } else {
                p.dist = vlength(to);
                p.o = p.origin;
                p.d = vdiv(to, p.dist);
                p.tmin = eps;
                p.tmax = p.dist + 2.0f * eps;
                p.kind = K_EMIT;
                out = A_TRACE;
                done = true;
            }
        }
            if (!done && act == A_FACE_DONE) {
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
        }
            if (!done && act == A_EMITTER_DONE) {
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
        }
        const bool again = !done && (act == A_START_FACE || act == A_BEGIN_EMITTER);  // the next face or emitter
        if (!again) break;
    }
    if (!done && act == A_EMIT_FINISH) {
        p.radiance = p.radiance + vmul(p.beta, val);
        act = A_FINISH_SURFACE;
    }
    if (!done && act == A_FINISH_SURFACE) {
        // integrator.rs:695-705.
        bool ends = false;
        if (p.bounces >= 3u) {
            float q_rr = clamp_r(max_elem(p.beta), 0.05f, 0.95f);
            if (rng_next(p.rng) > q_rr) ends = true;
            else p.beta = vdiv(p.beta, q_rr);
        }
        if (ends) {
            out = A_END;
            done = true;
        } else {
            p.d = cosine_hemisphere(p.n, p.rng);
            p.o = p.origin;
            p.tmin = 0.0f;
            p.specular = false;
            act = A_CONTINUE;
        }
    }
    if (!done && act == A_CONTINUE) {
        if (p.events >= MAX_EVENTS) {
            out = A_END;
        } else {
            p.kind = K_EXTEND;
            p.tmax = kINF;
            out = A_TRACE;
        }
        done = true;
    }
    return out;
}

// The result of the lane's last ray, by its kind (on_extend, on_shadow, on_emit).
template <bool REB = false>
LW_DI Act on_result(Path &p, const DevScene &S, const DevParams &P, const Hit &h, V3 &val) {
    if (p.kind == K_EXTEND) return on_extend<REB>(p, S, P, h);
    if (p.kind == K_SHADOW) return on_shadow(p, S, P, h);
    return on_emit(p, S, P, h, val);
}

template <bool REB = false>
LW_DI Act shade(Path &p, const DevScene &S, const DevParams &P, const Hit &h) {
    V3 val = v3(0.0f, 0.0f, 0.0f);
    Act a = on_result<REB>(p, S, P, h, val);
    return advance<REB>(p, S, P, a, val);
}

LW_DI void kahan_add(float &s, float &c, float x) {
    float y = x - c;
    float t = s + y;
    c = (t - s) - y;
    s = t;
}

LW_DI bool finite3(V3 v) { return isfinite(v.x) && isfinite(v.y) && isfinite(v.z); }

// The index of the job whose range [begin, next begin) holds `x` (begins ascending, first 0).
LW_DI uint32_t find_job(const uint32_t *begins, uint32_t n, uint32_t x) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (ldg(begins + mid) <= x) lo = mid;
        else hi = mid;
    }
    return lo;
}

}  // namespace lw
