// The differentiable form: the hq path tracer with parameters theta (a linear albedo per atlas
// texel, an intensity per emitter group, the sky cache and sun direction of a sun azimuth, altitude
// and turbidity), its adjoint by path replay, and paired finite differences.
//
// Forward: render_sample (crates/lumenwright-kernel/src/integrator.rs:539-709) with two changes
// that leave it unchanged at the nominal parameters: a hit's albedo is the parameter of its atlas
// texel (the value gamma_to_linear gives for the texel's bytes, :27-34, :634) times the decoded tint,
// and an emitting surface's intensity misc_f.x is multiplied by the intensity of its emitter group
// (a hash of the emitting block's voxel, 32 groups).
//
// Adjoint (path replay backpropagation, Vicini, Speierer and Jakob, SIGGRAPH 2021): each sample's
// path is replayed twice with its random stream. Replay 1 gives the path's radiance L. Replay 2
// walks the path again; every radiance term added after a vertex carries that vertex's albedo, so
// at a diffuse vertex i with texel parameter a_i
//   dL(c) / da_i(c) = (L(c) - L_before_i(c) + E_i(c)) / a_i(c)
// where L_before_i is the radiance before vertex i and E_i its emitted term (Chunky's emission is
// albedo squared, so it counts twice). The Russian roulette probability is detached: it is a
// function of the throughput, and the estimator's expectation does not depend on it, so replay 2
// treats it as a constant (the estimate of the gradient stays unbiased). The emitter terms give the
// gradients of the emitters' colours and group intensities; the sky terms the gradient of the sky
// cache entries (through the bilinear HSL lookup and rgb_from_hsl); the sun's next-event terms the
// gradient of the sun direction through sample_sun, the cosine and the water crossed by the shadow
// ray. Visibility changes (shadow edges, alpha tests) are discontinuities with no interior
// derivative; their boundary terms are not estimated.
//
// Finite differences: every sample is rendered with theta+ and theta-, with the roulette's
// probability and decisions taken from the nominal throughput and the shadow rays traced along the
// nominal sun direction (the crossed water's length follows the perturbed direction through the
// same surfaces), so the pair differs only through the parameters and the difference is the
// derivative the adjoint estimates.
#include "device_path.cuh"
#include "internal.h"

namespace lw {
namespace adj {

enum { M_FWD = 0, M_GRAD = 1, M_FD = 2 };

// Blocks of 128 threads per SM the compiler must fit, which bounds the registers: the forward pass
// at 128 (4 blocks; unbounded it takes 141), the backward pass at 168 (3 blocks; 208 with 176 B of
// stack unbounded). More warps hide more of the paths' latency: forward -16 %, backward -27 % at the
// differentiation workload.
#ifndef LW_ADJ_FWD_MINB
#define LW_ADJ_FWD_MINB 4
#endif
#ifndef LW_ADJ_BWD_MINB
#define LW_ADJ_BWD_MINB 3
#endif
#define LW_ADJ_BOUNDS(minb) __launch_bounds__(128, (minb) > 0 ? (minb) : 1)

struct Theta {
    AdjFrame F;
    const float *albedo0;  // nominal albedo (the roulette's throughput in M_FD)
    float4 sun0;           // nominal sun direction and cone (the shadow rays' direction in M_FD)
};

constexpr int kGroups = LW_ADJ_EMITTER_GROUPS;

// The emitter group of the block at voxel (x, y, z).
LW_DI uint32_t emitter_group(int x, int y, int z) {
    return pcg_hash((uint32_t)x * 73856093u ^ (uint32_t)y * 19349663u ^ (uint32_t)z * 83492791u) & (kGroups - 1);
}

// The atlas index quad_texel reads for a hit at (s, tt) (trace.rs:62-69).
LW_DI uint32_t texel_index(const DevParams &P, const DevQuad *q, float s, float tt) {
    float4 uv = ldg(&q->uv), uvt = ldg(&q->uvt);
    float sc = fmin_r(fmax_r(s, 0.0005f), 0.9995f);
    float tc = fmin_r(fmax_r(tt, 0.0005f), 0.9995f);
    float u = uv.x + sc * uv.z + tc * uvt.x;
    float v = uv.y + sc * uv.w + tc * uvt.y;
    int w = (int)P.off2.y, h = (int)P.off2.z;
    int x = clamp_i(to_i32(floorf(u)), 0, w - 1);
    int y = clamp_i(to_i32(floorf(v)), 0, h - 1);
    return (uint32_t)(y * w + x);
}

LW_DI V3 load3(const float *p, int i) { return v3(ldg(p + 3 * i), ldg(p + 3 * i + 1), ldg(p + 3 * i + 2)); }

// The linear colour of a hit's texel under theta, and its parameter (-1: the decoded texel).
LW_DI V3 texel_albedo(const DevScene &S, const AdjFrame &F, const DevQuad *q, const Hit &h, int &param) {
    param = ldg(F.texel_param + texel_index(F.P, q, h.s, h.tt));
    return param < 0 ? linear_rgb(S.gamma, h.texel) : load3(F.albedo, param);
}

// sample_sun (integrator.rs:291-302) about `axis` with the two draws given.
LW_DI V3 cone_dir(V3 axis, float cos_max, float r1, float r2) {
    float cos_t = 1.0f - r1 * (1.0f - cos_max);
    float sin_t = __fsqrt_rn(fmax_r(1.0f - cos_t * cos_t, 0.0f));
    float sin_phi, cos_phi;
    sin_cos_turns(r2, sin_phi, cos_phi);
    V3 t, b;
    onb(axis, t, b);
    return normalize(t * (sin_t * cos_phi) + b * (sin_t * sin_phi) + axis * cos_t);
}

// ---- forward-mode duals for the derivative of cone_dir with respect to its axis -------------------
struct D3 {
    float v, g[3];
};
LW_DI D3 dconst(float v) { return D3{v, {0.0f, 0.0f, 0.0f}}; }
LW_DI D3 operator+(D3 a, D3 b) { return D3{a.v + b.v, {a.g[0] + b.g[0], a.g[1] + b.g[1], a.g[2] + b.g[2]}}; }
LW_DI D3 operator*(D3 a, D3 b) {
    D3 r;
    r.v = a.v * b.v;
    for (int i = 0; i < 3; i++) r.g[i] = a.g[i] * b.v + a.v * b.g[i];
    return r;
}
LW_DI D3 operator*(D3 a, float s) { return D3{a.v * s, {a.g[0] * s, a.g[1] * s, a.g[2] * s}}; }
LW_DI D3 dinv(D3 a) {
    D3 r;
    r.v = __fdiv_rn(1.0f, a.v);
    for (int i = 0; i < 3; i++) r.g[i] = -a.g[i] * r.v * r.v;
    return r;
}
LW_DI D3 dsqrt(D3 a) {
    D3 r;
    r.v = __fsqrt_rn(a.v);
    for (int i = 0; i < 3; i++) r.g[i] = r.v > 0.0f ? a.g[i] * __fdiv_rn(0.5f, r.v) : 0.0f;
    return r;
}

// J[i][j] = d cone_dir(axis)_i / d axis_j for fixed draws (the axis moves, the cone sample with it).
LW_DI void cone_dir_jacobian(V3 axis, float cos_max, float r1, float r2, float J[3][3]) {
    D3 x{axis.x, {1.0f, 0.0f, 0.0f}}, y{axis.y, {0.0f, 1.0f, 0.0f}}, z{axis.z, {0.0f, 0.0f, 1.0f}};
    float cos_t = 1.0f - r1 * (1.0f - cos_max);
    float sin_t = __fsqrt_rn(fmax_r(1.0f - cos_t * cos_t, 0.0f));
    float sin_phi, cos_phi;
    sin_cos_turns(r2, sin_phi, cos_phi);
    // onb (math.rs:348-356); the sign is locally constant.
    float sign = axis.z >= 0.0f ? 1.0f : -1.0f;
    D3 a = dinv(dconst(sign) + z) * -1.0f;
    D3 bb = x * y * a;
    D3 t0 = dconst(1.0f) + x * x * a * sign, t1 = bb * sign, t2 = x * -sign;
    D3 b0 = bb, b1 = dconst(sign) + y * y * a, b2 = y * -1.0f;
    float ca = sin_t * cos_phi, cb = sin_t * sin_phi;
    D3 v0 = t0 * ca + b0 * cb + x * cos_t, v1 = t1 * ca + b1 * cb + y * cos_t, v2 = t2 * ca + b2 * cb + z * cos_t;
    D3 il = dinv(dsqrt(v0 * v0 + v1 * v1 + v2 * v2));
    D3 l0 = v0 * il, l1 = v1 * il, l2 = v2 * il;
    for (int j = 0; j < 3; j++) {
        J[0][j] = l0.g[j];
        J[1][j] = l1.g[j];
        J[2][j] = l2.g[j];
    }
}

// d rgb_from_hsl / d (hue, saturation, lightness) (integrator.rs:108-127), per output channel.
LW_DI void rgb_from_hsl_grad(float hue, float sat, float light, V3 &dh, V3 &ds, V3 &dl) {
    float k = 1.0f - fabs_r(2.0f * light - 1.0f);
    float craw = k * sat;
    float dc_ds = craw < 1.0f ? k : 0.0f;
    float dc_dl = craw < 1.0f ? -2.0f * sat * (2.0f * light - 1.0f > 0.0f ? 1.0f : -1.0f) : 0.0f;
    float c = fmin_r(1.0f, craw);
    float h = hue * 6.0f;
    float md = fmodf(h, 2.0f);
    float fx = 1.0f - fabs_r(md - 1.0f);
    float dx_dh = -c * (md - 1.0f > 0.0f ? 1.0f : -1.0f) * 6.0f;
    float dx_ds = dc_ds * fx, dx_dl = dc_dl * fx;
    int ci, xi;  // the channels holding c and x
    if (h < 1.0f) ci = 0, xi = 1;
    else if (h < 2.0f) ci = 1, xi = 0;
    else if (h < 3.0f) ci = 1, xi = 2;
    else if (h < 4.0f) ci = 2, xi = 1;
    else if (h < 5.0f) ci = 2, xi = 0;
    else ci = 0, xi = 2;
    float gh[3] = {0.0f, 0.0f, 0.0f}, gs[3] = {0.0f, 0.0f, 0.0f}, gl[3] = {0.0f, 0.0f, 0.0f};
    gh[xi] = dx_dh;
    gs[ci] = dc_ds;
    gs[xi] = dx_ds;
    gl[ci] = dc_dl;
    gl[xi] = dx_dl;
    float mraw = light - 0.5f * c;
    float dm_ds = mraw > 0.0f ? -0.5f * dc_ds : 0.0f;
    float dm_dl = mraw > 0.0f ? 1.0f - 0.5f * dc_dl : 0.0f;
    dh = v3(gh[0], gh[1], gh[2]);
    ds = v3(gs[0] + dm_ds, gs[1] + dm_ds, gs[2] + dm_ds);
    dl = v3(gl[0] + dm_dl, gl[1] + dm_dl, gl[2] + dm_dl);
}

// Adds the gradient of sum_c wb(c) sky_radiance(d)(c) with respect to the cache entries it reads
// (integrator.rs:158-188) to g.
LW_DI void sky_cache_grad(const DevScene &S, const DevParams &P, V3 d, V3 wb, double *g) {
    float n = P.misc_f.z;
    if (n < 1.0f) return;
    float theta = __fdiv_rn(atan2_r(d.z, d.x), 2.0f * kPI);
    theta = fmodf(fmodf(theta, 1.0f) + 1.0f, 1.0f);
    float phi = 1.0f - __fdiv_rn(acos_r(clamp_r(d.y, -1.0f, 1.0f)), kPI);
    float x = theta * n, y = phi * n;
    float fx = floorf(clamp_r(x, 0.0f, n - 1.0f));
    float fy = floorf(clamp_r(y, 0.0f, n - 1.0f));
    uint32_t m = to_u32(n) + 1u;
    uint32_t a00 = (to_u32(fx) * m + to_u32(fy)) * 3u, a10 = (to_u32(fx + 1.0f) * m + to_u32(fy)) * 3u;
    uint32_t a01 = (to_u32(fx) * m + to_u32(fy + 1.0f)) * 3u, a11 = (to_u32(fx + 1.0f) * m + to_u32(fy + 1.0f)) * 3u;
    float tx = x - fx, ty = y - fy;
    float hsl[3];
    for (int k = 0; k < 3; k++) {
        float s00 = ldg(S.sky + a00 + k), s10 = ldg(S.sky + a10 + k), s01 = ldg(S.sky + a01 + k), s11 = ldg(S.sky + a11 + k);
        float y0 = s00 + tx * (s10 - s00), y1 = s01 + tx * (s11 - s01);
        hsl[k] = y0 + ty * (y1 - y0);
    }
    V3 dh, ds, dl;
    rgb_from_hsl_grad(hsl[0], hsl[1], hsl[2], dh, ds, dl);
    double scale = P.sky_sun.w;
    double gk[3] = {dot(wb, dh) * scale, dot(wb, ds) * scale, dot(wb, dl) * scale};
    for (int k = 0; k < 3; k++) {
        atomicAdd(g + a00 + k, gk[k] * (1.0 - tx) * (1.0 - ty));
        atomicAdd(g + a10 + k, gk[k] * tx * (1.0 - ty));
        atomicAdd(g + a01 + k, gk[k] * (1.0 - tx) * ty);
        atomicAdd(g + a11 + k, gk[k] * tx * ty);
    }
}

// Adds w(c) term(c) lambda(c) to entry c of parameter `param`, lambda(c) being the log-derivative
// of the term with respect to the parameter's channel c.
LW_DI void add_albedo(const AdjGrad &go, int param, V3 w, V3 term, V3 lambda) {
    double v[3] = {(double)w.x * term.x * lambda.x, (double)w.y * term.y * lambda.y, (double)w.z * term.z * lambda.z};
    for (int c = 0; c < 3; c++)
        if (v[c] != 0.0 && isfinite(v[c])) atomicAdd(go.albedo + 3 * param + c, v[c]);
}

// A path's radiance, summed in FP64 so that a difference of two sums (the radiance after a vertex,
// the change a parameter step makes) keeps the precision of its terms.
struct DV {
    double x, y, z;
};
LW_DI void acc(DV &r, V3 t) {
    r.x += t.x;
    r.y += t.y;
    r.z += t.z;
}
LW_DI V3 vsub(DV a, DV b) { return v3((float)(a.x - b.x), (float)(a.y - b.y), (float)(a.z - b.z)); }
LW_DI bool finite_dv(DV v) { return isfinite(v.x) && isfinite(v.y) && isfinite(v.z); }

LW_DI V3 inv3(V3 a) {
    return v3(a.x != 0.0f ? __fdiv_rn(1.0f, a.x) : 0.0f, a.y != 0.0f ? __fdiv_rn(1.0f, a.y) : 0.0f,
              a.z != 0.0f ? __fdiv_rn(1.0f, a.z) : 0.0f);
}

// One path sample with theta. M_FWD: its radiance. M_GRAD: replay 2, with the sample's radiance L
// (replay 1) and the loss weights w = dLoss/dI(pixel) / spp; adds the gradients to `go`. M_FD: the
// radiance with the roulette and the shadow rays of the nominal theta.
template <int M>
LW_DI DV path(const DevScene &S0, const Theta &T, uint32_t px, uint32_t py, uint32_t sample, DV L, V3 w,
              const AdjGrad &go) {
    constexpr bool GRAD = M == M_GRAD, FD = M == M_FD;
    const DevParams &P = T.F.P;
    DevScene S = S0;
    S.sky = T.F.sky;
    const float eps = P.misc_f.y;
    uint32_t rng = rng_new(py * P.frame.x + px, sample, P.misc_u.x);
    float jx = rng_next(rng);
    float jy = rng_next(rng);
    float sx = (__fdiv_rn(2.0f * ((float)px + jx), (float)P.frame.x) - 1.0f) * P.cam_fwd.w * P.cam_pos.w;
    float sy = (1.0f - __fdiv_rn(2.0f * ((float)py + jy), (float)P.frame.y)) * P.cam_pos.w;
    V3 d = normalize(f4v(P.cam_fwd) + f4v(P.cam_right) * sx + f4v(P.cam_up) * sy);
    V3 o = f4v(P.cam_pos);
    DV radiance{0.0, 0.0, 0.0};
    V3 beta = v3(1.0f, 1.0f, 1.0f), beta0 = beta;
    uint32_t bounces = 0;
    bool specular = true, in_water = false;
    const uint32_t strategy = strategy_of(P);
    float tmin = 0.0f;
    const V3 sigma = f4v(P.water_color);
    for (uint32_t ev = 0; ev < MAX_EVENTS; ev++) {
        Hit h = trace<false>(S, P, o, d, tmin, kINF);
        bool found = h.quad != NO_QUAD, forced = false;
        if (bounces == 0 && P.see_through.y > 0u && found && !is_see_through(P, h.quad)) {
            Hit st = see_through_hit(S, P, o, d, h.t);
            if (st.quad != NO_QUAD) {
                uint32_t sf = __float_as_uint(ldg(&S.quads[st.quad].p0_flags).w);
                if ((sf & FLAG_ALPHA_MASK) == ALPHA_TRANSLUCENT) {
                    if (rng_next(rng) < __fdiv_rn((float)(st.texel >> 24), 255.0f)) {
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
            if (in_water) {
                V3 tr = transmittance(sigma, tp);
                beta = vmul(beta, tr);
                beta0 = vmul(beta0, tr);
            }
            bool front = d.y < 0.0f;
            V3 nd, no;
            in_water = water_interface(P, o + d * tp, d, v3(0.0f, front ? 1.0f : -1.0f, 0.0f), front, in_water, eps, rng, nd, no);
            d = nd;
            o = no;
            specular = true;
            tmin = 0.0f;
            continue;
        }
        if (!found) {
            if (!in_water && !under_water_plane(P, o, d)) {
                V3 sk = bounces == 0 ? sky_lens(S, P, d) : sky_light(S, P, d);
                acc(radiance, vmul(beta, sk));
                if (GRAD && P.sky_map.x < 1.0f) sky_cache_grad(S, P, d, vmul(w, beta), go.cache);
                if (specular && bounces == 0) acc(radiance, vmul(beta, sun_texture(S, P, d)));
            }
            break;
        }
        if (in_water) {
            V3 tr = transmittance(sigma, h.t);
            beta = vmul(beta, tr);
            beta0 = vmul(beta0, tr);
        }
        const DevQuad *q = S.quads + h.quad;
        uint32_t flags = __float_as_uint(ldg(&q->p0_flags).w);
        V3 pos = o + d * h.t;
        float alpha = __fdiv_rn((float)(h.texel >> 24), 255.0f);
        int param;
        V3 a = texel_albedo(S, T.F, q, h, param);
        V3 tintl = linear_rgb(S.gamma, __float_as_uint(ldg(&q->eu_tint).w));
        V3 albedo = vmul(a, tintl);
        V3 albedo0 = albedo;
        if (FD && param >= 0) albedo0 = vmul(load3(T.albedo0, param), tintl);
        V3 n = normalize(-f4v(ldg(&q->n_nn)));
        bool front = true;
        if (!(dot(n, d) < 0.0f)) {
            n = -n;
            front = false;
        }
        if (flags & FLAG_WATER) {
            V3 nd, no;
            in_water = water_interface(P, pos, d, n, front, in_water, eps, rng, nd, no);
            d = nd;
            o = no;
            specular = true;
            tmin = 0.0f;
            continue;
        }
        if (!forced && (flags & FLAG_ALPHA_MASK) == ALPHA_TRANSLUCENT && rng_next(rng) >= alpha) {
            V3 f = lerp(v3(1.0f, 1.0f, 1.0f), albedo, alpha);
            // Every later term carries f, whose log-derivative is alpha tint / f.
            if (GRAD && param >= 0) add_albedo(go, param, w, vsub(L, radiance), vmul(tintl * alpha, inv3(f)));
            beta = vmul(beta, f);
            beta0 = FD ? vmul(beta0, lerp(v3(1.0f, 1.0f, 1.0f), albedo0, alpha)) : beta;
            o = pos + d * eps;
            tmin = 0.0f;
            continue;
        }
        if (bounces >= P.frame.w) break;
        const DV l_before = radiance;
        float emittance = ldg(&q->ev_em).w * P.misc_f.x;
        bool emits = emittance > 0.0f && (P.emitter.y == 0u || strategy == EMITTER_SAMPLING_NONE || bounces == 0u);
        V3 e_term = v3(0.0f, 0.0f, 0.0f);
        if (emits) {
            V3 inside = pos - n * 1e-3f;
            uint32_t g = emitter_group(to_i32(floorf(inside.x)), to_i32(floorf(inside.y)), to_i32(floorf(inside.z)));
            float mult = ldg(T.F.emit_mult + g);
            e_term = vmul(beta, vmul(albedo, albedo)) * (emittance * mult);
            acc(radiance, e_term);
            if (GRAD && mult != 0.0f) atomicAdd(go.emit + g, (double)dot(w, e_term) / mult);
        }
        bounces += 1;
        V3 origin = pos + n * eps;
        V3 beta_a = vmul(beta, albedo);

        V3 sun = f4v(P.sun_dir);
        float sin_r = __fsqrt_rn(fmax_r(1.0f - P.sun_dir.w * P.sun_dir.w, 0.0f));
        bool lit = P.sun_color.x > 0.0f || P.sun_color.y > 0.0f || P.sun_color.z > 0.0f;
        if (lit && dot(n, sun) > -sin_r && P.sun_dir.y > -sin_r) {
            float r1 = rng_next(rng);
            float r2 = rng_next(rng);
            V3 l = cone_dir(sun, P.sun_dir.w, r1, r2);
            V3 l0 = FD ? cone_dir(f4v(T.sun0), T.sun0.w, r1, r2) : l;
            float cos_l = dot(n, l);
            if (cos_l > 0.0f && l.y >= 0.0f) {
                // shadow (integrator.rs:319-346) along l0. u: distance from `origin` to the current
                // hit along the ray; du: its derivative with respect to the direction.
                V3 tr = v3(1.0f, 1.0f, 1.0f), so = origin;
                float tmax = kINF, ucum = 0.0f, ul_prev = 0.0f;
                V3 du_prev = v3(0.0f, 0.0f, 0.0f), vw = v3(0.0f, 0.0f, 0.0f);
                int tparam[8];
                V3 tlam[8];
                int nt = 0;
                for (int sg = 0; sg < 8; sg++) {
                    Hit sh = trace<false>(S, P, so, l0, eps, tmax);
                    if (sh.quad == NO_QUAD) break;
                    const DevQuad *sq = S.quads + sh.quad;
                    uint32_t sf = __float_as_uint(ldg(&sq->p0_flags).w);
                    V3 nq = f4v(ldg(&sq->n_nn));
                    float u = ucum + sh.t;
                    float ul = 0.0f;
                    if (FD) ul = __fdiv_rn(dot((so + l0 * sh.t) - origin, nq), dot(l, nq));
                    V3 du = v3(0.0f, 0.0f, 0.0f);
                    if (GRAD) du = nq * __fdiv_rn(-u, dot(l, nq));
                    if (sf & FLAG_WATER) {
                        if (-dot(nq, l0) > 0.0f) {
                            float t = FD ? (sg == 0 ? ul : ul - (ul_prev + eps)) : sh.t;
                            tr = vmul(tr, transmittance(sigma, t));
                            if (GRAD) vw = vw + (du - du_prev);
                        }
                    } else if ((sf & FLAG_ALPHA_MASK) == ALPHA_TRANSLUCENT) {
                        float sa = __fdiv_rn((float)(sh.texel >> 24), 255.0f);
                        int sp;
                        V3 sa3 = texel_albedo(S, T.F, sq, sh, sp);
                        V3 stint = linear_rgb(S.gamma, __float_as_uint(ldg(&sq->eu_tint).w));
                        V3 f = lerp(v3(1.0f, 1.0f, 1.0f), vmul(sa3, stint), sa);
                        tr = vmul(tr, f);
                        if (GRAD && sp >= 0 && nt < 8) {
                            tparam[nt] = sp;
                            tlam[nt] = vmul(stint * sa, inv3(f));
                            nt++;
                        }
                    } else {
                        tr = v3(0.0f, 0.0f, 0.0f);
                        break;
                    }
                    so = so + l0 * (sh.t + eps);
                    tmax -= sh.t + eps;
                    ucum = u + eps;
                    ul_prev = ul;
                    du_prev = du;
                }
                V3 s_term = vmul(vmul(beta_a, f4v(P.sun_color)), tr) * cos_l;
                acc(radiance, s_term);
                if (GRAD && (s_term.x != 0.0f || s_term.y != 0.0f || s_term.z != 0.0f)) {
                    V3 ws = vmul(w, s_term);
                    // d s_term(c) / dl = s_term(c) (n / cos_l - sigma(c) sum over water segments of dt/dl)
                    V3 gl = n * __fdiv_rn(ws.x + ws.y + ws.z, cos_l) - vw * dot(ws, sigma);
                    float J[3][3];
                    cone_dir_jacobian(sun, P.sun_dir.w, r1, r2, J);
                    for (int j = 0; j < 3; j++) {
                        double gj = (double)gl.x * J[0][j] + (double)gl.y * J[1][j] + (double)gl.z * J[2][j];
                        if (gj != 0.0 && isfinite(gj)) atomicAdd(go.sun + j, gj);
                    }
                    for (int k = 0; k < nt; k++) add_albedo(go, tparam[k], w, s_term, tlam[k]);
                }
            }
        }
        if (!emits && strategy != EMITTER_SAMPLING_NONE) {
            // sample_emitters (integrator.rs:441-469), each face's term kept for its gradients.
            uint32_t start, count;
            emitter_cell(S, pos, start, count);
            V3 esum = v3(0.0f, 0.0f, 0.0f);
            if (count > 0) {
                const uint32_t *eg = S.emitter_grid;
                uint32_t list = EMITTER_GRID_HEADER + ldg(eg + 1) * ldg(eg + 2) * ldg(eg + 3) * 2u + start;
                uint32_t k0 = 0, k1 = count;
                float escale = kPI;
                if (strategy == EMITTER_SAMPLING_ONE || strategy == EMITTER_SAMPLING_ONE_BLOCK) {
                    k0 = pick(count, rng_next(rng));
                    k1 = k0 + 1;
                } else if (strategy == EMITTER_SAMPLING_ALL) {
                    escale = __fdiv_rn(kPI, (float)count);
                } else {
                    k1 = 0;
                }
                for (uint32_t kk = k0; kk < k1; kk++) {
                    uint32_t ei = ldg(eg + list + kk);
                    float4 e0 = ldg(S.emitters + 2u * ei), e1 = ldg(S.emitters + 2u * ei + 1u);
                    uint32_t faces = __float_as_uint(e1.x);
                    if (faces == 0) continue;
                    uint32_t g = emitter_group(to_i32(e0.x), to_i32(e0.y), to_i32(e0.z));
                    float mult = ldg(T.F.emit_mult + g);
                    uint32_t f0 = 0, f1 = faces;
                    float scaler = __fdiv_rn(1.0f, (float)faces);
                    if (P.emitter.x == EMITTER_SAMPLING_ONE) {
                        f0 = pick(faces, rng_next(rng));
                        f1 = f0 + 1;
                        scaler = 1.0f;
                    }
                    V3 fsum = v3(0.0f, 0.0f, 0.0f);
                    for (uint32_t f = f0; f < f1; f++) {
                        const DevQuad *eq = S.quads + __float_as_uint(e0.w) + f;
                        float s = rng_next(rng);
                        float t = rng_next(rng);
                        V3 at = f4v(e0) + f4v(ldg(&eq->p0_flags)) + f4v(ldg(&eq->eu_tint)) * s + f4v(ldg(&eq->ev_em)) * t;
                        V3 to = at - origin;
                        V3 val = v3(0.0f, 0.0f, 0.0f);
                        if (dot(to, n) > 0.0f) {
                            float dist = vlength(to);
                            V3 ll = vdiv(to, dist);
                            Hit eh = trace<false>(S, P, origin, ll, eps, dist + 2.0f * eps);
                            if (eh.quad != NO_QUAD && !(fabs_r(eh.t - dist) >= 2.0f * eps)) {
                                V3 nq = -f4v(ldg(&eq->n_nn));
                                float area = vlength(nq);
                                float cos_e = __fdiv_rn(fabs_r(dot(nq, ll)), area);
                                const DevQuad *hq = S.quads + eh.quad;
                                int eparam;
                                V3 ea = texel_albedo(S, T.F, hq, eh, eparam);
                                V3 c = vmul(ea, linear_rgb(S.gamma, __float_as_uint(ldg(&hq->eu_tint).w)));
                                val = c * (__fdiv_rn(cos_e, fmax_r(dist * dist, 1.0f)) * area * ldg(&eq->ev_em).w *
                                           (P.misc_f.x * mult) * scaler);
                                if (GRAD) {
                                    V3 term = vmul(beta_a, val) * escale;  // this face's share of the radiance
                                    if (eparam >= 0) add_albedo(go, eparam, w, term, inv3(ea));
                                    if (mult != 0.0f) atomicAdd(go.emit + g, (double)dot(w, term) / mult);
                                }
                            }
                        }
                        fsum = (P.emitter.x == EMITTER_SAMPLING_ONE) ? val : fsum + val;
                    }
                    esum = (strategy == EMITTER_SAMPLING_ALL) ? esum + fsum : fsum;
                }
                esum = esum * escale;
            }
            acc(radiance, vmul(beta_a, esum));
        }
        beta = beta_a;
        beta0 = FD ? vmul(beta0, albedo0) : beta;
        // Every term from this vertex's emission on carries its albedo (the emission twice).
        if (GRAD && param >= 0) add_albedo(go, param, w, vsub(L, l_before) + e_term, inv3(a));
        if (bounces >= 3u) {
            float q_rr = clamp_r(max_elem(FD ? beta0 : beta), 0.05f, 0.95f);
            if (rng_next(rng) > q_rr) break;
            beta = vdiv(beta, q_rr);
            beta0 = FD ? vdiv(beta0, q_rr) : beta;
        }
        d = cosine_hemisphere(n, rng);
        o = origin;
        tmin = 0.0f;
        specular = false;
    }
    return radiance;
}

// One thread per (pixel, run of `chunk` samples).
struct Cell {
    uint32_t px, py, pix, s0, s1;
};
LW_DI bool cell_of(const DevParams &P, uint32_t spp, uint32_t chunk, Cell &c) {
    uint32_t w = P.frame.x, h = P.frame.y;
    uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t npix = (uint64_t)w * h;
    uint32_t chunks = (spp + chunk - 1) / chunk;
    if (g >= npix * chunks) return false;
    c.pix = (uint32_t)(g % npix);
    uint32_t ck = (uint32_t)(g / npix);
    c.px = c.pix % w;
    c.py = c.pix / w;
    c.s0 = ck * chunk;
    c.s1 = min(spp, c.s0 + chunk);
    return true;
}

// The per-pixel mean radiance of samples [0, spp) with theta (non-finite samples left out of the
// sum, every sample counted).
// With `Ls`, each sample's radiance is kept there ([pixel * spp + sample]) for the backward pass.
__global__ void LW_ADJ_BOUNDS(LW_ADJ_FWD_MINB) k_adj_forward(const DevScene S, const Theta T, uint32_t spp, uint32_t chunk, double *img, DV *Ls) {
    Cell c;
    if (!cell_of(T.F.P, spp, chunk, c)) return;
    const AdjGrad none{};
    double a0 = 0, a1 = 0, a2 = 0;
    for (uint32_t s = c.s0; s < c.s1; s++) {
        DV r = path<M_FWD>(S, T, c.px, c.py, s, DV{}, V3{}, none);
        if (Ls) Ls[(size_t)c.pix * spp + s] = r;
        if (finite_dv(r)) {
            a0 += r.x;
            a1 += r.y;
            a2 += r.z;
        }
    }
    atomicAdd(img + 3 * c.pix, a0 / spp);
    atomicAdd(img + 3 * c.pix + 1, a1 / spp);
    atomicAdd(img + 3 * c.pix + 2, a2 / spp);
}

// Replay 1 (or the forward pass's kept radiance `Ls`) then replay 2 per sample; d_img = dLoss/dI
// per pixel.
__global__ void LW_ADJ_BOUNDS(LW_ADJ_BWD_MINB) k_adj_backward(const DevScene S, const Theta T, uint32_t spp, uint32_t chunk, const double *d_img,
                               const AdjGrad go, const DV *Ls) {
    Cell c;
    if (!cell_of(T.F.P, spp, chunk, c)) return;
    V3 w = v3((float)(d_img[3 * c.pix] / spp), (float)(d_img[3 * c.pix + 1] / spp), (float)(d_img[3 * c.pix + 2] / spp));
    if (w.x == 0.0f && w.y == 0.0f && w.z == 0.0f) return;
    for (uint32_t s = c.s0; s < c.s1; s++) {
        DV L = Ls ? Ls[(size_t)c.pix * spp + s] : path<M_FWD>(S, T, c.px, c.py, s, DV{}, V3{}, go);
        if (!finite_dv(L)) continue;
        (void)path<M_GRAD>(S, T, c.px, c.py, s, L, w, go);
    }
}

// Every sample with theta+ and theta-: per pixel the means of the paired differences and of the
// pairs' midpoints (f64).
__global__ void k_adj_fd(const DevScene S, const Theta Tp, const Theta Tm, uint32_t spp, uint32_t chunk, double *diff,
                         double *mean) {
    Cell c;
    if (!cell_of(Tp.F.P, spp, chunk, c)) return;
    const AdjGrad none{};
    double d0 = 0, d1 = 0, d2 = 0, m0 = 0, m1 = 0, m2 = 0;
    for (uint32_t s = c.s0; s < c.s1; s++) {
        DV a = path<M_FD>(S, Tp, c.px, c.py, s, DV{}, V3{}, none);
        DV b = path<M_FD>(S, Tm, c.px, c.py, s, DV{}, V3{}, none);
        if (!finite_dv(a) || !finite_dv(b)) continue;
        d0 += a.x - b.x;
        d1 += a.y - b.y;
        d2 += a.z - b.z;
        m0 += 0.5 * (a.x + b.x);
        m1 += 0.5 * (a.y + b.y);
        m2 += 0.5 * (a.z + b.z);
    }
    atomicAdd(diff + 3 * c.pix, d0 / spp);
    atomicAdd(diff + 3 * c.pix + 1, d1 / spp);
    atomicAdd(diff + 3 * c.pix + 2, d2 / spp);
    atomicAdd(mean + 3 * c.pix, m0 / spp);
    atomicAdd(mean + 3 * c.pix + 1, m1 / spp);
    atomicAdd(mean + 3 * c.pix + 2, m2 / spp);
}

}  // namespace adj

namespace {
constexpr uint32_t kAdjChunk = 4;
constexpr int kAdjThreads = 128;
unsigned adj_blocks(const DevParams &P, uint32_t spp) {
    uint64_t n = (uint64_t)P.frame.x * P.frame.y * ((spp + kAdjChunk - 1) / kAdjChunk);
    return (unsigned)((n + kAdjThreads - 1) / kAdjThreads);
}
}  // namespace

cudaError_t launch_adj_forward(const DevScene &S, const AdjFrame &F, uint32_t spp, double *img, double *Ls,
                               cudaStream_t st) {
    adj::Theta t{F, F.albedo, F.P.sun_dir};
    adj::k_adj_forward<<<adj_blocks(F.P, spp), kAdjThreads, 0, st>>>(S, t, spp, kAdjChunk, img, (adj::DV *)Ls);
    return cudaGetLastError();
}

cudaError_t launch_adj_backward(const DevScene &S, const AdjFrame &F, uint32_t spp, const double *d_img,
                                const AdjGrad &G, const double *Ls, cudaStream_t st) {
    adj::Theta t{F, F.albedo, F.P.sun_dir};
    adj::k_adj_backward<<<adj_blocks(F.P, spp), kAdjThreads, 0, st>>>(S, t, spp, kAdjChunk, d_img, G,
                                                                      (const adj::DV *)Ls);
    return cudaGetLastError();
}

cudaError_t launch_adj_fd(const DevScene &S, const AdjFrame &plus, const AdjFrame &minus, const float *albedo0,
                          float4 sun0, uint32_t spp, double *diff, double *mean, cudaStream_t st) {
    adj::Theta a{plus, albedo0, sun0};
    adj::Theta b{minus, albedo0, sun0};
    adj::k_adj_fd<<<adj_blocks(plus.P, spp), kAdjThreads, 0, st>>>(S, a, b, spp, kAdjChunk, diff, mean);
    return cudaGetLastError();
}

}  // namespace lw
