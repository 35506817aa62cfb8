/*
 * The oracle kernel, written once for two arithmetic types. kernel32.c includes it with
 * REAL = float (the reference's own arithmetic), kernel64.c with REAL = double (the FP64
 * twin). Each function cites the reference function it restates; operation order,
 * parenthesisation and comparisons follow the reference so the FP32 build rounds alike.
 *
 * Test infrastructure only (see lw_oracle.h).
 *
 * The including file defines:
 *   REAL, PFX(name), K(lit)                 type, symbol prefix, literal of type REAL
 *   R_SQRT, R_FLOOR, R_EXP, R_FMOD          libm functions of type REAL
 *   R_TEXP                                  the exponential of the water transmittance
 *   R_ACOS, R_ATAN2, R_GAMMA, R_SINCOS_TURNS the kernel's transcendental functions
 *   LWO_F64                                  defined in the double build
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "lw_oracle.h"

/* ---- scene layout constants (crates/lumenwright-kernel/src/scene.rs:16-37, 144-155) ---- */
#define EMPTY 0xFFFFFFFFu
#define UNIFORM 0x80000000u
#define BRICK_WORDS 2048u
#define OV_CELL_WORDS 8192u
#define ALPHA_CUTOUT 1u
#define ALPHA_TRANSLUCENT 2u
#define FLAG_ALPHA_MASK 3u
#define FLAG_WATER 4u
#define FLAG_FRONT_ONLY 16u
#define EMITTER_SAMPLING_NONE 0u
#define EMITTER_SAMPLING_ONE 1u
#define EMITTER_SAMPLING_ONE_BLOCK 2u
#define EMITTER_SAMPLING_ALL 3u
#define EMITTER_GRID_HEADER 8u
#define MAX_STEPS 65536u /* trace.rs:31 */
#define MAX_EVENTS 48u   /* integrator.rs:24 */

extern uint64_t lwo_bounds_error_count;
extern __thread lwo_counters *lwo_cnt;
#define CNT(f)                \
    do {                      \
        if (lwo_cnt) lwo_cnt->f++; \
    } while (0)

/* The differentiable form's theta (FP64 build only; the FP32 build never has one). */
#ifdef LWO_F64
extern __thread const lwo_theta *lwo_th;
#define TH lwo_th
#else
#define TH ((const lwo_theta *)0)
#endif

static inline float f32_of(uint32_t u) {
    float f;
    memcpy(&f, &u, 4);
    return f;
}
static inline uint32_t bits_of(float f) {
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
}

/* Rust's saturating float-to-int casts (`as i32`, `as u32`): NaN gives 0. */
static inline int32_t to_i32(REAL x) {
    if (x != x) return 0;
    if (x <= (REAL)-2147483648.0) return INT32_MIN;
    if (x >= (REAL)2147483647.0) return INT32_MAX;
    return (int32_t)x;
}
static inline uint32_t to_u32(REAL x) {
    if (x != x || x <= (REAL)0) return 0;
    if (x >= (REAL)4294967295.0) return UINT32_MAX;
    return (uint32_t)x;
}
static inline int32_t clamp_i32(int32_t v, int32_t lo, int32_t hi) {
    return v < lo ? lo : (v > hi ? hi : v);
}

/* Bounds-checked buffer reads: an out-of-range index is counted and reads 0, where the
 * reference would panic. Valid scenes never trigger it (tests check the count). */
static inline void bounds_error(void) {
    __atomic_fetch_add(&lwo_bounds_error_count, 1, __ATOMIC_RELAXED);
    CNT(bounds_errors);
}
static inline uint32_t GRID(const lwo_scene *s, uint64_t i) {
    if (i >= s->grid_len) { bounds_error(); return 0; }
    return s->grid[i];
}
static inline uint32_t EGRID(const lwo_scene *s, uint64_t i) {
    if (i >= s->emitter_grid_len) { bounds_error(); return 0; }
    return s->emitter_grid[i];
}
static const lwo_quad zero_quad;
static inline const lwo_quad *QUAD(const lwo_scene *s, uint64_t i) {
    if (i >= s->quads_len) { bounds_error(); return &zero_quad; }
    return &s->quads[i];
}
static inline lwo_model MODEL(const lwo_scene *s, uint64_t i) {
    lwo_model z = {0, 0, 0, 0};
    if (i >= s->models_len) { bounds_error(); return z; }
    return s->models[i];
}
static inline lwo_emitter EMITTER(const lwo_scene *s, uint64_t i) {
    lwo_emitter z;
    memset(&z, 0, sizeof z);
    if (i >= s->emitters_len) { bounds_error(); return z; }
    return s->emitters[i];
}
static inline REAL SKY(const lwo_scene *s, uint64_t i) {
    if (TH && TH->sky64) {
        if (i >= TH->sky64_len) { bounds_error(); return 0; }
        return (REAL)TH->sky64[i];
    }
    if (i >= s->sky_len) { bounds_error(); return 0; }
    return (REAL)s->sky[i];
}
static inline uint32_t ATLAS(const lwo_scene *s, uint64_t i) {
    if (i >= s->atlas_len) { bounds_error(); return 0; }
    return s->atlas[i];
}

/* ---- V3 (math.rs:218-344) ------------------------------------------------------------ */
typedef struct { REAL x, y, z; } V3;
static inline V3 v3(REAL x, REAL y, REAL z) { V3 r = {x, y, z}; return r; }
static inline V3 v3f4(const float a[4]) { return v3((REAL)a[0], (REAL)a[1], (REAL)a[2]); }
static inline V3 vadd(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 vsub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 vmuls(V3 a, REAL s) { return v3(a.x * s, a.y * s, a.z * s); }
static inline V3 vmul(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline V3 vneg(V3 a) { return v3(-a.x, -a.y, -a.z); }
static inline REAL vdot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3 vcross(V3 a, V3 o) {
    return v3(a.y * o.z - a.z * o.y, a.z * o.x - a.x * o.z, a.x * o.y - a.y * o.x);
}
static inline REAL vlength(V3 a) { return R_SQRT(vdot(a, a)); }
static inline V3 vnormalize(V3 a) {
    REAL l = vlength(a);
    return l > K(0.0) ? vmuls(a, K(1.0) / l) : a;
}
static inline V3 vdivs(V3 a, REAL s) { return vmuls(a, K(1.0) / s); }
static inline REAL rmin(REAL a, REAL b) { return a < b ? a : b; } /* math.rs:155 */
static inline REAL rmax(REAL a, REAL b) { return a > b ? a : b; } /* math.rs:161 */
static inline REAL rabs(REAL x) { return x < K(0.0) ? -x : x; }   /* math.rs:149 */
static inline REAL rclamp(REAL x, REAL lo, REAL hi) { return rmin(rmax(x, lo), hi); }
static inline REAL vmax_elem(V3 a) { return rmax(a.x, rmax(a.y, a.z)); }
static inline REAL vget(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
static inline V3 vlerp(V3 a, V3 o, REAL t) { return vadd(a, vmuls(vsub(o, a), t)); }
static inline V3 vtransmittance(V3 a, REAL t) { /* math.rs:300 */
    return v3(R_TEXP(-a.x * t), R_TEXP(-a.y * t), R_TEXP(-a.z * t));
}
static const V3 V3_ZERO = {0, 0, 0};
static const V3 V3_ONE = {1, 1, 1};

/* Duff et al. 2017 basis (math.rs:348-356). */
static inline void onb(V3 n, V3 *t, V3 *b) {
    REAL sign = n.z >= K(0.0) ? K(1.0) : K(-1.0);
    REAL a = K(-1.0) / (sign + n.z);
    REAL bb = n.x * n.y * a;
    *t = v3(K(1.0) + sign * n.x * n.x * a, sign * bb, -sign * n.x);
    *b = v3(bb, sign + n.y * n.y * a, -n.y);
}

/* ---- RNG (rng.rs:5-34) ---------------------------------------------------------------- */
static inline uint32_t pcg_hash(uint32_t v) {
    uint32_t state = v * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28) + 4u)) ^ state) * 277803737u;
    return (word >> 22) ^ word;
}
static inline uint32_t rng_new(uint32_t pixel, uint32_t sample, uint32_t seed) {
    return pcg_hash(pixel ^ pcg_hash(sample + pcg_hash(seed)));
}
static inline REAL rng_next(uint32_t *st) {
    *st = pcg_hash(*st);
    /* (state >> 8) as f32 * (1 / 2^24): exact in both types. */
    return (REAL)(*st >> 8) * (K(1.0) / K(16777216.0));
}

/* unpack_rgba (scene.rs:299-306) and linear_rgb (integrator.rs:27-34). */
static inline REAL unpack_c(uint32_t c, int k) { return (REAL)((c >> (8 * k)) & 0xFFu) / K(255.0); }
static inline V3 linear_rgb(uint32_t c) {
    return v3(R_GAMMA(unpack_c(c, 0)), R_GAMMA(unpack_c(c, 1)), R_GAMMA(unpack_c(c, 2)));
}

/* ---- quad accessors (scene.rs:59-97) ---------------------------------------------------- */
static inline uint32_t q_flags(const lwo_quad *q) { return bits_of(q->p0[3]); }
static inline uint32_t q_tint(const lwo_quad *q) { return bits_of(q->eu[3]); }
static inline REAL q_emittance(const lwo_quad *q) { return (REAL)q->ev[3]; }
static inline V3 q_origin(const lwo_quad *q) { return v3f4(q->p0); }
static inline V3 q_eu(const lwo_quad *q) { return v3f4(q->eu); }
static inline V3 q_ev(const lwo_quad *q) { return v3f4(q->ev); }
static inline V3 q_normal(const lwo_quad *q) { return vcross(q_ev(q), q_eu(q)); }

static inline V3 grid_size(const lwo_scene *s) { /* scene.rs:264-267 */
    const uint32_t *d = s->params->grid_dims;
    return v3((REAL)(d[0] * 16u), (REAL)(d[1] * 16u), (REAL)(d[2] * 16u));
}

/* SceneView::voxel (scene.rs:271-284). */
static uint32_t voxel(const lwo_scene *s, int32_t x, int32_t y, int32_t z) {
    const uint32_t *d = s->params->grid_dims;
    uint32_t b = (((uint32_t)(y >> 4) * d[2] + (uint32_t)(z >> 4)) * d[0] + (uint32_t)(x >> 4));
    uint32_t e = GRID(s, (uint64_t)s->params->off[0] + b);
    if (e == EMPTY) return 0;
    if (e & UNIFORM) return e & ~UNIFORM;
    uint32_t local = (uint32_t)((((y & 15) * 16 + (z & 15)) * 16) + (x & 15));
    uint32_t w = GRID(s, (uint64_t)(s->params->off[1] + e * BRICK_WORDS + (local >> 1)));
    return (w >> ((local & 1u) * 16u)) & 0xFFFFu;
}

/* SceneView::texel (scene.rs:288-294). */
static inline uint32_t texel(const lwo_scene *s, REAL u, REAL v) {
    int32_t w = (int32_t)s->params->off2[1];
    int32_t h = (int32_t)s->params->off2[2];
    int32_t x = clamp_i32(to_i32(R_FLOOR(u)), 0, w - 1);
    int32_t y = clamp_i32(to_i32(R_FLOOR(v)), 0, h - 1);
    CNT(texel_fetches);
    return ATLAS(s, (uint64_t)(uint32_t)(y * w + x));
}

/* ---- trace.rs ---------------------------------------------------------------------------- */
typedef struct { REAL t; uint32_t quad, texel; REAL s, tt; } Hit;
#define NO_QUAD 0xFFFFFFFFu
static inline Hit no_hit(void) {
    Hit h = {(REAL)INFINITY, NO_QUAD, 0, K(0.0), K(0.0)};
    return h;
}

/* ---- chunk-origin frames (the library's precision option; the reference has none) -------- */
/* With Params.see_through[2] = 1 the library holds a path's positions relative to a chunk corner
 * A of the grid (a multiple of 16 blocks per axis), the corner nearest the path's current origin,
 * starting from the camera's corner packed in see_through[3] (chunk indices, two's complement: x in
 * bits 0-10, y in 11-20, z in 21-31); the grid's cell c is the frame's integer c - A. Restated from
 * the library's kernels (csrc/device_scene.cuh `Frame`, `rebase`). The sample being rendered sets
 * the frame here, per thread; every other entry point runs in the grid's frame (A = 0). */
static __thread int lwo_reb;
static __thread int32_t lwo_fa[3];
static inline void frame_unpack(uint32_t w, int32_t a[3]) {
    a[0] = ((int32_t)(w << 21) >> 21) * 16;
    a[1] = ((int32_t)(w << 11) >> 22) * 16;
    a[2] = ((int32_t)w >> 21) * 16;
}
static inline V3 frame_origin(const int32_t a[3]) { return v3((REAL)a[0], (REAL)a[1], (REAL)a[2]); }
/* rint(x / 16), kept within +-4096 (NaN to -4096). */
static inline int32_t chunk_step(REAL x) {
    double r = rint((double)(x * K(0.0625)));
    if (!(r >= -4096.0)) r = -4096.0;
    if (r > 4096.0) r = 4096.0;
    return (int32_t)r;
}
/* x (in the current frame) moved to the frame of the chunk corner nearest it, which becomes the
 * current frame: k = rint(x / 16) chunks per axis (the frame within the packable chunk range),
 * x - 16 k, exactly (16 k and x are multiples of x's ulp, and |x - 16 k| <= |x| when k != 0). */
static inline V3 rebase(V3 x) {
    const int32_t c[3] = {lwo_fa[0] >> 4, lwo_fa[1] >> 4, lwo_fa[2] >> 4};
    const int32_t n[3] = {clamp_i32(c[0] + chunk_step(x.x), -1024, 1023), clamp_i32(c[1] + chunk_step(x.y), -512, 511),
                          clamp_i32(c[2] + chunk_step(x.z), -1024, 1023)};
    V3 r = v3(x.x - (REAL)((n[0] - c[0]) * 16), x.y - (REAL)((n[1] - c[1]) * 16), x.z - (REAL)((n[2] - c[2]) * 16));
    for (int a = 0; a < 3; a++) lwo_fa[a] = n[a] * 16;
    return r;
}

/* intersect_quad (trace.rs:37-58). Returns 1 and (t, s, tt) on a hit. With `pb` the quad's p0 is
 * taken relative to *pb (a quad given in grid coordinates, a ray in a chunk frame). */
static inline int intersect_quad(const lwo_quad *q, V3 o, V3 d, REAL tmin, REAL tmax, REAL *pt,
                                 REAL *ps, REAL *ptt, const V3 *pb) {
    V3 eu = q_eu(q), ev = q_ev(q);
    V3 n = vcross(eu, ev);
    REAL denom = vdot(n, d);
    if (rabs(denom) < K(1e-12)) return 0;
    V3 p0 = q_origin(q);
    if (pb) p0 = vsub(p0, *pb);
    REAL t = vdot(n, vsub(p0, o)) / denom;
    if (!(t > tmin && t < tmax)) return 0;
    V3 p = vsub(vadd(o, vmuls(d, t)), p0);
    REAL nn = vdot(n, n);
    REAL s = vdot(vcross(p, ev), n) / nn;
    REAL tt = vdot(vcross(eu, p), n) / nn;
    if (s < K(0.0) || s > K(1.0) || tt < K(0.0) || tt > K(1.0)) return 0;
    *pt = t;
    *ps = s;
    *ptt = tt;
    return 1;
}

/* quad_texel (trace.rs:62-69). */
static inline uint32_t quad_texel(const lwo_scene *s, const lwo_quad *q, REAL ss, REAL t) {
    ss = rmin(rmax(ss, K(0.0005)), K(0.9995));
    t = rmin(rmax(t, K(0.0005)), K(0.9995));
    REAL u = (REAL)q->uv[0] + ss * (REAL)q->uv[2] + t * (REAL)q->uvt[0];
    REAL v = (REAL)q->uv[1] + ss * (REAL)q->uv[3] + t * (REAL)q->uvt[1];
    return texel(s, u, v);
}

/* The atlas index quad_texel reads. */
static inline uint64_t quad_texel_index(const lwo_scene *s, const lwo_quad *q, REAL ss, REAL t) {
    ss = rmin(rmax(ss, K(0.0005)), K(0.9995));
    t = rmin(rmax(t, K(0.0005)), K(0.9995));
    REAL u = (REAL)q->uv[0] + ss * (REAL)q->uv[2] + t * (REAL)q->uvt[0];
    REAL v = (REAL)q->uv[1] + ss * (REAL)q->uv[3] + t * (REAL)q->uvt[1];
    int32_t w = (int32_t)s->params->off2[1];
    int32_t h = (int32_t)s->params->off2[2];
    int32_t x = clamp_i32(to_i32(R_FLOOR(u)), 0, w - 1);
    int32_t y = clamp_i32(to_i32(R_FLOOR(v)), 0, h - 1);
    return (uint64_t)(uint32_t)(y * w + x);
}

#define COPLANAR K(1e-5) /* trace.rs:73 */

/* test_quad (trace.rs:81-109). */
static inline void test_quad(const lwo_scene *s, uint32_t qi, V3 o, V3 d, REAL tmin, Hit *best, const V3 *pb) {
    const lwo_quad *q = QUAD(s, qi);
    CNT(quad_tests);
    REAL reach = (best->quad != NO_QUAD && qi > best->quad) ? best->t + COPLANAR : best->t;
    REAL t, ss, tt;
    if (intersect_quad(q, o, d, tmin, reach, &t, &ss, &tt, pb)) {
        if ((q_flags(q) & FLAG_FRONT_ONLY) && vdot(q_normal(q), d) >= K(0.0)) return;
        uint32_t tx = quad_texel(s, q, ss, tt);
        uint32_t alpha = tx >> 24;
        uint32_t mode = q_flags(q) & FLAG_ALPHA_MASK;
        if ((mode == ALPHA_CUTOUT && alpha < 128u) || (mode == ALPHA_TRANSLUCENT && alpha == 0u)) return;
        best->t = t;
        best->quad = qi;
        best->texel = tx;
        best->s = ss;
        best->tt = tt;
    }
}

/* is_see_through (trace.rs:113-116). */
static inline int is_see_through(const lwo_scene *s, uint32_t qi) {
    const uint32_t *st = s->params->see_through;
    return qi >= st[0] && qi - st[0] < st[1];
}

/* see_through_hit (trace.rs:120-131); in a chunk frame the quads' p0 relative to its origin. */
static Hit see_through_hit(const lwo_scene *s, V3 o, V3 d, REAL tmin) {
    const uint32_t *st = s->params->see_through;
    Hit best = no_hit();
    V3 fo = frame_origin(lwo_fa);
    for (uint32_t i = 0; i < st[1]; i++) test_quad(s, st[0] + i, o, d, tmin, &best, lwo_reb ? &fo : NULL);
    return best;
}

static inline REAL safe_inv(REAL x) { /* trace.rs:293-299 */
    if (rabs(x) < K(1e-12)) return x < K(0.0) ? K(-1e12) : K(1e12);
    return K(1.0) / x;
}
static inline int32_t sgn(REAL x) { return x > K(0.0) ? 1 : (x < K(0.0) ? -1 : 0); }
/* `a`: the frame's origin on this axis (grid cell c's boundary is at c - a in the frame). */
static inline REAL next_boundary(REAL o, REAL inv, int32_t cell, int32_t step, int32_t a) { /* :313-319 */
    if (step == 0) return (REAL)INFINITY;
    REAL bound = (REAL)((step > 0 ? cell + 1 : cell) - a);
    return (bound - o) * inv;
}

/* trace (trace.rs:137-290), with o in the current frame: the grid spans [-A, size - A) there. */
static Hit trace(const lwo_scene *s, V3 o, V3 d, REAL tmin, REAL tmax) {
    const lwo_params *p = s->params;
    const uint32_t *dims = p->grid_dims;
    const int32_t A[3] = {lwo_reb ? lwo_fa[0] : 0, lwo_reb ? lwo_fa[1] : 0, lwo_reb ? lwo_fa[2] : 0};
    V3 lo = v3((REAL)(-A[0]), (REAL)(-A[1]), (REAL)(-A[2]));
    V3 hi = v3((REAL)((int32_t)(dims[0] * 16u) - A[0]), (REAL)((int32_t)(dims[1] * 16u) - A[1]),
               (REAL)((int32_t)(dims[2] * 16u) - A[2]));
    CNT(traces);

    V3 inv = v3(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z));
    V3 ta = vmul(vsub(lo, o), inv);
    V3 tb = vmul(vsub(hi, o), inv);
    REAL t_enter = rmax(rmax(rmin(ta.x, tb.x), rmin(ta.y, tb.y)), rmin(ta.z, tb.z));
    REAL t_exit = rmin(rmin(rmax(ta.x, tb.x), rmax(ta.y, tb.y)), rmax(ta.z, tb.z));
    REAL t = rmax(t_enter, K(0.0));
    REAL t_end = rmin(t_exit, tmax);
    if (t > t_end) return no_hit();

    V3 start = vadd(o, vmuls(d, t + K(1e-4)));
    int32_t gs[3] = {(int32_t)dims[0] * 16, (int32_t)dims[1] * 16, (int32_t)dims[2] * 16};
    int32_t cell[3] = {clamp_i32(to_i32(R_FLOOR(start.x)) + A[0], 0, gs[0] - 1),
                       clamp_i32(to_i32(R_FLOOR(start.y)) + A[1], 0, gs[1] - 1),
                       clamp_i32(to_i32(R_FLOOR(start.z)) + A[2], 0, gs[2] - 1)};
    int32_t step[3] = {sgn(d.x), sgn(d.y), sgn(d.z)};
    REAL next[3];
    for (int a = 0; a < 3; a++) next[a] = next_boundary(vget(o, a), vget(inv, a), cell[a], step[a], A[a]);

    uint32_t top_off = p->off[0];
    uint32_t ov_top_off = p->off[2];
    REAL best_t = t_end + K(1e-3);

    for (uint32_t it = 0; it < MAX_STEPS; it++) {
        CNT(dda_steps);
        uint32_t bx = (uint32_t)(cell[0] >> 4), by = (uint32_t)(cell[1] >> 4), bz = (uint32_t)(cell[2] >> 4);
        uint32_t b = (by * dims[2] + bz) * dims[0] + bx;
        uint32_t entry = GRID(s, (uint64_t)(top_off + b));
        uint32_t ov = GRID(s, (uint64_t)(ov_top_off + b));

        if (entry == EMPTY && ov == EMPTY) {
            CNT(brick_skips);
            int32_t bc[3] = {(int32_t)bx, (int32_t)by, (int32_t)bz};
            REAL t_out = (REAL)INFINITY;
            int axis = 0;
            for (int a = 0; a < 3; a++) {
                if (step[a] != 0) {
                    int32_t bound = step[a] > 0 ? (bc[a] + 1) * 16 : bc[a] * 16;
                    REAL tt = ((REAL)(bound - A[a]) - vget(o, a)) * vget(inv, a);
                    if (tt < t_out) { t_out = tt; axis = a; }
                }
            }
            if (t_out > t_end) break;
            V3 pos = vadd(o, vmuls(d, t_out));
            for (int a = 0; a < 3; a++) {
                if (a == axis)
                    cell[a] = step[a] > 0 ? (bc[a] + 1) * 16 : bc[a] * 16 - 1;
                else
                    cell[a] = clamp_i32(to_i32(R_FLOOR(vget(pos, a))) + A[a], bc[a] * 16, bc[a] * 16 + 15);
            }
            if (cell[axis] < 0 || cell[axis] >= gs[axis]) break;
            for (int a = 0; a < 3; a++) next[a] = next_boundary(vget(o, a), vget(inv, a), cell[a], step[a], A[a]);
            t = t_out;
            continue;
        }

        REAL t_cell_exit = rmin(next[0], rmin(next[1], next[2]));
        REAL t_lo = rmax(t - K(1e-4), tmin);
        REAL t_hi = t_cell_exit + K(1e-4);

        uint32_t model;
        if (entry == EMPTY) {
            model = 0;
        } else if (entry & UNIFORM) {
            model = entry & ~UNIFORM;
        } else {
            uint32_t local = (uint32_t)((((cell[1] & 15) * 16 + (cell[2] & 15)) * 16) + (cell[0] & 15));
            CNT(voxel_lookups);
            uint32_t w = GRID(s, (uint64_t)(p->off[1] + entry * BRICK_WORDS + (local >> 1)));
            model = (w >> ((local & 1u) * 16u)) & 0xFFFFu;
        }
        Hit cand = no_hit();
        cand.t = rmin(t_hi, best_t);
        /* the origin relative to the cell: o - (c - A) */
        V3 olo = vsub(o, v3((REAL)(cell[0] - A[0]), (REAL)(cell[1] - A[1]), (REAL)(cell[2] - A[2])));
        if (model != 0) {
            lwo_model m = MODEL(s, model);
            CNT(model_fetches);
            for (uint32_t i = 0; i < m.quad_count; i++) test_quad(s, m.quad_offset + i, olo, d, t_lo, &cand, NULL);
        }
        if (ov != EMPTY) {
            uint32_t local = (uint32_t)((((cell[1] & 15) * 16 + (cell[2] & 15)) * 16) + (cell[0] & 15));
            uint64_t base = (uint64_t)(p->off[3] + ov * OV_CELL_WORDS + local * 2u);
            uint32_t off = GRID(s, base);
            uint32_t count = GRID(s, base + 1);
            CNT(overlay_reads);
            /* in a chunk frame relative to the cell, like a model's quads: the quads' p0 - c */
            V3 cv = v3((REAL)cell[0], (REAL)cell[1], (REAL)cell[2]);
            for (uint32_t i = 0; i < count; i++) {
                uint32_t qi = GRID(s, (uint64_t)(p->off2[0] + off + i));
                if (lwo_reb) test_quad(s, qi, olo, d, t_lo, &cand, &cv);
                else test_quad(s, qi, o, d, t_lo, &cand, NULL);
            }
        }
        if (cand.quad != NO_QUAD) return cand;

        int axis = next[0] < next[1] ? (next[0] < next[2] ? 0 : 2) : (next[1] < next[2] ? 1 : 2);
        t = next[axis];
        if (t > t_end) break;
        cell[axis] += step[axis];
        if (cell[axis] < 0 || cell[axis] >= gs[axis]) break;
        next[axis] = next_boundary(vget(o, axis), vget(inv, axis), cell[axis], step[axis], A[axis]);
    }
    return no_hit();
}

/* ---- integrator.rs ---------------------------------------------------------------------- */
#define PI_R K(3.14159265358979323846)

/* preetham_radiance (integrator.rs:44-74). */
static V3 preetham_radiance(const lwo_scene *s, V3 d) {
    const lwo_params *p = s->params;
    V3 sun = v3f4(p->sky_sun);
    REAL cos_theta = rmax(d.y + (REAL)p->sky_zenith[3], K(0.0));
    REAL cos_gamma = rclamp(vdot(d, sun), K(-1.0), K(1.0));
    REAL gamma = R_ACOS(cos_gamma);
    REAL cos2_gamma = cos_gamma * cos_gamma;
    REAL perez[3];
    for (int k = 0; k < 3; k++) {
        REAL a = cos_theta > K(0.0) ? (REAL)p->perez_a[k] * R_EXP((REAL)p->perez_b[k] / cos_theta) : K(0.0);
        perez[k] = (K(1.0) + a) *
                   (K(1.0) + (REAL)p->perez_c[k] * R_EXP((REAL)p->perez_d[k] * gamma) + (REAL)p->perez_e[k] * cos2_gamma);
    }
    REAL x = (REAL)p->sky_zenith[0] * perez[0];
    REAL y = (REAL)p->sky_zenith[1] * perez[1];
    REAL lum = (REAL)p->sky_zenith[2] * perez[2];
    if (y <= K(5e-8)) return V3_ZERO;
    REAL f = lum / y;
    REAL cx = x * f, cy = lum, cz = (K(1.0) - x - y) * f;
    return vmuls(v3(K(2.3706743) * cx - K(0.9000405) * cy - K(0.4706338) * cz,
                    K(-0.513885) * cx + K(1.4253036) * cy + K(0.0885814) * cz,
                    K(0.0052982) * cx - K(0.0146949) * cy + K(1.0093968) * cz),
                 K(0.045));
}

/* rgb_to_hsl (integrator.rs:79-104). */
static void rgb_to_hsl(V3 c, REAL out[3]) {
    REAL r = rclamp(c.x, K(0.0), K(1.0)), g = rclamp(c.y, K(0.0), K(1.0)), b = rclamp(c.z, K(0.0), K(1.0));
    REAL cmax = rmax(rmax(r, g), b);
    REAL cmin = rmin(rmin(r, g), b);
    REAL delta = cmax - cmin;
    REAL lightness = (cmax + cmin) / K(2.0);
    REAL hue;
    if (delta == K(0.0)) hue = K(0.0);
    else if (cmax == r) hue = R_FMOD((g - b) / delta, K(6.0)) / K(6.0);
    else if (cmax == g) hue = (((b - r) / delta) + K(2.0)) / K(6.0);
    else hue = (((r - g) / delta) + K(4.0)) / K(6.0);
    REAL saturation = delta < K(5e-8) ? K(0.0) : delta / (K(1.0) - rabs(K(2.0) * lightness - K(1.0)));
    out[0] = hue;
    out[1] = saturation;
    out[2] = lightness;
}

/* rgb_from_hsl (integrator.rs:108-127). */
static inline V3 rgb_from_hsl(REAL hue, REAL saturation, REAL lightness) {
    REAL c = rmin(K(1.0), (K(1.0) - rabs(K(2.0) * lightness - K(1.0))) * saturation);
    REAL h = hue * K(6.0);
    REAL x = c * (K(1.0) - rabs(R_FMOD(h, K(2.0)) - K(1.0)));
    V3 rgb;
    if (h < K(1.0)) rgb = v3(c, x, K(0.0));
    else if (h < K(2.0)) rgb = v3(x, c, K(0.0));
    else if (h < K(3.0)) rgb = v3(K(0.0), c, x);
    else if (h < K(4.0)) rgb = v3(K(0.0), x, c);
    else if (h < K(5.0)) rgb = v3(x, K(0.0), c);
    else rgb = v3(c, K(0.0), x);
    REAL m = rmax(K(0.0), lightness - K(0.5) * c);
    return vadd(rgb, v3(m, m, m));
}

/* build_sky_cache (integrator.rs:133-148). */
static void build_sky_cache(const lwo_scene *s, uint32_t n, float *out) {
    uint32_t m = n + 1;
    for (uint32_t i = 0; i < m; i++) {
        REAL sin_t, cos_t;
        R_SINCOS_TURNS((REAL)i / (REAL)n, &sin_t, &cos_t);
        for (uint32_t j = 0; j < m; j++) {
            REAL sin_p, cos_p;
            R_SINCOS_TURNS((REAL)j / (REAL)(2 * n) - K(0.25), &sin_p, &cos_p);
            REAL r = rabs(cos_p);
            REAL hsl[3];
            rgb_to_hsl(preetham_radiance(s, v3(cos_t * r, sin_p, sin_t * r)), hsl);
            uint64_t at = (uint64_t)(i * m + j) * 3u;
            out[at] = (float)hsl[0];
            out[at + 1] = (float)hsl[1];
            out[at + 2] = (float)hsl[2];
        }
    }
}

/* sky_radiance (integrator.rs:158-188). */
static V3 sky_radiance(const lwo_scene *s, V3 d) {
    const lwo_params *p = s->params;
    REAL n = (REAL)p->misc_f[2];
    if (n < K(1.0)) return V3_ZERO;
    CNT(sky_reads);
    REAL theta = R_ATAN2(d.z, d.x) / (K(2.0) * PI_R);
    theta = R_FMOD(R_FMOD(theta, K(1.0)) + K(1.0), K(1.0));
    REAL phi = K(1.0) - R_ACOS(rclamp(d.y, K(-1.0), K(1.0))) / PI_R;
    REAL x = theta * n, y = phi * n;
    REAL fx = R_FLOOR(rclamp(x, K(0.0), n - K(1.0)));
    REAL fy = R_FLOOR(rclamp(y, K(0.0), n - K(1.0)));
    uint32_t m = to_u32(n) + 1u;
#define AT(i, j) ((uint64_t)((to_u32(i) * m + to_u32(j)) * 3u))
    uint64_t a00 = AT(fx, fy), a10 = AT(fx + K(1.0), fy), a01 = AT(fx, fy + K(1.0)), a11 = AT(fx + K(1.0), fy + K(1.0));
#undef AT
    REAL hsl[3];
    for (int k = 0; k < 3; k++) {
        REAL y0 = SKY(s, a00 + k) + (x - fx) * (SKY(s, a10 + k) - SKY(s, a00 + k));
        REAL y1 = SKY(s, a01 + k) + (x - fx) * (SKY(s, a11 + k) - SKY(s, a01 + k));
        hsl[k] = y0 + (y - fy) * (y1 - y0);
    }
    return vmuls(rgb_from_hsl(hsl[0], hsl[1], hsl[2]), (REAL)p->sky_sun[3]);
}

/* map_lookup (integrator.rs:196-217). */
static V3 map_lookup(const lwo_scene *s, uint32_t base, REAL w, REAL h, V3 d) {
    CNT(map_reads);
    REAL u = R_ATAN2(d.z, d.x) / (K(2.0) * PI_R);
    u = R_FMOD(R_FMOD(u, K(1.0)) + K(1.0), K(1.0));
    REAL v = K(1.0) - R_ACOS(rclamp(d.y, K(-1.0), K(1.0))) / PI_R;
    REAL x = u * w - K(0.5);
    REAL y = rclamp(v * h - K(0.5), K(0.0), h - K(1.0));
    REAL fx = R_FLOOR(x), fy = R_FLOOR(y);
    REAL tx = x - fx, ty = y - fy;
    REAL i0 = fx < K(0.0) ? w - K(1.0) : fx;
    REAL i1 = fx + K(1.0) >= w ? K(0.0) : fx + K(1.0);
    REAL j1 = rmin(fy + K(1.0), h - K(1.0));
    uint32_t wu = to_u32(w);
#define AT(i, j) ({ uint64_t k_ = (uint64_t)(base + (to_u32(j) * wu + to_u32(i)) * 3u); v3(SKY(s, k_), SKY(s, k_ + 1), SKY(s, k_ + 2)); })
    V3 top = vadd(vmuls(AT(i0, fy), K(1.0) - tx), vmuls(AT(i1, fy), tx));
    V3 bottom = vadd(vmuls(AT(i0, j1), K(1.0) - tx), vmuls(AT(i1, j1), tx));
#undef AT
    return vadd(vmuls(top, K(1.0) - ty), vmuls(bottom, ty));
}

/* sky_lens / sky_light (integrator.rs:225-243). */
static V3 sky_lens(const lwo_scene *s, V3 d) {
    const float *m = s->params->sky_map;
    if ((REAL)m[0] < K(1.0)) return sky_radiance(s, d);
    return map_lookup(s, 0, (REAL)m[0], (REAL)m[1], d);
}
static V3 sky_light(const lwo_scene *s, V3 d) {
    const float *m = s->params->sky_map;
    if ((REAL)m[0] < K(1.0)) return sky_radiance(s, d);
    /* (m[0] * m[1]) as u32 * 3, in f32 as the reference computes it. */
    return map_lookup(s, to_u32((REAL)(m[0] * m[1])) * 3u, (REAL)m[2], (REAL)m[3], d);
}

/* sun_texture (integrator.rs:252-277). */
static V3 sun_texture(const lwo_scene *s, V3 d) {
    const lwo_params *p = s->params;
    const float *sprite = p->sun_sprite;
    if ((REAL)sprite[2] <= K(0.0) || vdot(d, v3f4(p->sun_dir)) < K(0.5)) return V3_ZERO;
    REAL width = (REAL)p->sun_sv[3];
    REAL width2 = width * K(2.0);
    REAL a = K(0.5) * PI_R - R_ACOS(vdot(d, v3f4(p->sun_su))) + width;
    REAL b = K(0.5) * PI_R - R_ACOS(vdot(d, v3f4(p->sun_sv))) + width;
    if (a < K(0.0) || a >= width2 || b < K(0.0) || b >= width2) return V3_ZERO;
    REAL x = rclamp(R_FLOOR(a / width2 * (REAL)sprite[2] - K(5e-8)), K(0.0), (REAL)sprite[2] - K(1.0));
    REAL y = rclamp(R_FLOOR((K(1.0) - b / width2) * (REAL)sprite[3] - K(5e-8)), K(0.0), (REAL)sprite[3] - K(1.0));
    return vmuls(linear_rgb(texel(s, (REAL)sprite[0] + x + K(0.5), (REAL)sprite[1] + y + K(0.5))), (REAL)p->sun_su[3]);
}

/* cosine_hemisphere (integrator.rs:280-287). */
static inline V3 cosine_hemisphere(V3 n, uint32_t *rng) {
    REAL r1 = rng_next(rng);
    REAL r2 = rng_next(rng);
    REAL r = R_SQRT(r1);
    REAL sin_phi, cos_phi;
    R_SINCOS_TURNS(r2, &sin_phi, &cos_phi);
    V3 t, b;
    onb(n, &t, &b);
    return vnormalize(vadd(vadd(vmuls(t, r * cos_phi), vmuls(b, r * sin_phi)), vmuls(n, R_SQRT(rmax(K(1.0) - r1, K(0.0))))));
}

/* sample_sun (integrator.rs:291-302). */
static inline V3 sample_sun(const lwo_scene *s, uint32_t *rng) {
    const lwo_params *p = s->params;
    V3 sun = v3f4(p->sun_dir);
    REAL cos_max = (REAL)p->sun_dir[3];
    REAL r1 = rng_next(rng);
    REAL r2 = rng_next(rng);
    REAL cos_t = K(1.0) - r1 * (K(1.0) - cos_max);
    REAL sin_t = R_SQRT(rmax(K(1.0) - cos_t * cos_t, K(0.0)));
    REAL sin_phi, cos_phi;
    R_SINCOS_TURNS(r2, &sin_phi, &cos_phi);
    V3 t, b;
    onb(sun, &t, &b);
    return vnormalize(vadd(vadd(vmuls(t, sin_t * cos_phi), vmuls(b, sin_t * sin_phi)), vmuls(sun, cos_t)));
}

/* shading_normal (integrator.rs:308-315). */
static inline V3 shading_normal(const lwo_quad *q, V3 d, int *front) {
    V3 n = vnormalize(q_normal(q));
    if (vdot(n, d) < K(0.0)) { *front = 1; return n; }
    *front = 0;
    return vneg(n);
}

/* shadow (integrator.rs:319-346). */
static V3 shadow(const lwo_scene *s, V3 o, V3 d, REAL tmax) {
    REAL eps = (REAL)s->params->misc_f[1];
    V3 tr = V3_ONE;
    for (int i = 0; i < 8; i++) {
        Hit h = trace(s, o, d, eps, tmax);
        if (h.quad == NO_QUAD) return tr;
        const lwo_quad *q = QUAD(s, h.quad);
        uint32_t flags = q_flags(q);
        if (flags & FLAG_WATER) {
            if (vdot(q_normal(q), d) > K(0.0)) tr = vmul(tr, vtransmittance(v3f4(s->params->water_color), h.t));
        } else if ((flags & FLAG_ALPHA_MASK) == ALPHA_TRANSLUCENT) {
            REAL a = (REAL)(h.texel >> 24) / K(255.0);
            V3 col = vmul(linear_rgb(h.texel), linear_rgb(q_tint(q)));
            tr = vmul(tr, vlerp(V3_ONE, col, a));
        } else {
            return V3_ZERO;
        }
        o = vadd(o, vmuls(d, h.t + eps));
        tmax -= h.t + eps;
    }
    return tr;
}

/* ---- the differentiable form's theta (test infrastructure for the reference gradient) ---- */
/* The emitter group of the block at voxel (x, y, z). */
static inline uint32_t emitter_group(int32_t x, int32_t y, int32_t z) {
    return pcg_hash((uint32_t)x * 73856093u ^ (uint32_t)y * 19349663u ^ (uint32_t)z * 83492791u) & 31u;
}

/* A hit's linear texel colour under theta and its parameter (-1: the decoded texel). */
static inline V3 theta_texel(const lwo_scene *s, const lwo_quad *q, const Hit *h, int32_t *param) {
    *param = -1;
    if (TH) {
        uint64_t i = quad_texel_index(s, q, h->s, h->tt);
        if (i < TH->texel_param_len) *param = TH->texel_param[i];
        else bounds_error();
        if (*param >= (int32_t)TH->n_params) { bounds_error(); *param = -1; }
        if (*param >= 0) return v3((REAL)TH->albedo[3 * *param], (REAL)TH->albedo[3 * *param + 1], (REAL)TH->albedo[3 * *param + 2]);
    }
    return linear_rgb(h->texel);
}

/* sample_sun's cone direction about `axis` for the draws r1, r2 (integrator.rs:291-302). */
static inline V3 cone_dir(V3 axis, REAL cos_max, REAL r1, REAL r2) {
    REAL cos_t = K(1.0) - r1 * (K(1.0) - cos_max);
    REAL sin_t = R_SQRT(rmax(K(1.0) - cos_t * cos_t, K(0.0)));
    REAL sin_phi, cos_phi;
    R_SINCOS_TURNS(r2, &sin_phi, &cos_phi);
    V3 t, b;
    onb(axis, &t, &b);
    return vnormalize(vadd(vadd(vmuls(t, sin_t * cos_phi), vmuls(b, sin_t * sin_phi)), vmuls(axis, cos_t)));
}

/* shadow (integrator.rs:319-346) with the visibility of direction l0: the segments are traced
 * along l0, and the water they cross is measured along l through the same surfaces (each hit
 * surface's plane, met from `o` along l). */
static V3 shadow_frozen(const lwo_scene *s, V3 o, V3 l0, V3 l) {
    REAL eps = (REAL)s->params->misc_f[1];
    V3 tr = V3_ONE, so = o;
    REAL tmax = (REAL)INFINITY, u_prev = K(0.0);
    for (int i = 0; i < 8; i++) {
        Hit h = trace(s, so, l0, eps, tmax);
        if (h.quad == NO_QUAD) return tr;
        const lwo_quad *q = QUAD(s, h.quad);
        uint32_t flags = q_flags(q);
        V3 nq = q_normal(q);
        REAL u = vdot(vsub(vadd(so, vmuls(l0, h.t)), o), nq) / vdot(l, nq);
        if (flags & FLAG_WATER) {
            if (vdot(nq, l0) > K(0.0)) {
                REAL t = i == 0 ? u : u - (u_prev + eps);
                tr = vmul(tr, vtransmittance(v3f4(s->params->water_color), t));
            }
        } else if ((flags & FLAG_ALPHA_MASK) == ALPHA_TRANSLUCENT) {
            REAL a = (REAL)(h.texel >> 24) / K(255.0);
            int32_t param;
            V3 col = vmul(theta_texel(s, q, &h, &param), linear_rgb(q_tint(q)));
            tr = vmul(tr, vlerp(V3_ONE, col, a));
        } else {
            return V3_ZERO;
        }
        so = vadd(so, vmuls(l0, h.t + eps));
        tmax -= h.t + eps;
        u_prev = u;
    }
    return tr;
}

/* pick (integrator.rs:350-353). */
static inline uint32_t pick(uint32_t n, REAL u) {
    uint32_t i = to_u32(u * (REAL)n);
    return i < n ? i : n - 1;
}

/* floor(b / cell) for an integer block coordinate b and integer cell: exact for |b| < 2^24 (the
 * quotient's rounding error stays below 1 / cell, its least distance to an integer it is not). */
static inline int32_t cell_of_block(int32_t b, REAL cell) { return to_i32(R_FLOOR((REAL)b / cell)); }

/* emitter_cell (integrator.rs:358-373). In a chunk frame the cell of p's block in the grid,
 * floor(p) + A, in integers (floor((b + f) / size) = floor(b / size) for f in [0, 1)). */
static void emitter_cell(const lwo_scene *s, V3 p, uint32_t *start, uint32_t *count) {
    REAL cell = (REAL)EGRID(s, 0);
    int32_t size[3] = {(int32_t)EGRID(s, 1), (int32_t)EGRID(s, 2), (int32_t)EGRID(s, 3)};
    int32_t c[3];
    if (lwo_reb) {
        c[0] = cell_of_block(to_i32(R_FLOOR(p.x)) + lwo_fa[0], cell) - (int32_t)EGRID(s, 4);
        c[1] = cell_of_block(to_i32(R_FLOOR(p.y)) + lwo_fa[1], cell) - (int32_t)EGRID(s, 5);
        c[2] = cell_of_block(to_i32(R_FLOOR(p.z)) + lwo_fa[2], cell) - (int32_t)EGRID(s, 6);
    } else {
        c[0] = to_i32(R_FLOOR(p.x / cell)) - (int32_t)EGRID(s, 4);
        c[1] = to_i32(R_FLOOR(p.y / cell)) - (int32_t)EGRID(s, 5);
        c[2] = to_i32(R_FLOOR(p.z / cell)) - (int32_t)EGRID(s, 6);
    }
    CNT(emitter_cell_reads);
    if (c[0] < 0 || c[1] < 0 || c[2] < 0 || c[0] >= size[0] || c[1] >= size[1] || c[2] >= size[2]) {
        *start = 0;
        *count = 0;
        return;
    }
    uint32_t i = (uint32_t)((c[1] * size[2] + c[2]) * size[0] + c[0]);
    uint64_t at = (uint64_t)(EMITTER_GRID_HEADER + i * 2u);
    *start = EGRID(s, at);
    *count = EGRID(s, at + 1);
}

/* sample_emitter_face (integrator.rs:381-414). */
static V3 sample_emitter_face(const lwo_scene *s, V3 origin, V3 n, const lwo_emitter *e, uint32_t face,
                              REAL scaler, uint32_t *rng) {
    const lwo_params *p = s->params;
    const lwo_quad *q = QUAD(s, (uint64_t)(bits_of(e->pos[3]) + face));
    REAL ss = rng_next(rng);
    REAL t = rng_next(rng);
    V3 epos = v3f4(e->pos);
    if (lwo_reb) epos = vsub(epos, frame_origin(lwo_fa));  /* the block's corner in the frame: exact */
    V3 at = vadd(vadd(vadd(epos, q_origin(q)), vmuls(q_eu(q), ss)), vmuls(q_ev(q), t));
    V3 to = vsub(at, origin);
    if (vdot(to, n) <= K(0.0)) return V3_ZERO;
    REAL dist = vlength(to);
    V3 l = vdivs(to, dist);
    REAL eps = (REAL)p->misc_f[1];
    Hit h = trace(s, origin, l, eps, dist + K(2.0) * eps);
    if (h.quad == NO_QUAD) return V3_ZERO;
    if (rabs(h.t - dist) >= K(2.0) * eps) return V3_ZERO;
    V3 nq = q_normal(q);
    REAL area = vlength(nq);
    REAL cos_l = rabs(vdot(nq, l)) / area;
    const lwo_quad *hq = QUAD(s, h.quad);
    int32_t param;
    V3 c = vmul(theta_texel(s, hq, &h, &param), linear_rgb(q_tint(hq)));
    REAL intensity = (REAL)p->misc_f[0];
    if (TH) intensity = intensity * (REAL)TH->emit_mult[emitter_group(to_i32((REAL)e->pos[0]), to_i32((REAL)e->pos[1]), to_i32((REAL)e->pos[2]))];
    return vmuls(c, cos_l / rmax(dist * dist, K(1.0)) * area * q_emittance(q) * intensity * scaler);
}

/* sample_emitter (integrator.rs:419-433). */
static V3 sample_emitter(const lwo_scene *s, V3 origin, V3 n, const lwo_emitter *e, uint32_t *rng) {
    uint32_t faces = e->faces[0];
    if (faces == 0) return V3_ZERO;
    if (s->params->emitter[0] == EMITTER_SAMPLING_ONE) {
        uint32_t f = pick(faces, rng_next(rng));
        return sample_emitter_face(s, origin, n, e, f, K(1.0), rng);
    }
    V3 sum = V3_ZERO;
    for (uint32_t f = 0; f < faces; f++)
        sum = vadd(sum, sample_emitter_face(s, origin, n, e, f, K(1.0) / (REAL)faces, rng));
    return sum;
}

/* sample_emitters (integrator.rs:441-469) on the emitters of a cell emitter_cell found. */
static V3 sample_cell_emitters(const lwo_scene *s, uint32_t start, uint32_t count, V3 origin, V3 n, uint32_t *rng) {
    if (count == 0) return V3_ZERO;
    uint64_t list = (uint64_t)EMITTER_GRID_HEADER +
                    (uint64_t)EGRID(s, 1) * (uint64_t)EGRID(s, 2) * (uint64_t)EGRID(s, 3) * 2u + start;
    uint32_t strategy = s->params->emitter[0];
    if (strategy == EMITTER_SAMPLING_ONE || strategy == EMITTER_SAMPLING_ONE_BLOCK) {
        uint32_t i = EGRID(s, list + pick(count, rng_next(rng)));
        CNT(emitter_index_reads);
        lwo_emitter e = EMITTER(s, i);
        CNT(emitter_reads);
        return vmuls(sample_emitter(s, origin, n, &e, rng), PI_R);
    }
    if (strategy == EMITTER_SAMPLING_ALL) {
        V3 sum = V3_ZERO;
        for (uint32_t k = 0; k < count; k++) {
            uint32_t i = EGRID(s, list + k);
            CNT(emitter_index_reads);
            lwo_emitter e = EMITTER(s, i);
            CNT(emitter_reads);
            sum = vadd(sum, sample_emitter(s, origin, n, &e, rng));
        }
        return vmuls(sum, PI_R / (REAL)count);
    }
    return V3_ZERO;
}

/* sample_emitters (integrator.rs:441-469). */
static V3 sample_emitters(const lwo_scene *s, V3 pos, V3 origin, V3 n, uint32_t *rng) {
    uint32_t start, count;
    emitter_cell(s, pos, &start, &count);
    return sample_cell_emitters(s, start, count, origin, n, rng);
}

/* water_interface (integrator.rs:477-505). Writes the new direction and origin. */
static int water_interface(const lwo_params *p, V3 pos, V3 d, V3 n, int front, int in_water, REAL eps,
                           uint32_t *rng, V3 *nd, V3 *no) {
    REAL ior = (REAL)p->water_color[3];
    REAL eta = front ? K(1.0) / ior : ior;
    REAL cos_i = -vdot(n, d);
    REAL sin2_t = eta * eta * rmax(K(1.0) - cos_i * cos_i, K(0.0));
    REAL r0 = (K(1.0) - ior) / (K(1.0) + ior);
    r0 = r0 * r0;
    REAL m = K(1.0) - cos_i;
    REAL fresnel = r0 + (K(1.0) - r0) * m * m * m * m * m;
    if (sin2_t >= K(1.0) || rng_next(rng) < fresnel) {
        *nd = vnormalize(vadd(d, vmuls(n, K(2.0) * cos_i)));
        *no = vadd(pos, vmuls(n, eps));
        return in_water;
    }
    REAL cos_t = R_SQRT(K(1.0) - sin2_t);
    *nd = vnormalize(vadd(vmuls(d, eta), vmuls(n, eta * cos_i - cos_t)));
    *no = vsub(pos, vmuls(n, eps));
    return front;
}

/* The water plane's height in the current frame. */
static inline REAL water_height(const lwo_params *p) {
    return lwo_reb ? (REAL)p->water_plane[0] - (REAL)lwo_fa[1] : (REAL)p->water_plane[0];
}

/* water_plane (integrator.rs:511-526). Returns 1 and the distance when met. In the current frame
 * the grid's columns span [-A, size - A). */
static int water_plane(const lwo_scene *s, V3 o, V3 d, REAL *tp) {
    const lwo_params *p = s->params;
    if ((REAL)p->water_plane[1] == K(0.0) || d.y == K(0.0)) return 0;
    REAL t = (water_height(p) - o.y) / d.y;
    if (!(t > K(0.0) && t < (REAL)INFINITY)) return 0;
    V3 at = vadd(o, vmuls(d, t));
    const int32_t ax = lwo_reb ? lwo_fa[0] : 0, az = lwo_reb ? lwo_fa[2] : 0;
    REAL x0 = (REAL)(-ax), z0 = (REAL)(-az);
    REAL sx = (REAL)((int32_t)(p->grid_dims[0] * 16u) - ax), sz = (REAL)((int32_t)(p->grid_dims[2] * 16u) - az);
    if (at.x >= x0 && at.z >= z0 && at.x < sx && at.z < sz) return 0;
    *tp = t;
    return 1;
}

/* under_water_plane (integrator.rs:531-534). */
static inline int under_water_plane(const lwo_scene *s, V3 o, V3 d) {
    const lwo_params *p = s->params;
    return (REAL)p->water_plane[1] != K(0.0) && o.y < water_height(p) && d.y <= K(0.0);
}

/* The camera a sample starts from: Params in the FP32 build, the f64 camera in the FP64
 * twin when one is given. `framed`: pos is relative to the chunk corner of `frame` (Params'
 * see_through[2] and [3]); otherwise to the grid origin. */
typedef struct { V3 pos, fwd, right, up; REAL tan_half, aspect; uint32_t framed, frame; } Cam;

static V3 render_path(const lwo_scene *s, const Cam *cam, uint32_t px, uint32_t py, uint32_t sample);

/* render_sample (integrator.rs:539-709), in the camera's frame. */
static V3 render_sample(const lwo_scene *s, const Cam *cam, uint32_t px, uint32_t py, uint32_t sample) {
    lwo_reb = cam->framed != 0;
    if (lwo_reb) frame_unpack(cam->frame, lwo_fa);
    V3 r = render_path(s, cam, px, py, sample);
    lwo_reb = 0;
    lwo_fa[0] = lwo_fa[1] = lwo_fa[2] = 0;
    return r;
}

static V3 render_path(const lwo_scene *s, const Cam *cam, uint32_t px, uint32_t py, uint32_t sample) {
    const lwo_params *p = s->params;
    uint32_t width = p->frame[0], height = p->frame[1], max_bounces = p->frame[3];
    REAL eps = (REAL)p->misc_f[1];
    uint32_t rng = rng_new(py * width + px, sample, p->misc_u[0]);
    CNT(samples);

    REAL tan_half = cam->tan_half, aspect = cam->aspect;
    REAL jx = rng_next(&rng);
    REAL jy = rng_next(&rng);
    REAL sx = (K(2.0) * ((REAL)px + jx) / (REAL)width - K(1.0)) * aspect * tan_half;
    REAL sy = (K(1.0) - K(2.0) * ((REAL)py + jy) / (REAL)height) * tan_half;
    V3 d = vnormalize(vadd(vadd(cam->fwd, vmuls(cam->right, sx)), vmuls(cam->up, sy)));
    V3 o = cam->pos;

    V3 radiance = V3_ZERO, beta = V3_ONE, beta0 = V3_ONE; /* beta0: the frozen roulette's throughput */
    uint32_t bounces = 0;
    int specular = 1, in_water = 0;
    uint32_t strategy = p->misc_u[3] > 0 ? p->emitter[0] : EMITTER_SAMPLING_NONE;
    REAL tmin = K(0.0);
    V3 sigma = v3f4(p->water_color);

    for (uint32_t ev_i = 0; ev_i < MAX_EVENTS; ev_i++) {
        CNT(events);
        Hit hit = trace(s, o, d, tmin, (REAL)INFINITY);
        int found = hit.quad != NO_QUAD;
        int forced = 0;
        if (bounces == 0 && p->see_through[1] > 0 && found && !is_see_through(s, hit.quad)) {
            Hit st = see_through_hit(s, o, d, hit.t);
            if (st.quad != NO_QUAD) {
                const lwo_quad *sq = QUAD(s, st.quad);
                if ((q_flags(sq) & FLAG_ALPHA_MASK) == ALPHA_TRANSLUCENT) {
                    if (rng_next(&rng) < (REAL)(st.texel >> 24) / K(255.0)) {
                        hit = st;
                        forced = 1;
                    }
                } else {
                    hit = st;
                }
            }
        }
        REAL tp;
        if (water_plane(s, o, d, &tp) && (!found || tp < hit.t)) {
            if (in_water) {
                beta = vmul(beta, vtransmittance(sigma, tp));
                if (TH) beta0 = vmul(beta0, vtransmittance(sigma, tp));
            }
            int front = d.y < K(0.0);
            V3 n = v3(K(0.0), front ? K(1.0) : K(-1.0), K(0.0));
            V3 nd, no;
            in_water = water_interface(p, vadd(o, vmuls(d, tp)), d, n, front, in_water, eps, &rng, &nd, &no);
            d = nd;
            o = no;
            if (lwo_reb) o = rebase(o);
            specular = 1;
            tmin = K(0.0);
            continue;
        }
        if (!found) {
            if (!in_water && !under_water_plane(s, o, d)) {
                if (bounces == 0) radiance = vadd(radiance, vmul(beta, sky_lens(s, d)));
                else radiance = vadd(radiance, vmul(beta, sky_light(s, d)));
                if (specular && bounces == 0) radiance = vadd(radiance, vmul(beta, sun_texture(s, d)));
            }
            break;
        }
        if (in_water) {
            beta = vmul(beta, vtransmittance(sigma, hit.t));
            if (TH) beta0 = vmul(beta0, vtransmittance(sigma, hit.t));
        }
        const lwo_quad *q = QUAD(s, hit.quad);
        uint32_t flags = q_flags(q);
        V3 pos = vadd(o, vmuls(d, hit.t));
        REAL alpha = (REAL)(hit.texel >> 24) / K(255.0);
        int32_t param;
        V3 albedo = vmul(theta_texel(s, q, &hit, &param), linear_rgb(q_tint(q)));
        V3 albedo0 = albedo;
        if (TH && TH->frozen && param >= 0)
            albedo0 = vmul(v3((REAL)TH->albedo0[3 * param], (REAL)TH->albedo0[3 * param + 1], (REAL)TH->albedo0[3 * param + 2]),
                           linear_rgb(q_tint(q)));
        int front;
        V3 n = shading_normal(q, d, &front);

        if (flags & FLAG_WATER) {
            V3 nd, no;
            in_water = water_interface(p, pos, d, n, front, in_water, eps, &rng, &nd, &no);
            d = nd;
            o = no;
            if (lwo_reb) o = rebase(o);
            specular = 1;
            tmin = K(0.0);
            continue;
        }
        if (!forced && (flags & FLAG_ALPHA_MASK) == ALPHA_TRANSLUCENT && rng_next(&rng) >= alpha) {
            beta = vmul(beta, vlerp(V3_ONE, albedo, alpha));
            if (TH) beta0 = vmul(beta0, vlerp(V3_ONE, albedo0, alpha));
            o = vadd(pos, vmuls(d, eps));
            if (lwo_reb) o = rebase(o);
            tmin = K(0.0);
            continue;
        }
        if (bounces >= max_bounces) break;
        REAL emittance = q_emittance(q) * (REAL)p->misc_f[0];
        int emits = emittance > K(0.0) && (p->emitter[1] == 0 || strategy == EMITTER_SAMPLING_NONE || bounces == 0);
        if (emits && TH) {
            V3 inside = vsub(pos, vmuls(n, K(1e-3)));
            emittance = emittance * (REAL)TH->emit_mult[emitter_group(to_i32(R_FLOOR(inside.x)), to_i32(R_FLOOR(inside.y)),
                                                                       to_i32(R_FLOOR(inside.z)))];
        }
        if (emits) radiance = vadd(radiance, vmuls(vmul(beta, vmul(albedo, albedo)), emittance));
        bounces += 1;

        V3 origin = vadd(pos, vmuls(n, eps));
        /* the emitters' cell, found in the hit's frame before the origin moves to its own */
        const int sample_e = !emits && strategy != EMITTER_SAMPLING_NONE;
        uint32_t e_start = 0, e_count = 0;
        if (sample_e) emitter_cell(s, pos, &e_start, &e_count);
        if (lwo_reb) origin = rebase(origin);
        V3 sun = TH ? v3((REAL)TH->sun[0], (REAL)TH->sun[1], (REAL)TH->sun[2]) : v3f4(p->sun_dir);
        REAL sd3 = TH ? (REAL)TH->sun[3] : (REAL)p->sun_dir[3];
        REAL sin_r = R_SQRT(rmax(K(1.0) - sd3 * sd3, K(0.0)));
        int lit = p->sun_color[0] > 0.0f || p->sun_color[1] > 0.0f || p->sun_color[2] > 0.0f;
        if (lit && vdot(n, sun) > -sin_r && sun.y > -sin_r) {
            V3 l, l0;
            if (TH) {
                REAL r1 = rng_next(&rng);
                REAL r2 = rng_next(&rng);
                l = cone_dir(sun, sd3, r1, r2);
                l0 = TH->frozen ? cone_dir(v3((REAL)TH->sun0[0], (REAL)TH->sun0[1], (REAL)TH->sun0[2]), (REAL)TH->sun0[3], r1, r2) : l;
            } else {
                l = sample_sun(s, &rng);
                l0 = l;
            }
            REAL cos_l = vdot(n, l);
            if (cos_l > K(0.0) && l.y >= K(0.0)) {
                V3 tr = TH && TH->frozen ? shadow_frozen(s, origin, l0, l) : shadow(s, origin, l, (REAL)INFINITY);
                radiance = vadd(radiance, vmuls(vmul(vmul(vmul(beta, albedo), v3f4(p->sun_color)), tr), cos_l));
            }
        }
        if (sample_e)
            radiance = vadd(radiance, vmul(vmul(beta, albedo), sample_cell_emitters(s, e_start, e_count, origin, n, &rng)));

        beta = vmul(beta, albedo);
        if (TH) beta0 = vmul(beta0, albedo0);
        if (bounces >= 3) {
            REAL q_rr = rclamp(vmax_elem(TH && TH->frozen ? beta0 : beta), K(0.05), K(0.95));
            if (rng_next(&rng) > q_rr) break;
            beta = vdivs(beta, q_rr);
            if (TH) beta0 = vdivs(beta0, q_rr);
        }
        d = cosine_hemisphere(n, &rng);
        o = origin;
        tmin = K(0.0);
        specular = 0;
    }
    return radiance;
}
