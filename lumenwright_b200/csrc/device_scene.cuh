// The scene as the B200 kernels read it, and the reference's traversal on it.
//
// Layout in HBM (built by lw_scene_upload from the reference's `HqScene` buffers):
//   top     uint2[nb]            (top entry, overlay entry) per brick: one 8-byte load per brick
//                                where the reference reads two words (trace.rs:181-182)
//   bricks  uint16[n * 4096]     the voxel ids of each non-uniform brick (a model without quads
//                                re-laid as air, 0: csrc/scene.cu), 4x4x4-sub-block-major:
//                                sub-block ((y>>2)*4 + (z>>2))*4 + (x>>2), then ((y&3)*4+(z&3))*4+(x&3)
//                                inside it, so one sub-block is one 128-byte line
//   occ     uint2[n]             a 64-bit mask per non-uniform brick: bit s set when sub-block s
//                                holds a voxel whose model has quads
//   quads   DevQuad[q]           96-byte records with the normal eu x ev and |n|^2 precomputed
//   grid    uint32[]             the reference's grid, read for the overlay cells and ov_quads and
//                                by the voxel lookup
//   models, atlas, emitters, emitter_grid, sky: the reference's buffers unchanged
//   gamma   float[256]           gamma_to_linear(k / 255) for every byte k (math.rs:214-216)
#pragma once

#include "device_math.cuh"

namespace lw {

constexpr uint32_t EMPTY = 0xFFFFFFFFu;
constexpr uint32_t UNIFORM = 0x80000000u;
constexpr uint32_t OV_CELL_WORDS = 8192u;
constexpr uint32_t ALPHA_CUTOUT = 1u;
constexpr uint32_t ALPHA_TRANSLUCENT = 2u;
constexpr uint32_t FLAG_ALPHA_MASK = 3u;
constexpr uint32_t FLAG_WATER = 4u;
constexpr uint32_t FLAG_FRONT_ONLY = 16u;
constexpr uint32_t EMITTER_SAMPLING_NONE = 0u;
constexpr uint32_t EMITTER_SAMPLING_ONE = 1u;
constexpr uint32_t EMITTER_SAMPLING_ONE_BLOCK = 2u;
constexpr uint32_t EMITTER_SAMPLING_ALL = 3u;
constexpr uint32_t EMITTER_GRID_HEADER = 8u;
constexpr uint32_t MAX_STEPS = 65536u;  // trace.rs:31
constexpr uint32_t MAX_EVENTS = 48u;    // integrator.rs:24
constexpr uint32_t NO_QUAD = 0xFFFFFFFFu;
constexpr float COPLANAR = 1e-5f;       // trace.rs:73


struct __align__(16) DevQuad {
    float4 n_nn;      // n = eu x ev, w = n . n
    float4 p0_flags;  // p0, w = flags (bit cast)
    float4 eu_tint;   // eu, w = tint (bit cast)
    float4 ev_em;     // ev, w = emittance
    float4 uv;        // uv0.xy, uvs.xy
    float4 uvt;       // uvt.xy, 0, 0
};
static_assert(sizeof(DevQuad) == 96, "DevQuad is 96 bytes");

// The frame parameters as the kernels use them (a copy of `Params` plus derived values).
struct __align__(16) DevParams {
    float4 cam_pos, cam_fwd, cam_right, cam_up, sun_dir, sun_color, sky_sun, sky_zenith;
    float4 perez_a, perez_b, perez_c, perez_d, perez_e, water_color, misc_f;
    uint4 grid_dims, off, off2, frame, misc_u, see_through, emitter;
    float4 sun_su, sun_sv, sun_sprite, sky_map, water_plane;
};
static_assert(sizeof(DevParams) == 432, "Params is 432 bytes");

struct DevScene {
    const uint2 *top;
    const uint16_t *bricks;
    const uint2 *occ;
    const uint32_t *grid;
    const uint4 *models;
    const DevQuad *quads;
    const uint32_t *atlas;
    const float4 *emitters;  // two float4 per emitter: (offset, first quad), (faces, -, -, -)
    const uint32_t *emitter_grid;
    const float *sky;
    const float *gamma;
    // The lowest brick row above which every brick is empty (no block, no overlay): a ray in an
    // empty brick at or above it that does not go down meets nothing more.
    uint32_t sky_brick_y;
    uint32_t n_top, n_occ;  // entries of `top` and `occ` (what a block stages in shared memory)
};

// A top-level entry or occupancy mask: from global memory through the read-only path, or (STAGED)
// from the block's copy in shared memory, which `top` and `occ` then point into.
template <bool STAGED>
LW_DI uint2 scene_word(const uint2 *p) {
    if (STAGED) return *p;
    return __ldg(p);
}

template <typename T>
LW_DI T ldg(const T *p) { return __ldg(p); }

struct Hit {
    float t;
    uint32_t quad, texel;
    float s, tt;
};
LW_DI Hit no_hit() { return Hit{kINF, NO_QUAD, 0u, 0.0f, 0.0f}; }

// ---- chunk-origin frames ------------------------------------------------------------------------
// With chunk-origin rebasing (Params.see_through.z = 1) a path's positions are held relative to a
// chunk corner A of the grid (a multiple of 16 blocks on each axis), the corner nearest the path's
// current origin, so every origin is within 8 blocks of its frame's origin: an f32 step of 2^-20
// block at most, where a grid-relative coordinate of a 32-chunk grid has steps of 2^-15. The word
// packs A's chunk indices in two's complement: x in bits 0-10, y in 11-20, z in 21-31. The grid's
// cell c is the frame's integer c - A, so the traversal forms its boundaries in the frame from
// integers, exactly, and reads the grid at the grid's own indices. In the grid's own frame
// (rebasing off) A is 0 and every expression below reduces to the reference's.
// The frame is kept as its packed word (one register in the kernels' loops) and unpacked where it
// is used; the grid's frame is word 0, for which every use below folds to the reference's
// expression.
struct Frame {
    uint32_t w;  // the packed chunk indices (frame_word)
    // the frame's origin in the grid, in blocks (16 x the chunk index, sign-extended)
    LW_DI int x() const { return (int)(w << 21) >> 17; }
    LW_DI int y() const { return ((int)(w << 11) >> 18) & ~15; }
    LW_DI int z() const { return ((int)w >> 17) & ~15; }
};
LW_DI Frame frame_of(uint32_t w) { return Frame{w}; }
LW_DI uint32_t frame_word(int cx, int cy, int cz) {
    return ((uint32_t)cx & 0x7FFu) | (((uint32_t)cy & 0x3FFu) << 11) | (((uint32_t)cz & 0x7FFu) << 21);
}
LW_DI V3 frame_origin(const Frame &A) { return v3((float)A.x(), (float)A.y(), (float)A.z()); }

// Moves position x, held in the frame of word w, to the frame of the chunk corner nearest it:
// k = rint(x / 16) chunks per axis (the frame kept within the packable chunk range), x - 16 k. Both
// steps are exact: x / 16 is a scaling by a power of two, 16 k and x are multiples of x's ulp, and
// |x - 16 k| <= |x| whenever k != 0, so the difference is representable.
LW_DI int chunk_step(float x) { return to_i32(fminf(fmaxf(rintf(x * 0.0625f), -4096.0f), 4096.0f)); }
LW_DI void rebase(V3 &x, uint32_t &w) {
    const Frame f = frame_of(w);
    const int cx = f.x() >> 4, cy = f.y() >> 4, cz = f.z() >> 4;
    const int nx = clamp_i(cx + chunk_step(x.x), -1024, 1023);
    const int ny = clamp_i(cy + chunk_step(x.y), -512, 511);
    const int nz = clamp_i(cz + chunk_step(x.z), -1024, 1023);
    x = v3(x.x - (float)((nx - cx) * 16), x.y - (float)((ny - cy) * 16), x.z - (float)((nz - cz) * 16));
    w = frame_word(nx, ny, nz);
}

// SceneView::texel (scene.rs:288-294).
LW_DI uint32_t texel(const DevScene &S, const DevParams &P, float u, float v) {
    int w = (int)P.off2.y, h = (int)P.off2.z;
    int x = clamp_i(to_i32(floorf(u)), 0, w - 1);
    int y = clamp_i(to_i32(floorf(v)), 0, h - 1);
    return ldg(S.atlas + (uint32_t)(y * w + x));
}

// linear_rgb (integrator.rs:27-34) through the byte table.
LW_DI V3 linear_rgb(const float *gamma, uint32_t c) {
    return v3(gamma[c & 0xFFu], gamma[(c >> 8) & 0xFFu], gamma[(c >> 16) & 0xFFu]);
}

// intersect_quad (trace.rs:37-58) with quad_texel (:62-69) and the alpha test of test_quad
// (:81-109): whether quad qi is met at a t in (tmin, t_limit), inside its bounds, on a texel that
// is not cut out; the hit in `h`. The normal eu x ev and n . n come precomputed; a front-only quad
// met from behind is rejected before the division instead of after it: `normal() . d` is exactly
// `-(n . d)`, and intersect_quad has no side effects, so the outcome is the reference's.
// SHIFT: the quad's p0 is taken relative to `pb` (p0 - pb), for a quad given in grid coordinates
// and a ray in another frame.
template <bool SHIFT = false>
LW_DI bool quad_candidate(const DevScene &S, const DevParams &P, uint32_t qi, V3 o, V3 d, float tmin, float t_limit,
                          Hit &h, V3 pb = V3{0.0f, 0.0f, 0.0f}) {
    const DevQuad *q = S.quads + qi;
    float4 a = ldg(&q->n_nn);
    V3 n = f4v(a);
    float denom = dot(n, d);
    if (fabs_r(denom) < 1e-12f) return false;
    float4 b = ldg(&q->p0_flags);
    uint32_t flags = __float_as_uint(b.w);
    if ((flags & FLAG_FRONT_ONLY) && -denom >= 0.0f) return false;
    V3 p0 = f4v(b);
    if (SHIFT) p0 = p0 - pb;
    float t = __fdiv_rn(dot(n, p0 - o), denom);
    if (!(t > tmin && t < t_limit)) return false;
    V3 eu = f4v(ldg(&q->eu_tint));
    V3 ev = f4v(ldg(&q->ev_em));
    V3 p = (o + d * t) - p0;
    float nn = a.w;
    float s = __fdiv_rn(dot(cross(p, ev), n), nn);
    float tt = __fdiv_rn(dot(cross(eu, p), n), nn);
    if (s < 0.0f || s > 1.0f || tt < 0.0f || tt > 1.0f) return false;
    float4 uv = ldg(&q->uv);
    float4 uvt = ldg(&q->uvt);
    float sc = fmin_r(fmax_r(s, 0.0005f), 0.9995f);
    float tc = fmin_r(fmax_r(tt, 0.0005f), 0.9995f);
    float u = uv.x + sc * uv.z + tc * uvt.x;
    float v = uv.y + sc * uv.w + tc * uvt.y;
    uint32_t tx = texel(S, P, u, v);
    uint32_t alpha = tx >> 24;
    uint32_t mode = flags & FLAG_ALPHA_MASK;
    if ((mode == ALPHA_CUTOUT && alpha < 128u) || (mode == ALPHA_TRANSLUCENT && alpha == 0u)) return false;
    h = Hit{t, qi, tx, s, tt};
    return true;
}

// The acceptance rule of test_quad (trace.rs:81-109): a quad is taken when it is met before the
// best hit so far, or (a later quad, coplanar with it) less than COPLANAR behind it.
LW_DI float reach_of(const Hit &best, uint32_t qi) {
    return (best.quad != NO_QUAD && qi > best.quad) ? best.t + COPLANAR : best.t;
}

// test_quad (trace.rs:81-109).
template <bool SHIFT = false>
LW_DI void test_quad(const DevScene &S, const DevParams &P, uint32_t qi, V3 o, V3 d, float tmin, Hit &best,
                     V3 pb = V3{0.0f, 0.0f, 0.0f}) {
    const float reach = reach_of(best, qi);
    quad_candidate<SHIFT>(S, P, qi, o, d, tmin, reach, best, pb);  // writes `best` only when the quad is taken
}

// SceneView::voxel (scene.rs:271-284) on the re-laid grid.
LW_DI uint32_t brick_voxel(const DevScene &S, uint32_t entry, int lx, int ly, int lz) {
    uint32_t sb = (uint32_t)(((ly >> 2) * 4 + (lz >> 2)) * 4 + (lx >> 2));
    uint32_t v = (uint32_t)(((ly & 3) * 4 + (lz & 3)) * 4 + (lx & 3));
    return ldg(S.bricks + ((size_t)entry * 4096u + sb * 64u + v));
}
// The reference's voxel id, from the reference's grid (the traversal's bricks re-lay models
// without quads as air).
LW_DI uint32_t voxel(const DevScene &S, const DevParams &P, int x, int y, int z) {
    uint32_t b = ((uint32_t)(y >> 4) * P.grid_dims.z + (uint32_t)(z >> 4)) * P.grid_dims.x + (uint32_t)(x >> 4);
    uint32_t e = ldg(S.grid + (size_t)P.off.x + b);
    if (e == EMPTY) return 0;
    if (e & UNIFORM) return e & ~UNIFORM;
    uint32_t local = (uint32_t)((((y & 15) * 16 + (z & 15)) * 16) + (x & 15));
    uint32_t w = ldg(S.grid + (size_t)P.off.y + (size_t)e * 2048u + (local >> 1));
    return (w >> ((local & 1u) * 16u)) & 0xFFFFu;
}

LW_DI float safe_inv(float x) {  // trace.rs:293-299
    if (fabs_r(x) < 1e-12f) return x < 0.0f ? -1e12f : 1e12f;
    return __fdiv_rn(1.0f, x);
}
LW_DI int sgn(float x) { return x > 0.0f ? 1 : (x < 0.0f ? -1 : 0); }
// `a`: the frame's origin on this axis (the boundary of grid cell c is at c - a in the frame).
LW_DI float next_boundary(float o, float inv, int cell, int step, int a = 0) {  // trace.rs:313-319
    if (step == 0) return kINF;
    float bound = (float)((step > 0 ? cell + 1 : cell) - a);
    return (bound - o) * inv;
}

// One DDA step (trace.rs:267-287): to the next voxel along the axis whose boundary is nearest.
// Written with selects so the lanes of a warp take no branch on the axis. False when the ray
// leaves the range or the grid.
struct Dda {
    int c0, c1, c2;    // the current cell
    float n0, n1, n2;  // distances to its next boundary along each axis
    float t;           // distance at which the ray entered the cell
};
LW_DI bool dda_advance(Dda &s, V3 o, V3 inv, int s0, int s1, int s2, int gs0, int gs1, int gs2, float t_end,
                       const Frame &A = Frame{}) {
    int axis = s.n0 < s.n1 ? (s.n0 < s.n2 ? 0 : 2) : (s.n1 < s.n2 ? 1 : 2);
    bool ax0 = axis == 0, ax1 = axis == 1;
    s.t = ax0 ? s.n0 : (ax1 ? s.n1 : s.n2);
    if (s.t > t_end) return false;
    int st = ax0 ? s0 : (ax1 ? s1 : s2);
    int c = (ax0 ? s.c0 : (ax1 ? s.c1 : s.c2)) + st;
    int g = ax0 ? gs0 : (ax1 ? gs1 : gs2);
    if (c < 0 || c >= g) return false;
    float nb = next_boundary(ax0 ? o.x : (ax1 ? o.y : o.z), ax0 ? inv.x : (ax1 ? inv.y : inv.z), c, st,
                             ax0 ? A.x() : (ax1 ? A.y() : A.z()));
    s.c0 = ax0 ? c : s.c0;
    s.c1 = ax1 ? c : s.c1;
    s.c2 = (!ax0 && !ax1) ? c : s.c2;
    s.n0 = ax0 ? nb : s.n0;
    s.n1 = ax1 ? nb : s.n1;
    s.n2 = (!ax0 && !ax1) ? nb : s.n2;
    return true;
}

// The state of a traversal between two calls of trace_run: the DDA, the inverse direction, the
// end of the range and the visit count. Everything else (the signs of the direction, the brick
// cached in registers) is derived again when the traversal resumes.
struct TraceState {
    Dda s;
    V3 inv;
    float t_end;
    uint32_t it;
};

// The set-up of trace (trace.rs:137-174): the slab test against the grid and the first cell.
// False when the range misses the grid (trace returns None at once).
// In frame A the grid spans [-A, size - A).
LW_DI bool trace_begin(TraceState &ts, const DevParams &P, V3 o, V3 d, float tmax, const Frame &A = Frame{}) {
    const uint32_t dx = P.grid_dims.x, dy = P.grid_dims.y, dz = P.grid_dims.z;
    V3 lo = v3((float)(-A.x()), (float)(-A.y()), (float)(-A.z()));
    V3 hi = v3((float)((int)(dx * 16u) - A.x()), (float)((int)(dy * 16u) - A.y()), (float)((int)(dz * 16u) - A.z()));
    V3 inv = v3(safe_inv(d.x), safe_inv(d.y), safe_inv(d.z));
    V3 ta = vmul(lo - o, inv);
    V3 tb = vmul(hi - o, inv);
    float t_enter = fmax_r(fmax_r(fmin_r(ta.x, tb.x), fmin_r(ta.y, tb.y)), fmin_r(ta.z, tb.z));
    float t_exit = fmin_r(fmin_r(fmax_r(ta.x, tb.x), fmax_r(ta.y, tb.y)), fmax_r(ta.z, tb.z));
    float t0 = fmax_r(t_enter, 0.0f);
    float t_end = fmin_r(t_exit, tmax);
    if (t0 > t_end) return false;
    V3 start = o + d * (t0 + 1e-4f);
    const int s0 = sgn(d.x), s1 = sgn(d.y), s2 = sgn(d.z);
    ts.s.c0 = clamp_i(to_i32(floorf(start.x)) + A.x(), 0, (int)dx * 16 - 1);
    ts.s.c1 = clamp_i(to_i32(floorf(start.y)) + A.y(), 0, (int)dy * 16 - 1);
    ts.s.c2 = clamp_i(to_i32(floorf(start.z)) + A.z(), 0, (int)dz * 16 - 1);
    ts.s.n0 = next_boundary(o.x, inv.x, ts.s.c0, s0, A.x());
    ts.s.n1 = next_boundary(o.y, inv.y, ts.s.c1, s1, A.y());
    ts.s.n2 = next_boundary(o.z, inv.z, ts.s.c2, s2, A.z());
    ts.s.t = t0;
    ts.inv = inv;
    ts.t_end = t_end;
    ts.it = 0;
    return true;
}

// The brick a traversal is in: its top and overlay entries and its occupancy mask, loaded once
// when the ray enters the brick and kept in registers.
struct BrickCache {
    uint32_t b, entry, ov;
    uint2 occ;
};
LW_DI BrickCache no_brick() { return BrickCache{0xFFFFFFFFu, EMPTY, EMPTY, make_uint2(0u, 0u)}; }

// The per-ray constants of the traversal loop.
struct RayDda {
    int s0, s1, s2;     // signs of the direction
    int gs0, gs1, gs2;  // the grid's size in voxels
};
LW_DI RayDda ray_dda(const DevParams &P, V3 d) {
    return RayDda{sgn(d.x), sgn(d.y), sgn(d.z), (int)P.grid_dims.x * 16, (int)P.grid_dims.y * 16, (int)P.grid_dims.z * 16};
}

// One iteration of trace's loop (trace.rs:176-241) up to the quad tests. Returns -1 when the ray
// leaves the range or the grid (or the visit limit is reached), 0 when it stepped past an empty
// brick or voxel, 1 when the cell has quads to test: its model in `model`, its brick's overlay
// entry in bc.ov; the DDA then stays in that cell.
//  * A voxel in an empty 4^3 sub-block of a brick without overlay is not read (its model is 0, it
//    tests no quad).
//  * An empty brick is crossed in one step; with RUNS, so is a whole run of them. A ray in an
//    empty brick above the last occupied brick row that does not go down ends there, no hit.
//  * Every visit (brick skip, empty voxel, voxel with quads) counts towards MAX_STEPS as one
//    iteration of the reference's loop does.
template <bool RUNS = true, bool STAGED = false>
LW_DI int visit(const DevScene &S, const DevParams &P, TraceState &ts, V3 o, V3 d, const RayDda &R, BrickCache &bc,
                uint32_t &model, const Frame &A = Frame{}) {
    const uint32_t dx = P.grid_dims.x, dz = P.grid_dims.z;
    Dda &s = ts.s;
    if (ts.it >= MAX_STEPS) return -1;
    ts.it++;
    uint32_t bx = (uint32_t)(s.c0 >> 4), by = (uint32_t)(s.c1 >> 4), bz = (uint32_t)(s.c2 >> 4);
    uint32_t b = (by * dz + bz) * dx + bx;
    if (b != bc.b) {
        bc.b = b;
        uint2 e = scene_word<STAGED>(S.top + b);
        bc.entry = e.x;
        bc.ov = e.y;
        if (bc.entry != EMPTY && !(bc.entry & UNIFORM)) bc.occ = scene_word<STAGED>(S.occ + bc.entry);
    }
    const V3 inv = ts.inv;
    if (bc.entry == EMPTY && bc.ov == EMPTY) {
        // Above the last row with anything in it, a ray that does not go down stays in empty
        // bricks until it leaves the grid: the reference's loop skips them one by one and ends
        // without a hit, which is the result here at once.
        if (R.s1 >= 0 && by >= S.sky_brick_y) return -1;
        if (!RUNS) {
            // Skip the whole brick: jump to its exit face (trace.rs:184-226).
            int bc0 = (int)bx, bc1 = (int)by, bc2 = (int)bz;
            float t_out = kINF;
            int axis = 0;
            if (R.s0 != 0) {
                float tt = ((float)((R.s0 > 0 ? (bc0 + 1) * 16 : bc0 * 16) - A.x()) - o.x) * inv.x;
                if (tt < t_out) { t_out = tt; axis = 0; }
            }
            if (R.s1 != 0) {
                float tt = ((float)((R.s1 > 0 ? (bc1 + 1) * 16 : bc1 * 16) - A.y()) - o.y) * inv.y;
                if (tt < t_out) { t_out = tt; axis = 1; }
            }
            if (R.s2 != 0) {
                float tt = ((float)((R.s2 > 0 ? (bc2 + 1) * 16 : bc2 * 16) - A.z()) - o.z) * inv.z;
                if (tt < t_out) { t_out = tt; axis = 2; }
            }
            if (t_out > ts.t_end) return -1;
            V3 pos = o + d * t_out;
            s.c0 = axis == 0 ? (R.s0 > 0 ? (bc0 + 1) * 16 : bc0 * 16 - 1) : clamp_i(to_i32(floorf(pos.x)) + A.x(), bc0 * 16, bc0 * 16 + 15);
            s.c1 = axis == 1 ? (R.s1 > 0 ? (bc1 + 1) * 16 : bc1 * 16 - 1) : clamp_i(to_i32(floorf(pos.y)) + A.y(), bc1 * 16, bc1 * 16 + 15);
            s.c2 = axis == 2 ? (R.s2 > 0 ? (bc2 + 1) * 16 : bc2 * 16 - 1) : clamp_i(to_i32(floorf(pos.z)) + A.z(), bc2 * 16, bc2 * 16 + 15);
            int ca = axis == 0 ? s.c0 : (axis == 1 ? s.c1 : s.c2);
            int ga = axis == 0 ? R.gs0 : (axis == 1 ? R.gs1 : R.gs2);
            if (ca < 0 || ca >= ga) return -1;
            s.n0 = next_boundary(o.x, inv.x, s.c0, R.s0, A.x());
            s.n1 = next_boundary(o.y, inv.y, s.c1, R.s1, A.y());
            s.n2 = next_boundary(o.z, inv.z, s.c2, R.s2, A.z());
            s.t = t_out;
            return 0;
        }
        // Skip the whole brick: jump to its exit face (trace.rs:184-226). The brick after a skip
        // is the neighbour along the exit axis (the other axes' cells are clamped into the brick
        // skipped), and the exit distances depend on the bricks alone, so a run of empty bricks is
        // stepped brick by brick here, each one counted as the reference's loop counts it, and
        // the cell, next boundaries and distance are formed once, as the last skip forms them.
        int bc0 = (int)bx, bc1 = (int)by, bc2 = (int)bz;
        float e0 = R.s0 != 0 ? ((float)((R.s0 > 0 ? (bc0 + 1) * 16 : bc0 * 16) - A.x()) - o.x) * inv.x : kINF;
        float e1 = R.s1 != 0 ? ((float)((R.s1 > 0 ? (bc1 + 1) * 16 : bc1 * 16) - A.y()) - o.y) * inv.y : kINF;
        float e2 = R.s2 != 0 ? ((float)((R.s2 > 0 ? (bc2 + 1) * 16 : bc2 * 16) - A.z()) - o.z) * inv.z : kINF;
        float t_out;
        int axis;
        for (;;) {
            // The first axis with the smallest exit distance (trace.rs's strict comparisons).
            t_out = kINF;
            axis = 0;
            if (R.s0 != 0 && e0 < t_out) { t_out = e0; axis = 0; }
            if (R.s1 != 0 && e1 < t_out) { t_out = e1; axis = 1; }
            if (R.s2 != 0 && e2 < t_out) { t_out = e2; axis = 2; }
            if (t_out > ts.t_end) return -1;
            const int nb0 = bc0 + (axis == 0 ? R.s0 : 0), nb1 = bc1 + (axis == 1 ? R.s1 : 0), nb2 = bc2 + (axis == 2 ? R.s2 : 0);
            const int na = axis == 0 ? nb0 : (axis == 1 ? nb1 : nb2);
            const int da = (int)(axis == 0 ? dx : (axis == 1 ? P.grid_dims.y : dz));
            if (na < 0 || na >= da) return -1;  // the exit cell leaves the grid
            const uint32_t nb = ((uint32_t)nb1 * dz + (uint32_t)nb2) * dx + (uint32_t)nb0;
            const uint2 e = scene_word<STAGED>(S.top + nb);
            if (e.x != EMPTY || e.y != EMPTY) {
                bc.b = nb;
                bc.entry = e.x;
                bc.ov = e.y;
                if (bc.entry != EMPTY && !(bc.entry & UNIFORM)) bc.occ = scene_word<STAGED>(S.occ + bc.entry);
                break;
            }
            // The next brick is empty too: the reference's next visit, counted, skips it.
            if (ts.it >= MAX_STEPS) return -1;
            ts.it++;
            if (R.s1 >= 0 && nb1 >= (int)S.sky_brick_y) return -1;
            bc0 = nb0;
            bc1 = nb1;
            bc2 = nb2;
            if (axis == 0) e0 = ((float)((R.s0 > 0 ? (bc0 + 1) * 16 : bc0 * 16) - A.x()) - o.x) * inv.x;
            else if (axis == 1) e1 = ((float)((R.s1 > 0 ? (bc1 + 1) * 16 : bc1 * 16) - A.y()) - o.y) * inv.y;
            else e2 = ((float)((R.s2 > 0 ? (bc2 + 1) * 16 : bc2 * 16) - A.z()) - o.z) * inv.z;
        }
        V3 pos = o + d * t_out;
        s.c0 = axis == 0 ? (R.s0 > 0 ? (bc0 + 1) * 16 : bc0 * 16 - 1) : clamp_i(to_i32(floorf(pos.x)) + A.x(), bc0 * 16, bc0 * 16 + 15);
        s.c1 = axis == 1 ? (R.s1 > 0 ? (bc1 + 1) * 16 : bc1 * 16 - 1) : clamp_i(to_i32(floorf(pos.y)) + A.y(), bc1 * 16, bc1 * 16 + 15);
        s.c2 = axis == 2 ? (R.s2 > 0 ? (bc2 + 1) * 16 : bc2 * 16 - 1) : clamp_i(to_i32(floorf(pos.z)) + A.z(), bc2 * 16, bc2 * 16 + 15);
        s.n0 = next_boundary(o.x, inv.x, s.c0, R.s0, A.x());
        s.n1 = next_boundary(o.y, inv.y, s.c1, R.s1, A.y());
        s.n2 = next_boundary(o.z, inv.z, s.c2, R.s2, A.z());
        s.t = t_out;
        return 0;
    }
    // Block model in this voxel (trace.rs:233-241).
    model = 0u;
    if (bc.entry != EMPTY) {
        if (bc.entry & UNIFORM) {
            model = bc.entry & ~UNIFORM;
        } else {
            int lx = s.c0 & 15, ly = s.c1 & 15, lz = s.c2 & 15;
            uint32_t sb = (uint32_t)(((ly >> 2) * 4 + (lz >> 2)) * 4 + (lx >> 2));
            uint32_t word = sb < 32u ? bc.occ.x : bc.occ.y;
            if ((word >> (sb & 31u)) & 1u) model = brick_voxel(S, bc.entry, lx, ly, lz);
        }
    }
    if (model != 0u || bc.ov != EMPTY) return 1;
    return dda_advance(s, o, inv, R.s0, R.s1, R.s2, R.gs0, R.gs1, R.gs2, ts.t_end, A) ? 0 : -1;
}

// The overlay quads of the cell: in the grid's frame with the ray's own origin (trace.rs:243-263);
// in a chunk frame (REB) relative to the cell, like a model's quads: the origin o - (c - A) and the
// quads' p0 - c.
template <bool REB>
LW_DI void test_overlay(const DevScene &S, const DevParams &P, const Dda &s, uint32_t ov, V3 o, V3 olo, V3 d, float t_lo,
                        Hit &best) {
    uint32_t local = (uint32_t)((((s.c1 & 15) * 16 + (s.c2 & 15)) * 16) + (s.c0 & 15));
    size_t base = (size_t)P.off.w + (size_t)ov * OV_CELL_WORDS + local * 2u;
    uint32_t off = ldg(S.grid + base);
    uint32_t count = ldg(S.grid + base + 1);
    const V3 cell = v3((float)s.c0, (float)s.c1, (float)s.c2);
    for (uint32_t i = 0; i < count; i++) {
        uint32_t qi = ldg(S.grid + (size_t)P.off2.x + off + i);
        if (REB) test_quad<true>(S, P, qi, olo, d, t_lo, best, cell);
        else test_quad(S, P, qi, o, d, t_lo, best);
    }
}

// The origin relative to the cell the DDA is in: o - (c - A).
LW_DI V3 cell_origin(V3 o, const Dda &s, const Frame &A) {
    return o - v3((float)(s.c0 - A.x()), (float)(s.c1 - A.y()), (float)(s.c2 - A.z()));
}

// The quads of the cell the DDA is in (trace.rs:228-264): true with the closest hit in `out`.
template <bool REB = false>
LW_DI bool test_cell(const DevScene &S, const DevParams &P, const TraceState &ts, V3 o, V3 d, float tmin, uint32_t model,
                     uint32_t ov, Hit &out, const Frame &A = Frame{}) {
    const Dda &s = ts.s;
    float t_cell_exit = fmin_r(s.n0, fmin_r(s.n1, s.n2));
    float t_lo = fmax_r(s.t - 1e-4f, tmin);
    float t_hi = t_cell_exit + 1e-4f;
    Hit cand = no_hit();
    cand.t = fmin_r(t_hi, ts.t_end + 1e-3f);
    const V3 lo = cell_origin(o, s, A);
    if (model != 0u) {
        uint4 m = ldg(S.models + model);
        for (uint32_t i = 0; i < m.y; i++) test_quad(S, P, m.x + i, lo, d, t_lo, cand);
    }
    if (ov != EMPTY) test_overlay<REB>(S, P, s, ov, o, lo, d, t_lo, cand);
    if (cand.quad == NO_QUAD) return false;
    out = cand;
    return true;
}

// The traversal loop of trace (trace.rs:176-289), run for at most `budget` voxel visits (0: no
// limit). Returns 1 with the hit, -1 when the ray leaves without one, 0 when the budget ran out
// first; trace_run then continues from `ts` exactly where it stopped.
//
// The DDA is the reference's step for step; what differs is where the words come from (visit) and
// how the lanes of a warp are kept together: the loop is split in two (a "while-while" traversal),
// an inner loop that steps through empty bricks and empty voxels until the ray reaches a cell with
// quads, then the quads of that cell, so the lanes of a warp reach the quad tests together.
template <bool RUNS = true, bool REB = false>
LW_DI int trace_run(const DevScene &S, const DevParams &P, TraceState &ts, V3 o, V3 d, float tmin, uint32_t budget,
                    Hit &out, const Frame &A = Frame{}) {
    const RayDda R = ray_dda(P, d);
    BrickCache bc = no_brick();
    uint32_t n = 0;
    for (;;) {
        uint32_t model = 0;
        for (;;) {
            if (budget != 0u && n >= budget) return 0;
            n++;
            int r = visit<RUNS>(S, P, ts, o, d, R, bc, model, A);
            if (r < 0) return -1;
            if (r > 0) break;
        }
        if (test_cell<REB>(S, P, ts, o, d, tmin, model, bc.ov, out, A)) return 1;
        if (!dda_advance(ts.s, o, ts.inv, R.s0, R.s1, R.s2, R.gs0, R.gs1, R.gs2, ts.t_end, A)) return -1;
    }
}

// The quad tests of the cells the lanes of a warp reached in a round, spread over the warp. Every
// lane calls it (a lane without a cell passes pending = false). The quads of the pending lanes'
// models form one list in lane order; entry k runs quad_candidate on lane k % 32 (in chunks of
// 32), with its owner's ray fetched by shuffles, and writes its candidate hit to `sq` (32 entries
// for this warp). Each owner then takes its own quads' candidates in quad order under trace's
// acceptance rule (reach_of), exactly as the sequential loop of test_cell would, and tests its
// cell's overlay quads, if any, after them. Returns true with the closest hit in `out`.
template <bool REB = false>
LW_DI bool warp_test_cells(const DevScene &S, const DevParams &P, const TraceState &ts, V3 o, V3 d, float tmin,
                           bool pending, uint32_t model, uint32_t ov, Hit &out, float4 *sq, const Frame &A = Frame{}) {
    const unsigned FULL = 0xFFFFFFFFu;
    const uint32_t lane = threadIdx.x & 31u;
    const Dda &s = ts.s;
    float t_lo = 0.0f;
    uint32_t qbase = 0u, cnt = 0u;
    Hit best = no_hit();
    if (pending) {
        float t_cell_exit = fmin_r(s.n0, fmin_r(s.n1, s.n2));
        t_lo = fmax_r(s.t - 1e-4f, tmin);
        best.t = fmin_r(t_cell_exit + 1e-4f, ts.t_end + 1e-3f);
        if (model != 0u) {
            uint4 m = ldg(S.models + model);
            qbase = m.x;
            cnt = m.y;
        }
    }
    // Exclusive scan of the lanes' quad counts.
    uint32_t incl = cnt;
    for (uint32_t off = 1; off < 32u; off <<= 1) {
        uint32_t v = __shfl_up_sync(FULL, incl, off);
        if (lane >= off) incl += v;
    }
    const uint32_t pre = incl - cnt;
    const uint32_t total = __shfl_sync(FULL, incl, 31);
    for (uint32_t base = 0; base < total; base += 32u) {
        const uint32_t k = base + lane;
        // The entry's owner: the highest lane whose list starts at or before k (a lane with no
        // quads starts where the next one does, so the owner of an entry k < total has quads).
        uint32_t L = 0;
        for (uint32_t step = 16; step != 0u; step >>= 1) {
            uint32_t p = __shfl_sync(FULL, pre, L + step);
            if (p <= k) L += step;
        }
        // the owner's origin relative to its cell, formed here from its origin and cell (fewer
        // registers live across the loop than keeping it in the owner)
        const V3 olo = v3(__shfl_sync(FULL, o.x, L), __shfl_sync(FULL, o.y, L), __shfl_sync(FULL, o.z, L)) -
                       v3((float)__shfl_sync(FULL, s.c0 - A.x(), L), (float)__shfl_sync(FULL, s.c1 - A.y(), L),
                          (float)__shfl_sync(FULL, s.c2 - A.z(), L));
        const V3 od = v3(__shfl_sync(FULL, d.x, L), __shfl_sync(FULL, d.y, L), __shfl_sync(FULL, d.z, L));
        const float otlo = __shfl_sync(FULL, t_lo, L);
        const uint32_t oq = __shfl_sync(FULL, qbase, L) + (k - __shfl_sync(FULL, pre, L));
        Hit h;
        // No upper bound on t here: the owner applies the exact reach when it takes the entry.
        const bool valid = k < total && quad_candidate(S, P, oq, olo, od, otlo, kINF, h);
        if (valid) sq[lane] = make_float4(h.t, h.s, h.tt, __uint_as_float(h.texel));
        const unsigned vm = __ballot_sync(FULL, valid);
        __syncwarp();
        // This lane's entries in the chunk, in order; only valid candidates can be taken.
        if (cnt != 0u && pre < base + 32u && pre + cnt > base) {
            const uint32_t a = pre > base ? pre - base : 0u;
            const uint32_t b = min(pre + cnt - base, 32u);
            unsigned mine = vm & (b >= 32u ? FULL : ((1u << b) - 1u)) & ~((1u << a) - 1u);
            while (mine) {
                const uint32_t j = (uint32_t)(__ffs(mine) - 1);
                mine &= mine - 1u;
                const float4 c = sq[j];
                const uint32_t qi = qbase + (base + j - pre);
                if (c.x < reach_of(best, qi)) best = Hit{c.x, qi, __float_as_uint(c.w), c.y, c.z};
            }
        }
        __syncwarp();
    }
    if (pending && ov != EMPTY) test_overlay<REB>(S, P, s, ov, o, REB ? cell_origin(o, s, A) : o, d, t_lo, best);
    if (!pending || best.quad == NO_QUAD) return false;
    out = best;
    return true;
}

// One round of a traversal for the lanes of a warp that trace rays together; every lane calls it
// (a lane without a ray passes have = false and gets 0). Each lane makes at most `budget` (>= 1)
// visits through empty space, up to the first cell with quads; then one warp_test_cells tests the
// cells the lanes reached, so a warp runs one phase of quad tests per round, spread over its 32
// lanes. Returns as trace_run does (1 hit, -1 no hit, 0 the round ended first); after 0 the next
// round continues from `ts`. The visits and quad tests are trace_run's, in the same order.
template <bool STAGED = false, bool REB = false>
LW_DI int trace_round_warp(const DevScene &S, const DevParams &P, TraceState &ts, V3 o, V3 d, float tmin,
                           uint32_t budget, bool have, Hit &out, float4 *sq, const Frame &A = Frame{}) {
    const RayDda R = ray_dda(P, d);
    BrickCache bc = no_brick();
    uint32_t model = 0;
    int r = 0;
    if (have) {
        uint32_t more = budget - 1u;  // visits left in this round after the next one
        for (;;) {
            r = visit<true, STAGED>(S, P, ts, o, d, R, bc, model, A);
            if (r != 0 || more == 0u) break;
            more--;
        }
    }
    const bool pending = have && r > 0;
    if (__any_sync(0xFFFFFFFFu, pending)) {
        const bool hit = warp_test_cells<REB>(S, P, ts, o, d, tmin, pending, model, bc.ov, out, sq, A);
        if (pending) r = hit ? 1 : (dda_advance(ts.s, o, ts.inv, R.s0, R.s1, R.s2, R.gs0, R.gs1, R.gs2, ts.t_end, A) ? 0 : -1);
    }
    return have ? r : 0;
}

// trace (trace.rs:137-290): the closest hit along o + t d, t in (tmin, tmax), in one go.
// RUNS: whether a visit steps a whole run of empty bricks (the adjoint's kernels, whose registers
// are bounded tighter, run 10 % faster with one brick per visit).
// REB: o is in frame A (chunk-origin rebasing).
template <bool RUNS = true, bool REB = false>
LW_DI Hit trace(const DevScene &S, const DevParams &P, V3 o, V3 d, float tmin, float tmax, const Frame &A = Frame{}) {
    TraceState ts;
    if (!trace_begin(ts, P, o, d, tmax, A)) return no_hit();
    Hit h;
    if (trace_run<RUNS, REB>(S, P, ts, o, d, tmin, 0u, h, A) == 1) return h;
    return no_hit();
}

// is_see_through / see_through_hit (trace.rs:113-131).
LW_DI bool is_see_through(const DevParams &P, uint32_t qi) {
    return qi >= P.see_through.x && qi - P.see_through.x < P.see_through.y;
}
// REB: o in frame A, the quads' p0 taken relative to A.
template <bool REB = false>
LW_COLD Hit see_through_hit(const DevScene &S, const DevParams &P, V3 o, V3 d, float tmin, const Frame &A = Frame{}) {
    Hit best = no_hit();
    for (uint32_t i = 0; i < P.see_through.y; i++) {
        if (REB) test_quad<true>(S, P, P.see_through.x + i, o, d, tmin, best, frame_origin(A));
        else test_quad(S, P, P.see_through.x + i, o, d, tmin, best);
    }
    return best;
}

}  // namespace lw
