/*
 * CPU oracle for the hq path tracer: a plain-C restatement of the reference kernel crate
 * `crates/lumenwright-kernel` (rng.rs, math.rs, scene.rs, trace.rs, integrator.rs) and of
 * the CPU backend's per-pixel loop (`crates/lumenwright/src/render/cpu/mod.rs:39-87`).
 *
 * THIS IS TEST INFRASTRUCTURE. Only the tests, the smoke check and the CPU-baseline leg of
 * the benchmark may load it, and only as the checker or the timed CPU baseline; the
 * product path (lumenwright_b200) never calls it.
 *
 * Two builds share one source (kernel_impl.h):
 *   - FP32 (`lwo32_*`): the reference's f32 arithmetic, operation for operation, compiled
 *     with -ffp-contract=off so no FMA is formed, with the reference's own f32 polynomials
 *     for sin/cos in turns, acos, atan2 and ln, and the platform libm `expf` (the
 *     reference's host build calls Rust std `f32::exp`, which is the platform libm's).
 *   - FP64 (`lwo64_*`): the same algorithm and the same random draws in double precision
 *     with libm's double functions, the converged-image reference.
 *
 * Parity pins: the FP32 build reproduces every known-answer test of
 * `crates/lumenwright-kernel/src/tests.rs` (tests/test_oracle_kernel.py).
 */
#ifndef LW_ORACLE_H
#define LW_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* `GpuQuad` (crates/lumenwright-kernel/src/scene.rs:46-57), 80 bytes. */
typedef struct {
    float p0[4];  /* xyz corner, w = flags (bit cast) */
    float eu[4];  /* xyz edge along s, w = tint RGBA8 (bit cast) */
    float ev[4];  /* xyz edge along t, w = emittance */
    float uv[4];  /* uv0.xy, uvs.xy */
    float uvt[4]; /* uvt.xy, 0, 0 */
} lwo_quad;

/* `GpuModel` (scene.rs:103-112), 16 bytes. */
typedef struct {
    uint32_t quad_offset, quad_count, flags, pad;
} lwo_model;

/* `GpuEmitter` (scene.rs:119-124), 32 bytes. */
typedef struct {
    float pos[4];      /* xyz offset, w = first quad (bit cast) */
    uint32_t faces[4]; /* x = face count */
} lwo_emitter;

/* `Params` (scene.rs:160-228), 27 x 16 = 432 bytes. */
typedef struct {
    float cam_pos[4], cam_fwd[4], cam_right[4], cam_up[4];
    float sun_dir[4], sun_color[4], sky_sun[4], sky_zenith[4];
    float perez_a[4], perez_b[4], perez_c[4], perez_d[4], perez_e[4];
    float water_color[4], misc_f[4];
    uint32_t grid_dims[4], off[4], off2[4], frame[4], misc_u[4], see_through[4], emitter[4];
    float sun_su[4], sun_sv[4], sun_sprite[4], sky_map[4], water_plane[4];
} lwo_params;

/* `SceneView` (scene.rs:232-259): borrowed buffers with their lengths in elements. */
typedef struct {
    const lwo_params *params;
    const uint32_t *grid;
    uint64_t grid_len;
    const lwo_model *models;
    uint64_t models_len;
    const lwo_quad *quads;
    uint64_t quads_len;
    const uint32_t *atlas;
    uint64_t atlas_len;
    const lwo_emitter *emitters;
    uint64_t emitters_len;
    const uint32_t *emitter_grid;
    uint64_t emitter_grid_len;
    const float *sky;
    uint64_t sky_len;
} lwo_scene;

/* `Hit` (trace.rs:11-22). `found` is 0 for `None`. */
typedef struct {
    float t;
    uint32_t quad, texel;
    float s, tt;
    int32_t found;
} lwo_hit;

/* The FP64 oracle's camera: eye relative to the grid origin and the basis, in double
 * precision (the reference forms the eye in f64 before casting, request.rs:640-644). */
typedef struct {
    double eye[3], fwd[3], right[3], up[3];
    double tan_half, aspect;
} lwo_camera64;

/* Parameters theta of the differentiable form, for the FP64 build's reference gradient. With a
 * theta, a hit's albedo is the parameter of its atlas texel (texel_param, -1 = the decoded
 * texel) times the decoded tint; an emitter's intensity is scaled by its group's entry of
 * emit_mult (group = pcg_hash of its voxel, 32 groups); the sun direction is `sun` and the Chunky
 * sky cache `sky64`. With `frozen`, the Russian roulette takes its probability and decision from
 * the `albedo0` throughput and the shadow rays run along `sun0` (the crossed water's length
 * follows `sun` through the same surfaces): the estimator whose derivative the adjoint forms. */
typedef struct {
    const double *albedo;      /* n_params * 3 */
    const double *albedo0;     /* n_params * 3, the nominal albedos (frozen roulette) */
    uint32_t n_params;
    int32_t frozen;
    const int32_t *texel_param; /* one per atlas texel */
    uint64_t texel_param_len;
    const double *emit_mult;   /* 32 */
    const double *sky64;       /* the sky cache under theta, or NULL for the scene's sky */
    uint64_t sky64_len;
    double sun[4];             /* sun direction, cos of the sun's angular radius */
    double sun0[4];            /* nominal sun direction (frozen shadow rays) */
} lwo_theta;

/* Work counters of the instrumented FP32 build (algorithmic bytes per sample). */
typedef struct {
    uint64_t samples, events, traces, dda_steps, brick_skips, voxel_lookups, model_fetches,
        quad_tests, texel_fetches, overlay_reads, sky_reads, map_reads, emitter_cell_reads,
        emitter_index_reads, emitter_reads, bounds_errors;
} lwo_counters;

/* ---- FP32 build ---------------------------------------------------------------------- */
uint32_t lwo32_pcg_hash(uint32_t v);
uint32_t lwo32_rng_new(uint32_t pixel, uint32_t sample, uint32_t seed);
float lwo32_rng_next(uint32_t *state);
void lwo32_sin_cos_turns(float u, float *s, float *c);
float lwo32_acos(float x);
float lwo32_atan2(float y, float x);
float lwo32_ln(float x);
float lwo32_gamma_to_linear(float c);
uint32_t lwo32_voxel(const lwo_scene *s, int32_t x, int32_t y, int32_t z);
lwo_hit lwo32_trace(const lwo_scene *s, const float o[3], const float d[3], float tmin, float tmax);
lwo_hit lwo32_see_through_hit(const lwo_scene *s, const float o[3], const float d[3], float tmin);
void lwo32_render_sample(const lwo_scene *s, uint32_t px, uint32_t py, uint32_t sample,
                         float out[3]);
void lwo32_sample_emitters(const lwo_scene *s, const float pos[3], const float origin[3],
                           const float n[3], uint32_t *rng_state, float out[3]);
void lwo32_emitter_cell(const lwo_scene *s, const float p[3], uint32_t *start, uint32_t *count);
/* One step of chunk-origin rebasing (the library's precision option): x, held in the frame of
 * chunk corner *word, moved to the frame of the corner nearest it; *word becomes that corner. */
void lwo32_rebase(float x[3], uint32_t *word);
void lwo32_preetham_radiance(const lwo_scene *s, const float d[3], float out[3]);
void lwo32_build_sky_cache(const lwo_scene *s, uint32_t n, float *out);
void lwo32_sky_radiance(const lwo_scene *s, const float d[3], float out[3]);
void lwo32_sky_lens(const lwo_scene *s, const float d[3], float out[3]);
void lwo32_sky_light(const lwo_scene *s, const float d[3], float out[3]);
void lwo32_sun_texture(const lwo_scene *s, const float d[3], float out[3]);
/* sky_radiance for n directions (d: 3n floats, out: 3n floats), over all host threads. */
void lwo32_sky_radiance_many(const lwo_scene *s, uint64_t n, const float *d, float *out);

/* Per-sample radiance of `count` samples starting at `sample_start` for every pixel of the
 * rectangle [x0, x0+w) x [y0, y0+h): out[((py*w + px) * count + k) * 3 + c]. */
void lwo32_render_samples(const lwo_scene *s, uint32_t x0, uint32_t y0, uint32_t w, uint32_t h,
                          uint32_t sample_start, uint32_t count, float *out, int threads);

/* The CPU backend's per-pixel mean (cpu/mod.rs:39-87): f64 sums of finite samples divided by
 * spp, for the rectangle; out[(py*w+px)*3+c]. Rows run in parallel over `threads`. */
void lwo32_render_mean(const lwo_scene *s, uint32_t x0, uint32_t y0, uint32_t w, uint32_t h,
                       uint32_t spp, float *out, int threads);

/* Instrumented run: the same as lwo32_render_mean, counting work. */
void lwo32_count_work(const lwo_scene *s, uint32_t x0, uint32_t y0, uint32_t w, uint32_t h,
                      uint32_t spp, lwo_counters *out);

/* Number of out-of-range buffer reads the FP32/FP64 builds have seen (0 for valid scenes). */
uint64_t lwo_bounds_errors(void);
void lwo_reset_bounds_errors(void);

/* ---- the display pass (post.c) ------------------------------------------------------- */
/* post::tonemap (mix = 0) or post::tonemap_mix, n pixels of 3 floats to RGBA8 words. */
void lwo_tonemap(const float *hdr, uint64_t n, float exposure, uint32_t op, uint32_t mix, uint32_t op_b, float weight,
                 uint32_t *out);
void lwo_game_tone_curve(float out[7]);

/* `QuickSky` (crates/lumenwright/src/render/sky.rs:274-305), 608 bytes: the record the game
 * sky's per-texel pass reads. */
typedef struct {
    float sky_color[4], fog_color[4], fog_dist[4], sunrise[4], flags[4];
    float sun[4][4], moon[4][4], star_rot[3][4], fan[18][4];
    float cam_forward[4], cam_right[4], cam_up[4], cam_misc[4];
} lwo_quick_sky;
/* `draw_map` (sky.rs:861-878): QuickSky::background for every texel of a w x h equirectangular
 * map, decoded to linear, into out (w * h * 3 floats, row 0 at the nadir). */
void lwo_draw_sky_map(const lwo_quick_sky *q, const uint32_t *atlas, uint32_t atlas_w, const uint32_t *stars, uint32_t w,
                      uint32_t h, float *out, int threads);
double lwo_mid_grey_gain(void);
double lwo_game_before_gamma(double x);

/* ---- FP64 build ---------------------------------------------------------------------- */
void lwo64_render_sample(const lwo_scene *s, const lwo_camera64 *cam, uint32_t px, uint32_t py,
                         uint32_t sample, double out[3]);
/* Per-sample radiance of the FP64 twin, (h, w, count, 3) doubles. */
void lwo64_render_samples(const lwo_scene *s, const lwo_camera64 *cam, uint32_t x0, uint32_t y0, uint32_t w, uint32_t h,
                          uint32_t sample_start, uint32_t count, double *out, int threads);
void lwo64_render_mean(const lwo_scene *s, const lwo_camera64 *cam, uint32_t x0, uint32_t y0,
                       uint32_t w, uint32_t h, uint32_t spp, double *out, int threads);
/* lwo64_render_mean under a theta. */
void lwo64_render_mean_theta(const lwo_scene *s, const lwo_camera64 *cam, const lwo_theta *th, uint32_t x0,
                             uint32_t y0, uint32_t w, uint32_t h, uint32_t spp, double *out, int threads);
/* Every sample under `plus` and under `minus`: per pixel the mean of the paired differences and
 * of the pairs' midpoints (the FP64 reference gradient's finite differences). */
void lwo64_render_fd_theta(const lwo_scene *s, const lwo_camera64 *cam, const lwo_theta *plus,
                           const lwo_theta *minus, uint32_t x0, uint32_t y0, uint32_t w, uint32_t h,
                           uint32_t spp, double *diff, double *mean, int threads);

#ifdef __cplusplus
}
#endif
#endif
