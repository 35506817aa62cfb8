/*
 * lumenwright_b200: the hq path tracer of Lumenwright (brick-grid traversal, block shading,
 * Chunky/game sky with sun shadow rays, emitter sampling, per-pixel sample accumulation),
 * written for NVIDIA B200 (sm_100a), behind a C ABI.
 *
 * It replaces the reference's CUDA entry `pt_render`
 * (crates/lumenwright-ptx/src/lib.rs:37-87) and its host launcher `CudaBackend::render_hq`
 * (crates/lumenwright/src/render/cuda.rs:77-184); a Rust `Backend` implementation calls these
 * functions through an FFI crate.
 *
 * Conventions: every length is in elements of its buffer, as `pt_render` takes them; the caller
 * owns every host buffer; the library owns device memory inside an `lw_ctx`. No function traps
 * or aborts: each returns an `lw_status`, and `lw_last_error` gives the text of the last failure.
 * A context is used from one thread at a time.
 */
#ifndef LUMENWRIGHT_B200_H
#define LUMENWRIGHT_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- records shared with the reference (crates/lumenwright-kernel/src/scene.rs) ---------- */

/* `GpuQuad` (scene.rs:46-57), 80 bytes. */
typedef struct {
    float p0[4];  /* xyz corner, w = flags (bit cast) */
    float eu[4];  /* xyz edge along s, w = tint RGBA8 (bit cast) */
    float ev[4];  /* xyz edge along t, w = emittance */
    float uv[4];  /* uv0.xy, uvs.xy */
    float uvt[4]; /* uvt.xy, unused, unused */
} lw_quad;

/* `GpuModel` (scene.rs:103-112), 16 bytes. */
typedef struct {
    uint32_t quad_offset, quad_count, flags, pad;
} lw_model;

/* `GpuEmitter` (scene.rs:119-124), 32 bytes. */
typedef struct {
    float pos[4];      /* xyz offset into grid space, w = first quad (bit cast) */
    uint32_t faces[4]; /* x = face count */
} lw_emitter;

/* `Params` (scene.rs:160-228), 27 x 16 = 432 bytes, layout-identical. Two of its unused words
 * carry this library's chunk-origin rebasing (the precision form): see_through[2] = 1 holds every
 * position of a path relative to the chunk corner nearest its current origin instead of the grid
 * origin, starting from the camera's chunk corner packed in see_through[3] (chunk indices in two's
 * complement, x in bits 0-10, y in 11-20, z in 21-31), cam_pos.xyz then being the eye relative to
 * that corner. lw_rebase_camera sets the three from the eye in f64. see_through[2] = 0 (the
 * reference's value) renders in the grid's frame, as the reference does. The batched and
 * differentiable forms, and lw_trace_rays, take the grid's frame only. */
typedef struct {
    float cam_pos[4], cam_fwd[4], cam_right[4], cam_up[4];
    float sun_dir[4], sun_color[4], sky_sun[4], sky_zenith[4];
    float perez_a[4], perez_b[4], perez_c[4], perez_d[4], perez_e[4];
    float water_color[4], misc_f[4];
    uint32_t grid_dims[4], off[4], off2[4], frame[4], misc_u[4], see_through[4], emitter[4];
    float sun_su[4], sun_sv[4], sun_sprite[4], sky_map[4], water_plane[4];
} lw_params;

/* `Hit` (crates/lumenwright-kernel/src/trace.rs:11-22); found = 0 for `None`. */
typedef struct {
    float t;
    uint32_t quad, texel;
    float s, tt;
    int32_t found;
} lw_hit;

/* ---- status ------------------------------------------------------------------------------ */
typedef enum {
    LW_OK = 0,
    LW_ERR_INVALID_ARGUMENT = 1, /* a null pointer, a zero size, an unknown option */
    LW_ERR_BUFFER_LENGTH = 2,    /* a buffer shorter than the layout it must hold, or an index
                                    in one buffer that points outside another */
    LW_ERR_OUT_OF_MEMORY = 3,
    LW_ERR_DEVICE_TIMEOUT = 4, /* a wait for the GPU ran past the deadline of lw_set_timeout */
    LW_ERR_LAUNCH = 5,         /* a CUDA launch or copy failed */
    LW_ERR_CANCELLED = 6,      /* lw_cancel was called during the render */
    LW_ERR_NO_DEVICE = 7,      /* no CUDA device, or not an sm_100 one */
    LW_ERR_NO_SCENE = 8        /* a render before lw_scene_upload */
} lw_status;

typedef struct lw_ctx lw_ctx;

/* The scene a frame is drawn in: `HqScene` (crates/lumenwright/src/scene/voxel.rs:19-49).
 * `dims` is the grid in bricks and `offsets` the word offsets of top, bricks, ov_top,
 * ov_cells, ov_quads in `grid` (the reference's `HqScene.dims` / `offsets`). */
typedef struct {
    const uint32_t *grid;
    uint64_t grid_len;
    const lw_model *models;
    uint64_t models_len;
    const lw_quad *quads;
    uint64_t quads_len;
    const uint32_t *atlas;
    uint64_t atlas_len;
    const lw_emitter *emitters;
    uint64_t emitters_len;
    const uint32_t *emitter_grid;
    uint64_t emitter_grid_len;
    uint32_t dims[3];
    uint32_t offsets[5];
    uint32_t atlas_size[2];
} lw_scene_desc;

/* Progress after each batch of samples: (samples done, samples total, user). Called on the
 * thread that called lw_render_hq, between launches; never from a CUDA callback thread. */
typedef void (*lw_progress_fn)(uint32_t done, uint32_t total, void *user);

/* Launch statistics of the last render on a context. */
typedef struct {
    double kernel_ms;        /* CUDA-event time of the path-tracing launches */
    double upload_ms;        /* host-to-device copies and the grid re-layout of the last upload */
    uint32_t launches;       /* kernel launches of the render (path tracing and reductions) */
    uint32_t blocks, threads; /* launch shape of the megakernel (blocks = SMs x resident blocks) */
    uint64_t samples;        /* path samples traced */
    /* the wavefront engine: CUDA-event time and launches of its tracing and shading kernels */
    double trace_ms, shade_ms;
    uint32_t trace_launches, shade_launches;
    uint64_t rays;           /* rays traced (path, shadow and emitter rays) */
} lw_stats;

/* Launch tuning of the render (the autotuner's knobs).
 * engine: how lw_render_hq / lw_render_device run: LW_ENGINE_WAVEFRONT (the default) keeps each
 *   path in a slot of a pool in device memory and alternates a shading kernel with a tracing kernel
 *   whose lanes take the next queued ray as soon as theirs ends; LW_ENGINE_MEGAKERNEL runs one
 *   persistent kernel in which each lane follows its own paths. For the same samples per work
 *   item (sub) both give the same image, bit for bit; left at 0, sub is 1 for the wavefront and
 *   chosen from the frame for the megakernel, so the images then differ by the rounding of the
 *   item sums. The batched form runs the engine named here too (the wavefront as one CUDA graph); the
 *   per-sample entry point and lw_render_accumulate_noalloc always run the megakernel.
 * threads: threads per block of the megakernel (64, 128 or 256).
 * budget: voxel visits a ray advances before its lane may take up other work: the megakernel's
 *   regrouping period (0 = a whole traversal at once), the wavefront's visits through empty
 *   space per round, between queue fetches (0 = 8).
 * sub: samples per work item (0: one for the wavefront; for the megakernel and the batched form
 *   chosen from the frame so every lane gets many items).
 * paths: path slots of the wavefront (0: sized from each launch's sample count, 2^16 to 2^23). */
#define LW_ENGINE_WAVEFRONT 0u
#define LW_ENGINE_MEGAKERNEL 1u
typedef struct {
    uint32_t threads;
    uint32_t budget;
    uint32_t sub;
    uint32_t engine;
    uint32_t paths;
} lw_tuning;

/* ---- context ------------------------------------------------------------------------------
 * Replaces CudaBackend::new (crates/lumenwright/src/render/cuda.rs:55-63): opens `device`,
 * checks it is sm_100, creates the context's streams. */
lw_status lw_ctx_create(int device, lw_ctx **out);
void lw_ctx_destroy(lw_ctx *ctx);
/* Text of the last failure on `ctx` (or of the last lw_ctx_create failure when ctx is null). */
const char *lw_last_error(const lw_ctx *ctx);
/* The CUDA stream (cudaStream_t) the context launches its path-tracing kernels on. */
void *lw_stream(lw_ctx *ctx);
lw_status lw_get_stats(const lw_ctx *ctx, lw_stats *out);
/* Sets / reads the launch tuning of a context (defaults: wavefront engine with automatic path
 * slots, 128 threads, budget 0, sub automatic). */
lw_status lw_set_tuning(lw_ctx *ctx, const lw_tuning *tuning);
lw_status lw_get_tuning(const lw_ctx *ctx, lw_tuning *out);
/* Asks a running render on `ctx` to stop; safe from any thread. The render's call returns
 * LW_ERR_CANCELLED, or, where that call returns before its kernels end (lw_render_device,
 * lw_batch_run), the call that waits for its results does (lw_read_accumulator,
 * lw_read_accumulator_rgba, lw_batch_read). A render is cut into launches (a batch of samples
 * each); a launch that a cancel reaches adds nothing to the accumulator, so every pixel keeps the
 * whole launches done before it and its count says how many samples that is (a cancelled batch
 * leaves its images at zero). A cancel also stops the kernels of lw_render_accumulate_noalloc,
 * which returns before they run and so cannot report it: the caller's accumulator then holds the
 * launches done before the cancel, and each record's count (its fourth float) tells how many
 * samples. The next render on `ctx` starts uncancelled. */
void lw_cancel(lw_ctx *ctx);
/* A deadline, in seconds, for every wait of a call on `ctx` for its render's work on the GPU
 * (0, the default: no limit). The reference's CUDA backend waits without a limit for each batch
 * (crates/lumenwright/src/render/cuda.rs:154-159). With a deadline, a wait polls the work's
 * completion; if the deadline passes first, the render's kernels are cancelled as lw_cancel
 * cancels them, the call waits at most 10 s more for them to end, and it returns
 * LW_ERR_DEVICE_TIMEOUT (the accumulator then holds the launches done before, as after a cancel).
 * The next render on `ctx` starts uncancelled. */
lw_status lw_set_timeout(lw_ctx *ctx, double seconds);
/* Records timing mark `slot` (0..7), a CUDA event on the context's stream, and reads the time
 * between two marks once both are reached (the device's clock, not the host's). */
lw_status lw_mark(lw_ctx *ctx, uint32_t slot);
lw_status lw_elapsed_ms(lw_ctx *ctx, uint32_t from, uint32_t to, double *ms);

/* ---- scene ---------------------------------------------------------------------------------
 * Replaces the seven `clone_htod` copies of CudaBackend::render_hq (cuda.rs:96-111): validates
 * every buffer length and every cross-buffer index (what the reference's slice bounds checks
 * would trap on), copies the buffers and re-lays the brick grid for the B200 kernels. The scene
 * stays resident across renders until the next upload. */
lw_status lw_scene_upload(lw_ctx *ctx, const lw_scene_desc *scene);

/* ---- the grid build on the device -----------------------------------------------------------
 * `voxel::build_hq` (crates/lumenwright/src/scene/voxel.rs:111-491, with `emitter_list`, :542-607)
 * for a block volume, producing the same buffers word for word as the host build, resident as the
 * context's scene (as after lw_scene_upload). Two calls around the caller's model generation:
 *   1. lw_scene_build_keys: the volume's distinct model-instance keys (a block state `s` gives
 *      key s << 8, a fluid state s << 8 | its face mask, `Scene::fluid_face_mask`,
 *      crates/lumenwright/src/scene/mod.rs:586-609; an invisible state none) in the order the
 *      build interns them (bricks in brick order, voxels in (y, z, x) order inside a brick);
 *   2. lw_scene_build_grid, with the caller's models and quads for those keys (models[0] air,
 *      models[i] the instance of keys[i - 1], quads as the build lays them out, model_emits[i] 1 for
 *      an emitting instance) and the atlas: instance ids, buried / uniform / stored bricks, the
 *      grid, the emitters and the emitter grid, then the B200 re-layout. */
#define LW_STATE_OCCLUDES 1u
#define LW_STATE_INVISIBLE 2u
#define LW_STATE_FLUID 4u
typedef struct {
    const uint16_t *blocks;     /* voxel states, index (y * size[2] + z) * size[0] + x */
    uint32_t size[3];           /* x, y, z in voxels, multiples of 16 */
    const uint8_t *state_flags; /* per state: LW_STATE_* bits */
    uint32_t n_states;          /* at most 65536 */
} lw_world_desc;
typedef struct {
    const lw_model *models;
    uint64_t models_len;
    const lw_quad *quads;
    uint64_t quads_len;
    const uint8_t *model_emits;
    const uint32_t *atlas;
    uint64_t atlas_len;
    uint32_t atlas_size[2];
} lw_instances_desc;
typedef struct {
    uint32_t dims[3];      /* the grid in bricks */
    uint32_t offsets[5];   /* top, bricks, ov_top, ov_cells, ov_quads */
    uint64_t grid_len, emitter_grid_len;
    uint32_t bricks, uniform_bricks, buried_bricks, emitters;
    double keys_ms, grid_ms; /* wall time of the two calls */
} lw_build_info;
lw_status lw_scene_build_keys(lw_ctx *ctx, const lw_world_desc *world, uint32_t *keys, uint32_t cap, uint32_t *n_keys);
lw_status lw_scene_build_grid(lw_ctx *ctx, const lw_world_desc *world, const lw_instances_desc *inst, lw_build_info *info);
/* Reads the context's scene back: the grid, the emitters and the emitter grid (each skipped when
 * NULL; each capacity in elements must hold the scene's length). */
lw_status lw_scene_read(lw_ctx *ctx, uint32_t *grid, uint64_t grid_cap, lw_emitter *emitters, uint64_t emitters_cap,
                        uint32_t *emitter_grid, uint64_t emitter_grid_cap);

/* ---- rendering -----------------------------------------------------------------------------
 * `Backend::render_hq` (crates/lumenwright/src/render/mod.rs:98-102) on the uploaded scene:
 * `params` is the frame's `Params`, `sky` the frame's sky buffer (`HqFrame.sky`), `spp` the
 * samples per pixel (at least 1). Writes the mean linear radiance per pixel, row-major, top row
 * first, to `out_rgb` (frame[0] * frame[1] * 3 floats). Non-finite samples are left out of the
 * sum and counted, as `pt_render` does (crates/lumenwright-ptx/src/lib.rs:76-84). The sums are
 * Kahan-compensated FP32. The samples run in as few launches as keep a launch's item sums (16
 * bytes a pixel sample with the wavefront's one-sample items) within 16 GiB, or a quarter of the
 * device memory free when the context was made if that is less; `progress` is called after each
 * launch. */
lw_status lw_render_hq(lw_ctx *ctx, const lw_params *params, const float *sky, uint64_t sky_len, uint32_t spp,
                       lw_progress_fn progress, void *user, float *out_rgb);

/* The same render with every buffer already on the device: the scene uploaded, the sky
 * uploaded by lw_sky_upload, the result left in the context's device accumulator (read it with
 * lw_read_accumulator). Samples [sample_start, sample_start + spp) are added to the
 * accumulator; clear it with lw_clear_accumulator. No host copies happen inside. */
lw_status lw_sky_upload(lw_ctx *ctx, const float *sky, uint64_t sky_len);
lw_status lw_clear_accumulator(lw_ctx *ctx, uint32_t width, uint32_t height);
lw_status lw_render_device(lw_ctx *ctx, const lw_params *params, uint32_t sample_start, uint32_t spp);
lw_status lw_read_accumulator(lw_ctx *ctx, float *out_rgb);

/* One shard of a frame split over GPUs (one process and context per GPU): the samples
 * [sample_start, sample_start + spp) of the frame's 8x4-pixel tiles shard, shard + shards,
 * shard + 2 shards, ... (tiles numbered row by row), added to the context's accumulator. Every
 * (pixel, sample) is independent (crates/lumenwright-kernel/src/rng.rs:23-27) and a pixel's sums
 * depend only on its own samples, so a pixel's record is the one a render of the whole frame
 * gives, bit for bit; the other pixels' records are left as they are (zero after
 * lw_clear_accumulator), so a sum of the shards' accumulators over the GPUs (an NCCL reduce of the
 * records lw_accumulator_device names) is exactly the whole frame's accumulator. */
lw_status lw_render_device_shard(lw_ctx *ctx, const lw_params *params, uint32_t sample_start, uint32_t spp, uint32_t shard,
                                 uint32_t shards);
/* The context's device accumulator: frame[0] * frame[1] records of 8 floats (Kahan sum r, g, b,
 * sample count; compensation r, g, b, unused), valid until the next lw_clear_accumulator or
 * render of another frame size; for a caller that combines accumulators across GPUs. */
lw_status lw_accumulator_device(lw_ctx *ctx, void **records, uint32_t *width, uint32_t *height);

/* ---- the batched form ----------------------------------------------------------------------
 * Many cameras of uneven resolution and spp over the uploaded scene in one persistent launch:
 * every camera's work items go into one queue, so the GPU stays full until the last sample of
 * the last camera. lw_batch_prepare uploads the cameras' skies (once per distinct host buffer),
 * lays out their accumulators and partial sums, and captures clear + render + reduce into a CUDA
 * graph; lw_batch_run replays the graph (asynchronously, on lw_stream); lw_batch_read waits and
 * copies each camera's mean radiance to its `out_rgb` (skipped when NULL). lw_render_batch does
 * all three. A camera's image is what lw_render_hq gives for the same Params, sky and spp. With
 * the wavefront engine and automatic items (lw_tuning.sub 0), every work item is one sample and
 * the graph runs the batch in as many passes as keep a pass's item sums (16 bytes an item) within
 * 40 GiB and a third of the free device memory (LUMENWRIGHT_BATCH_SUMS_MB in the environment
 * lowers that cap), each pass an equal slice of every camera's samples; a camera's pixel sums run
 * on across the passes in sample order. */
typedef struct {
    lw_params params;      /* the camera's frame: camera, frame size, bounces, sky and sun settings */
    const float *sky;      /* the camera's sky buffer (HqFrame.sky) */
    uint64_t sky_len;
    uint32_t spp;          /* samples per pixel (at least 1) */
    uint32_t sample_start; /* first sample index (0 for a fresh frame) */
    float *out_rgb;        /* frame[0] * frame[1] * 3 floats, or NULL */
} lw_camera_job;
lw_status lw_batch_prepare(lw_ctx *ctx, const lw_camera_job *jobs, uint32_t n);
lw_status lw_batch_run(lw_ctx *ctx);
lw_status lw_batch_read(lw_ctx *ctx);
lw_status lw_render_batch(lw_ctx *ctx, const lw_camera_job *jobs, uint32_t n);

/* ---- allocation-free rendering ---------------------------------------------------------------
 * No counterpart in the reference. For callers that must not allocate device memory once they run
 * (an application that owns the GPU's memory budget, a per-frame loop that must not stall on
 * cudaMalloc/cudaFree): after lw_ctx_create, lw_scene_upload and lw_sky_upload (which allocate),
 * this adds samples [sample_start, sample_start + spp) of every pixel to `accum`, a device buffer
 * the caller owns of frame[0] * frame[1] records of 8 floats (Kahan sum r, g, b, sample count;
 * compensation r, g, b, unused; zero it before the first call), and allocates nothing: the
 * render kernel's work counter and item sums live in a fixed 32 MiB array inside the library.
 * The mean of a pixel is (sum - compensation) / count. Frames of more than 2,097,152 pixel slots
 * (8x4-pixel tiles, about 1920x1088) are refused with LW_ERR_INVALID_ARGUMENT, and so is an `accum`
 * that is not device (or managed) memory of the context's GPU. The work is queued on the context's
 * stream (lw_stream) and the call returns without waiting for the GPU (an earlier lw_cancel's
 * write is waited for on the device, not on the host). Every call on every
 * context of a device shares the one array: calls whose work overlaps on the GPU (from several
 * threads, contexts or streams) race on it and must be serialised by the caller. The first call on
 * a device looks the array's address up (cudaGetSymbolAddress); make that first call before any
 * stream capture. */
lw_status lw_render_accumulate_noalloc(lw_ctx *ctx, const lw_params *params, uint32_t sample_start, uint32_t spp,
                                       void *accum);

/* ---- parity entry points (the reference's kernel functions, one call per query) ----------
 * Per-sample radiance of `render_sample` (crates/lumenwright-kernel/src/integrator.rs:539-709)
 * for samples [sample_start, sample_start + count) of every pixel of the rectangle
 * [x0, x0+w) x [y0, y0+h): out[((py*w + px) * count + k) * 3 + c]. */
lw_status lw_render_samples(lw_ctx *ctx, const lw_params *params, uint32_t x0, uint32_t y0, uint32_t w,
                            uint32_t h, uint32_t sample_start, uint32_t count, float *out);
/* `trace` (crates/lumenwright-kernel/src/trace.rs:137-290) for n rays: o, d are 3n floats. */
lw_status lw_trace_rays(lw_ctx *ctx, const lw_params *params, uint32_t n, const float *o, const float *d,
                        float tmin, float tmax, lw_hit *out);
/* `SceneView::voxel` (crates/lumenwright-kernel/src/scene.rs:271-284) on the re-laid grid, for n
 * voxels given as 3n int32 coordinates. */
lw_status lw_voxel_lookup(lw_ctx *ctx, uint32_t n, const int32_t *xyz, uint32_t *out);

/* The exponential the kernels apply in the water's Beer-Lambert transmittance, exp(-sigma * t)
 * (`transmittance`, crates/lumenwright-kernel/src/math.rs:300), for n arguments: exp(x[i]) rounded
 * to the nearest f32 (the project's own correctly rounded exponential, which the CPU oracle calls
 * too), in out[i]. */
lw_status lw_water_exp(lw_ctx *ctx, uint64_t n, const float *x, float *out);

/* ---- sky precompute on the device -----------------------------------------------------------
 * Chunky's sky cache for the sky in `params` (sky_sun, sky_zenith, perez_a..e) at resolution n:
 * `build_sky_cache` (crates/lumenwright-kernel/src/integrator.rs:133-148), which the reference
 * runs on the host per frame (crates/lumenwright/src/render/sky.rs:593-611). Writes (n+1)^2 * 3
 * floats to `out`. */
lw_status lw_build_sky_cache(lw_ctx *ctx, const lw_params *params, uint32_t n, float *out);
/* `blend_chunky_sky` (crates/lumenwright/src/render/sky.rs:836-850): mixes Chunky's sky, read
 * through `cache` at params->misc_f[2] as the kernel reads it, into the lens map then the light
 * map in `maps` (sizes lens w, h, light w, h), in place: weight * chunky + (1 - weight) * map. */
lw_status lw_blend_chunky_sky(lw_ctx *ctx, const lw_params *params, const float *cache, uint64_t cache_len,
                              float *maps, const float sizes[4], float weight);

/* The game's sky (SkyLook::Game, or a day weight below 1): the client's sky drawn into the two
 * equirectangular maps the kernel's `sky_lens` / `sky_light` read (crates/lumenwright/src/render/
 * sky.rs:855-952), which the reference draws on the host per frame. `lw_quick_sky` is `QuickSky`
 * (sky.rs:274-305), 608 bytes, as `QuickSky::new` packs it (its camera fields are not read). */
typedef struct {
    float sky_color[4], fog_color[4], fog_dist[4], sunrise[4], flags[4];
    float sun[4][4], moon[4][4], star_rot[3][4], fan[18][4];
    float cam_forward[4], cam_right[4], cam_up[4], cam_misc[4];
} lw_quick_sky;
/* `draw_map` (sky.rs:861-878): `QuickSky::background` (sky.rs:509-530: the fog colour, the sky
 * disc, the sunrise glow, the sun and moon sprites from `atlas`, the stars of `stars`, the table
 * `star_table` builds, sky.rs:158-217) for the direction of every texel of a w x h map (row 0 at
 * the nadir, `map_direction`, sky.rs:853-858), decoded to linear with c^2.2, into out (w * h * 3
 * floats). `atlas` is atlas_len RGBA8 texels, atlas_w a row; the sun's and moon's rectangles must
 * lie inside it. */
lw_status lw_draw_sky_map(lw_ctx *ctx, const lw_quick_sky *sky, const uint32_t *stars, uint64_t stars_len,
                          const uint32_t *atlas, uint64_t atlas_len, uint32_t atlas_w, uint32_t w, uint32_t h,
                          float *out);

/* ---- the display pass ---------------------------------------------------------------------------
 * `post::tonemap` / `post::tonemap_mix` (crates/lumenwright/src/render/post.rs:152-217) on the
 * device: exposure, the operator, the display gamma v^(1/2.2) and the 8-bit rounding, packed as
 * RGBA8 with alpha 255 (byte 0 red). With mix = 0 it is tonemap(hdr, exposure, op); otherwise
 * tonemap_mix(hdr, exposure, op, op_b, weight), the two curves mixed in display values (the
 * reference's default for an hq frame: op = gamma, op_b = the game curve, weight = the day
 * weight, crates/lumenwright/src/request.rs:938-947). */
#define LW_TONEMAP_GAMMA 0u            /* Tonemap::Gamma */
#define LW_TONEMAP_ACES 1u             /* Tonemap::Aces */
#define LW_TONEMAP_FILMIC 2u           /* Tonemap::Filmic (Chunky's Hable preset FILMIC_WORLDS) */
#define LW_TONEMAP_FILMIC_MID_GREY 3u  /* Tonemap::FilmicMidGrey (the game's curve) */
typedef struct {
    float exposure;
    uint32_t op;
    uint32_t mix;
    uint32_t op_b;
    float weight;
} lw_tonemap;
/* The display bytes of n linear RGB values (3n floats) into out_rgba (n words). */
lw_status lw_tonemap_rgba(lw_ctx *ctx, const float *hdr, uint64_t n, const lw_tonemap *tm, uint32_t *out_rgba);
/* The last render's mean radiance (the accumulator of lw_render_hq / lw_render_device) tone-mapped
 * in the same pass that divides the sums, read back as frame[0] * frame[1] words; the linear means
 * are read too when out_rgb is not NULL. Waits for the render. */
lw_status lw_read_accumulator_rgba(lw_ctx *ctx, const lw_tonemap *tm, uint32_t *out_rgba, float *out_rgb);

/* ---- the differentiable form ------------------------------------------------------------------
 * No counterpart in the reference: the forward/backward pair of an image loss's gradient with
 * respect to parameters theta of an hq frame on the uploaded scene. theta is
 *   - a linear RGB albedo per texel parameter, replacing gamma_to_linear of the texel's bytes
 *     (crates/lumenwright-kernel/src/integrator.rs:27-34, :634) for every atlas texel mapped to it,
 *   - an intensity per emitter group (LW_EMITTER_GROUPS groups, a hash of the emitting block's
 *     voxel) multiplying the emitter intensity params->misc_f[0],
 *   - the frame's sun direction (params->sun_dir) and sky buffer, which the caller derives from a
 *     sun azimuth, altitude and turbidity.
 * At the decoded albedos, unit group intensities and the frame's own sky the forward image is
 * lw_render_hq's. The adjoint replays each sample's path (path replay backpropagation) with the
 * Russian roulette probability detached; visibility changes have no interior derivative and
 * their boundary terms are not estimated. Sums are FP64. */
#define LW_EMITTER_GROUPS 32
typedef struct {
    const lw_params *params;      /* the frame under theta */
    const float *sky;             /* its sky buffer under theta (the Chunky cache, or game-sky maps) */
    uint64_t sky_len;
    const float *albedo;          /* n_params * 3 linear RGB albedos */
    uint32_t n_params;
    const int32_t *texel_param;   /* one per atlas texel: its parameter, or -1 to decode the texel */
    uint64_t texel_param_len;     /* the atlas's texel count */
    const float *emitter_scale;   /* LW_EMITTER_GROUPS group intensities */
} lw_adj_frame;

/* d loss / d theta. */
typedef struct {
    double *albedo;        /* n_params * 3 */
    double *emitter_scale; /* LW_EMITTER_GROUPS */
    double *sky;           /* sky_len: per sky float (the Chunky cache's entries; zeros for game-sky maps) */
    double sun_dir[3];     /* per component of params->sun_dir, through the sun's next-event estimates */
} lw_gradient;

/* The mean radiance per pixel of samples [0, spp) under theta, FP64, frame[0] * frame[1] * 3. */
lw_status lw_adjoint_forward(lw_ctx *ctx, const lw_adj_frame *frame, uint32_t spp, double *out_rgb);
/* The gradient of a loss whose derivative with respect to the forward image is `d_rgb`
 * (frame[0] * frame[1] * 3 doubles), over the same samples; overwrites `out`. Called after
 * lw_adjoint_forward with the same inputs (params, sky, theta, spp: compared by a digest of their
 * bytes), it reads each sample's radiance the forward pass kept on the device (up to 4 GiB of
 * them) instead of replaying every path a first time. */
lw_status lw_adjoint_backward(lw_ctx *ctx, const lw_adj_frame *frame, uint32_t spp, const double *d_rgb,
                              lw_gradient *out);
/* Paired finite differences: every sample under `plus` and under `minus` (same size, same
 * parameter count), with the roulette's probabilities and decisions of the `nominal` albedos and
 * the shadow rays along nominal->params->sun_dir; writes per pixel the mean of the paired
 * differences (plus - minus) and of the pairs' midpoints. */
lw_status lw_adjoint_fd(lw_ctx *ctx, const lw_adj_frame *plus, const lw_adj_frame *minus, const lw_adj_frame *nominal,
                        uint32_t spp, double *diff_rgb, double *mean_rgb);
/* Chunk-origin rebasing of a frame's camera, on the host, in f64: the eye (relative to the grid
 * origin, as request.rs:640-644 rebases it from the world) is split into the chunk corner nearest
 * it, 16 * rint(eye / 16) per axis, and the remainder, at most 8 blocks on each axis, which is
 * rounded once to f32 into params->cam_pos.xyz; see_through[2] and [3] are set as `lw_params`
 * describes. The kernels then hold each path origin relative to its own nearest chunk corner,
 * moving between corners by exact integer offsets. LW_ERR_INVALID_ARGUMENT for a non-finite eye
 * or one whose chunk is outside the packed range (x and z within +-1024 chunks, y +-512). No GPU
 * is used. */
lw_status lw_rebase_camera(lw_params *params, const double eye[3]);

/* The byte-to-linear table the kernels decode texels with: gamma_to_linear(k / 255) for k in
 * 0..255 (crates/lumenwright-kernel/src/math.rs:183-216), so a caller can form nominal albedos. */
lw_status lw_gamma_table(float out[256]);

#ifdef __cplusplus
}
#endif
#endif
