// Declarations shared by the library's translation units (not part of the C ABI).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "device_scene.cuh"

namespace lw {

// One render launch: samples [sample_start, sample_start + spp) of every pixel of the rectangle
// [x0, x0+w) x [y0, y0+h), cut into items of `sub` consecutive samples of one pixel.
struct WorkDesc {
    uint32_t x0, y0, w, h;       // the rectangle
    uint32_t tiles_x;            // 8x4-pixel tiles per rectangle row
    uint32_t tile_step, tile_first;  // the launch's tiles: tile_first, tile_first + tile_step, ...
                                     // (one shard of a frame split over GPUs; 1, 0 for all tiles)
    uint32_t n_slots;            // pixel slots: the launch's tiles * 32
    uint32_t sample_start, spp;  // the launch's samples
    uint32_t sub;                // samples per item
    uint32_t n_sub;              // items per pixel: ceil(spp / sub)
    uint32_t n_items;            // n_slots * n_sub
    uint32_t budget;             // voxel visits per ray per loop iteration (0: no limit)
    uint32_t *counter;           // work counter (zeroed before the launch)
    float4 *partials;            // [n_sub][n_slots] compensated item sums (accumulating mode)
    float *samples_out;          // per-sample radiance (sample mode), [(py*w+px)*spp + k][3]
    const volatile uint32_t *cancel;  // device cancel word: the kernel stops taking items when set
};

// Per-pixel accumulator: Kahan (sum, compensation), with the sample count in sum.w.
struct __align__(16) Accum {
    float4 sum;
    float4 comp;
};

enum { MODE_ACCUM = 0, MODE_SAMPLES = 1 };

// One camera of the batched form: its frame, its sky, where its items, sums and image live.
struct __align__(16) DevJob {
    DevParams P;
    const float *sky;
    Accum *acc;
    float *out;             // its image, w * h * 3 floats
    uint64_t partial_off;   // first item sum of the camera in the batch's partial sums
    uint32_t item_begin;    // first item of the camera in the batch's queue
    uint32_t slot_begin;    // first pixel slot of the camera among all cameras' slots
    uint32_t w, h, tiles_x, n_slots, sample_start, spp, sub, n_sub;
};

struct BatchDesc {
    const DevJob *jobs;
    const uint32_t *item_begin;  // the jobs' item_begin, ascending (for the binary search)
    const uint32_t *slot_begin;  // the jobs' slot_begin, ascending
    uint32_t n_jobs, n_items, n_slots;
    uint32_t budget;  // regrouping period (0: whole traversals)
    uint32_t *counter;
    float4 *partials;
    const volatile uint32_t *cancel;
};

struct LaunchShape {
    int blocks, threads;
};

// render.cu
cudaError_t launch_render(int mode, const DevScene &S, const DevParams &P, const WorkDesc &W, LaunchShape shape,
                          cudaStream_t st);
LaunchShape render_shape(int mode, int device, int threads);
cudaError_t launch_reduce(const WorkDesc &W, Accum *acc, uint32_t frame_w, cudaStream_t st);
cudaError_t launch_finalize(const Accum *acc, uint32_t n, float *out_rgb, cudaStream_t st);
cudaError_t launch_trace_rays(const DevScene &S, const DevParams &P, uint32_t n, const float *o, const float *d,
                              float tmin, float tmax, void *out_hits, cudaStream_t st);
cudaError_t launch_voxel_lookup(const DevScene &S, const DevParams &P, uint32_t n, const int32_t *xyz, uint32_t *out,
                                cudaStream_t st);
cudaError_t launch_water_exp(uint64_t n, const float *x, float *out, cudaStream_t st);

// sky.cu
cudaError_t launch_sky_cache(const DevParams &P, uint32_t n, float *out, cudaStream_t st);
cudaError_t launch_blend_chunky(const DevScene &S, const DevParams &P, float *map, uint32_t w, uint32_t h, float weight,
                                cudaStream_t st);
cudaError_t launch_sky_map(const void *quick_sky, const uint32_t *atlas, uint32_t atlas_w, const uint32_t *stars,
                           uint32_t w, uint32_t h, float *out, cudaStream_t st);

// batch.cu
LaunchShape batch_shape(int device, int threads, bool resume);
cudaError_t launch_render_batch(const DevScene &S, const BatchDesc &B, LaunchShape shape, cudaStream_t st);
cudaError_t launch_reduce_batch(const BatchDesc &B, cudaStream_t st);

// wavefront.cu: the render as shade / trace iterations over a pool of path slots.
constexpr int kWfWords = 16;
struct WfState {
    float4 *state;    // kWfWords float4 per slot, word k of slot i at state[k * n + i]
    uint32_t n;       // slots
    uint32_t *queue;  // 3 sets of n slot ids: the rays of iterations t % 3
    float4 *hit0;     // per slot: t, quad, texel, s of its last ray
    float *hit1;      // per slot: tt
    uint32_t *ctr;    // per queue set s: [4s] its length, [4s + 1] the trace fetch counter; [12]: the
                      // iteration; [14..15]: rays traced (64-bit, 8-byte aligned)
    float4 *ts;       // 3 float4 per slot (word k at ts[k * n + i]): a carried-over traversal
    uint32_t *frame;  // per slot: the frame word of its path (chunk-origin rebasing only)
};
// The path slots' word with an item's camera in the batched form (j, pixel slot, camera, -), which
// the batched form clears with the core word before a pass: a slot that has not taken an item yet
// then names camera 0, so the shading kernel reads the camera table within its bounds.
constexpr int kWfItemCameraWord = 13;
// Visits through empty space per round of the wavefront's tracing kernel when the tuning leaves it
// at 0: 8, since cells without quads count as air (a 256-spp C2 frame traced in 118.0, 115.4, 114.0,
// 113.3 and 114.0 ms at 4, 5, 6, 8 and 10; the 8-spp C5 frame in 90.0 at 5 and 87.7 at 8).
constexpr uint32_t kWfBudget = 8u;
#ifndef LW_SHADE_THREADS
#define LW_SHADE_THREADS 256
#endif
// Threads per block of the shading kernel (256: shading -2.6 % against 128 at c2; 64 is slower).
constexpr uint32_t kShadeThreads = LW_SHADE_THREADS;
// The tracing kernel can stage the scene's top level and occupancy masks in shared memory, per
// block, when they take at most LW_TRACE_STAGE_MAX bytes. Off (0) by default: the tables stay in
// L1 anyway, and staged the c2 frame's tracing took 147.2 ms a 256-spp frame against 124.8 (29 KB
// a block leaves 7 blocks a SM instead of 8), the c4 frame's 19.3 against 19.0 (same occupancy).
#ifndef LW_TRACE_STAGE_MAX
#define LW_TRACE_STAGE_MAX 0
#endif
// The persistent tracing kernel's grid: its resident blocks per SM x the SMs (reb: the form with
// chunk-origin rebasing).
LaunchShape wf_trace_shape(int device, size_t stage_bytes = 0, bool reb = false);
cudaError_t launch_wf_shade(const DevScene &S, const DevParams &P, const WorkDesc &W, const WfState &F, uint32_t blocks,
                            cudaStream_t st);
cudaError_t launch_wf_shade_batch(const DevScene &S, const DevParams &P0, const BatchDesc &B, const WfState &F,
                                  uint32_t blocks, cudaStream_t st);
cudaError_t launch_wf_trace(const DevScene &S, const DevParams &P, const WfState &F, LaunchShape trace_shape,
                            uint32_t budget, uint32_t tail, size_t stage_bytes, cudaStream_t st);
cudaError_t launch_wf_advance(const WfState &F, cudaStream_t st);
cudaError_t launch_wf_advance_graph(const WfState &F, cudaGraphConditionalHandle loop, cudaStream_t st);

// build.cu: the hq grid build on the device.
struct BuildVol {
    const uint16_t *blocks;  // voxel states, (y * size_z + z) * size_x + x
    uint32_t size[3];        // x, y, z in voxels
    const uint8_t *flags;    // per state: 1 occludes, 2 invisible, 4 fluid
    uint32_t n_states;
    uint32_t *error;         // bit 0: a voxel names a state out of range
};
cudaError_t launch_keys_first(const BuildVol &v, uint32_t *keys, uint32_t *first, cudaStream_t st);
cudaError_t launch_bricks_scan(const BuildVol &v, const uint32_t *keys, const uint32_t *key_id, const uint8_t *model_emits,
                               uint16_t *ids, uint4 *cls, uint32_t nb, cudaStream_t st);
cudaError_t launch_bricks_pack(const BuildVol &v, const uint16_t *ids, const uint8_t *model_emits, const uint32_t *slot,
                               const uint32_t *emit_off, uint32_t *brick_words, uint4 *sites, uint32_t nb, cudaStream_t st);

// post.cu: the display pass (tone mapping to RGBA8).
struct ToneCurve {  // a Hable curve as HableCurve::h reads it: f32 products widened, and 1 / h(W)
    double a, b, cb, de, df, ef, white;
};
struct TonemapDesc {
    float exposure;
    uint32_t op_a, op_b, mix;  // operators (0 gamma, 1 ACES, 2 Hable preset, 3 game curve); mix: tonemap_mix
    float weight;              // the mix weight of op_a
    float inv_gamma;           // 1 / 2.2 in f32
    ToneCurve preset, game;
};
cudaError_t launch_finalize_tonemap(const Accum *acc, uint32_t n, const TonemapDesc &t, uint32_t *rgba, float *hdr,
                                    cudaStream_t st);
cudaError_t launch_tonemap(const float *hdr, uint32_t n, const TonemapDesc &t, uint32_t *rgba, cudaStream_t st);

// adjoint.cu: the differentiable form.
#define LW_ADJ_EMITTER_GROUPS 32
struct AdjFrame {
    DevParams P;                 // the frame with this theta's sun and sky
    const float *sky;            // the sky buffer of this theta
    const float *albedo;         // [params][3] linear albedo per texel parameter
    const int32_t *texel_param;  // per atlas texel: its parameter, or -1 (the decoded texel)
    const float *emit_mult;      // [LW_ADJ_EMITTER_GROUPS] emitter group intensities
};
struct AdjGrad {
    double *albedo;  // [params][3]
    double *emit;    // [LW_ADJ_EMITTER_GROUPS]
    double *cache;   // one per sky float
    double *sun;     // [3]: d / d sun_dir.xyz
};
// Ls: per-sample radiance, 3 doubles per sample at [pixel * spp + sample] (kept by the forward
// pass, read by the backward pass in place of its first replay), or null.
cudaError_t launch_adj_forward(const DevScene &S, const AdjFrame &F, uint32_t spp, double *img, double *Ls,
                               cudaStream_t st);
cudaError_t launch_adj_backward(const DevScene &S, const AdjFrame &F, uint32_t spp, const double *d_img,
                                const AdjGrad &G, const double *Ls, cudaStream_t st);
cudaError_t launch_adj_fd(const DevScene &S, const AdjFrame &plus, const AdjFrame &minus, const float *albedo0,
                          float4 sun0, uint32_t spp, double *diff, double *mean, cudaStream_t st);

// noalloc.cu: the fixed scratch array of the allocation-free entry point.
extern const size_t kNoallocPartials;
cudaError_t noalloc_scratch(int device, float4 **out);

// scene.cu
struct SceneUploadDesc {
    const uint32_t *grid;  // device copy of the reference grid
    uint32_t nb, n_bricks, off_top, off_bricks, off_ov_top;
    uint32_t n_models, n_ov_bricks;
    const uint4 *models;   // device copy of the models (quad offset, quad count, flags, -)
    uint2 *top;
    uint16_t *bricks;
    uint2 *occ;
    uint32_t *error;  // device error word: bit 0 a top entry out of range, bit 1 a voxel id out of range
};
cudaError_t launch_relayout(const SceneUploadDesc &d, cudaStream_t st);
cudaError_t launch_quads(const void *ref_quads, DevQuad *out, uint32_t n, cudaStream_t st);

}  // namespace lw
