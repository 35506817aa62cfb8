// The C ABI (include/lumenwright_b200.h): contexts, scene upload and validation, the render
// loop that replaces CudaBackend::render_hq (crates/lumenwright/src/render/cuda.rs:77-184), and
// the parity entry points.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/lumenwright_b200.h"
#include "internal.h"

using namespace lw;

static_assert(sizeof(lw_params) == sizeof(DevParams), "Params layout");
static_assert(sizeof(lw_quad) == 80 && sizeof(lw_model) == 16 && sizeof(lw_emitter) == 32, "record layout");
static_assert(sizeof(lw_quick_sky) == 608, "QuickSky layout");

// The item sums a launch may fill (16 B each): 16 GiB, or a quarter of the device memory free when
// the context is made if that is less. One launch then covers the 1024-spp C2 frame (15.1 GB of
// one-sample items), which in four launches of the 4 GiB cap before took 2.1 % longer (808.0 ms
// against 791.6: each launch ends in a drain of the path pool).
#ifndef LW_PARTIALS_CAP_GIB
#define LW_PARTIALS_CAP_GIB 16
#endif
namespace {

thread_local std::string g_create_error;

template <typename T>
struct DBuf {
    T *p = nullptr;
    size_t n = 0;  // elements allocated
    void free_() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

// The reference's `gamma_to_linear` (crates/lumenwright-kernel/src/math.rs:183-216), exp(2.2 ln c)
// with its own f32 `ln` and the platform expf, evaluated once per byte value on the host.
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
    float s = (m - 1.0f) / (m + 1.0f);
    float s2 = s * s;
    float series = 2.0f * s * (1.0f + s2 * (1.0f / 3.0f + s2 * (1.0f / 5.0f + s2 * (1.0f / 7.0f + s2 * (1.0f / 9.0f)))));
    return (float)e * 0.693147180559945309417f + series;
}
float ref_gamma_to_linear(float c) { return c <= 0.0f ? 0.0f : expf(2.2f * ref_ln(c)); }

}  // namespace

struct lw_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    LaunchShape shape_accum{}, shape_samples{};
    cudaEvent_t ev_a = nullptr, ev_b = nullptr;
    cudaEvent_t marks[8] = {};
    // scene
    bool has_scene = false;
    uint32_t dims[3] = {}, offsets[5] = {}, atlas_size[2] = {};
    uint32_t sky_brick_y = 0;  // DevScene::sky_brick_y of the uploaded scene
    uint32_t nb = 0, n_bricks = 0, n_ov_bricks = 0;
    DBuf<uint32_t> grid, atlas, egrid;
    DBuf<uint2> top, occ;
    DBuf<uint16_t> bricks;
    DBuf<uint4> models;
    DBuf<DevQuad> quads;
    DBuf<float4> emitters;
    DBuf<uint8_t> ref_quads;  // the reference's 80-byte quads, re-laid into `quads` at upload
    uint64_t grid_len = 0, models_len = 0, quads_len = 0, atlas_len = 0, emitters_len = 0, egrid_len = 0;
    // frame
    DBuf<float> sky, gamma, out_rgb;
    DBuf<uint32_t> out_rgba;
    uint64_t sky_len = 0;
    DBuf<Accum> acc;
    uint32_t acc_w = 0, acc_h = 0;
    DBuf<float4> partials;
    DBuf<uint32_t> counter, error;
    DBuf<float> samples;
    DBuf<float> rays;
    DBuf<uint8_t> hits;
    DBuf<int32_t> xyz;
    DBuf<uint32_t> vox;
    int *cancel_host = nullptr;      // host flag, read between launches
    DBuf<uint32_t> cancel_word;      // device word the render kernel polls; set by lw_cancel
    cudaStream_t aux = nullptr;      // lw_cancel's stream, so the write lands while a render runs
    cudaEvent_t cancel_ev = nullptr; // recorded on `aux` after each cancel's write
    double timeout_s = 0.0;          // deadline of every wait on the render's work (0: none)
    cudaEvent_t wait_ev = nullptr;   // marks the work a bounded wait waits for
    cudaStream_t cap = nullptr;      // the stream a graph's loop body is captured on
    lw_stats stats{};
    lw_tuning tuning{128, 0, 0, LW_ENGINE_WAVEFRONT, 0};
    // the batched form
    struct BatchSky { const float *host; uint64_t len; DBuf<float> dev; };
    std::vector<BatchSky *> batch_skies;
    DBuf<DevJob> batch_jobs;
    DBuf<uint32_t> batch_item_begin, batch_slot_begin;
    DBuf<Accum> batch_acc;
    DBuf<float> batch_out;
    DBuf<float4> batch_partials;
    std::vector<lw_camera_job> batch_host;
    std::vector<size_t> batch_out_off;
    cudaGraphExec_t batch_graph = nullptr;
    uint64_t batch_samples = 0;
    uint32_t batch_passes = 1;  // passes of the prepared batch (the wavefront's one-sample items)
    size_t partials_cap_bytes = size_t(LW_PARTIALS_CAP_GIB) << 30;
    // the wavefront engine: path slots (grown to the largest pool used), queue fetch settings
#ifndef LW_WF_TAIL
#define LW_WF_TAIL 12
#endif
    uint32_t wf_tail = LW_WF_TAIL;
    // kernel_ms of the launches already timed when the last one is still running (stats.kernel_ms
    // is then -1 until lw_get_stats adds the last launch's event time)
    double kernel_ms_base = 0.0;
    LaunchShape shape_wf{};        // the tracing kernel reading the scene from global memory
    LaunchShape shape_wf_reb{};    // ... with chunk-origin rebasing
    LaunchShape shape_wf_staged{}; // ... and staging it in shared memory (stage_bytes of it)
    size_t stage_bytes = 0;
    struct WfBufs {
        DBuf<float4> state, hit0, ts;
        DBuf<float> hit1;
        DBuf<uint32_t> queue, ctr, frame;
        void free_() {
            frame.free_();
            state.free_();
            hit0.free_();
            ts.free_();
            hit1.free_();
            queue.free_();
            ctr.free_();
        }
    };
    WfBufs wf, bwf;  // the single-frame renders' pool; the batch graph's own (its pointers are baked in)
    uint32_t *wf_host = nullptr;  // pinned word the iteration count is read into
    cudaEvent_t wf_ev[48] = {};   // per iteration of a 16-iteration window: before shade, between, after trace
    // the grid build on the device
    DBuf<uint16_t> bv_blocks, bv_ids;
    DBuf<uint8_t> bv_flags, bv_emits;
    DBuf<uint32_t> bv_keys, bv_first, bv_key_id, bv_slot, bv_emit_off;
    DBuf<uint4> bv_cls, bv_sites;
    std::vector<uint32_t> bv_order;  // the keys of the last lw_scene_build_keys, in interning order
    uint32_t bv_size[3] = {}, bv_states = 0;
    // the differentiable form: per frame slot (0 and 1: the frames, 2: the nominal frame)
    DBuf<float> adj_albedo[3], adj_sky[3], adj_emit[3];
    DBuf<int32_t> adj_tparam[3];
    DBuf<double> adj_img, adj_img2, adj_g, adj_L;
    uint64_t adj_L_key = 0;  // the inputs the kept per-sample radiance belongs to (0: none)
};

namespace {

lw_status fail(lw_ctx *c, lw_status s, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    else g_create_error = buf;
    return s;
}

lw_status cuda_fail(lw_ctx *c, cudaError_t e, const char *what) {
    lw_status s = e == cudaErrorMemoryAllocation ? LW_ERR_OUT_OF_MEMORY : LW_ERR_LAUNCH;
    return fail(c, s, "%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
}

#define CK(c, call, what)                                  \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return cuda_fail(c, e_, what); \
    } while (0)

// The start of a render: clears the cancel flag and the device cancel word. lw_cancel writes the
// word on its own stream, so the clear is ordered after the write of every cancel made before
// this call (the render's stream waits for the event recorded after it, on the device; the host
// does not wait): landing after the clear, such a write would stop this render's kernels unseen.
lw_status begin_render(lw_ctx *c) {
    CK(c, cudaStreamWaitEvent(c->stream, c->cancel_ev, 0), "ordering after an earlier cancel");
    __atomic_store_n(c->cancel_host, 0, __ATOMIC_RELAXED);
    CK(c, cudaMemsetAsync(c->cancel_word.p, 0, 4, c->stream), "clearing the cancel word");
    return LW_OK;
}

// The device half of lw_cancel: the cancel word on the aux stream, which the render kernels poll.
void cancel_device(lw_ctx *c) {
    __atomic_store_n(c->cancel_host, 1, __ATOMIC_RELAXED);
    cudaMemsetAsync(c->cancel_word.p, 0xFF, 4, c->aux);  // lands while a render kernel runs
    cudaEventRecord(c->cancel_ev, c->aux);               // the next render's clear waits for it
}

// How long a wait that ran out gives the cancelled kernels to end before it returns anyway.
constexpr double kDrainSeconds = 10.0;

// Waits for event `ev`. With a deadline set (lw_set_timeout) the wait is a poll of the event
// against it: spinning briefly, then sleeping 50 us between polls. If the deadline passes first,
// the render's kernels are cancelled (they stop taking work at their next poll of the cancel
// word), the wait goes on for at most kDrainSeconds more for them to end, and the call returns
// LW_ERR_DEVICE_TIMEOUT; the results of the render are then incomplete.
lw_status wait_event(lw_ctx *c, cudaEvent_t ev, const char *what) {
    if (c->timeout_s <= 0.0) {
        CK(c, cudaEventSynchronize(ev), what);
        return LW_OK;
    }
    using clock = std::chrono::steady_clock;
    const auto deadline = clock::now() + std::chrono::duration<double>(c->timeout_s);
    for (unsigned polls = 0;; polls++) {
        cudaError_t e = cudaEventQuery(ev);
        if (e == cudaSuccess) return LW_OK;
        if (e != cudaErrorNotReady) return cuda_fail(c, e, what);
        if (clock::now() >= deadline) break;
        if (polls < 64) std::this_thread::yield();
        else std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
    cancel_device(c);
    const auto drain = clock::now() + std::chrono::duration<double>(kDrainSeconds);
    cudaError_t e = cudaEventQuery(ev);
    while (e == cudaErrorNotReady && clock::now() < drain) {
        std::this_thread::sleep_for(std::chrono::milliseconds(1));
        e = cudaEventQuery(ev);
    }
    if (e != cudaSuccess && e != cudaErrorNotReady) return cuda_fail(c, e, what);
    return fail(c, LW_ERR_DEVICE_TIMEOUT, "%s: not done within the %.6g s deadline; %s", what, c->timeout_s,
                e == cudaSuccess ? "its kernels were stopped and have ended"
                                 : "its kernels were asked to stop and had not ended 10 s later");
}

// Waits for the work queued on the context's stream so far (see wait_event).
lw_status wait_stream(lw_ctx *c, const char *what) {
    CK(c, cudaEventRecord(c->wait_ev, c->stream), "recording an event");
    return wait_event(c, c->wait_ev, what);
}

#define WAIT(c, what)                                \
    do {                                             \
        lw_status ws_ = wait_stream((c), (what));    \
        if (ws_ != LW_OK) return ws_;                \
    } while (0)

// After the wait for a render's results: a cancel that came while the kernels ran (after the last
// check between launches) may have stopped them before the last sample, so the results are
// incomplete and the call reports the cancel.
lw_status check_cancelled(lw_ctx *c) {
    if (__atomic_load_n(c->cancel_host, __ATOMIC_RELAXED))
        return fail(c, LW_ERR_CANCELLED, "cancelled: the render may have stopped before its last sample");
    return LW_OK;
}

template <typename T>
cudaError_t ensure(DBuf<T> &b, size_t n) {
    if (n == 0) n = 1;
    if (b.n >= n) return cudaSuccess;
    b.free_();
    cudaError_t e = cudaMalloc(&b.p, n * sizeof(T));
    if (e == cudaSuccess) b.n = n;
    else b.p = nullptr;
    return e;
}

template <typename T>
cudaError_t upload(lw_ctx *c, DBuf<T> &b, const void *src, size_t n_elems, size_t elem_bytes) {
    size_t bytes = n_elems * elem_bytes;
    cudaError_t e = ensure(b, (bytes + sizeof(T) - 1) / sizeof(T));
    if (e != cudaSuccess || bytes == 0) return e;
    return cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, c->stream);
}

DevScene dev_scene(const lw_ctx *c) {
    DevScene S;
    S.top = c->top.p;
    S.bricks = c->bricks.p;
    S.occ = c->occ.p;
    S.grid = c->grid.p;
    S.models = c->models.p;
    S.quads = c->quads.p;
    S.atlas = c->atlas.p;
    S.emitters = c->emitters.p;
    S.emitter_grid = c->egrid.p;
    S.sky = c->sky.p;
    S.gamma = c->gamma.p;
    S.sky_brick_y = c->sky_brick_y;
    S.n_top = c->nb;
    S.n_occ = c->n_bricks;
    return S;
}

// Checks a frame's Params against the uploaded scene and sky: every index the kernels form from
// them stays inside its buffer.
lw_status check_params(lw_ctx *c, const lw_params *p, bool need_frame, uint64_t sky_len = UINT64_MAX) {
    if (sky_len == UINT64_MAX) sky_len = c->sky_len;
    if (!p) return fail(c, LW_ERR_INVALID_ARGUMENT, "params is null");
    if (!c->has_scene) return fail(c, LW_ERR_NO_SCENE, "no scene uploaded");
    for (int a = 0; a < 3; a++)
        if (p->grid_dims[a] != c->dims[a])
            return fail(c, LW_ERR_INVALID_ARGUMENT, "params.grid_dims[%d] = %u, the scene has %u", a, p->grid_dims[a], c->dims[a]);
    for (int a = 0; a < 4; a++)
        if (p->off[a] != c->offsets[a])
            return fail(c, LW_ERR_INVALID_ARGUMENT, "params.off[%d] = %u, the scene has %u", a, p->off[a], c->offsets[a]);
    if (p->off2[0] != c->offsets[4] || p->off2[1] != c->atlas_size[0] || p->off2[2] != c->atlas_size[1])
        return fail(c, LW_ERR_INVALID_ARGUMENT, "params.off2 does not match the scene (ov_quads offset, atlas size)");
    if (need_frame && (p->frame[0] == 0 || p->frame[1] == 0))
        return fail(c, LW_ERR_INVALID_ARGUMENT, "frame size %ux%u", p->frame[0], p->frame[1]);
    if (p->see_through[2] > 1u)
        return fail(c, LW_ERR_INVALID_ARGUMENT, "params.see_through[2] = %u: the origin frames are 0 (the grid's) or 1 (chunk "
                    "corners)", p->see_through[2]);
    if ((uint64_t)p->see_through[0] + p->see_through[1] > c->quads_len)
        return fail(c, LW_ERR_BUFFER_LENGTH, "see-through quads [%u, +%u) outside %llu quads", p->see_through[0],
                    p->see_through[1], (unsigned long long)c->quads_len);
    if (p->sky_map[0] >= 1.0f) {
        double lens = (double)(uint64_t)p->sky_map[0] * (uint64_t)p->sky_map[1];
        double light = (double)(uint64_t)p->sky_map[2] * (uint64_t)p->sky_map[3];
        if (!(p->sky_map[1] >= 1.0f && p->sky_map[2] >= 1.0f && p->sky_map[3] >= 1.0f) ||
            (lens + light) * 3.0 > (double)sky_len || p->sky_map[0] * p->sky_map[1] >= 4294967040.0f)
            return fail(c, LW_ERR_BUFFER_LENGTH, "sky maps %gx%g + %gx%g need more than the %llu sky floats", p->sky_map[0],
                        p->sky_map[1], p->sky_map[2], p->sky_map[3], (unsigned long long)sky_len);
    } else if (p->misc_f[2] >= 1.0f) {
        double n = std::floor((double)p->misc_f[2]);
        if ((n + 1.0) * (n + 1.0) * 3.0 > (double)sky_len)
            return fail(c, LW_ERR_BUFFER_LENGTH, "sky cache of resolution %g needs %g floats, %llu given", n,
                        (n + 1.0) * (n + 1.0) * 3.0, (unsigned long long)sky_len);
    }
    return LW_OK;
}

DevParams dev_params(const lw_params *p) {
    DevParams d;
    std::memcpy(&d, p, sizeof d);
    return d;
}

// Splits [sample_start, sample_start + spp) over a rectangle into launches whose partial sums fit
// the context's buffer; `sub` samples per item, chosen so each lane gets many items.
struct Plan {
    uint32_t sub, batch;
};
Plan plan(const lw_ctx *c, uint64_t n_slots, uint32_t spp, uint32_t sub_override = 0) {
    uint64_t lanes = (uint64_t)c->shape_accum.blocks * c->shape_accum.threads;
    uint64_t total = n_slots * spp;
    uint64_t sub = total / (lanes * 16ull + 1ull);
    sub = sub < 1 ? 1 : (sub > 16 ? 16 : sub);
    if (sub_override) sub = sub_override;
    if (c->tuning.sub) sub = c->tuning.sub;
    uint64_t max_items = c->partials_cap_bytes / sizeof(float4);
    uint64_t max_sub_per_launch = max_items / (n_slots ? n_slots : 1);
    if (max_sub_per_launch < 1) max_sub_per_launch = 1;
    uint64_t batch = max_sub_per_launch * sub;
    if (batch > spp) batch = spp;
    return Plan{(uint32_t)sub, (uint32_t)batch};
}

// A launch over the rectangle's 8x4-pixel tiles shard, shard + shards, shard + 2 shards, ...
// (all of them for shard 0 of 1).
WorkDesc work(lw_ctx *c, uint32_t x0, uint32_t y0, uint32_t w, uint32_t h, uint32_t s0, uint32_t spp, uint32_t sub,
              uint32_t shard = 0, uint32_t shards = 1) {
    WorkDesc W{};
    W.x0 = x0;
    W.y0 = y0;
    W.w = w;
    W.h = h;
    W.tiles_x = (w + 7) / 8;
    uint32_t tiles_y = (h + 3) / 4;
    const uint32_t tiles = W.tiles_x * tiles_y;
    W.tile_step = shards;
    W.tile_first = shard;
    W.n_slots = (tiles > shard ? (tiles - shard + shards - 1) / shards : 0u) * 32u;
    W.sample_start = s0;
    W.spp = spp;
    W.sub = sub;
    W.n_sub = (spp + sub - 1) / sub;
    W.n_items = W.n_slots * W.n_sub;
    W.budget = c->tuning.budget;
    W.counter = c->counter.p;
    W.partials = c->partials.p;
    W.samples_out = c->samples.p;
    W.cancel = c->cancel_word.p;
    return W;
}

lw_status ensure_accum(lw_ctx *c, uint32_t w, uint32_t h) {
    CK(c, ensure(c->acc, (size_t)w * h), "allocating the accumulator");
    c->acc_w = w;
    c->acc_h = h;
    return LW_OK;
}

// The wavefront's pool of n path slots, its queue and counters, cleared on `st` for a new render.
lw_status wf_setup(lw_ctx *c, lw_ctx::WfBufs &b, uint32_t n, WfState &F, cudaStream_t st) {
    CK(c, ensure(b.state, (size_t)kWfWords * n), "allocating the path slots");
    CK(c, ensure(b.hit0, n), "allocating the hits");
    CK(c, ensure(b.ts, (size_t)3 * n), "allocating the carried traversals");
    CK(c, ensure(b.hit1, n), "allocating the hits");
    CK(c, ensure(b.queue, (size_t)3 * n), "allocating the ray queues");
    CK(c, ensure(b.frame, n), "allocating the path frames");
    CK(c, ensure(b.ctr, 16), "allocating the queue counters");
    if (!c->wf_host) CK(c, cudaMallocHost((void **)&c->wf_host, 4), "allocating a pinned word");
    F = WfState{b.state.p, n, b.queue.p, b.hit0.p, b.hit1.p, b.ctr.p, b.ts.p, b.frame.p};
    // the slots' core words (flags 0: no item yet), the counters and the iteration, the hits
    CK(c, cudaMemsetAsync(b.state.p + (size_t)4 * n, 0, (size_t)n * sizeof(float4), st), "clearing the slots");
    CK(c, cudaMemsetAsync(b.ctr.p, 0, 16 * sizeof(uint32_t), st), "clearing the queue counters");
    CK(c, cudaMemsetAsync(b.hit0.p, 0, (size_t)n * sizeof(float4), st), "clearing the hits");
    return LW_OK;
}

// Blocks of the shading kernel: one thread per slot.
uint32_t wf_shade_blocks(const lw_ctx *, uint32_t n) { return (n + kShadeThreads - 1u) / kShadeThreads; }

// Path slots for a render of `samples` samples in `items` work items: one per 16 samples, a power
// of two from 2^16 to 2^23, no more than the items (or the tuning's count).
uint32_t wf_slots(const lw_ctx *c, uint64_t samples, uint64_t items, uint32_t cap = 1u << 23) {
    if (c->tuning.paths) return c->tuning.paths;
    uint64_t want = samples / 16u;
    uint32_t n = 1u << 16;
    while (n < want && n < cap) n <<= 1;
    while (n > (1u << 10) && (n >> 1) >= items) n >>= 1;
    return n;
}

// The tone curves as post.rs computes them: Chunky's Hable preset FILMIC_WORLDS (post.rs:57-65),
// its white scale in f32 (:74-88), and the game's curve: the preset brightened (:113-120) by the gain
// that holds mid-grey 0.18 (:125-137).
struct HableF {
    float a, b, c, d, e, f, w;
};
float white_scale(const HableF &k) {
    float num = k.w * (k.a * k.w + k.c * k.b) + k.d * k.e;
    float den = k.w * (k.a * k.w + k.b) + k.d * k.f;
    return 1.0f / (num / den - k.e / k.f);
}
ToneCurve tone_curve(const HableF &k) {
    return ToneCurve{(double)k.a, (double)k.b, (double)(k.c * k.b), (double)(k.d * k.e), (double)(k.d * k.f),
                     (double)(k.e / k.f), (double)white_scale(k)};
}
double mid_grey_gain(const HableF &k, double m) {
    ToneCurve t = tone_curve(k);
    double q = m / (double)white_scale(k) + t.ef;
    double qa = t.a * (1.0 - q), qb = t.cb - q * t.b, qc = t.de - q * t.df;
    double y = (-qb + std::sqrt(qb * qb - 4.0 * qa * qc)) / (2.0 * qa);
    return y / (2.0 * m);
}
HableF brightened(const HableF &k, double g) {
    HableF r = k;
    r.a = (float)((double)k.a * g * g);
    r.b = (float)((double)k.b * g);
    r.w = (float)((double)k.w / g);
    return r;
}
lw_status tonemap_desc(lw_ctx *c, const lw_tonemap *tm, TonemapDesc &t) {
    if (!tm || tm->op > 3u || (tm->mix && tm->op_b > 3u)) return fail(c, LW_ERR_INVALID_ARGUMENT, "unknown tone map");
    const HableF preset{0.15f, 0.5f, 0.1f, 0.2f, 0.02f, 0.3f, 11.2f};
    t.exposure = tm->exposure;
    t.op_a = tm->op;
    t.op_b = tm->mix ? tm->op_b : tm->op;
    t.mix = tm->mix ? 1u : 0u;
    t.weight = tm->weight;
    t.inv_gamma = 1.0f / 2.2f;
    t.preset = tone_curve(preset);
    t.game = tone_curve(brightened(preset, mid_grey_gain(preset, 0.18)));
    return LW_OK;
}

lw_status install_scene(lw_ctx *c, const lw_scene_desc *d, uint32_t n_bricks, uint32_t n_ov);

void reset_stats(lw_ctx *c) {
    double up = c->stats.upload_ms;
    c->stats = lw_stats{};
    c->stats.upload_ms = up;
}

// One launch's items through the wavefront iterations, until no slot has a ray left. The pool
// holds one slot per 16 samples of the launch (a power of two from 2^16 to 2^23, and no more slots
// than items): a larger pool keeps more rays in each iteration, so the iterations' fixed costs and
// their last long traversals weigh less, at 328 bytes of device memory per slot.
lw_status run_wavefront(lw_ctx *c, const DevScene &S, const DevParams &P, const WorkDesc &W) {
    const uint32_t n = wf_slots(c, (uint64_t)W.w * W.h * W.spp, W.n_items);
    const uint32_t budget = c->tuning.budget ? c->tuning.budget : kWfBudget;
    WfState F;
    lw_status s = wf_setup(c, c->wf, n, F, c->stream);
    if (s != LW_OK) return s;
    if (!c->wf_ev[0])
        for (auto &e : c->wf_ev) CK(c, cudaEventCreate(&e), "creating events");
    // Iterations in windows of 16: the host reads the last queue length of each window and stops
    // after the first window whose last iteration had nothing to trace.
    for (uint32_t t = 0;; t++) {
        cudaEvent_t *e = c->wf_ev + 3 * (t & 15u);
        CK(c, cudaEventRecord(e[0], c->stream), "recording an event");
        CK(c, launch_wf_shade(S, P, W, F, wf_shade_blocks(c, n), c->stream), "launching the shading kernel");
        CK(c, cudaEventRecord(e[1], c->stream), "recording an event");
        const bool staged = c->stage_bytes && P.see_through.z == 0u;  // the rebased tracing kernel is unstaged
        const LaunchShape &shape = staged ? c->shape_wf_staged : (P.see_through.z ? c->shape_wf_reb : c->shape_wf);
        CK(c, launch_wf_trace(S, P, F, shape, budget, c->wf_tail, staged ? c->stage_bytes : 0,
                              c->stream), "launching the tracing kernel");
        CK(c, cudaEventRecord(e[2], c->stream), "recording an event");
        CK(c, launch_wf_advance(F, c->stream), "launching the iteration step");
        c->stats.shade_launches++;
        c->stats.trace_launches++;
        c->stats.launches += 3;
        if ((t & 15u) == 15u) {
            CK(c, cudaMemcpyAsync(c->wf_host, F.ctr + 4 * (t % 3u), 4, cudaMemcpyDeviceToHost, c->stream),
               "reading the queue length");
            WAIT(c, "running the iterations");
            for (int k = 0; k < 16; k++) {
                float a = 0.f, b = 0.f;
                cudaEventElapsedTime(&a, c->wf_ev[3 * k], c->wf_ev[3 * k + 1]);
                cudaEventElapsedTime(&b, c->wf_ev[3 * k + 1], c->wf_ev[3 * k + 2]);
                c->stats.shade_ms += a;
                c->stats.trace_ms += b;
            }
            if (*(volatile uint32_t *)c->wf_host == 0u) break;
        }
    }
    uint64_t rays = 0;
    CK(c, cudaMemcpy(&rays, F.ctr + 14, 8, cudaMemcpyDeviceToHost), "reading the ray count");
    c->stats.rays += rays;
    return LW_OK;
}

// Launches the accumulating render of samples [s0, s0 + spp) over the whole frame, in batches.
// With `progress`, each batch is waited for and reported; without it nothing waits.
lw_status render_batches(lw_ctx *c, const lw_params *params, uint32_t s0, uint32_t spp, lw_progress_fn progress,
                         void *user, uint32_t progress_total, uint32_t shard = 0, uint32_t shards = 1) {
    const uint32_t w = params->frame[0], h = params->frame[1];
    WorkDesc probe = work(c, 0, 0, w, h, 0, 1, 1, shard, shards);
    if (probe.n_slots == 0) return LW_OK;  // a shard with no tile of the frame
    Plan pl = plan(c, probe.n_slots, spp);
    if (c->tuning.engine == LW_ENGINE_WAVEFRONT && c->tuning.sub == 0) {
        // Items of one sample: a slot that ends a sample takes the next item at once, and when the
        // items run out no slot has more than one sample left, so the pool drains in few
        // iterations (against items of up to 16 samples: c2 +8 % at 256 spp, +4.5 % at 1024 spp
        // in the launches of 291 spp that a 4 GiB item-sum cap allowed; c4 +8 %).
        pl = plan(c, probe.n_slots, spp, 1u);
    }
    CK(c, ensure(c->partials, (size_t)probe.n_slots * ((pl.batch + pl.sub - 1) / pl.sub)), "allocating partial sums");
    DevScene S = dev_scene(c);
    DevParams P = dev_params(params);
    uint32_t done = 0;
    while (done < spp) {
        uint32_t n = spp - done < pl.batch ? spp - done : pl.batch;
        WorkDesc W = work(c, 0, 0, w, h, s0 + done, n, pl.sub, shard, shards);
        CK(c, cudaMemsetAsync(c->counter.p, 0, sizeof(uint32_t), c->stream), "clearing the work counter");
        CK(c, cudaEventRecord(c->ev_a, c->stream), "recording an event");
        if (c->tuning.engine == LW_ENGINE_WAVEFRONT) {
            lw_status ws = run_wavefront(c, S, P, W);
            if (ws != LW_OK) return ws;
        } else {
            CK(c, launch_render(MODE_ACCUM, S, P, W, c->shape_accum, c->stream), "launching the render kernel");
        }
        CK(c, cudaEventRecord(c->ev_b, c->stream), "recording an event");
        CK(c, launch_reduce(W, c->acc.p, w, c->stream), "launching the reduction");
        c->stats.launches += c->tuning.engine == LW_ENGINE_WAVEFRONT ? 1u : 2u;
        c->stats.samples += (uint64_t)w * h * n;
        done += n;
        if (progress || done < spp) {
            {
                lw_status ws = wait_event(c, c->ev_b, "waiting for the render kernel");
                if (ws != LW_OK) return ws;
            }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, c->ev_a, c->ev_b);
            c->stats.kernel_ms += ms;
            if (progress) progress(done, progress_total, user);
            if (__atomic_load_n(c->cancel_host, __ATOMIC_RELAXED))
                return fail(c, LW_ERR_CANCELLED, "cancelled after %u of %u samples", done, spp);
        } else {
            c->kernel_ms_base = c->stats.kernel_ms;  // the earlier launches of this call
            c->stats.kernel_ms = -1.0;               // read by lw_get_stats once the last launch is done
        }
    }
    return LW_OK;
}

// The batched form on the wavefront engine as one CUDA graph: clear the accumulators; then per pass
// clear the work counter and the path slots, a loop node (a conditional WHILE node) whose body is
// one iteration (shade every slot, trace the queue, advance) and which runs again while the last
// iteration had rays to trace, all decided on the device, and the pass's per-camera reduction,
// which carries every pixel's Kahan sums on from the pass before.
lw_status batch_graph_wavefront(lw_ctx *c, const std::vector<BatchDesc> &Bs, const DevParams &P0, uint64_t pixels,
                               uint32_t slots) {
    if (!c->cap) CK(c, cudaStreamCreateWithFlags(&c->cap, cudaStreamNonBlocking), "creating a capture stream");
    const uint32_t budget = c->tuning.budget ? c->tuning.budget : kWfBudget;
    // The buffers first (cleared outside the graph too, which is harmless).
    WfState F;
    lw_status s = wf_setup(c, c->bwf, slots, F, c->stream);
    if (s != LW_OK) return s;
    CK(c, cudaStreamSynchronize(c->stream), "preparing the path slots");
    DevScene S = dev_scene(c);
    cudaGraph_t graph = nullptr;
    CK(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal), "starting the graph capture");
    cudaError_t e = cudaMemsetAsync(c->batch_acc.p, 0, sizeof(Accum) * pixels, c->stream);
    // Per pass: clear the work counter and the path slots, the loop node, the pass's reduction.
    for (size_t k = 0; k < Bs.size() && e == cudaSuccess; k++) {
        const BatchDesc &B = Bs[k];
        e = cudaMemsetAsync(B.counter, 0, 4, c->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(F.state + (size_t)4 * F.n, 0, (size_t)F.n * sizeof(float4), c->stream);
        if (e == cudaSuccess)
            e = cudaMemsetAsync(F.state + (size_t)kWfItemCameraWord * F.n, 0, (size_t)F.n * sizeof(float4), c->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(F.ctr, 0, 16 * sizeof(uint32_t), c->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(F.hit0, 0, (size_t)F.n * sizeof(float4), c->stream);
        cudaGraphNode_t loop_node = nullptr;
        if (e == cudaSuccess) {
            cudaStreamCaptureStatus status;
            cudaGraph_t g = nullptr;
            const cudaGraphNode_t *deps = nullptr;
            size_t ndeps = 0;
            e = cudaStreamGetCaptureInfo(c->stream, &status, nullptr, &g, &deps, &ndeps);
            cudaGraphConditionalHandle loop{};
            if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&loop, g, 1u, cudaGraphCondAssignDefault);
            cudaGraphNodeParams np{};
            np.type = cudaGraphNodeTypeConditional;
            np.conditional.handle = loop;
            np.conditional.type = cudaGraphCondTypeWhile;
            np.conditional.size = 1;
            if (e == cudaSuccess) e = cudaGraphAddNode(&loop_node, g, deps, ndeps, &np);
            if (e == cudaSuccess) {
                cudaGraph_t body = np.conditional.phGraph_out[0];
                e = cudaStreamBeginCaptureToGraph(c->cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
                if (e == cudaSuccess) {
                    cudaError_t eb = launch_wf_shade_batch(S, P0, B, F, wf_shade_blocks(c, F.n), c->cap);
                    if (eb == cudaSuccess)
                        eb = launch_wf_trace(S, P0, F, c->stage_bytes ? c->shape_wf_staged : c->shape_wf, budget, c->wf_tail,
                                             c->stage_bytes, c->cap);
                    if (eb == cudaSuccess) eb = launch_wf_advance_graph(F, loop, c->cap);
                    cudaGraph_t done = nullptr;
                    e = cudaStreamEndCapture(c->cap, &done);
                    if (eb != cudaSuccess) e = eb;
                }
            }
            if (e == cudaSuccess) e = cudaStreamUpdateCaptureDependencies(c->stream, &loop_node, 1, cudaStreamSetCaptureDependencies);
        }
        if (e == cudaSuccess) e = launch_reduce_batch(B, c->stream);
    }
    cudaError_t e2 = cudaStreamEndCapture(c->stream, &graph);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&c->batch_graph, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_fail(c, e, "building the batch graph");
    return LW_OK;
}

}  // namespace

extern "C" {

lw_status lw_ctx_create(int device, lw_ctx **out) {
    if (!out) return fail(nullptr, LW_ERR_INVALID_ARGUMENT, "out is null");
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return fail(nullptr, LW_ERR_NO_DEVICE, "no CUDA device");
    if (device < 0 || device >= n) return fail(nullptr, LW_ERR_NO_DEVICE, "device %d of %d", device, n);
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, device);
    if (prop.major != 10) return fail(nullptr, LW_ERR_NO_DEVICE, "device %d (%s) is sm_%d%d; this library is built for sm_100a", device, prop.name, prop.major, prop.minor);
    lw_ctx *c = new lw_ctx();
    c->device = device;
    auto bail = [&](cudaError_t e, const char *what) {
        g_create_error = std::string(what) + ": " + cudaGetErrorString(e);
        lw_ctx_destroy(c);
        return e == cudaErrorMemoryAllocation ? LW_ERR_OUT_OF_MEMORY : LW_ERR_LAUNCH;
    };
    cudaError_t e;
    if ((e = cudaSetDevice(device)) != cudaSuccess) return bail(e, "cudaSetDevice");
    if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess) return bail(e, "creating a stream");
    if ((e = cudaEventCreate(&c->ev_a)) != cudaSuccess || (e = cudaEventCreate(&c->ev_b)) != cudaSuccess)
        return bail(e, "creating events");
    for (auto &m : c->marks)
        if ((e = cudaEventCreate(&m)) != cudaSuccess) return bail(e, "creating events");
    c->cancel_host = new int(0);
    if ((e = cudaStreamCreateWithFlags(&c->aux, cudaStreamNonBlocking)) != cudaSuccess) return bail(e, "creating a stream");
    if ((e = cudaEventCreateWithFlags(&c->cancel_ev, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&c->wait_ev, cudaEventDisableTiming)) != cudaSuccess)
        return bail(e, "creating events");
    if ((e = ensure(c->cancel_word, 1)) != cudaSuccess) return bail(e, "allocating the cancel word");
    if ((e = cudaMemset(c->cancel_word.p, 0, 4)) != cudaSuccess) return bail(e, "clearing the cancel word");
    float lut[256];
    for (int k = 0; k < 256; k++) lut[k] = ref_gamma_to_linear((float)k / 255.0f);
    if ((e = ensure(c->gamma, 256)) != cudaSuccess) return bail(e, "allocating the gamma table");
    if ((e = cudaMemcpy(c->gamma.p, lut, sizeof lut, cudaMemcpyHostToDevice)) != cudaSuccess) return bail(e, "uploading the gamma table");
    if ((e = ensure(c->counter, 1)) != cudaSuccess || (e = ensure(c->error, 1)) != cudaSuccess) return bail(e, "allocating counters");
    {
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess && free_b / 4 < c->partials_cap_bytes)
            c->partials_cap_bytes = free_b / 4 > (size_t(1) << 28) ? free_b / 4 : size_t(1) << 28;
    }
    c->shape_wf = wf_trace_shape(device);
    c->shape_wf_reb = wf_trace_shape(device, 0, true);
    c->shape_accum = render_shape(MODE_ACCUM, device, (int)c->tuning.threads);
    c->shape_samples = render_shape(MODE_SAMPLES, device, (int)c->tuning.threads);
    *out = c;
    return LW_OK;
}

void lw_ctx_destroy(lw_ctx *c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (auto *b : {&c->grid, &c->atlas, &c->egrid, &c->counter, &c->error, &c->vox}) b->free_();
    c->top.free_();
    c->occ.free_();
    c->bricks.free_();
    c->models.free_();
    c->quads.free_();
    c->emitters.free_();
    c->partials.free_();
    c->ref_quads.free_();
    if (c->batch_graph) cudaGraphExecDestroy(c->batch_graph);
    for (auto *b : c->batch_skies) { b->dev.free_(); delete b; }
    c->batch_jobs.free_();
    c->batch_item_begin.free_();
    c->batch_slot_begin.free_();
    c->batch_acc.free_();
    c->batch_out.free_();
    c->batch_partials.free_();
    for (int k = 0; k < 3; k++) {
        c->adj_albedo[k].free_();
        c->adj_sky[k].free_();
        c->adj_emit[k].free_();
        c->adj_tparam[k].free_();
    }
    for (auto *b : {&c->adj_img, &c->adj_img2, &c->adj_g, &c->adj_L}) b->free_();
    c->wf.free_();
    c->bwf.free_();
    c->bv_blocks.free_();
    c->bv_ids.free_();
    c->bv_flags.free_();
    c->bv_emits.free_();
    for (auto *b : {&c->bv_keys, &c->bv_first, &c->bv_key_id, &c->bv_slot, &c->bv_emit_off}) b->free_();
    c->bv_cls.free_();
    c->bv_sites.free_();
    if (c->wf_host) cudaFreeHost(c->wf_host);
    for (auto e : c->wf_ev)
        if (e) cudaEventDestroy(e);
    for (auto *b : {&c->sky, &c->gamma, &c->out_rgb, &c->samples, &c->rays}) b->free_();
    c->out_rgba.free_();
    c->acc.free_();
    c->hits.free_();
    c->xyz.free_();
    delete c->cancel_host;
    c->cancel_word.free_();
    if (c->aux) cudaStreamDestroy(c->aux);
    if (c->cancel_ev) cudaEventDestroy(c->cancel_ev);
    if (c->wait_ev) cudaEventDestroy(c->wait_ev);
    if (c->cap) cudaStreamDestroy(c->cap);
    if (c->ev_a) cudaEventDestroy(c->ev_a);
    if (c->ev_b) cudaEventDestroy(c->ev_b);
    for (auto m : c->marks)
        if (m) cudaEventDestroy(m);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

const char *lw_last_error(const lw_ctx *c) { return c ? c->err.c_str() : g_create_error.c_str(); }

void *lw_stream(lw_ctx *c) { return c ? (void *)c->stream : nullptr; }

void lw_cancel(lw_ctx *c) {
    if (!c || !c->cancel_host) return;
    cudaSetDevice(c->device);
    cancel_device(c);
}

lw_status lw_set_timeout(lw_ctx *c, double seconds) {
    if (!c) return LW_ERR_INVALID_ARGUMENT;
    if (!(seconds >= 0.0) || seconds > 1e6) return fail(c, LW_ERR_INVALID_ARGUMENT, "timeout %g s", seconds);
    c->timeout_s = seconds;
    return LW_OK;
}

lw_status lw_set_tuning(lw_ctx *c, const lw_tuning *t) {
    if (!c || !t) return LW_ERR_INVALID_ARGUMENT;
    if (t->threads != 64 && t->threads != 128 && t->threads != 256)
        return fail(c, LW_ERR_INVALID_ARGUMENT, "threads per block %u (64, 128 or 256)", t->threads);
    if (t->sub > 4096) return fail(c, LW_ERR_INVALID_ARGUMENT, "sub %u", t->sub);
    if (t->engine != LW_ENGINE_WAVEFRONT && t->engine != LW_ENGINE_MEGAKERNEL)
        return fail(c, LW_ERR_INVALID_ARGUMENT, "engine %u", t->engine);
    if (t->paths > (1u << 26)) return fail(c, LW_ERR_INVALID_ARGUMENT, "paths %u (at most 2^26)", t->paths);
    cudaSetDevice(c->device);
    c->tuning = *t;
    c->shape_accum = render_shape(MODE_ACCUM, c->device, (int)t->threads);
    c->shape_samples = render_shape(MODE_SAMPLES, c->device, (int)t->threads);
    return LW_OK;
}

lw_status lw_get_tuning(const lw_ctx *c, lw_tuning *out) {
    if (!c || !out) return LW_ERR_INVALID_ARGUMENT;
    *out = c->tuning;
    return LW_OK;
}

lw_status lw_mark(lw_ctx *c, uint32_t slot) {
    if (!c || slot >= 8) return fail(c, LW_ERR_INVALID_ARGUMENT, "mark slot %u", slot);
    cudaSetDevice(c->device);
    CK(c, cudaEventRecord(c->marks[slot], c->stream), "recording a mark");
    return LW_OK;
}

lw_status lw_elapsed_ms(lw_ctx *c, uint32_t from, uint32_t to, double *ms) {
    if (!c || !ms || from >= 8 || to >= 8) return fail(c, LW_ERR_INVALID_ARGUMENT, "bad mark");
    cudaSetDevice(c->device);
    CK(c, cudaEventSynchronize(c->marks[to]), "waiting for a mark");
    float f = 0.f;
    CK(c, cudaEventElapsedTime(&f, c->marks[from], c->marks[to]), "reading marks");
    *ms = f;
    return LW_OK;
}

lw_status lw_get_stats(const lw_ctx *cc, lw_stats *out) {
    lw_ctx *c = const_cast<lw_ctx *>(cc);
    if (!c || !out) return LW_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    if (c->stats.kernel_ms < 0.0) {
        if (cudaEventSynchronize(c->ev_b) != cudaSuccess) return LW_ERR_LAUNCH;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev_a, c->ev_b);
        c->stats.kernel_ms = c->kernel_ms_base + ms;
        c->kernel_ms_base = 0.0;
    }
    *out = c->stats;
    out->blocks = (uint32_t)c->shape_accum.blocks;
    out->threads = (uint32_t)c->shape_accum.threads;
    return LW_OK;
}

lw_status lw_scene_upload(lw_ctx *c, const lw_scene_desc *d) {
    if (!c || !d) return fail(c, LW_ERR_INVALID_ARGUMENT, "null argument");
    cudaSetDevice(c->device);
    auto t0 = std::chrono::steady_clock::now();
    c->has_scene = false;
    if (!d->grid || !d->models || !d->quads || !d->atlas || !d->emitters || !d->emitter_grid)
        return fail(c, LW_ERR_INVALID_ARGUMENT, "a scene buffer is null");
    if (!d->models_len || !d->quads_len || !d->emitters_len)
        return fail(c, LW_ERR_BUFFER_LENGTH, "models, quads and emitters hold at least one entry each");
    const uint64_t nb = (uint64_t)d->dims[0] * d->dims[1] * d->dims[2];
    if (nb == 0 || nb > 0x7FFFFFFFull) return fail(c, LW_ERR_INVALID_ARGUMENT, "grid of %ux%ux%u bricks", d->dims[0], d->dims[1], d->dims[2]);
    if ((uint64_t)d->dims[0] * 16 > 0x7FFFFFF || (uint64_t)d->dims[1] * 16 > 0x7FFFFFF || (uint64_t)d->dims[2] * 16 > 0x7FFFFFF)
        return fail(c, LW_ERR_INVALID_ARGUMENT, "grid too large");
    const uint32_t *o = d->offsets;
    if (o[0] + nb > d->grid_len || o[2] + nb > d->grid_len)
        return fail(c, LW_ERR_BUFFER_LENGTH, "top or ov_top entries outside the %llu grid words", (unsigned long long)d->grid_len);
    if (o[1] > o[2] || (o[2] - o[1]) % 2048u != 0 || o[3] > o[4] || (o[4] - o[3]) % 8192u != 0 || o[4] > d->grid_len || o[3] < o[2] + nb)
        return fail(c, LW_ERR_BUFFER_LENGTH, "grid offsets %u %u %u %u %u are not [top | bricks | ov_top | ov_cells | ov_quads]", o[0], o[1], o[2], o[3], o[4]);
    const uint32_t n_bricks = (o[2] - o[1]) / 2048u, n_ov = (o[4] - o[3]) / 8192u;
    const uint64_t ovq_len = d->grid_len - o[4];
    // Cross-buffer indices the kernels follow (the reference's slice bounds checks).
    for (uint64_t i = 0; i < d->models_len; i++)
        if ((uint64_t)d->models[i].quad_offset + d->models[i].quad_count > d->quads_len)
            return fail(c, LW_ERR_BUFFER_LENGTH, "model %llu's quads [%u, +%u) outside %llu quads", (unsigned long long)i,
                        d->models[i].quad_offset, d->models[i].quad_count, (unsigned long long)d->quads_len);
    for (uint64_t i = 0; i < d->emitters_len; i++) {
        uint32_t first;
        std::memcpy(&first, &d->emitters[i].pos[3], 4);
        if ((uint64_t)first + d->emitters[i].faces[0] > d->quads_len)
            return fail(c, LW_ERR_BUFFER_LENGTH, "emitter %llu's faces outside the quads", (unsigned long long)i);
    }
    if (d->emitter_grid_len < 8) return fail(c, LW_ERR_BUFFER_LENGTH, "emitter grid shorter than its header");
    {
        const uint32_t *g = d->emitter_grid;
        uint64_t cells = (uint64_t)g[1] * g[2] * g[3];
        if (8 + 2 * cells > d->emitter_grid_len) return fail(c, LW_ERR_BUFFER_LENGTH, "emitter grid cells outside the buffer");
        uint64_t list_len = d->emitter_grid_len - 8 - 2 * cells;
        for (uint64_t k = 0; k < cells; k++)
            if ((uint64_t)g[8 + 2 * k] + g[9 + 2 * k] > list_len)
                return fail(c, LW_ERR_BUFFER_LENGTH, "emitter grid cell %llu's list outside the buffer", (unsigned long long)k);
        for (uint64_t k = 0; k < list_len; k++)
            if (g[8 + 2 * cells + k] >= d->emitters_len)
                return fail(c, LW_ERR_BUFFER_LENGTH, "emitter grid names emitter %u of %llu", g[8 + 2 * cells + k], (unsigned long long)d->emitters_len);
    }
    for (uint64_t k = 0; k < (uint64_t)n_ov * 4096u; k++) {
        uint64_t off = d->grid[o[3] + 2 * k], cnt = d->grid[o[3] + 2 * k + 1];
        if (off + cnt > ovq_len) return fail(c, LW_ERR_BUFFER_LENGTH, "overlay cell %llu's quads outside ov_quads", (unsigned long long)k);
    }
    for (uint64_t k = 0; k < (uint64_t)n_ov * 4096u; k++) {
        uint64_t off = d->grid[o[3] + 2 * k], cnt = d->grid[o[3] + 2 * k + 1];
        for (uint64_t i = 0; i < cnt; i++)
            if (d->grid[o[4] + off + i] >= d->quads_len) return fail(c, LW_ERR_BUFFER_LENGTH, "an overlay cell names a quad out of range");
    }
    if ((uint64_t)d->atlas_size[0] * d->atlas_size[1] > d->atlas_len || d->atlas_size[0] == 0 || d->atlas_size[1] == 0)
        return fail(c, LW_ERR_BUFFER_LENGTH, "atlas %ux%u needs more than %llu texels", d->atlas_size[0], d->atlas_size[1], (unsigned long long)d->atlas_len);

    CK(c, upload(c, c->grid, d->grid, d->grid_len, 4), "uploading the grid");
    lw_status s = install_scene(c, d, n_bricks, n_ov);
    if (s != LW_OK) return s;
    c->stats.upload_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return LW_OK;
}

}  // extern "C"

namespace {

// The scene's buffers other than the grid (already in c->grid) to the device, the B200 re-layout,
// and the context's scene description.
lw_status install_scene(lw_ctx *c, const lw_scene_desc *d, uint32_t n_bricks, uint32_t n_ov) {
    const uint64_t nb = (uint64_t)d->dims[0] * d->dims[1] * d->dims[2];
    const uint32_t *o = d->offsets;
    CK(c, upload(c, c->models, d->models, d->models_len, 16), "uploading the models");
    CK(c, upload(c, c->atlas, d->atlas, d->atlas_len, 4), "uploading the atlas");
    CK(c, upload(c, c->emitters, d->emitters, d->emitters_len, 32), "uploading the emitters");
    CK(c, upload(c, c->egrid, d->emitter_grid, d->emitter_grid_len, 4), "uploading the emitter grid");
    CK(c, upload(c, c->ref_quads, d->quads, d->quads_len, 80), "uploading the quads");
    CK(c, ensure(c->quads, d->quads_len), "allocating the quads");
    CK(c, launch_quads(c->ref_quads.p, c->quads.p, (uint32_t)d->quads_len, c->stream), "re-laying the quads");
    CK(c, ensure(c->top, nb), "allocating the top level");
    CK(c, ensure(c->bricks, (size_t)n_bricks * 4096u), "allocating the bricks");
    CK(c, ensure(c->occ, n_bricks), "allocating the occupancy masks");
    CK(c, cudaMemsetAsync(c->error.p, 0, 4, c->stream), "clearing the error word");
    SceneUploadDesc u{c->grid.p, (uint32_t)nb, n_bricks, o[0], o[1], o[2], (uint32_t)d->models_len, n_ov,
                      (const uint4 *)c->models.p, c->top.p, c->bricks.p, c->occ.p, c->error.p};
    CK(c, launch_relayout(u, c->stream), "re-laying the grid");
    uint32_t err = 0;
    CK(c, cudaMemcpyAsync(&err, c->error.p, 4, cudaMemcpyDeviceToHost, c->stream), "reading the error word");
    CK(c, cudaStreamSynchronize(c->stream), "uploading the scene");
    if (err & 1u) return fail(c, LW_ERR_BUFFER_LENGTH, "a top-level entry names a brick, model or overlay brick out of range");
    if (err & 2u) return fail(c, LW_ERR_BUFFER_LENGTH, "a voxel names a model out of range");
    // The lowest brick row with nothing at or above it (bricks of the top level are (y, z, x)-major).
    {
        std::vector<uint2> top(nb);
        CK(c, cudaMemcpy(top.data(), c->top.p, nb * sizeof(uint2), cudaMemcpyDeviceToHost), "reading the top level");
        const uint64_t row = (uint64_t)d->dims[0] * d->dims[2];
        uint32_t sky_y = 0;
        for (uint64_t b = 0; b < nb; b++)
            if (top[b].x != 0xFFFFFFFFu || top[b].y != 0xFFFFFFFFu) sky_y = (uint32_t)(b / row) + 1u;
        c->sky_brick_y = sky_y;
    }
    std::memcpy(c->dims, d->dims, sizeof c->dims);
    std::memcpy(c->offsets, d->offsets, sizeof c->offsets);
    std::memcpy(c->atlas_size, d->atlas_size, sizeof c->atlas_size);
    c->nb = (uint32_t)nb;
    c->n_bricks = n_bricks;
    // The tracing kernel stages the top level and the occupancy masks per block when they are small.
    c->stage_bytes = (nb + n_bricks) * sizeof(uint2) <= (uint64_t)LW_TRACE_STAGE_MAX ? (nb + n_bricks) * sizeof(uint2) : 0;
    if (c->stage_bytes) c->shape_wf_staged = wf_trace_shape(c->device, c->stage_bytes);
    c->n_ov_bricks = n_ov;
    c->grid_len = d->grid_len;
    c->models_len = d->models_len;
    c->quads_len = d->quads_len;
    c->atlas_len = d->atlas_len;
    c->emitters_len = d->emitters_len;
    c->egrid_len = d->emitter_grid_len;
    c->has_scene = true;
    return LW_OK;
}

}  // namespace

extern "C" {

lw_status lw_sky_upload(lw_ctx *c, const float *sky, uint64_t sky_len) {
    if (!c) return LW_ERR_INVALID_ARGUMENT;
    if (sky_len && !sky) return fail(c, LW_ERR_INVALID_ARGUMENT, "sky is null");
    cudaSetDevice(c->device);
    CK(c, upload(c, c->sky, sky, sky_len, 4), "uploading the sky");
    c->sky_len = sky_len;
    return LW_OK;
}

lw_status lw_clear_accumulator(lw_ctx *c, uint32_t w, uint32_t h) {
    if (!c || !w || !h) return fail(c, LW_ERR_INVALID_ARGUMENT, "bad frame size");
    cudaSetDevice(c->device);
    lw_status s = ensure_accum(c, w, h);
    if (s != LW_OK) return s;
    CK(c, cudaMemsetAsync(c->acc.p, 0, sizeof(Accum) * (size_t)w * h, c->stream), "clearing the accumulator");
    return LW_OK;
}

lw_status lw_render_device(lw_ctx *c, const lw_params *params, uint32_t sample_start, uint32_t spp) {
    if (!c) return LW_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    lw_status s = check_params(c, params, true);
    if (s != LW_OK) return s;
    if (c->acc_w != params->frame[0] || c->acc_h != params->frame[1])
        return fail(c, LW_ERR_INVALID_ARGUMENT, "the accumulator is %ux%u, the frame %ux%u", c->acc_w, c->acc_h, params->frame[0], params->frame[1]);
    if (spp == 0) return fail(c, LW_ERR_INVALID_ARGUMENT, "spp is 0");
    s = begin_render(c);
    if (s != LW_OK) return s;
    reset_stats(c);
    return render_batches(c, params, sample_start, spp, nullptr, nullptr, spp);
}

lw_status lw_render_device_shard(lw_ctx *c, const lw_params *params, uint32_t sample_start, uint32_t spp, uint32_t shard,
                                 uint32_t shards) {
    if (!c) return LW_ERR_INVALID_ARGUMENT;
    if (shards == 0 || shard >= shards) return fail(c, LW_ERR_INVALID_ARGUMENT, "shard %u of %u", shard, shards);
    cudaSetDevice(c->device);
    lw_status s = check_params(c, params, true);
    if (s != LW_OK) return s;
    if (c->acc_w != params->frame[0] || c->acc_h != params->frame[1])
        return fail(c, LW_ERR_INVALID_ARGUMENT, "the accumulator is %ux%u, the frame %ux%u", c->acc_w, c->acc_h, params->frame[0], params->frame[1]);
    if (spp == 0) return fail(c, LW_ERR_INVALID_ARGUMENT, "spp is 0");
    s = begin_render(c);
    if (s != LW_OK) return s;
    reset_stats(c);
    return render_batches(c, params, sample_start, spp, nullptr, nullptr, spp, shard, shards);
}

lw_status lw_accumulator_device(lw_ctx *c, void **records, uint32_t *width, uint32_t *height) {
    if (!c || !records) return fail(c, LW_ERR_INVALID_ARGUMENT, "null argument");
    if (!c->acc_w) return fail(c, LW_ERR_INVALID_ARGUMENT, "no accumulator");
    *records = c->acc.p;
    if (width) *width = c->acc_w;
    if (height) *height = c->acc_h;
    return LW_OK;
}

lw_status lw_render_accumulate_noalloc(lw_ctx *c, const lw_params *params, uint32_t sample_start, uint32_t spp,
                                       void *accum) {
    if (!c || !params || !accum || spp == 0) return fail(c, LW_ERR_INVALID_ARGUMENT, "null argument or spp 0");
    cudaSetDevice(c->device);
    lw_status s = check_params(c, params, true);
    if (s != LW_OK) return s;
    const uint32_t w = params->frame[0], h = params->frame[1];
    WorkDesc probe = work(c, 0, 0, w, h, 0, 1, 1);
    if ((size_t)probe.n_slots > kNoallocPartials)
        return fail(c, LW_ERR_INVALID_ARGUMENT,
                    "a %ux%u frame needs %u pixel slots; the allocation-free entry point holds %zu (about 1920x1088)",
                    w, h, probe.n_slots, kNoallocPartials);
    // The accumulator must be device memory of this context's GPU (a host pointer or another GPU's
    // buffer would fault in the reduction); cudaPointerGetAttributes allocates nothing.
    {
        cudaPointerAttributes pa{};
        cudaError_t e = cudaPointerGetAttributes(&pa, accum);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(c, LW_ERR_INVALID_ARGUMENT, "accum is not a CUDA pointer: %s", cudaGetErrorString(e));
        }
        if ((pa.type != cudaMemoryTypeDevice && pa.type != cudaMemoryTypeManaged) || pa.device != c->device)
            return fail(c, LW_ERR_INVALID_ARGUMENT, "accum must be device memory on device %d (it is of type %d on device %d)",
                        c->device, (int)pa.type, pa.device);
    }
    float4 *scratch = nullptr;
    CK(c, noalloc_scratch(c->device, &scratch), "looking up the scratch array");
    Plan pl = plan(c, probe.n_slots, spp);
    uint64_t subs = kNoallocPartials / probe.n_slots;
    uint64_t batch = subs * pl.sub < spp ? subs * pl.sub : spp;
    DevScene S = dev_scene(c);
    DevParams P = dev_params(params);
    s = begin_render(c);
    if (s != LW_OK) return s;
    for (uint32_t done = 0; done < spp;) {
        uint32_t n = spp - done < batch ? spp - done : (uint32_t)batch;
        WorkDesc W = work(c, 0, 0, w, h, sample_start + done, n, pl.sub);
        W.counter = (uint32_t *)scratch;  // the header's first word; the item sums follow it
        W.partials = scratch + 16;
        CK(c, cudaMemsetAsync(W.counter, 0, sizeof(uint32_t), c->stream), "clearing the work counter");
        CK(c, launch_render(MODE_ACCUM, S, P, W, c->shape_accum, c->stream), "launching the render kernel");
        CK(c, launch_reduce(W, (Accum *)accum, w, c->stream), "launching the reduction");
        done += n;
    }
    return LW_OK;
}

lw_status lw_read_accumulator(lw_ctx *c, float *out_rgb) {
    if (!c || !out_rgb) return fail(c, LW_ERR_INVALID_ARGUMENT, "null argument");
    cudaSetDevice(c->device);
    size_t n = (size_t)c->acc_w * c->acc_h;
    if (!n) return fail(c, LW_ERR_INVALID_ARGUMENT, "no accumulator");
    CK(c, ensure(c->out_rgb, 3 * n), "allocating the output");
    CK(c, launch_finalize(c->acc.p, (uint32_t)n, c->out_rgb.p, c->stream), "launching the finalize kernel");
    CK(c, cudaMemcpyAsync(out_rgb, c->out_rgb.p, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, c->stream), "reading the image");
    WAIT(c, "reading the image");
    return check_cancelled(c);
}

lw_status lw_render_hq(lw_ctx *c, const lw_params *params, const float *sky, uint64_t sky_len, uint32_t spp,
                       lw_progress_fn progress, void *user, float *out_rgb) {
    if (!c || !out_rgb) return fail(c, LW_ERR_INVALID_ARGUMENT, "null argument");
    cudaSetDevice(c->device);
    if (spp < 1) spp = 1;  // `f.spp.max(1)` (cuda.rs:85)
    lw_status s = lw_sky_upload(c, sky, sky_len);
    if (s != LW_OK) return s;
    s = check_params(c, params, true);
    if (s != LW_OK) return s;
    s = lw_clear_accumulator(c, params->frame[0], params->frame[1]);
    if (s != LW_OK) return s;
    s = begin_render(c);
    if (s != LW_OK) return s;
    reset_stats(c);
    s = render_batches(c, params, 0, spp, progress, user, spp);
    if (s != LW_OK) return s;
    return lw_read_accumulator(c, out_rgb);
}

lw_status lw_render_samples(lw_ctx *c, const lw_params *params, uint32_t x0, uint32_t y0, uint32_t w, uint32_t h,
                            uint32_t sample_start, uint32_t count, float *out) {
    if (!c || !out || !w || !h || !count) return fail(c, LW_ERR_INVALID_ARGUMENT, "bad argument");
    cudaSetDevice(c->device);
    lw_status s = check_params(c, params, true);
    if (s != LW_OK) return s;
    if ((uint64_t)x0 + w > params->frame[0] || (uint64_t)y0 + h > params->frame[1])
        return fail(c, LW_ERR_INVALID_ARGUMENT, "rectangle outside the frame");
    size_t n = (size_t)w * h * count * 3;
    CK(c, ensure(c->samples, n), "allocating the samples");
    WorkDesc W = work(c, x0, y0, w, h, sample_start, count, 1);
    W.samples_out = c->samples.p;
    s = begin_render(c);
    if (s != LW_OK) return s;
    CK(c, cudaMemsetAsync(c->counter.p, 0, 4, c->stream), "clearing the work counter");
    CK(c, launch_render(MODE_SAMPLES, dev_scene(c), dev_params(params), W, c->shape_samples, c->stream), "launching the render kernel");
    CK(c, cudaMemcpyAsync(out, c->samples.p, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream), "reading the samples");
    WAIT(c, "rendering samples");
    return check_cancelled(c);
}

lw_status lw_trace_rays(lw_ctx *c, const lw_params *params, uint32_t n, const float *o, const float *d, float tmin,
                        float tmax, lw_hit *out) {
    if (!c || !o || !d || !out || !n) return fail(c, LW_ERR_INVALID_ARGUMENT, "bad argument");
    cudaSetDevice(c->device);
    lw_status s = check_params(c, params, false);
    if (s != LW_OK) return s;
    CK(c, ensure(c->rays, (size_t)6 * n), "allocating rays");
    CK(c, ensure(c->hits, sizeof(lw_hit) * (size_t)n), "allocating hits");
    CK(c, cudaMemcpyAsync(c->rays.p, o, 12 * (size_t)n, cudaMemcpyHostToDevice, c->stream), "uploading rays");
    CK(c, cudaMemcpyAsync(c->rays.p + 3 * (size_t)n, d, 12 * (size_t)n, cudaMemcpyHostToDevice, c->stream), "uploading rays");
    CK(c, launch_trace_rays(dev_scene(c), dev_params(params), n, c->rays.p, c->rays.p + 3 * (size_t)n, tmin, tmax, c->hits.p, c->stream),
       "launching the trace kernel");
    CK(c, cudaMemcpyAsync(out, c->hits.p, sizeof(lw_hit) * (size_t)n, cudaMemcpyDeviceToHost, c->stream), "reading hits");
    WAIT(c, "tracing rays");
    return LW_OK;
}

lw_status lw_voxel_lookup(lw_ctx *c, uint32_t n, const int32_t *xyz, uint32_t *out) {
    if (!c || !xyz || !out || !n) return fail(c, LW_ERR_INVALID_ARGUMENT, "bad argument");
    if (!c->has_scene) return fail(c, LW_ERR_NO_SCENE, "no scene uploaded");
    cudaSetDevice(c->device);
    for (uint32_t i = 0; i < n; i++)
        for (int a = 0; a < 3; a++)
            if (xyz[3 * i + a] < 0 || (uint32_t)xyz[3 * i + a] >= c->dims[a] * 16u)
                return fail(c, LW_ERR_INVALID_ARGUMENT, "voxel %u outside the grid", i);
    lw_params p{};
    std::memcpy(p.grid_dims, c->dims, sizeof c->dims);
    std::memcpy(p.off, c->offsets, sizeof p.off);  // the reference grid's top and brick offsets
    CK(c, ensure(c->xyz, (size_t)3 * n), "allocating coordinates");
    CK(c, ensure(c->vox, n), "allocating ids");
    CK(c, cudaMemcpyAsync(c->xyz.p, xyz, 12 * (size_t)n, cudaMemcpyHostToDevice, c->stream), "uploading coordinates");
    CK(c, launch_voxel_lookup(dev_scene(c), dev_params(&p), n, c->xyz.p, c->vox.p, c->stream), "launching the lookup kernel");
    CK(c, cudaMemcpyAsync(out, c->vox.p, 4 * (size_t)n, cudaMemcpyDeviceToHost, c->stream), "reading ids");
    CK(c, cudaStreamSynchronize(c->stream), "looking up voxels");
    return LW_OK;
}

lw_status lw_water_exp(lw_ctx *c, uint64_t n, const float *x, float *out) {
    if (!c || !x || !out || !n || n > (uint64_t(1) << 31)) return fail(c, LW_ERR_INVALID_ARGUMENT, "bad argument");
    cudaSetDevice(c->device);
    CK(c, ensure(c->rays, (size_t)2 * n), "allocating the arguments");
    CK(c, cudaMemcpyAsync(c->rays.p, x, 4 * (size_t)n, cudaMemcpyHostToDevice, c->stream), "uploading the arguments");
    CK(c, launch_water_exp(n, c->rays.p, c->rays.p + n, c->stream), "launching the exponential");
    CK(c, cudaMemcpyAsync(out, c->rays.p + n, 4 * (size_t)n, cudaMemcpyDeviceToHost, c->stream), "reading the results");
    CK(c, cudaStreamSynchronize(c->stream), "evaluating the exponential");
    return LW_OK;
}

lw_status lw_batch_prepare(lw_ctx *c, const lw_camera_job *jobs, uint32_t n) {
    if (!c || !jobs || n == 0) return fail(c, LW_ERR_INVALID_ARGUMENT, "no cameras");
    cudaSetDevice(c->device);
    if (c->batch_graph) {
        cudaGraphExecDestroy(c->batch_graph);
        c->batch_graph = nullptr;
    }
    // Skies: one device copy per distinct host buffer.
    std::vector<const float *> sky_dev(n);
    for (uint32_t i = 0; i < n; i++) {
        lw_ctx::BatchSky *found = nullptr;
        for (auto *b : c->batch_skies)
            if (b->host == jobs[i].sky && b->len == jobs[i].sky_len) found = b;
        if (!found) {
            found = new lw_ctx::BatchSky{jobs[i].sky, jobs[i].sky_len, {}};
            c->batch_skies.push_back(found);
            if (jobs[i].sky_len) {
                CK(c, ensure(found->dev, jobs[i].sky_len), "allocating a sky");
                CK(c, cudaMemcpyAsync(found->dev.p, jobs[i].sky, jobs[i].sky_len * 4, cudaMemcpyHostToDevice, c->stream),
                   "uploading a sky");
            }
        }
        sky_dev[i] = found->dev.p;
        lw_status s = check_params(c, &jobs[i].params, true, jobs[i].sky_len);
        if (s != LW_OK) return s;
        if (jobs[i].spp == 0) return fail(c, LW_ERR_INVALID_ARGUMENT, "camera %u has spp 0", i);
        if (jobs[i].params.see_through[2])
            return fail(c, LW_ERR_INVALID_ARGUMENT, "camera %u: the batched form renders in the grid's frame only", i);
    }
    // Layout: items, slots, accumulators, images, item sums.
    uint64_t total_samples = 0;
    for (uint32_t i = 0; i < n; i++) total_samples += (uint64_t)jobs[i].params.frame[0] * jobs[i].params.frame[1] * jobs[i].spp;
    // Samples per item and passes. The item sums (16 B each) of a pass must fit 40 GiB and a third
    // of the device memory free now. The wavefront engine with automatic items takes one sample per
    // item (a slot that ends a sample takes the next item at once, so the pool drains fastest) and
    // as many passes as the cap needs, each covering an equal slice of every camera's samples; with
    // items of `sub` samples (the tuning's, or the megakernel's) the batch is one pass of items as
    // small as fit.
    size_t free_b = 0, total_b = 0;
    uint64_t sums_cap = 40ull << 30;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess && free_b / 3 < sums_cap) sums_cap = free_b / 3;
    if (const char *mb = std::getenv("LUMENWRIGHT_BATCH_SUMS_MB")) sums_cap = std::min<uint64_t>(sums_cap, std::strtoull(mb, nullptr, 10) << 20);
    const uint64_t max_items = sums_cap / sizeof(float4) > 0 ? sums_cap / sizeof(float4) : 1;
    uint64_t sub = (total_samples + max_items - 1) / max_items;
    sub = sub < 1 ? 1 : (sub > 64 ? 64 : sub);
    uint32_t passes = 1;
    if (c->tuning.engine == LW_ENGINE_WAVEFRONT && c->tuning.sub == 0) {
        passes = (uint32_t)std::min<uint64_t>((total_samples + max_items - 1) / max_items, 64);
        if (passes < 1) passes = 1;
        sub = 1;
    }
    if (c->tuning.sub) sub = c->tuning.sub;
    // Per pass and camera: the camera's share of the pass's items, item sums and samples.
    std::vector<DevJob> dj((size_t)n * passes);
    std::vector<uint32_t> ib((size_t)n * passes), sb(n);
    std::vector<uint64_t> pass_items(passes, 0), pass_samples(passes, 0);
    uint64_t slots = 0, pixels = 0, max_partials = 0;
    c->batch_out_off.assign(n, 0);
    for (uint32_t i = 0; i < n; i++) {
        const lw_params &p = jobs[i].params;
        c->batch_out_off[i] = (size_t)pixels;
        pixels += (uint64_t)p.frame[0] * p.frame[1];
    }
    for (uint32_t k = 0; k < passes; k++) {
        uint64_t items = 0, partials = 0;
        slots = 0;
        for (uint32_t i = 0; i < n; i++) {
            const lw_params &p = jobs[i].params;
            DevJob &J = dj[(size_t)k * n + i];
            J.P = dev_params(&p);
            J.sky = sky_dev[i];
            J.w = p.frame[0];
            J.h = p.frame[1];
            J.tiles_x = (J.w + 7) / 8;
            J.n_slots = J.tiles_x * ((J.h + 3) / 4) * 32u;
            // this pass's slice of the camera's samples
            const uint64_t s0 = (uint64_t)jobs[i].spp * k / passes, s1 = (uint64_t)jobs[i].spp * (k + 1) / passes;
            J.sample_start = jobs[i].sample_start + (uint32_t)s0;
            J.spp = (uint32_t)(s1 - s0);
            J.sub = J.spp == 0 ? 1u : (uint32_t)(sub < J.spp ? sub : J.spp);
            J.n_sub = (J.spp + J.sub - 1) / J.sub;
            J.item_begin = (uint32_t)items;
            J.slot_begin = (uint32_t)slots;
            J.partial_off = partials;
            J.acc = c->batch_acc.p;  // set below, once the accumulators are allocated
            J.out = nullptr;
            ib[(size_t)k * n + i] = J.item_begin;
            sb[i] = J.slot_begin;
            items += (uint64_t)J.n_slots * J.n_sub;
            slots += J.n_slots;
            partials += (uint64_t)J.n_slots * J.n_sub;
            pass_samples[k] += (uint64_t)J.w * J.h * J.spp;
        }
        if (items >= 0xFFFFFFFFull || slots >= 0xFFFFFFFFull)
            return fail(c, LW_ERR_INVALID_ARGUMENT, "a pass of the batch has %llu work items; at most 2^32 - 1 fit one launch",
                        (unsigned long long)items);
        pass_items[k] = items;
        max_partials = std::max(max_partials, partials);
    }
    CK(c, ensure(c->batch_acc, pixels), "allocating the accumulators");
    CK(c, ensure(c->batch_out, 3 * pixels), "allocating the images");
    CK(c, ensure(c->batch_partials, max_partials), "allocating the item sums");
    for (size_t q = 0; q < dj.size(); q++) {
        const size_t i = q % n;
        dj[q].acc = c->batch_acc.p + c->batch_out_off[i];
        dj[q].out = c->batch_out.p + 3 * c->batch_out_off[i];
    }
    CK(c, ensure(c->batch_jobs, dj.size()), "allocating the job table");
    CK(c, ensure(c->batch_item_begin, ib.size()), "allocating the job table");
    CK(c, ensure(c->batch_slot_begin, n), "allocating the job table");
    CK(c, cudaMemcpyAsync(c->batch_jobs.p, dj.data(), sizeof(DevJob) * dj.size(), cudaMemcpyHostToDevice, c->stream),
       "uploading jobs");
    CK(c, cudaMemcpyAsync(c->batch_item_begin.p, ib.data(), 4 * ib.size(), cudaMemcpyHostToDevice, c->stream),
       "uploading jobs");
    CK(c, cudaMemcpyAsync(c->batch_slot_begin.p, sb.data(), 4 * n, cudaMemcpyHostToDevice, c->stream), "uploading jobs");
    CK(c, cudaStreamSynchronize(c->stream), "uploading jobs");
    std::vector<BatchDesc> Bs(passes);
    for (uint32_t k = 0; k < passes; k++)
        Bs[k] = BatchDesc{c->batch_jobs.p + (size_t)k * n, c->batch_item_begin.p + (size_t)k * n, c->batch_slot_begin.p, n,
                          (uint32_t)pass_items[k], (uint32_t)slots, c->tuning.budget, c->counter.p, c->batch_partials.p,
                          c->cancel_word.p};
    const BatchDesc &B = Bs[0];
    c->batch_passes = passes;
    if (c->tuning.engine == LW_ENGINE_WAVEFRONT) {
        uint64_t most = *std::max_element(pass_samples.begin(), pass_samples.end());
        uint64_t most_items = *std::max_element(pass_items.begin(), pass_items.end());
        // A pass that gives each of 2^24 slots at least 32 samples runs in a pool of 2^24 (the C3
        // batch at its full spp: 627.8 Msamples/s against 621.5 in 2^23 slots).
        const uint32_t cap = most >= (uint64_t(32) << 24) ? 1u << 24 : 1u << 23;
        lw_status ws = batch_graph_wavefront(c, Bs, dj[0].P, pixels, wf_slots(c, most, most_items, cap));
        if (ws != LW_OK) return ws;
        c->batch_host.assign(jobs, jobs + n);
        c->batch_samples = total_samples;
        return LW_OK;
    }
    LaunchShape shape = batch_shape(c->device, (int)c->tuning.threads, c->tuning.budget != 0);
    // Clear, render, reduce: one CUDA graph, replayed by lw_batch_run.
    cudaGraph_t graph = nullptr;
    CK(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal), "starting the graph capture");
    cudaError_t e = cudaMemsetAsync(c->counter.p, 0, 4, c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->batch_acc.p, 0, sizeof(Accum) * pixels, c->stream);
    if (e == cudaSuccess) e = launch_render_batch(dev_scene(c), B, shape, c->stream);
    if (e == cudaSuccess) e = launch_reduce_batch(B, c->stream);
    cudaError_t e2 = cudaStreamEndCapture(c->stream, &graph);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&c->batch_graph, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_fail(c, e, "capturing the batch graph");
    c->batch_host.assign(jobs, jobs + n);
    c->batch_samples = total_samples;
    return LW_OK;
}

lw_status lw_batch_run(lw_ctx *c) {
    if (!c || !c->batch_graph) return fail(c, LW_ERR_INVALID_ARGUMENT, "no batch prepared");
    cudaSetDevice(c->device);
    lw_status s = begin_render(c);
    if (s != LW_OK) return s;
    CK(c, cudaEventRecord(c->ev_a, c->stream), "recording an event");
    CK(c, cudaGraphLaunch(c->batch_graph, c->stream), "launching the batch graph");
    CK(c, cudaEventRecord(c->ev_b, c->stream), "recording an event");
    c->stats.launches = 1;
    c->stats.samples = c->batch_samples;
    c->kernel_ms_base = 0.0;
    c->stats.kernel_ms = -1.0;
    return LW_OK;
}

lw_status lw_batch_read(lw_ctx *c) {
    if (!c || !c->batch_graph) return fail(c, LW_ERR_INVALID_ARGUMENT, "no batch prepared");
    cudaSetDevice(c->device);
    for (size_t i = 0; i < c->batch_host.size(); i++) {
        const lw_camera_job &j = c->batch_host[i];
        if (!j.out_rgb) continue;
        size_t n = (size_t)j.params.frame[0] * j.params.frame[1] * 3;
        CK(c, cudaMemcpyAsync(j.out_rgb, c->batch_out.p + 3 * c->batch_out_off[i], n * 4, cudaMemcpyDeviceToHost, c->stream),
           "reading an image");
    }
    WAIT(c, "reading the images");
    return check_cancelled(c);
}

lw_status lw_render_batch(lw_ctx *c, const lw_camera_job *jobs, uint32_t n) {
    lw_status s = lw_batch_prepare(c, jobs, n);
    if (s == LW_OK) s = lw_batch_run(c);
    if (s == LW_OK) s = lw_batch_read(c);
    return s;
}

lw_status lw_build_sky_cache(lw_ctx *c, const lw_params *params, uint32_t n, float *out) {
    if (!c || !params || !out || n == 0 || n > 8192) return fail(c, LW_ERR_INVALID_ARGUMENT, "bad argument");
    cudaSetDevice(c->device);
    size_t cnt = (size_t)(n + 1) * (n + 1) * 3;
    DBuf<float> buf;
    CK(c, ensure(buf, cnt), "allocating the sky cache");
    cudaError_t e = launch_sky_cache(dev_params(params), n, buf.p, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, buf.p, cnt * 4, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    buf.free_();
    if (e != cudaSuccess) return cuda_fail(c, e, "building the sky cache");
    return LW_OK;
}

lw_status lw_blend_chunky_sky(lw_ctx *c, const lw_params *params, const float *cache, uint64_t cache_len, float *maps,
                              const float sizes[4], float weight) {
    if (!c || !params || !cache || !maps || !sizes) return fail(c, LW_ERR_INVALID_ARGUMENT, "null argument");
    cudaSetDevice(c->device);
    double n = std::floor((double)params->misc_f[2]);
    if (n < 1.0 || (n + 1.0) * (n + 1.0) * 3.0 > (double)cache_len)
        return fail(c, LW_ERR_BUFFER_LENGTH, "the sky cache does not hold resolution %g", n);
    uint32_t lw_ = (uint32_t)sizes[0], lh = (uint32_t)sizes[1], gw = (uint32_t)sizes[2], gh = (uint32_t)sizes[3];
    if (!lw_ || !lh || !gw || !gh) return fail(c, LW_ERR_INVALID_ARGUMENT, "empty map");
    size_t nmap = ((size_t)lw_ * lh + (size_t)gw * gh) * 3;
    DBuf<float> cbuf, mbuf;
    CK(c, ensure(cbuf, cache_len), "allocating the sky cache");
    if (ensure(mbuf, nmap) != cudaSuccess) {
        cbuf.free_();
        return fail(c, LW_ERR_OUT_OF_MEMORY, "allocating the maps");
    }
    cudaError_t e = cudaMemcpyAsync(cbuf.p, cache, cache_len * 4, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(mbuf.p, maps, nmap * 4, cudaMemcpyHostToDevice, c->stream);
    DevScene S = dev_scene(c);
    S.sky = cbuf.p;
    DevParams P = dev_params(params);
    if (e == cudaSuccess) e = launch_blend_chunky(S, P, mbuf.p, lw_, lh, weight, c->stream);
    if (e == cudaSuccess) e = launch_blend_chunky(S, P, mbuf.p + (size_t)lw_ * lh * 3, gw, gh, weight, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(maps, mbuf.p, nmap * 4, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cbuf.free_();
    mbuf.free_();
    if (e != cudaSuccess) return cuda_fail(c, e, "blending the sky maps");
    return LW_OK;
}

lw_status lw_draw_sky_map(lw_ctx *c, const lw_quick_sky *q, const uint32_t *stars, uint64_t stars_len,
                          const uint32_t *atlas, uint64_t atlas_len, uint32_t atlas_w, uint32_t w, uint32_t h, float *out) {
    if (!c || !q || !stars || !atlas || !out || !w || !h || !atlas_w || w > 16384 || h > 16384)
        return fail(c, LW_ERR_INVALID_ARGUMENT, "bad argument");
    cudaSetDevice(c->device);
    // The star table: bin starts (non-decreasing) and an end, then 9 words per entry.
    const uint64_t nb = 128u * 64u;
    if (stars_len < nb + 1) return fail(c, LW_ERR_BUFFER_LENGTH, "the star table is shorter than its bins");
    for (uint64_t b = 0; b < nb; b++)
        if (stars[b + 1] < stars[b]) return fail(c, LW_ERR_BUFFER_LENGTH, "star bin %llu ends before it starts", (unsigned long long)b);
    if (nb + 1 + (uint64_t)stars[nb] * 9u > stars_len)
        return fail(c, LW_ERR_BUFFER_LENGTH, "the star table's bins name %u entries it does not hold", stars[nb]);
    // The sun's and moon's sprite rectangles: every texel the quads can read lies in the atlas.
    for (const float(*b)[4] : {q->sun, q->moon}) {
        if (b[0][3] == 0.0f || !(b[3][2] > 0.0f)) continue;
        const double x = b[3][0], y = b[3][1], bw = b[3][2], bh = b[3][3];
        if (!(x >= 0.0 && y >= 0.0 && bh >= 0.0) || std::floor(x + bw) >= (double)atlas_w ||
            std::floor(y + bh) * atlas_w + std::floor(x + bw) >= (double)atlas_len)
            return fail(c, LW_ERR_BUFFER_LENGTH, "a sprite rectangle (%g, %g, %g, %g) reaches outside the %ux%llu atlas", x, y,
                        bw, bh, atlas_w, (unsigned long long)(atlas_len / atlas_w));
    }
    DBuf<uint32_t> dstars, datlas;
    DBuf<float> dout;
    cudaError_t e = ensure(dstars, stars_len);
    if (e == cudaSuccess) e = ensure(datlas, atlas_len);
    if (e == cudaSuccess) e = ensure(dout, (size_t)w * h * 3);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dstars.p, stars, stars_len * 4, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(datlas.p, atlas, atlas_len * 4, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = launch_sky_map(q, datlas.p, atlas_w, dstars.p, w, h, dout.p, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout.p, (size_t)w * h * 12, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    dstars.free_();
    datlas.free_();
    dout.free_();
    if (e != cudaSuccess) return cuda_fail(c, e, "drawing the sky map");
    return LW_OK;
}

lw_status lw_rebase_camera(lw_params *p, const double eye[3]) {
    if (!p || !eye) return LW_ERR_INVALID_ARGUMENT;
    const int lo[3] = {-1024, -512, -1024}, hi[3] = {1023, 511, 1023};
    int k[3];
    float local[3];
    for (int a = 0; a < 3; a++) {
        if (!std::isfinite(eye[a])) return LW_ERR_INVALID_ARGUMENT;
        const double ch = std::nearbyint(eye[a] / 16.0);  // exact scaling, rounding to the nearest (ties to even)
        if (ch < lo[a] || ch > hi[a]) return LW_ERR_INVALID_ARGUMENT;
        k[a] = (int)ch;
        local[a] = (float)(eye[a] - 16.0 * ch);  // exact in f64, rounded once to f32
    }
    for (int a = 0; a < 3; a++) p->cam_pos[a] = local[a];
    p->see_through[2] = 1u;
    p->see_through[3] = ((uint32_t)k[0] & 0x7FFu) | (((uint32_t)k[1] & 0x3FFu) << 11) | (((uint32_t)k[2] & 0x7FFu) << 21);
    return LW_OK;
}

lw_status lw_gamma_table(float out[256]) {
    if (!out) return LW_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < 256; k++) out[k] = ref_gamma_to_linear((float)k / 255.0f);
    return LW_OK;
}

}  // extern "C"

namespace {

// Checks one frame of the differentiable form and copies its theta and sky to slot `k`. A null
// `n_params_out` demands the frame's parameter count equal *n_params_in.
lw_status adj_upload(lw_ctx *c, const lw_adj_frame *f, int k, AdjFrame &out, uint32_t *n_params) {
    if (!f || !f->params || !f->texel_param || !f->emitter_scale || !f->sky || (f->n_params && !f->albedo))
        return fail(c, LW_ERR_INVALID_ARGUMENT, "adjoint frame %d: null argument", k);
    lw_status s = check_params(c, f->params, true, f->sky_len);
    if (s != LW_OK) return s;
    if (f->params->see_through[2])
        return fail(c, LW_ERR_INVALID_ARGUMENT, "adjoint frame %d: the differentiable form renders in the grid's frame only", k);
    if (f->params->misc_f[2] >= 1.0f && f->params->sky_map[0] < 1.0f) {
        double n = std::floor((double)f->params->misc_f[2]);
        if ((n + 1.0) * (n + 1.0) * 3.0 > (double)f->sky_len) return fail(c, LW_ERR_BUFFER_LENGTH, "sky cache too short");
    }
    if (f->texel_param_len != c->atlas_len)
        return fail(c, LW_ERR_BUFFER_LENGTH, "texel_param has %llu entries, the atlas %llu texels",
                    (unsigned long long)f->texel_param_len, (unsigned long long)c->atlas_len);
    if (*n_params != UINT32_MAX && *n_params != f->n_params)
        return fail(c, LW_ERR_INVALID_ARGUMENT, "frames with %u and %u parameters", *n_params, f->n_params);
    *n_params = f->n_params;
    for (uint64_t i = 0; i < f->texel_param_len; i++)
        if (f->texel_param[i] < -1 || f->texel_param[i] >= (int64_t)f->n_params)
            return fail(c, LW_ERR_BUFFER_LENGTH, "texel_param[%llu] = %d outside [-1, %u)", (unsigned long long)i,
                        f->texel_param[i], f->n_params);
    CK(c, upload(c, c->adj_albedo[k], f->albedo, (size_t)f->n_params * 3, 4), "uploading the albedo parameters");
    CK(c, upload(c, c->adj_tparam[k], f->texel_param, f->texel_param_len, 4), "uploading the texel parameters");
    CK(c, upload(c, c->adj_emit[k], f->emitter_scale, LW_EMITTER_GROUPS, 4), "uploading the emitter intensities");
    CK(c, upload(c, c->adj_sky[k], f->sky, f->sky_len, 4), "uploading the sky");
    out.P = dev_params(f->params);
    out.sky = c->adj_sky[k].p;
    out.albedo = c->adj_albedo[k].p;
    out.texel_param = c->adj_tparam[k].p;
    out.emit_mult = c->adj_emit[k].p;
    return LW_OK;
}

// A 64-bit digest of a frame of the differentiable form and its spp (the key of the kept
// per-sample radiance): every input byte through a multiply-xorshift mix.
uint64_t mix_bytes(uint64_t h, const void *p, uint64_t n) {
    const unsigned char *b = (const unsigned char *)p;
    uint64_t i = 0;
    for (; i + 8 <= n; i += 8) {
        uint64_t w;
        std::memcpy(&w, b + i, 8);
        h = (h ^ w) * 0x9E3779B97F4A7C15ull;
        h ^= h >> 29;
    }
    for (; i < n; i++) h = ((h ^ b[i]) * 0x100000001B3ull) ^ (h >> 31);
    return h ^ n;
}
uint64_t adj_key(const lw_adj_frame *f, uint32_t spp) {
    uint64_t h = 0x243F6A8885A308D3ull ^ spp;
    h = mix_bytes(h, f->params, sizeof(lw_params));
    h = mix_bytes(h, f->sky, f->sky_len * 4);
    h = mix_bytes(h, f->albedo, (uint64_t)f->n_params * 12);
    h = mix_bytes(h, f->texel_param, f->texel_param_len * 4);
    h = mix_bytes(h, f->emitter_scale, LW_EMITTER_GROUPS * 4);
    return h ? h : 1u;
}

lw_status adj_begin(lw_ctx *c) {
    if (!c) return LW_ERR_INVALID_ARGUMENT;
    if (!c->has_scene) return fail(c, LW_ERR_NO_SCENE, "no scene uploaded");
    cudaSetDevice(c->device);
    return LW_OK;
}

lw_status adj_timed(lw_ctx *c, cudaError_t (*launch)(lw_ctx *, void *), void *arg, uint64_t samples) {
    CK(c, cudaEventRecord(c->ev_a, c->stream), "recording an event");
    CK(c, launch(c, arg), "launching the adjoint kernel");
    CK(c, cudaEventRecord(c->ev_b, c->stream), "recording an event");
    {
        lw_status ws = wait_event(c, c->ev_b, "running the adjoint kernel");
        if (ws != LW_OK) return ws;
    }
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, c->ev_a, c->ev_b);
    c->stats.kernel_ms = ms;
    c->stats.launches = 1;
    c->stats.samples = samples;
    return LW_OK;
}

}  // namespace

extern "C" {

lw_status lw_adjoint_forward(lw_ctx *c, const lw_adj_frame *frame, uint32_t spp, double *out_rgb) {
    lw_status s = adj_begin(c);
    if (s != LW_OK) return s;
    if (!out_rgb || !spp) return fail(c, LW_ERR_INVALID_ARGUMENT, "bad argument");
    AdjFrame F;
    uint32_t np = UINT32_MAX;
    if ((s = adj_upload(c, frame, 0, F, &np)) != LW_OK) return s;
    size_t n = (size_t)F.P.frame.x * F.P.frame.y * 3;
    CK(c, ensure(c->adj_img, n), "allocating the image");
    CK(c, cudaMemsetAsync(c->adj_img.p, 0, n * 8, c->stream), "clearing the image");
    // Each sample's radiance is kept for a backward pass over the same inputs (up to 4 GiB).
    const uint64_t kept = (uint64_t)n / 3 * spp * 3;
    double *Ls = nullptr;
    c->adj_L_key = 0;
    if (kept * 8 <= (uint64_t(4) << 30) && ensure(c->adj_L, kept) == cudaSuccess) Ls = c->adj_L.p;
    struct A { DevScene S; AdjFrame F; uint32_t spp; double *img, *Ls; } a{dev_scene(c), F, spp, c->adj_img.p, Ls};
    s = adj_timed(c, [](lw_ctx *cc, void *p) {
        A &x = *(A *)p;
        return launch_adj_forward(x.S, x.F, x.spp, x.img, x.Ls, cc->stream);
    }, &a, (uint64_t)n / 3 * spp);
    if (s == LW_OK && Ls) c->adj_L_key = adj_key(frame, spp);
    if (s != LW_OK) return s;
    CK(c, cudaMemcpy(out_rgb, c->adj_img.p, n * 8, cudaMemcpyDeviceToHost), "reading the image");
    return LW_OK;
}

lw_status lw_adjoint_backward(lw_ctx *c, const lw_adj_frame *frame, uint32_t spp, const double *d_rgb, lw_gradient *out) {
    lw_status s = adj_begin(c);
    if (s != LW_OK) return s;
    if (!d_rgb || !out || !spp || !out->emitter_scale || !out->sky || (frame && frame->n_params && !out->albedo))
        return fail(c, LW_ERR_INVALID_ARGUMENT, "bad argument");
    AdjFrame F;
    uint32_t np = UINT32_MAX;
    if ((s = adj_upload(c, frame, 0, F, &np)) != LW_OK) return s;
    size_t n = (size_t)F.P.frame.x * F.P.frame.y * 3;
    size_t ng = (size_t)np * 3 + LW_EMITTER_GROUPS + frame->sky_len + 3;
    CK(c, ensure(c->adj_img, n), "allocating the image gradient");
    CK(c, ensure(c->adj_g, ng), "allocating the gradient");
    CK(c, cudaMemcpyAsync(c->adj_img.p, d_rgb, n * 8, cudaMemcpyHostToDevice, c->stream), "uploading the image gradient");
    CK(c, cudaMemsetAsync(c->adj_g.p, 0, ng * 8, c->stream), "clearing the gradient");
    AdjGrad G;
    G.albedo = c->adj_g.p;
    G.emit = G.albedo + (size_t)np * 3;
    G.cache = G.emit + LW_EMITTER_GROUPS;
    G.sun = G.cache + frame->sky_len;
    // The forward pass's per-sample radiance, when it was over these very inputs, replaces replay 1.
    const double *Ls = c->adj_L_key && c->adj_L_key == adj_key(frame, spp) ? c->adj_L.p : nullptr;
    struct A { DevScene S; AdjFrame F; uint32_t spp; const double *d; AdjGrad G; const double *Ls; } a{
        dev_scene(c), F, spp, c->adj_img.p, G, Ls};
    s = adj_timed(c, [](lw_ctx *cc, void *p) {
        A &x = *(A *)p;
        return launch_adj_backward(x.S, x.F, x.spp, x.d, x.G, x.Ls, cc->stream);
    }, &a, (uint64_t)n / 3 * spp * (Ls ? 1u : 2u));
    if (s != LW_OK) return s;
    if (np) CK(c, cudaMemcpy(out->albedo, G.albedo, (size_t)np * 3 * 8, cudaMemcpyDeviceToHost), "reading the gradient");
    CK(c, cudaMemcpy(out->emitter_scale, G.emit, LW_EMITTER_GROUPS * 8, cudaMemcpyDeviceToHost), "reading the gradient");
    CK(c, cudaMemcpy(out->sky, G.cache, frame->sky_len * 8, cudaMemcpyDeviceToHost), "reading the gradient");
    CK(c, cudaMemcpy(out->sun_dir, G.sun, 3 * 8, cudaMemcpyDeviceToHost), "reading the gradient");
    return LW_OK;
}

lw_status lw_adjoint_fd(lw_ctx *c, const lw_adj_frame *plus, const lw_adj_frame *minus, const lw_adj_frame *nominal,
                        uint32_t spp, double *diff_rgb, double *mean_rgb) {
    lw_status s = adj_begin(c);
    if (s != LW_OK) return s;
    if (!diff_rgb || !mean_rgb || !spp) return fail(c, LW_ERR_INVALID_ARGUMENT, "bad argument");
    AdjFrame Fp, Fm, F0;
    uint32_t np = UINT32_MAX;
    if ((s = adj_upload(c, plus, 0, Fp, &np)) != LW_OK) return s;
    if ((s = adj_upload(c, minus, 1, Fm, &np)) != LW_OK) return s;
    if ((s = adj_upload(c, nominal, 2, F0, &np)) != LW_OK) return s;
    for (int k = 0; k < 2; k++)
        if (Fm.P.frame.x != Fp.P.frame.x || Fm.P.frame.y != Fp.P.frame.y || F0.P.frame.x != Fp.P.frame.x ||
            F0.P.frame.y != Fp.P.frame.y)
            return fail(c, LW_ERR_INVALID_ARGUMENT, "the frames differ in size");
    size_t n = (size_t)Fp.P.frame.x * Fp.P.frame.y * 3;
    CK(c, ensure(c->adj_img, n), "allocating the differences");
    CK(c, ensure(c->adj_img2, n), "allocating the means");
    CK(c, cudaMemsetAsync(c->adj_img.p, 0, n * 8, c->stream), "clearing the differences");
    CK(c, cudaMemsetAsync(c->adj_img2.p, 0, n * 8, c->stream), "clearing the means");
    struct A { DevScene S; AdjFrame Fp, Fm; const float *a0; float4 sun0; uint32_t spp; double *d, *m; } a{
        dev_scene(c), Fp, Fm, F0.albedo, F0.P.sun_dir, spp, c->adj_img.p, c->adj_img2.p};
    s = adj_timed(c, [](lw_ctx *cc, void *p) {
        A &x = *(A *)p;
        return launch_adj_fd(x.S, x.Fp, x.Fm, x.a0, x.sun0, x.spp, x.d, x.m, cc->stream);
    }, &a, (uint64_t)n / 3 * spp * 2);
    if (s != LW_OK) return s;
    CK(c, cudaMemcpy(diff_rgb, c->adj_img.p, n * 8, cudaMemcpyDeviceToHost), "reading the differences");
    CK(c, cudaMemcpy(mean_rgb, c->adj_img2.p, n * 8, cudaMemcpyDeviceToHost), "reading the means");
    return LW_OK;
}

lw_status lw_tonemap_rgba(lw_ctx *c, const float *hdr, uint64_t n, const lw_tonemap *tm, uint32_t *out_rgba) {
    if (!c || !hdr || !out_rgba) return fail(c, LW_ERR_INVALID_ARGUMENT, "null argument");
    if (n == 0) return LW_OK;
    if (n > 0xFFFFFFFFull / 3u) return fail(c, LW_ERR_INVALID_ARGUMENT, "%llu pixels", (unsigned long long)n);
    cudaSetDevice(c->device);
    TonemapDesc t;
    lw_status s = tonemap_desc(c, tm, t);
    if (s != LW_OK) return s;
    CK(c, ensure(c->out_rgb, 3 * n), "allocating the pixels");
    CK(c, ensure(c->out_rgba, n), "allocating the pixels");
    CK(c, cudaMemcpyAsync(c->out_rgb.p, hdr, 12 * n, cudaMemcpyHostToDevice, c->stream), "uploading the pixels");
    CK(c, launch_tonemap(c->out_rgb.p, (uint32_t)n, t, c->out_rgba.p, c->stream), "launching the tone map");
    CK(c, cudaMemcpyAsync(out_rgba, c->out_rgba.p, 4 * n, cudaMemcpyDeviceToHost, c->stream), "reading the pixels");
    CK(c, cudaStreamSynchronize(c->stream), "reading the pixels");
    return LW_OK;
}

lw_status lw_read_accumulator_rgba(lw_ctx *c, const lw_tonemap *tm, uint32_t *out_rgba, float *out_rgb) {
    if (!c || !out_rgba) return fail(c, LW_ERR_INVALID_ARGUMENT, "null argument");
    cudaSetDevice(c->device);
    TonemapDesc t;
    lw_status s = tonemap_desc(c, tm, t);
    if (s != LW_OK) return s;
    size_t n = (size_t)c->acc_w * c->acc_h;
    if (n == 0) return fail(c, LW_ERR_INVALID_ARGUMENT, "no accumulator");
    CK(c, ensure(c->out_rgba, n), "allocating the pixels");
    if (out_rgb) CK(c, ensure(c->out_rgb, 3 * n), "allocating the output");
    CK(c, launch_finalize_tonemap(c->acc.p, (uint32_t)n, t, c->out_rgba.p, out_rgb ? c->out_rgb.p : nullptr, c->stream),
       "launching the display pass");
    CK(c, cudaMemcpyAsync(out_rgba, c->out_rgba.p, 4 * n, cudaMemcpyDeviceToHost, c->stream), "reading the pixels");
    if (out_rgb)
        CK(c, cudaMemcpyAsync(out_rgb, c->out_rgb.p, 12 * n, cudaMemcpyDeviceToHost, c->stream), "reading the image");
    WAIT(c, "reading the pixels");
    return check_cancelled(c);
}

static lw_status world_check(lw_ctx *c, const lw_world_desc *w) {
    if (!w || !w->blocks || !w->state_flags) return fail(c, LW_ERR_INVALID_ARGUMENT, "null argument");
    for (int a = 0; a < 3; a++)
        if (w->size[a] == 0 || w->size[a] % 16u || w->size[a] > (1u << 16))
            return fail(c, LW_ERR_INVALID_ARGUMENT, "volume size %u (a multiple of 16, at most 65536)", w->size[a]);
    if ((uint64_t)w->size[0] * w->size[1] * w->size[2] > 0xFFFFFFFFull)
        return fail(c, LW_ERR_INVALID_ARGUMENT, "volume of more than 2^32 voxels");
    if (w->n_states == 0 || w->n_states > 65536u) return fail(c, LW_ERR_INVALID_ARGUMENT, "%u states", w->n_states);
    return LW_OK;
}

static BuildVol build_vol(lw_ctx *c, const lw_world_desc *w) {
    return BuildVol{c->bv_blocks.p, {w->size[0], w->size[1], w->size[2]}, c->bv_flags.p, w->n_states, c->error.p};
}

lw_status lw_scene_build_keys(lw_ctx *c, const lw_world_desc *w, uint32_t *keys, uint32_t cap, uint32_t *n_keys) {
    if (!c || !n_keys) return fail(c, LW_ERR_INVALID_ARGUMENT, "null argument");
    lw_status s = world_check(c, w);
    if (s != LW_OK) return s;
    cudaSetDevice(c->device);
    auto t0 = std::chrono::steady_clock::now();
    const uint64_t n = (uint64_t)w->size[0] * w->size[1] * w->size[2];
    const uint64_t nk = (uint64_t)w->n_states * 256u;
    CK(c, upload(c, c->bv_blocks, w->blocks, n, 2), "uploading the blocks");
    CK(c, upload(c, c->bv_flags, w->state_flags, w->n_states, 1), "uploading the state flags");
    CK(c, ensure(c->bv_keys, n), "allocating the keys");
    CK(c, ensure(c->bv_first, nk), "allocating the key table");
    CK(c, cudaMemsetAsync(c->bv_first.p, 0xFF, nk * 4, c->stream), "clearing the key table");
    CK(c, cudaMemsetAsync(c->error.p, 0, 4, c->stream), "clearing the error word");
    CK(c, launch_keys_first(build_vol(c, w), c->bv_keys.p, c->bv_first.p, c->stream), "launching the key pass");
    std::vector<uint32_t> first(nk);
    uint32_t err = 0;
    CK(c, cudaMemcpyAsync(first.data(), c->bv_first.p, nk * 4, cudaMemcpyDeviceToHost, c->stream), "reading the key table");
    CK(c, cudaMemcpyAsync(&err, c->error.p, 4, cudaMemcpyDeviceToHost, c->stream), "reading the error word");
    CK(c, cudaStreamSynchronize(c->stream), "finding the keys");
    if (err) return fail(c, LW_ERR_BUFFER_LENGTH, "a voxel names a state beyond the %u states", w->n_states);
    std::vector<std::pair<uint32_t, uint32_t>> present;  // (first position, key)
    for (uint64_t k = 1; k < nk; k++)
        if (first[k] != 0xFFFFFFFFu) present.push_back({first[k], (uint32_t)k});
    std::sort(present.begin(), present.end());
    if (present.size() > 65535u) return fail(c, LW_ERR_INVALID_ARGUMENT, "more than 65535 distinct block model instances");
    c->bv_order.clear();
    for (auto &p : present) c->bv_order.push_back(p.second);
    std::memcpy(c->bv_size, w->size, sizeof c->bv_size);
    c->bv_states = w->n_states;
    *n_keys = (uint32_t)c->bv_order.size();
    if (keys) {
        if (cap < *n_keys) return fail(c, LW_ERR_BUFFER_LENGTH, "%u keys, room for %u", *n_keys, cap);
        std::memcpy(keys, c->bv_order.data(), 4 * (size_t)*n_keys);
    }
    c->stats.upload_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return LW_OK;
}

lw_status lw_scene_build_grid(lw_ctx *c, const lw_world_desc *w, const lw_instances_desc *in, lw_build_info *info) {
    if (!c || !in || !in->models || !in->quads || !in->model_emits || !in->atlas)
        return fail(c, LW_ERR_INVALID_ARGUMENT, "null argument");
    lw_status s = world_check(c, w);
    if (s != LW_OK) return s;
    if (std::memcmp(c->bv_size, w->size, sizeof c->bv_size) != 0 || c->bv_states != w->n_states)
        return fail(c, LW_ERR_INVALID_ARGUMENT, "call lw_scene_build_keys for this volume first");
    if (in->models_len != c->bv_order.size() + 1)
        return fail(c, LW_ERR_BUFFER_LENGTH, "%llu models for %zu keys (and air)", (unsigned long long)in->models_len,
                    c->bv_order.size());
    cudaSetDevice(c->device);
    auto t0 = std::chrono::steady_clock::now();
    c->has_scene = false;
    const uint32_t dims[3] = {w->size[0] / 16u, w->size[1] / 16u, w->size[2] / 16u};
    const uint32_t nb = dims[0] * dims[1] * dims[2];
    const uint64_t n = (uint64_t)w->size[0] * w->size[1] * w->size[2];
    const uint64_t nk = (uint64_t)w->n_states * 256u;
    // instance ids per key, emitting instances
    std::vector<uint32_t> key_id(nk, 0u);
    for (size_t i = 0; i < c->bv_order.size(); i++) key_id[c->bv_order[i]] = (uint32_t)i + 1u;
    CK(c, upload(c, c->bv_key_id, key_id.data(), nk, 4), "uploading the instance ids");
    CK(c, upload(c, c->bv_emits, in->model_emits, in->models_len, 1), "uploading the emitting instances");
    CK(c, ensure(c->bv_ids, n), "allocating the ids");
    CK(c, ensure(c->bv_cls, nb), "allocating the brick classes");
    BuildVol v = build_vol(c, w);
    CK(c, launch_bricks_scan(v, c->bv_keys.p, c->bv_key_id.p, c->bv_emits.p, c->bv_ids.p, c->bv_cls.p, nb, c->stream),
       "launching the brick pass");
    std::vector<uint4> cls(nb);
    CK(c, cudaMemcpyAsync(cls.data(), c->bv_cls.p, (size_t)nb * 16, cudaMemcpyDeviceToHost, c->stream), "reading the bricks");
    CK(c, cudaStreamSynchronize(c->stream), "classifying the bricks");
    // voxel.rs:345-392: buried (all occluding, every face neighbour inside and all occluding),
    // uniform, or stored; emitter sites of every brick in brick order.
    auto all_occ = [&](int64_t bx, int64_t by, int64_t bz) -> bool {
        if (bx < 0 || by < 0 || bz < 0 || bx >= dims[0] || by >= dims[1] || bz >= dims[2]) return false;
        return (cls[(by * dims[2] + bz) * dims[0] + bx].x & 2u) != 0u;
    };
    std::vector<uint32_t> top(nb, 0xFFFFFFFFu), slot(nb, 0xFFFFFFFFu), emit_off(nb, 0u);
    uint32_t n_bricks = 0, n_uniform = 0, n_buried = 0, n_emit = 0;
    for (uint32_t b = 0; b < nb; b++) {
        emit_off[b] = n_emit;
        n_emit += cls[b].w;
        if (!(cls[b].x & 1u)) continue;
        int64_t bx = b % dims[0], bz = (b / dims[0]) % dims[2], by = b / (dims[0] * dims[2]);
        bool buried = (cls[b].x & 2u) && all_occ(bx, by - 1, bz) && all_occ(bx, by + 1, bz) && all_occ(bx, by, bz - 1) &&
                      all_occ(bx, by, bz + 1) && all_occ(bx - 1, by, bz) && all_occ(bx + 1, by, bz);
        if (buried) {
            top[b] = UNIFORM | (cls[b].z ? cls[b].z : 1u);
            n_buried++;
        } else if (cls[b].x & 4u) {
            top[b] = UNIFORM | cls[b].y;
            n_uniform++;
        } else {
            top[b] = n_bricks;
            slot[b] = n_bricks++;
        }
    }
    // The grid: top | bricks | ov_top (no overlay) | a final 0 word.
    const uint64_t grid_len = (uint64_t)nb + (uint64_t)n_bricks * 2048u + nb + 1u;
    if (grid_len > 0xFFFFFFFFull) return fail(c, LW_ERR_INVALID_ARGUMENT, "grid of %llu words", (unsigned long long)grid_len);
    CK(c, ensure(c->grid, grid_len), "allocating the grid");
    CK(c, cudaMemcpyAsync(c->grid.p, top.data(), (size_t)nb * 4, cudaMemcpyHostToDevice, c->stream), "uploading the top level");
    CK(c, cudaMemsetAsync(c->grid.p + nb + (size_t)n_bricks * 2048u, 0xFF, (size_t)nb * 4, c->stream), "writing ov_top");
    CK(c, cudaMemsetAsync(c->grid.p + grid_len - 1, 0, 4, c->stream), "writing the last word");
    CK(c, upload(c, c->bv_slot, slot.data(), nb, 4), "uploading the brick slots");
    CK(c, upload(c, c->bv_emit_off, emit_off.data(), nb, 4), "uploading the emitter offsets");
    CK(c, ensure(c->bv_sites, n_emit ? n_emit : 1), "allocating the emitter sites");
    CK(c, launch_bricks_pack(v, c->bv_ids.p, c->bv_emits.p, c->bv_slot.p, c->bv_emit_off.p, c->grid.p + nb, c->bv_sites.p, nb,
                             c->stream), "launching the packing pass");
    std::vector<uint4> sites(n_emit);
    if (n_emit)
        CK(c, cudaMemcpyAsync(sites.data(), c->bv_sites.p, (size_t)n_emit * 16, cudaMemcpyDeviceToHost, c->stream),
           "reading the emitter sites");
    CK(c, cudaStreamSynchronize(c->stream), "packing the bricks");
    // emitter_list (voxel.rs:542-607): one emitter per site; the grid of 10-block cells, each
    // listing the emitters within one cell of it (27 neighbours), emitters in site order.
    const int64_t CELL = 10;
    std::vector<lw_emitter> em(n_emit ? n_emit : 1);
    std::vector<uint32_t> eg;
    if (n_emit == 0) {
        std::memset(em.data(), 0, sizeof(lw_emitter));
        eg.assign(8, 0u);
        eg[0] = (uint32_t)CELL;
    } else {
        int64_t lo[3] = {INT64_MAX, INT64_MAX, INT64_MAX}, hi[3] = {INT64_MIN, INT64_MIN, INT64_MIN};
        std::vector<int64_t> g(3 * (size_t)n_emit);
        for (uint32_t i = 0; i < n_emit; i++) {
            const uint32_t cc[3] = {sites[i].x, sites[i].y, sites[i].z};
            lw_emitter &e = em[i];
            std::memset(&e, 0, sizeof e);
            for (int a = 0; a < 3; a++) e.pos[a] = (float)cc[a];
            uint32_t off = in->models[sites[i].w].quad_offset;
            std::memcpy(&e.pos[3], &off, 4);
            e.faces[0] = in->models[sites[i].w].quad_count;
            for (int a = 0; a < 3; a++) {
                int64_t q = (int64_t)cc[a] / CELL;  // corners are non-negative: floor division
                g[3 * (size_t)i + a] = q;
                lo[a] = std::min(lo[a], q);
                hi[a] = std::max(hi[a], q);
            }
        }
        int64_t offset[3], size[3];
        for (int a = 0; a < 3; a++) {
            offset[a] = lo[a] - 1;
            size[a] = hi[a] - lo[a] + 3;
        }
        const uint64_t ncells = (uint64_t)size[0] * size[1] * size[2];
        std::vector<uint32_t> counts(ncells, 0u);
        auto cell = [&](uint32_t i, int dx, int dy, int dz) -> uint64_t {
            int64_t l0 = g[3 * (size_t)i] + dx - offset[0], l1 = g[3 * (size_t)i + 1] + dy - offset[1],
                    l2 = g[3 * (size_t)i + 2] + dz - offset[2];
            return (uint64_t)((l1 * size[2] + l2) * size[0] + l0);
        };
        for (uint32_t i = 0; i < n_emit; i++)
            for (int dy = -1; dy <= 1; dy++)
                for (int dz = -1; dz <= 1; dz++)
                    for (int dx = -1; dx <= 1; dx++) counts[cell(i, dx, dy, dz)]++;
        std::vector<uint32_t> start(ncells, 0u), fill(ncells, 0u);
        uint64_t acc = 0;
        for (uint64_t k = 0; k < ncells; k++) {
            start[k] = (uint32_t)acc;
            acc += counts[k];
        }
        eg.assign(8 + 2 * ncells + acc, 0u);
        eg[0] = (uint32_t)CELL;
        for (int a = 0; a < 3; a++) {
            eg[1 + a] = (uint32_t)size[a];
            eg[4 + a] = (uint32_t)(int32_t)offset[a];
        }
        for (uint64_t k = 0; k < ncells; k++) {
            eg[8 + 2 * k] = start[k];
            eg[9 + 2 * k] = counts[k];
        }
        // per cell, emitters in site order: sites are visited in order
        for (uint32_t i = 0; i < n_emit; i++)
            for (int dy = -1; dy <= 1; dy++)
                for (int dz = -1; dz <= 1; dz++)
                    for (int dx = -1; dx <= 1; dx++) {
                        uint64_t k = cell(i, dx, dy, dz);
                        eg[8 + 2 * ncells + start[k] + fill[k]++] = i;
                    }
    }
    lw_scene_desc d{};
    d.grid = nullptr;
    d.grid_len = grid_len;
    d.models = in->models;
    d.models_len = in->models_len;
    d.quads = in->quads;
    d.quads_len = in->quads_len;
    d.atlas = in->atlas;
    d.atlas_len = in->atlas_len;
    d.emitters = em.data();
    d.emitters_len = em.size();
    d.emitter_grid = eg.data();
    d.emitter_grid_len = eg.size();
    std::memcpy(d.dims, dims, sizeof dims);
    const uint32_t off_ov_top = nb + n_bricks * 2048u;
    const uint32_t offs[5] = {0u, nb, off_ov_top, off_ov_top + nb, off_ov_top + nb};
    std::memcpy(d.offsets, offs, sizeof offs);
    d.atlas_size[0] = in->atlas_size[0];
    d.atlas_size[1] = in->atlas_size[1];
    if ((uint64_t)in->atlas_size[0] * in->atlas_size[1] > in->atlas_len || !in->atlas_size[0] || !in->atlas_size[1])
        return fail(c, LW_ERR_BUFFER_LENGTH, "atlas size");
    for (uint64_t i = 0; i < in->models_len; i++)
        if ((uint64_t)in->models[i].quad_offset + in->models[i].quad_count > in->quads_len)
            return fail(c, LW_ERR_BUFFER_LENGTH, "model %llu's quads outside the quads", (unsigned long long)i);
    s = install_scene(c, &d, n_bricks, 0u);
    if (s != LW_OK) return s;
    if (info) {
        std::memcpy(info->dims, dims, sizeof dims);
        std::memcpy(info->offsets, offs, sizeof offs);
        info->grid_len = grid_len;
        info->emitter_grid_len = eg.size();
        info->bricks = n_bricks;
        info->uniform_bricks = n_uniform;
        info->buried_bricks = n_buried;
        info->emitters = n_emit;
        info->keys_ms = c->stats.upload_ms;
        info->grid_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return LW_OK;
}

lw_status lw_scene_read(lw_ctx *c, uint32_t *grid, uint64_t grid_cap, lw_emitter *emitters, uint64_t emitters_cap,
                        uint32_t *egrid, uint64_t egrid_cap) {
    if (!c) return LW_ERR_INVALID_ARGUMENT;
    if (!c->has_scene) return fail(c, LW_ERR_NO_SCENE, "no scene");
    cudaSetDevice(c->device);
    if ((grid && grid_cap < c->grid_len) || (emitters && emitters_cap < c->emitters_len) || (egrid && egrid_cap < c->egrid_len))
        return fail(c, LW_ERR_BUFFER_LENGTH, "the scene holds %llu grid words, %llu emitters, %llu emitter-grid words",
                    (unsigned long long)c->grid_len, (unsigned long long)c->emitters_len, (unsigned long long)c->egrid_len);
    if (grid) CK(c, cudaMemcpy(grid, c->grid.p, c->grid_len * 4, cudaMemcpyDeviceToHost), "reading the grid");
    if (emitters) CK(c, cudaMemcpy(emitters, c->emitters.p, c->emitters_len * 32, cudaMemcpyDeviceToHost), "reading the emitters");
    if (egrid) CK(c, cudaMemcpy(egrid, c->egrid.p, c->egrid_len * 4, cudaMemcpyDeviceToHost), "reading the emitter grid");
    return LW_OK;
}

}  // extern "C"
