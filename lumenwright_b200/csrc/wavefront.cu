// The wavefront form of the render: the persistent megakernel's lanes wait, at every ray, for the
// longest traversal of their warp (traversal lengths are heavy-tailed: a ray along the terrain
// visits hundreds of voxels, most visit a few). Here the path state lives in a pool of slots in
// device memory and each iteration runs two kernels:
//   k_wf_shade  one thread per slot: the state machine of device_path.cuh on the slot's last hit
//               (or a new item), up to the slot's next ray, whose slot id it appends to the queue;
//   k_wf_trace  a small persistent kernel: each lane takes the next queued ray as soon as its
//               current one is done (dynamic fetch, a few voxel visits between fetches), so the
//               warps stay full until the queue runs dry.
// Items, samples per item and the order of every Kahan addition are the megakernel's, so the
// partial sums and the image are bit-identical to it.
#include "device_path.cuh"
#include "internal.h"

namespace lw {
namespace {

// Queue entries a warp takes from the fetch counter at a time (one atomic per 32 rays, not per
// round); at least 32, the most a warp can need at once.
constexpr uint32_t kFetchChunk = 32u;
// Lanes of a warp without a ray take new ones once at least this many of them wait (or no lane has
// work left): fewer fetch phases, each with more lanes (-1 % tracing time at c2 and c4; 16 is
// slower).
#ifndef LW_FETCH_MIN
#define LW_FETCH_MIN 8
#endif
constexpr int kTraceThreads = 128;  // threads per block of the tracing kernel

enum : uint32_t { F_ACTIVE = 1u, F_DEAD = 2u };
// hit0.y of a slot whose ray is still being traversed (carried over to the next iteration).
constexpr uint32_t RESUME_MARK = 0xFFFFFFFEu;

// Slot words (float4, word k of slot i at state[k * n + i]). The core words are read and written
// at every shading step; the next-event words only while a shadow or emitter ray is on its way
// (before a step whose ray was one, after a step that queues one); the item words only when a
// sample ends.
enum {
    W_O = 0,       // o.xyz, tmin
    W_D = 1,       // d.xyz, tmax
    W_RAD = 2,     // radiance.xyz, kind
    W_BETA = 3,    // beta.xyz, rng
    W_CORE = 4,    // bounces, events, specular | in_water << 1, flags (F_ACTIVE, F_DEAD)
    W_N = 5,       // n.xyz, cos_l          (next-event words)
    W_ORIGIN = 6,  // origin.xyz, seg
    W_TR = 7,      // tr.xyz, dist
    W_ESUM = 8,    // esum.xyz, list
    W_FSUM = 9,    // fsum.xyz, count
    W_EOFF = 10,   // eoff.xyz, k
    W_E1 = 11,     // first, faces, f, emode | fmode << 1
    W_ITEM = 12,   // px, py, sample, s_end (item words)
    W_ITEM2 = 13,  // j, pixel slot, camera (batched form), -
    W_SUM = 14,    // s0, s1, s2, c0
    W_SUM2 = 15,   // c1, c2, -, -
};

static_assert(W_ITEM2 == kWfItemCameraWord, "the word the batched form clears");

LW_DI float4 ld(const WfState &F, int k, uint32_t i) { return F.state[(size_t)k * F.n + i]; }
LW_DI void st(const WfState &F, int k, uint32_t i, float4 v) { F.state[(size_t)k * F.n + i] = v; }
LW_DI float4 pk(V3 a, float w) { return make_float4(a.x, a.y, a.z, w); }
LW_DI float4 pku(V3 a, uint32_t w) { return make_float4(a.x, a.y, a.z, __uint_as_float(w)); }
LW_DI float4 u4(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    return make_float4(__uint_as_float(a), __uint_as_float(b), __uint_as_float(c), __uint_as_float(d));
}
LW_DI uint32_t fu(float x) { return __float_as_uint(x); }

LW_DI void unpack_core(Path &p, float4 a, float4 b, float4 c, float4 d, float4 core) {
    p.o = f4v(a);
    p.tmin = a.w;
    p.d = f4v(b);
    p.tmax = b.w;
    p.radiance = f4v(c);
    p.kind = fu(c.w);
    p.beta = f4v(d);
    p.rng = fu(d.w);
    p.bounces = fu(core.x);
    p.events = fu(core.y);
    p.specular = (fu(core.z) & 1u) != 0u;
    p.in_water = (fu(core.z) & 2u) != 0u;
}

LW_DI void load_nee(const WfState &F, uint32_t i, Path &p) {
    float4 a = ld(F, W_N, i), b = ld(F, W_ORIGIN, i), c = ld(F, W_TR, i), d = ld(F, W_ESUM, i);
    p.n = f4v(a);
    p.cos_l = a.w;
    p.origin = f4v(b);
    p.seg = fu(b.w);
    p.tr = f4v(c);
    p.dist = c.w;
    p.esum = f4v(d);
    p.list = fu(d.w);
    a = ld(F, W_FSUM, i), b = ld(F, W_EOFF, i), c = ld(F, W_E1, i);
    p.fsum = f4v(a);
    p.count = fu(a.w);
    p.eoff = f4v(b);
    p.k = fu(b.w);
    p.first = fu(c.x);
    p.faces = fu(c.y);
    p.f = fu(c.z);
    p.emode = fu(c.w) & 1u;
    p.fmode = fu(c.w) >> 1;
}

LW_DI void store_core(const WfState &F, uint32_t i, const Path &p, uint32_t flags) {
    st(F, W_O, i, pk(p.o, p.tmin));
    st(F, W_D, i, pk(p.d, p.tmax));
    st(F, W_RAD, i, pku(p.radiance, p.kind));
    st(F, W_BETA, i, pku(p.beta, p.rng));
    st(F, W_CORE, i, u4(p.bounces, p.events, (p.specular ? 1u : 0u) | (p.in_water ? 2u : 0u), flags));
}

LW_DI void store_nee(const WfState &F, uint32_t i, const Path &p) {
    st(F, W_N, i, pk(p.n, p.cos_l));
    st(F, W_ORIGIN, i, pku(p.origin, p.seg));
    st(F, W_TR, i, pk(p.tr, p.dist));
    st(F, W_ESUM, i, pku(p.esum, p.list));
    st(F, W_FSUM, i, pku(p.fsum, p.count));
    st(F, W_EOFF, i, pku(p.eoff, p.k));
    st(F, W_E1, i, u4(p.first, p.faces, p.f, p.emode | (p.fmode << 1)));
}

// One ticket per calling lane from `ctr`, one atomic per group of converged lanes.
LW_DI uint32_t ticket(uint32_t *ctr) {
    unsigned am = __activemask();
    uint32_t lane = threadIdx.x & 31u;
    int leader = __ffs(am) - 1;
    uint32_t base = 0;
    if ((int)lane == leader) base = atomicAdd(ctr, (uint32_t)__popc(am));
    base = __shfl_sync(am, base, leader);
    return base + (uint32_t)__popc(am & ((1u << lane) - 1u));
}

}  // namespace

// The slot's item: in the single-frame form one of W's, in the batched form one of B's cameras
// (found by a binary search over the cameras' item ranges).
struct ItemRef {
    uint32_t job, j, pslot, px, py, sample, s_end;
    bool valid;
};

template <bool BATCH>
LW_DI ItemRef decode_item(const WorkDesc &W, const BatchDesc &B, uint32_t item) {
    ItemRef r{};
    uint32_t n_slots, tiles_x, w, h, x0 = 0, y0 = 0, sample_start, spp, sub, local = item, step = 1, first = 0;
    if (BATCH) {
        r.job = find_job(B.item_begin, B.n_jobs, item);
        const DevJob &J = B.jobs[r.job];
        local = item - J.item_begin;
        n_slots = J.n_slots, tiles_x = J.tiles_x, w = J.w, h = J.h;
        sample_start = J.sample_start, spp = J.spp, sub = J.sub;
    } else {
        n_slots = W.n_slots, tiles_x = W.tiles_x, w = W.w, h = W.h, x0 = W.x0, y0 = W.y0;
        step = W.tile_step, first = W.tile_first;
        sample_start = W.sample_start, spp = W.spp, sub = W.sub;
    }
    r.j = local / n_slots;
    r.pslot = local - r.j * n_slots;
    uint32_t tile = (r.pslot >> 5) * step + first, in = r.pslot & 31u;
    uint32_t rx = (tile % tiles_x) * 8u + (in & 7u);
    uint32_t ry = (tile / tiles_x) * 4u + (in >> 3);
    r.valid = rx < w && ry < h;
    r.px = x0 + rx;
    r.py = y0 + ry;
    r.sample = sample_start + r.j * sub;
    r.s_end = min(r.sample + sub, sample_start + spp);
    return r;
}

// One shading step of slot i (none when valid is false); its next ray goes to queue set `cur`.
// Slots with nothing to shade (dead, or their ray still being traced) leave after the state
// machine rather than before it, so the kernel has one exit. REB: chunk-origin rebasing, the
// path's frame word in F.frame.
template <bool BATCH, bool REB = false>
LW_DI void shade_slot(bool valid, uint32_t i, const DevScene &S0, const DevParams &P0, const WorkDesc &W,
                      const BatchDesc &B, const WfState &F, uint32_t cur) {
    float4 core = valid ? ld(F, W_CORE, i) : u4(0u, 0u, 0u, F_DEAD);
    uint32_t flags = fu(core.w);
    bool live = !(flags & F_DEAD);
    // The item words: in the batched form the camera is needed at every step, otherwise only when
    // a sample ends.
    float4 it2 = BATCH && live ? ld(F, W_ITEM2, i) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    uint32_t job = BATCH ? fu(it2.z) : 0u;
    DevScene S = S0;
    if (BATCH) S.sky = B.jobs[job].sky;
    const DevParams &P = BATCH ? B.jobs[job].P : P0;
    Path p;
    Act a = A_END;
    bool part = false;
    V3 val = v3(0.0f, 0.0f, 0.0f);
    if (live && (flags & F_ACTIVE)) {
        float4 h0 = F.hit0[i];
        if (fu(h0.y) == RESUME_MARK) {
            live = false;  // its ray is still on its way: nothing to shade yet
        } else {
            float4 wo = ld(F, W_O, i), wd = ld(F, W_D, i), wr = ld(F, W_RAD, i), wb = ld(F, W_BETA, i);
            float h1 = F.hit1[i];
            unpack_core(p, wo, wd, wr, wb, core);
            if (REB) p.frame = F.frame[i];
            if (p.kind != K_EXTEND) load_nee(F, i, p);
            Hit h{h0.x, fu(h0.y), fu(h0.z), h0.w, h1};
            a = on_result<REB>(p, S, P, h, val);
            part = true;
        }
    }
    if (part) a = advance<REB>(p, S, P, a, val);
    if (!live) return;
    if (a == A_END) {
        // The sample is over: the item's sums, then its next sample or the next item.
        if (!BATCH) it2 = ld(F, W_ITEM2, i);
        float4 it = ld(F, W_ITEM, i), sa = ld(F, W_SUM, i), sb = ld(F, W_SUM2, i);
        uint32_t px = fu(it.x), py = fu(it.y), sample = fu(it.z), s_end = fu(it.w);
        uint32_t j = fu(it2.x), pslot = fu(it2.y);
        float s0 = sa.x, s1 = sa.y, s2 = sa.z, c0 = sa.w, c1 = sb.x, c2 = sb.y;
        while (a == A_END) {
            if (flags & F_ACTIVE) {
                if (finite3(p.radiance)) {
                    kahan_add(s0, c0, p.radiance.x);
                    kahan_add(s1, c1, p.radiance.y);
                    kahan_add(s2, c2, p.radiance.z);
                }
                sample++;
                if (sample < s_end) {
                    a = A_TRACE;  // the item's next sample
                    break;
                }
                float4 v = make_float4(s0 - c0, s1 - c1, s2 - c2, 0.0f);
                if (BATCH) {
                    const DevJob &J = B.jobs[job];
                    B.partials[J.partial_off + (size_t)j * J.n_slots + pslot] = v;
                } else {
                    W.partials[(size_t)j * W.n_slots + pslot] = v;
                }
                flags &= ~F_ACTIVE;
            }
            const uint32_t n_items = BATCH ? B.n_items : W.n_items;
            uint32_t item = ticket(BATCH ? B.counter : W.counter);
            // The cancel word is read when an item number crosses a multiple of 4096.
            if ((item & 4095u) == 0u && *(BATCH ? B.cancel : W.cancel)) atomicMax(BATCH ? B.counter : W.counter, n_items);
            if (item >= n_items) {
                flags |= F_DEAD;
                break;
            }
            ItemRef r = decode_item<BATCH>(W, B, item);
            job = r.job;
            j = r.j;
            pslot = r.pslot;
            if (r.valid) {
                px = r.px;
                py = r.py;
                sample = r.sample;
                s_end = r.s_end;
                s0 = s1 = s2 = c0 = c1 = c2 = 0.0f;
                flags |= F_ACTIVE;
                a = A_TRACE;
            }
        }
        if (a == A_TRACE) begin_sample<REB>(p, BATCH ? B.jobs[job].P : P0, px, py, sample);  // one call site
        st(F, W_ITEM, i, u4(px, py, sample, s_end));
        st(F, W_ITEM2, i, u4(j, pslot, job, 0u));
        st(F, W_SUM, i, make_float4(s0, s1, s2, c0));
        st(F, W_SUM2, i, make_float4(c1, c2, 0.0f, 0.0f));
    }
    if (a == A_TRACE) {
        F.queue[(size_t)cur * F.n + ticket(&F.ctr[4 * cur])] = i;
        store_core(F, i, p, flags);
        if (REB) F.frame[i] = p.frame;
        if (p.kind != K_EXTEND) store_nee(F, i, p);
    } else {
        st(F, W_CORE, i, u4(0u, 0u, 0u, flags));
    }
}

// One shading step for every slot that had a ray in the previous iteration. Iteration t's rays are queue set t % 3, filled by the shading of iteration t and by
// the rays the tracing of iteration t - 1 carried over; the shading of iteration t reads set
// (t - 1) % 3 and clears set (t + 1) % 3 for the next iteration. The iteration is the device word
// ctr[12], advanced by k_wf_advance after each trace.
// Blocks of 128 threads' worth per SM the shading kernel must fit: 6, so 80 registers a thread. The
// batched one (the camera's Params and sky read through its job, on top) spills 160 bytes a thread
// at 80, and none at 100 (LW_WF_SHADE_MINB_BATCH 4, two blocks a SM), but the occupancy counts for
// more: the full-spp 64-camera batch runs at 513.8 Msamples/s at 80 and 492.9 at 100.
#ifndef LW_WF_SHADE_MINB
#define LW_WF_SHADE_MINB 6
#endif
#ifndef LW_WF_SHADE_MINB_BATCH
#define LW_WF_SHADE_MINB_BATCH 6
#endif
// The same for the forms with chunk-origin rebasing (116 B of spills at 80 registers, but at 98
// registers and two blocks a SM the 8-spp C5 frame shaded in 51.7 ms against 44.0).
#ifndef LW_WF_SHADE_MINB_REB
#define LW_WF_SHADE_MINB_REB 6
#endif
template <bool BATCH, bool REB = false>
__global__ void __launch_bounds__(kShadeThreads,
                                  (BATCH ? LW_WF_SHADE_MINB_BATCH : (REB ? LW_WF_SHADE_MINB_REB : LW_WF_SHADE_MINB)) * 128 /
                                      kShadeThreads)
k_wf_shade(const DevScene S0, const DevParams P0, const WorkDesc W, const BatchDesc B, const WfState F) {
    const uint32_t t = *(volatile uint32_t *)&F.ctr[12];
    const uint32_t cur = t % 3u, prev = (t + 2u) % 3u, next = (t + 1u) % 3u;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        F.ctr[4 * next] = 0u;
        F.ctr[4 * next + 1] = 0u;
    }
    // While most slots have a ray, thread k shades slot k (coalesced loads of the slot words; slots
    // without a ray return at once); once the previous iteration traced fewer than an eighth of
    // the slots, as the pool drains, only the slots in its queue are visited.
    const uint32_t queued = *(volatile uint32_t *)&F.ctr[4 * prev];
    const bool dense = t == 0u || (uint64_t)queued * 8u > F.n;
    const uint32_t n = dense ? F.n : queued;
    const uint32_t *list = F.queue + (size_t)prev * F.n;
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;  // the grid covers every slot
    shade_slot<BATCH, REB>(k < n, k < n ? (dense ? k : list[k]) : 0u, S0, P0, W, B, F, cur);
}

// The end of an iteration: the next iteration's number; in a graph, whether to run another one (the
// loop stops after an iteration that had no ray to trace). ctr[14..15]: the rays traced so far
// (64-bit), for the statistics.
__global__ void k_wf_advance(const WfState F) {
    uint32_t t = F.ctr[12];
    *(unsigned long long *)&F.ctr[14] += F.ctr[4 * (t % 3u)];
    F.ctr[12] = t + 1u;
}
__global__ void k_wf_advance_graph(const WfState F, cudaGraphConditionalHandle loop) {
    uint32_t t = F.ctr[12];
    uint32_t n = F.ctr[4 * (t % 3u)];
    *(unsigned long long *)&F.ctr[14] += n;
    cudaGraphSetConditional(loop, n != 0u ? 1u : 0u);
    F.ctr[12] = t + 1u;
}

#ifndef LW_WF_TRACE_MINB
#define LW_WF_TRACE_MINB 8
#endif
// The tracing kernel with chunk-origin rebasing (the frame word held across the traversal): 7 blocks
// a SM, 72 registers, 20 B of spills; at 8 blocks (64 registers) it spills 44 B and took 99.7 ms on
// the 8-spp C5 frame against 95.5, at 6 blocks 101.5.
#ifndef LW_WF_TRACE_MINB_REB
#define LW_WF_TRACE_MINB_REB 7
#endif
// Traces the queued rays of this iteration: each lane takes a ray and advances it in rounds
// (trace_round: at most `budget` visits through empty space, then the quad tests of at most one
// cell, so the lanes of a warp run one phase of quad tests per round together), and takes the
// next queued ray as soon as its ray ends. Once the queue
// has run dry, a ray still on its way after `tail` more rounds saves its traversal state and goes
// to the next iteration's queue, so an iteration does not wait for its single longest ray.
// STAGED: the block first copies the scene's top level and occupancy masks (S0.n_top + S0.n_occ
// entries of 8 bytes, the dynamic shared memory of the launch) into shared memory and reads them
// there. REB: chunk-origin rebasing, each ray in the frame of its slot's frame word.
template <bool STAGED, bool REB = false>
__global__ void __launch_bounds__(kTraceThreads, REB ? LW_WF_TRACE_MINB_REB : LW_WF_TRACE_MINB) k_wf_trace(const DevScene S0, const DevParams P, const WfState F,
                                                                      uint32_t budget, uint32_t tail) {
    extern __shared__ uint2 s_scene[];
    DevScene S = S0;
    if (STAGED) {
        const uint32_t n = S0.n_top + S0.n_occ;
        for (uint32_t i = threadIdx.x; i < n; i += kTraceThreads)
            s_scene[i] = i < S0.n_top ? __ldg(S0.top + i) : __ldg(S0.occ + (i - S0.n_top));
        __syncthreads();
        S.top = s_scene;
        S.occ = s_scene + S0.n_top;
    }
    const unsigned FULL = 0xFFFFFFFFu;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t t = *(volatile uint32_t *)&F.ctr[12];
    const uint32_t cur = t % 3u, next = (t + 1u) % 3u;
    const uint32_t count = *(volatile uint32_t *)&F.ctr[4 * cur];
    uint32_t *fetch = &F.ctr[4 * cur + 1];
    const uint32_t *list = F.queue + (size_t)cur * F.n;
    TraceState ts;
    V3 o = v3(0.0f, 0.0f, 0.0f), d = o;
    Frame A = Frame{};
    float tmin = 0.0f;
    uint32_t slot = 0, rounds = 0;
    bool have = false, done = false;
    __shared__ float4 s_quads[kTraceThreads / 32][32];  // warp_test_cells' candidates, per warp
    uint32_t chunk_next = 0, chunk_end = 0;  // warp-uniform: queue entries this warp has taken
    for (;;) {
        bool need = !have && !done;
        unsigned m = __ballot_sync(FULL, need);
#if LW_FETCH_MIN > 1
        if (__popc(m) < LW_FETCH_MIN && __any_sync(FULL, have)) {
            m = 0u;
            need = false;
        }
#endif
        if (m) {
            const uint32_t rank = (uint32_t)__popc(m & ((1u << lane) - 1u));
            // The needing lanes take the warp's next entries in lane order: what is left of its
            // chunk first, then a new chunk (entries are handed out in increasing order, so once
            // one is past the queue's end every later one is too).
            const uint32_t want = (uint32_t)__popc(m), avail = chunk_end - chunk_next;
            uint32_t q = chunk_next + rank;
            if (avail < want) {
                uint32_t base = 0;
                if (lane == 0u) base = atomicAdd(fetch, kFetchChunk);
                base = __shfl_sync(FULL, base, 0);
                if (rank >= avail) q = base + (rank - avail);
                chunk_next = base + (want - avail);
                chunk_end = base + kFetchChunk;
            } else {
                chunk_next += want;
            }
            if (need) {
                if (q >= count) {
                    done = true;
                } else {
                    slot = list[q];
                    float4 a = ld(F, W_O, slot), b = ld(F, W_D, slot);
                    o = f4v(a);
                    tmin = a.w;
                    d = f4v(b);
                    if (REB) A = frame_of(F.frame[slot]);
                    if (fu(F.hit0[slot].y) == RESUME_MARK) {
                        // a ray carried over from the previous iteration
                        float4 t0 = F.ts[slot], t1 = F.ts[F.n + slot], t2 = F.ts[2 * (size_t)F.n + slot];
                        ts.s.c0 = (int)fu(t0.x);
                        ts.s.c1 = (int)fu(t0.y);
                        ts.s.c2 = (int)fu(t0.z);
                        ts.s.n0 = t0.w;
                        ts.s.n1 = t1.x;
                        ts.s.n2 = t1.y;
                        ts.s.t = t1.z;
                        ts.inv = v3(t1.w, t2.x, t2.y);
                        ts.t_end = t2.z;
                        ts.it = fu(t2.w);
                        have = true;
                    } else if (trace_begin(ts, P, o, d, b.w, A)) {
                        have = true;
                    } else {
                        F.hit0[slot] = make_float4(kINF, __uint_as_float(NO_QUAD), 0.0f, 0.0f);
                        F.hit1[slot] = 0.0f;
                    }
                }
            }
        }
        if (__all_sync(FULL, done && !have)) break;
        if (__any_sync(FULL, done)) rounds++;  // the queue is dry: count the tail rounds
        Hit h = no_hit();
        const int r = trace_round_warp<STAGED, REB>(S, P, ts, o, d, tmin, budget, have, h, s_quads[threadIdx.x >> 5], A);
        if (have) {
            if (r != 0) {
                if (r != 1) h = no_hit();
                F.hit0[slot] = make_float4(h.t, __uint_as_float(h.quad), __uint_as_float(h.texel), h.s);
                F.hit1[slot] = h.tt;
                have = false;
            } else if (rounds > tail) {
                F.ts[slot] = u4((uint32_t)ts.s.c0, (uint32_t)ts.s.c1, (uint32_t)ts.s.c2, fu(ts.s.n0));
                F.ts[F.n + slot] = make_float4(ts.s.n1, ts.s.n2, ts.s.t, ts.inv.x);
                F.ts[2 * (size_t)F.n + slot] = make_float4(ts.inv.y, ts.inv.z, ts.t_end, __uint_as_float(ts.it));
                F.hit0[slot] = make_float4(0.0f, __uint_as_float(RESUME_MARK), 0.0f, 0.0f);
                F.queue[(size_t)next * F.n + ticket(&F.ctr[4 * next])] = slot;
                have = false;
                done = true;
            }
        }
    }
}

LaunchShape wf_trace_shape(int device, size_t stage_bytes, bool reb) {
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const void *k = stage_bytes ? (const void *)k_wf_trace<true>
                                : (reb ? (const void *)k_wf_trace<false, true> : (const void *)k_wf_trace<false>);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kTraceThreads, stage_bytes);
    if (per_sm < 1) per_sm = 1;
    return LaunchShape{sms * per_sm, kTraceThreads};
}

cudaError_t launch_wf_shade(const DevScene &S, const DevParams &P, const WorkDesc &W, const WfState &F, uint32_t blocks,
                            cudaStream_t st) {
    BatchDesc none{};
    if (rebased(P)) k_wf_shade<false, true><<<blocks, kShadeThreads, 0, st>>>(S, P, W, none, F);
    else k_wf_shade<false><<<blocks, kShadeThreads, 0, st>>>(S, P, W, none, F);
    return cudaGetLastError();
}

cudaError_t launch_wf_shade_batch(const DevScene &S, const DevParams &P0, const BatchDesc &B, const WfState &F,
                                  uint32_t blocks, cudaStream_t st) {
    WorkDesc none{};
    k_wf_shade<true><<<blocks, kShadeThreads, 0, st>>>(S, P0, none, B, F);
    return cudaGetLastError();
}

cudaError_t launch_wf_trace(const DevScene &S, const DevParams &P, const WfState &F, LaunchShape trace_shape,
                            uint32_t budget, uint32_t tail, size_t stage_bytes, cudaStream_t st) {
    if (budget == 0u) budget = kWfBudget;  // a round makes at least one visit
    if (rebased(P))  // one form: unstaged
        k_wf_trace<false, true><<<trace_shape.blocks, trace_shape.threads, 0, st>>>(S, P, F, budget, tail);
    else if (stage_bytes)
        k_wf_trace<true><<<trace_shape.blocks, trace_shape.threads, stage_bytes, st>>>(S, P, F, budget, tail);
    else
        k_wf_trace<false><<<trace_shape.blocks, trace_shape.threads, 0, st>>>(S, P, F, budget, tail);
    return cudaGetLastError();
}

cudaError_t launch_wf_advance(const WfState &F, cudaStream_t st) {
    k_wf_advance<<<1, 1, 0, st>>>(F);
    return cudaGetLastError();
}

cudaError_t launch_wf_advance_graph(const WfState &F, cudaGraphConditionalHandle loop, cudaStream_t st) {
    k_wf_advance_graph<<<1, 1, 0, st>>>(F, loop);
    return cudaGetLastError();
}

}  // namespace lw
