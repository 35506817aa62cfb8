// The path-tracing kernels: the persistent render kernel with its per-lane path state machine
// (replacing `pt_render`, crates/lumenwright-ptx/src/lib.rs:37-87), the per-pixel reduction of
// its partial sums, and the parity kernels (trace, voxel lookup).
#include "device_path.cuh"
#include "internal.h"

namespace lw {


#ifndef LW_STATS
#define LW_STATS 0
#endif
#if LW_STATS
// Divergence counters of the instrumented build (not part of the product build):
// [0] loop iterations per warp, [1] lanes active in them, [2] lanes tracing, [3] lanes whose ray
// goes on to the next iteration, [4] warp shading passes, [5..7] lanes shading a path/shadow/emitter
// ray
__device__ unsigned long long g_stats[16];
#endif
#ifndef LW_MIN_BLOCKS
#define LW_MIN_BLOCKS 4
#endif

// The persistent render kernel. Each lane takes an item (sub consecutive samples of one pixel),
// traces its samples one after another, and takes the next item as soon as it is done. Each loop
// iteration traces one ray per active lane and shades it. With RESUME, an iteration advances each
// lane's ray by at most `W.budget` voxel visits instead (the regrouping period): a lane whose ray
// ends shades it and sets up its next ray, a lane whose ray is still on its way keeps it for the
// next iteration, so no lane waits longer than one budget for the longest traversal of its warp;
// the price is the traversal state kept live across iterations (more registers). REB: chunk-origin
// rebasing (the path's positions in the frame of p.frame).
template <int MODE, int THREADS, bool RESUME, bool REB = false>
__global__ void __launch_bounds__(THREADS, THREADS == 128 ? LW_MIN_BLOCKS : (THREADS == 64 ? 2 * LW_MIN_BLOCKS : 2))
k_render(const DevScene S, const DevParams P, const WorkDesc W) {
    const uint32_t lane = threadIdx.x & 31u;
    const unsigned FULL = 0xFFFFFFFFu;
    Path p;
    TraceState ts;  // only kept across iterations when RESUME
    bool active = false, exhausted = false, tracing = false;
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
                    uint32_t tile = (slot >> 5) * W.tile_step + W.tile_first, in = slot & 31u;
                    uint32_t rx = (tile % W.tiles_x) * 8u + (in & 7u);
                    uint32_t ry = (tile / W.tiles_x) * 4u + (in >> 3);
                    if (rx < W.w && ry < W.h) {
                        px = W.x0 + rx;
                        py = W.y0 + ry;
                        sample = W.sample_start + j * W.sub;
                        s_end = min(sample + W.sub, W.sample_start + W.spp);
                        s0 = s1 = s2 = c0 = c1 = c2 = 0.0f;
                        begin_sample<REB>(p, P, px, py, sample);
                        active = true;
                        tracing = false;
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
            }
        }
#endif
        if (!active) continue;

        Hit h = no_hit();
        int r = -1;
        if (!RESUME) {
            // The whole traversal at once: nothing of it lives on past this iteration.
            h = trace<true, REB>(S, P, p.o, p.d, p.tmin, p.tmax, REB ? frame_of(p.frame) : Frame{});
            r = h.quad != NO_QUAD ? 1 : -1;
        } else {
        const Frame A = REB ? frame_of(p.frame) : Frame{};
        if (!tracing) tracing = trace_begin(ts, P, p.o, p.d, p.tmax, A);
        if (tracing) {
            r = trace_run<true, REB>(S, P, ts, p.o, p.d, p.tmin, W.budget, h, A);
#if LW_STATS
            {
                unsigned am = __activemask();
                unsigned cont = __ballot_sync(am, r == 0);
                if ((int)lane == __ffs(am) - 1) {
                    atomicAdd(&g_stats[2], (unsigned long long)__popc(am));
                    atomicAdd(&g_stats[3], (unsigned long long)__popc(cont));
                }
            }
#endif
            if (r == 0) continue;  // the ray goes on in the next iteration
            tracing = false;
        }
        }
        if (r != 1) h = no_hit();
#if LW_STATS
        {
            unsigned am = __activemask();
            uint32_t kind = p.kind;
            unsigned k0 = __ballot_sync(am, kind == K_EXTEND), k1 = __ballot_sync(am, kind == K_SHADOW);
            unsigned k2 = __ballot_sync(am, kind == K_EMIT);
            if ((int)lane == __ffs(am) - 1) {
                atomicAdd(&g_stats[4], 1ull);
                atomicAdd(&g_stats[5], (unsigned long long)__popc(k0));
                atomicAdd(&g_stats[6], (unsigned long long)__popc(k1));
                atomicAdd(&g_stats[7], (unsigned long long)__popc(k2));
            }
        }
#endif
        Act a = shade<REB>(p, S, P, h);
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
                begin_sample<REB>(p, P, px, py, sample);
            } else {
                if (MODE == MODE_ACCUM) W.partials[(size_t)j * W.n_slots + slot] = make_float4(s0 - c0, s1 - c1, s2 - c2, 0.0f);
                active = false;
            }
        }
    }
}

// Adds the launch's item sums into the per-pixel accumulator, in item order (Kahan). After a
// cancel the render kernels may have left items unwritten (their sums then hold whatever an
// earlier launch left there), so a cancelled launch adds nothing: a pixel's record keeps whole
// launches only, and its count is the samples its sums hold.
__global__ void k_reduce(const WorkDesc W, Accum *acc, uint32_t frame_w) {
    uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= W.n_slots || *W.cancel) return;
    uint32_t tile = (slot >> 5) * W.tile_step + W.tile_first, in = slot & 31u;
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

__global__ void k_water_exp(uint64_t n, const float *x, float *out) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = lw_water_expf(x[i]);
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

template <int MODE, bool RESUME>
static const void *kernel_for_r(int threads) {
    if (threads == 64) return (const void *)k_render<MODE, 64, RESUME>;
    if (threads == 256) return (const void *)k_render<MODE, 256, RESUME>;
    return (const void *)k_render<MODE, 128, RESUME>;
}
// With chunk-origin rebasing one form: 128 threads, whole traversals.
template <int MODE>
static const void *kernel_for(int threads, bool resume = false, bool reb = false) {
    if (reb) return (const void *)k_render<MODE, 128, false, true>;
    return resume ? kernel_for_r<MODE, true>(threads) : kernel_for_r<MODE, false>(threads);
}

LaunchShape render_shape(int mode, int device, int threads) {
    if (threads != 64 && threads != 256) threads = 128;
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const void *k = mode == MODE_SAMPLES ? kernel_for<MODE_SAMPLES>(threads) : kernel_for<MODE_ACCUM>(threads);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, 0);
    if (per_sm < 1) per_sm = 1;
    return LaunchShape{sms * per_sm, threads};
}

cudaError_t launch_render(int mode, const DevScene &S, const DevParams &P, const WorkDesc &W, LaunchShape shape,
                          cudaStream_t st) {
    void *args[] = {(void *)&S, (void *)&P, (void *)&W};
    const bool resume = W.budget != 0u;
    const bool reb = rebased(P);
    LaunchShape sh = shape;
    if (reb && sh.threads != 128) {  // the same threads in blocks of 128 (the kernel is persistent)
        sh.blocks = sh.blocks * sh.threads / 128 > 0 ? sh.blocks * sh.threads / 128 : 1;
        sh.threads = 128;
    }
    const void *k = mode == MODE_SAMPLES ? kernel_for<MODE_SAMPLES>(sh.threads, resume, reb)
                                         : kernel_for<MODE_ACCUM>(sh.threads, resume, reb);
    return cudaLaunchKernel(k, dim3(sh.blocks), dim3(sh.threads), args, 0, st);
}

cudaError_t launch_reduce(const WorkDesc &W, Accum *acc, uint32_t frame_w, cudaStream_t st) {
    if (W.n_slots == 0) return cudaSuccess;
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

cudaError_t launch_water_exp(uint64_t n, const float *x, float *out, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    k_water_exp<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, x, out);
    return cudaGetLastError();
}

cudaError_t launch_voxel_lookup(const DevScene &S, const DevParams &P, uint32_t n, const int32_t *xyz, uint32_t *out,
                                cudaStream_t st) {
    k_voxel_lookup<<<(n + 255) / 256, 256, 0, st>>>(S, P, n, xyz, out);
    return cudaGetLastError();
}

}  // namespace lw
