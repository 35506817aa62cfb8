// The batched form: many cameras (each its own Params: frame size, spp, bounces, sky) rendered
// by one persistent launch. The work items of every camera form one queue: lanes take items from
// a single counter and find the camera an item belongs to by a binary search over the cameras'
// item ranges, so a small camera's last items and a large camera's first ones run side by side
// instead of each camera's launch ending in its own tail. The per-camera partial sums are reduced
// and finalised by one launch each; the host captures the whole sequence into a CUDA graph.
#include "device_path.cuh"
#include "internal.h"

namespace lw {

// RESUME: advance each ray by at most B.budget voxel visits per loop iteration (the regrouping
// period), as k_render does with it.
template <int THREADS, bool RESUME>
__global__ void __launch_bounds__(THREADS, THREADS == 128 ? 4 : (THREADS == 64 ? 8 : 2))
k_render_batch(const DevScene S, const BatchDesc B) {
    const uint32_t lane = threadIdx.x & 31u;
    const unsigned FULL = 0xFFFFFFFFu;
    Path p;
    TraceState ts;
    bool active = false, exhausted = false, tracing = false;
    uint32_t job = 0, px = 0, py = 0, slot = 0, j = 0, sample = 0, s_end = 0;
    float s0 = 0.f, s1 = 0.f, s2 = 0.f, c0 = 0.f, c1 = 0.f, c2 = 0.f;
    for (;;) {
        bool need = !active && !exhausted;
        unsigned mask = __ballot_sync(FULL, need);
        if (mask) {
            uint32_t base = 0;
            int leader = __ffs(mask) - 1;
            if ((int)lane == leader) {
                uint32_t n = (uint32_t)__popc(mask);
                base = atomicAdd(B.counter, n);
                if ((base & 4095u) < n && *B.cancel) base = B.n_items;
            }
            base = __shfl_sync(FULL, base, leader);
            if (need) {
                uint32_t item = base + (uint32_t)__popc(mask & ((1u << lane) - 1u));
                if (item >= B.n_items) {
                    exhausted = true;
                } else {
                    job = find_job(B.item_begin, B.n_jobs, item);
                    const DevJob &J = B.jobs[job];
                    uint32_t local = item - J.item_begin;
                    j = local / J.n_slots;
                    slot = local - j * J.n_slots;
                    uint32_t tile = slot >> 5, in = slot & 31u;
                    uint32_t rx = (tile % J.tiles_x) * 8u + (in & 7u);
                    uint32_t ry = (tile / J.tiles_x) * 4u + (in >> 3);
                    if (rx < J.w && ry < J.h) {
                        px = rx;
                        py = ry;
                        sample = J.sample_start + j * J.sub;
                        s_end = min(sample + J.sub, J.sample_start + J.spp);
                        s0 = s1 = s2 = c0 = c1 = c2 = 0.0f;
                        begin_sample(p, J.P, px, py, sample);
                        active = true;
                        tracing = false;
                    }
                }
            }
        }
        if (__all_sync(FULL, exhausted)) break;
        if (!active) continue;

        const DevJob &J = B.jobs[job];
        DevScene Sj = S;
        Sj.sky = J.sky;
        Hit h = no_hit();
        if (!RESUME) {
            h = trace(Sj, J.P, p.o, p.d, p.tmin, p.tmax);
        } else {
            int r = -1;
            if (!tracing) tracing = trace_begin(ts, J.P, p.o, p.d, p.tmax);
            if (tracing) {
                r = trace_run(Sj, J.P, ts, p.o, p.d, p.tmin, B.budget, h);
                if (r == 0) continue;
                tracing = false;
            }
            if (r != 1) h = no_hit();
        }
        Act a = shade(p, Sj, J.P, h);
        if (a == A_END) {
            if (finite3(p.radiance)) {
                kahan_add(s0, c0, p.radiance.x);
                kahan_add(s1, c1, p.radiance.y);
                kahan_add(s2, c2, p.radiance.z);
            }
            sample++;
            if (sample < s_end) {
                begin_sample(p, J.P, px, py, sample);
            } else {
                B.partials[J.partial_off + (size_t)j * J.n_slots + slot] = make_float4(s0 - c0, s1 - c1, s2 - c2, 0.0f);
                active = false;
            }
        }
    }
}

// Every camera's item sums into its accumulator (Kahan, in item order), then its image. A
// cancelled batch adds nothing (its item sums may be stale), so its images are left at zero.
__global__ void k_reduce_batch(const BatchDesc B) {
    uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= B.n_slots) return;
    uint32_t job = find_job(B.slot_begin, B.n_jobs, g);
    const DevJob &J = B.jobs[job];
    uint32_t slot = g - J.slot_begin;
    uint32_t tile = slot >> 5, in = slot & 31u;
    uint32_t rx = (tile % J.tiles_x) * 8u + (in & 7u);
    uint32_t ry = (tile / J.tiles_x) * 4u + (in >> 3);
    if (rx >= J.w || ry >= J.h) return;
    Accum &a = J.acc[(size_t)ry * J.w + rx];
    float4 s = a.sum, c = a.comp;
    if (!*B.cancel) {
        for (uint32_t jj = 0; jj < J.n_sub; jj++) {
            float4 v = B.partials[J.partial_off + (size_t)jj * J.n_slots + slot];
            kahan_add(s.x, c.x, v.x);
            kahan_add(s.y, c.y, v.y);
            kahan_add(s.z, c.z, v.z);
        }
        s.w += (float)J.spp;
    }
    a.sum = s;
    a.comp = c;
    float cnt = fmax_r(s.w, 1.0f);
    float *o = J.out + 3 * ((size_t)ry * J.w + rx);
    o[0] = __fdiv_rn(s.x - c.x, cnt);
    o[1] = __fdiv_rn(s.y - c.y, cnt);
    o[2] = __fdiv_rn(s.z - c.z, cnt);
}

template <bool RESUME>
static const void *batch_kernel(int threads) {
    if (threads == 64) return (const void *)k_render_batch<64, RESUME>;
    if (threads == 256) return (const void *)k_render_batch<256, RESUME>;
    return (const void *)k_render_batch<128, RESUME>;
}

LaunchShape batch_shape(int device, int threads, bool resume) {
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const void *k = resume ? batch_kernel<true>(threads) : batch_kernel<false>(threads);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, 0);
    if (per_sm < 1) per_sm = 1;
    return LaunchShape{sms * per_sm, threads};
}

cudaError_t launch_render_batch(const DevScene &S, const BatchDesc &B, LaunchShape shape, cudaStream_t st) {
    void *args[] = {(void *)&S, (void *)&B};
    const void *k = B.budget ? batch_kernel<true>(shape.threads) : batch_kernel<false>(shape.threads);
    return cudaLaunchKernel(k, dim3(shape.blocks), dim3(shape.threads), args, 0, st);
}

cudaError_t launch_reduce_batch(const BatchDesc &B, cudaStream_t st) {
    k_reduce_batch<<<(B.n_slots + 255) / 256, 256, 0, st>>>(B);
    return cudaGetLastError();
}

}  // namespace lw
