// Scene re-layout kernels run by lw_scene_upload: the fused (top, overlay) entries, the
// sub-block-major bricks with their occupancy masks, and the 96-byte quad records.
//
// In the traversal's copy a voxel whose model has no quads (a fluid block inside its fluid, every
// face culled) is re-laid as air, 0, and counts as empty in the occupancy masks. The traversal
// visits such a cell exactly as an air cell (one iteration of trace.rs's loop, the same DDA step,
// no quad to test), so the results are the reference's; the cell no longer stops its lane for a
// round of quad tests with nothing to test. A uniform brick of such a model keeps its entry as a
// uniform brick of air, which is still stepped voxel by voxel, not skipped as an empty brick. The
// reference's ids stay in the uploaded grid, which the voxel lookup reads.
#include "internal.h"

namespace lw {

// One entry per brick: (top, ov_top) from the reference grid; entries pointing outside the
// brick, model or overlay arrays raise bit 0 of the error word.
__global__ void k_top(SceneUploadDesc d) {
    uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= d.nb) return;
    uint32_t e = d.grid[d.off_top + b];
    uint32_t ov = d.grid[d.off_ov_top + b];
    bool bad = false;
    if (e != EMPTY) {
        if (e & UNIFORM) {
            const uint32_t m = e & ~UNIFORM;
            bad |= m >= d.n_models;
            if (!bad && d.models[m].y == 0u) e = UNIFORM;  // a uniform brick of air
        } else {
            bad |= e >= d.n_bricks;
        }
    }
    if (ov != EMPTY) bad |= ov >= d.n_ov_bricks;
    if (bad) {
        atomicOr(d.error, 1u);
        e = EMPTY;
        ov = EMPTY;
    }
    d.top[b] = make_uint2(e, ov);
}

// One block of 256 threads per non-uniform brick: each thread moves 16 voxel ids from the
// reference order (y*16+z)*16+x (two per word, the even voxel in the low half) to
// sub-block-major order, and the block ORs together the brick's occupancy mask.
__global__ void __launch_bounds__(256) k_bricks(SceneUploadDesc d) {
    __shared__ unsigned long long mask;
    uint32_t brick = blockIdx.x;
    if (threadIdx.x == 0) mask = 0ull;
    __syncthreads();
    const uint32_t *src = d.grid + d.off_bricks + (size_t)brick * 2048u;
    uint16_t *dst = d.bricks + (size_t)brick * 4096u;
    unsigned long long mine = 0ull;
    bool bad = false;
    for (uint32_t w = threadIdx.x; w < 2048u; w += 256u) {
        uint32_t word = src[w];
#pragma unroll
        for (uint32_t half = 0; half < 2; half++) {
            uint32_t local = 2u * w + half;
            uint32_t id = (word >> (16u * half)) & 0xFFFFu;
            uint32_t x = local & 15u, z = (local >> 4) & 15u, y = local >> 8;
            uint32_t sb = ((y >> 2) * 4u + (z >> 2)) * 4u + (x >> 2);
            uint32_t v = ((y & 3u) * 4u + (z & 3u)) * 4u + (x & 3u);
            bad |= id >= d.n_models;
            if (id != 0u && id < d.n_models && d.models[id].y == 0u) id = 0u;  // no quads: air
            dst[sb * 64u + v] = (uint16_t)id;
            if (id != 0u) mine |= 1ull << sb;
        }
    }
    atomicOr(&mask, mine);
    if (bad) atomicOr(d.error, 2u);
    __syncthreads();
    if (threadIdx.x == 0) d.occ[brick] = make_uint2((uint32_t)mask, (uint32_t)(mask >> 32));
}

cudaError_t launch_relayout(const SceneUploadDesc &d, cudaStream_t st) {
    if (d.nb) k_top<<<(d.nb + 255) / 256, 256, 0, st>>>(d);
    if (d.n_bricks) k_bricks<<<d.n_bricks, 256, 0, st>>>(d);
    return cudaGetLastError();
}

// GpuQuad (80 B) -> DevQuad (96 B) with n = eu x ev and n . n, computed in the kernels' own
// rounding (the library builds with --fmad=false), as intersect_quad computes them per test.
__global__ void k_quads(const float4 *ref, DevQuad *out, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 p0 = ref[5 * i], eu = ref[5 * i + 1], ev = ref[5 * i + 2], uv = ref[5 * i + 3], uvt = ref[5 * i + 4];
    V3 nn = cross(f4v(eu), f4v(ev));
    DevQuad q;
    q.n_nn = make_float4(nn.x, nn.y, nn.z, dot(nn, nn));
    q.p0_flags = p0;
    q.eu_tint = eu;
    q.ev_em = ev;
    q.uv = uv;
    q.uvt = make_float4(uvt.x, uvt.y, 0.0f, 0.0f);
    out[i] = q;
}

cudaError_t launch_quads(const void *ref_quads, DevQuad *out, uint32_t n, cudaStream_t st) {
    if (n) k_quads<<<(n + 127) / 128, 128, 0, st>>>((const float4 *)ref_quads, out, n);
    return cudaGetLastError();
}

}  // namespace lw
