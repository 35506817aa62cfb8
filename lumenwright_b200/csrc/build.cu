// The hq grid build on the device: `voxel::build_hq` (crates/lumenwright/src/scene/voxel.rs:111-491)
// for a block volume, in two phases around the host's model generation.
//
// Phase 1 (k_keys_first): each voxel's model-instance key — its block state, and for a fluid its
// face mask (`Scene::fluid_face_mask`, crates/lumenwright/src/scene/mod.rs:586-609: bit 7 and Up
// when the block above is the same fluid, each other face's bit when its neighbour is the same
// fluid or occludes; outside the volume is air); 0 for an invisible state. The build interns keys
// in the order it first meets them (bricks in brick order, voxels in (y, z, x) order inside a
// brick, voxel.rs:171-343), so each key's first position in that order is its rank: the kernel
// takes an atomicMin of the position per key, and the host sorts the keys present by it.
//
// Phase 2, after the host has built the instances' models and quads: k_bricks_scan gives every
// voxel its instance id and every brick its class (no visible voxel, all occluding, uniform, the
// first non-zero id, its emitting voxels); the host then decides buried / uniform / stored bricks
// (voxel.rs:345-392) and their offsets; k_bricks_pack writes the stored bricks' u16 ids (even voxel
// in the low half) into the grid and every brick's emitter sites in voxel order.
#include <cstdint>
#include <cuda_runtime.h>

#include "internal.h"

namespace lw {
namespace {

constexpr uint32_t SF_OCCLUDES = 1u, SF_INVISIBLE = 2u, SF_FLUID = 4u;
constexpr int DIR_DOWN = 0, DIR_UP = 1, DIR_NORTH = 2, DIR_SOUTH = 3, DIR_WEST = 4, DIR_EAST = 5;

struct Vol {
    const uint16_t *blocks;
    int sx, sy, sz;
    const uint8_t *flags;
    uint32_t n_states;
    uint32_t *error;
};

__device__ __forceinline__ uint32_t state_flags(const Vol &v, int x, int y, int z, uint16_t *state) {
    if (x < 0 || y < 0 || z < 0 || x >= v.sx || y >= v.sy || z >= v.sz) {
        *state = 0xFFFFu;  // outside the volume: air
        return SF_INVISIBLE;
    }
    uint16_t s = v.blocks[((size_t)y * v.sz + z) * v.sx + x];
    *state = s;
    if (s >= v.n_states) {
        atomicOr(v.error, 1u);
        return SF_INVISIBLE;
    }
    return v.flags[s];
}

// The voxel at (x, y, z) of brick order position `pos`.
__device__ __forceinline__ uint32_t key_of(const Vol &v, int x, int y, int z) {
    uint16_t s;
    uint32_t f = state_flags(v, x, y, z, &s);
    if (f & SF_INVISIBLE) return 0u;
    uint32_t mask = 0u;
    if (f & SF_FLUID) {
        const int off[6][3] = {{0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}, {-1, 0, 0}, {1, 0, 0}};
        uint16_t t;
        uint32_t g = state_flags(v, x, y + 1, z, &t);
        if (t == s && (g & SF_FLUID)) mask |= 0x80u | (1u << DIR_UP);
        const int dirs[5] = {DIR_DOWN, DIR_NORTH, DIR_SOUTH, DIR_WEST, DIR_EAST};
        for (int k = 0; k < 5; k++) {
            const int *o = off[dirs[k]];
            g = state_flags(v, x + o[0], y + o[1], z + o[2], &t);
            if ((t == s && (g & SF_FLUID)) || (g & SF_OCCLUDES)) mask |= 1u << dirs[k];
        }
    }
    return ((uint32_t)s << 8) | mask;
}

// One thread per voxel: its key, and the first brick-order position of every key.
__global__ void k_keys_first(const Vol v, uint32_t *keys, uint32_t *first) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    size_t n = (size_t)v.sx * v.sy * v.sz;
    if (i >= n) return;
    int x = (int)(i % v.sx), z = (int)((i / v.sx) % v.sz), y = (int)(i / ((size_t)v.sx * v.sz));
    uint32_t k = key_of(v, x, y, z);
    uint32_t dx = (uint32_t)v.sx / 16u, dz = (uint32_t)v.sz / 16u;
    uint32_t b = (((uint32_t)y >> 4) * dz + ((uint32_t)z >> 4)) * dx + ((uint32_t)x >> 4);
    uint32_t local = (((uint32_t)y & 15u) * 16u + ((uint32_t)z & 15u)) * 16u + ((uint32_t)x & 15u);
    uint32_t pos = b * 4096u + local;
    keys[pos] = k;
    if (k) atomicMin(first + k, pos);
}

// One 256-thread block per brick, 16 consecutive voxels per thread.
__global__ void __launch_bounds__(256) k_bricks_scan(const Vol v, const uint32_t *keys, const uint32_t *key_id,
                                                     const uint8_t *model_emits, uint16_t *ids, uint4 *cls) {
    const uint32_t b = blockIdx.x;
    __shared__ uint32_t s_any, s_all_occ, s_uniform, s_first, s_emit;
    if (threadIdx.x == 0) {
        s_any = 0u;
        s_all_occ = 1u;
        s_uniform = 1u;
        s_first = 0xFFFFFFFFu;
        s_emit = 0u;
    }
    __syncthreads();
    uint32_t dx = (uint32_t)v.sx / 16u, dz = (uint32_t)v.sz / 16u;
    uint32_t bx = b % dx, bz = (b / dx) % dz, by = b / (dx * dz);
    uint32_t id0 = key_id[keys[(size_t)b * 4096u]];
    uint32_t any = 0u, all_occ = 1u, uniform = 1u, first = 0xFFFFFFFFu, emit = 0u;
    for (uint32_t k = 0; k < 16; k++) {
        uint32_t local = threadIdx.x * 16u + k;
        uint32_t key = keys[(size_t)b * 4096u + local];
        uint32_t id = key_id[key];
        ids[(size_t)b * 4096u + local] = (uint16_t)id;
        any |= key != 0u;
        uniform &= id == id0;
        if (id != 0u && local < first) first = local;
        emit += model_emits[id];
        int x = (int)(bx * 16u + (local & 15u)), z = (int)(bz * 16u + ((local >> 4) & 15u)), y = (int)(by * 16u + (local >> 8));
        uint16_t s;
        all_occ &= (state_flags(v, x, y, z, &s) & SF_OCCLUDES) ? 1u : 0u;
    }
    if (any) atomicOr(&s_any, 1u);
    if (!all_occ) atomicAnd(&s_all_occ, 0u);
    if (!uniform) atomicAnd(&s_uniform, 0u);
    if (first != 0xFFFFFFFFu) atomicMin(&s_first, first);
    if (emit) atomicAdd(&s_emit, emit);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t first_id = s_first == 0xFFFFFFFFu ? 0u : (uint32_t)ids[(size_t)b * 4096u + s_first];
        uint32_t flags = s_any | (s_all_occ << 1) | (s_uniform << 2);
        cls[b] = make_uint4(flags, id0, first_id, s_emit);
    }
}

// One 256-thread block per brick: the stored bricks' packed ids, every brick's emitter sites in
// voxel order (site = voxel corner x, y, z, model id).
__global__ void __launch_bounds__(256) k_bricks_pack(const Vol v, const uint16_t *ids, const uint8_t *model_emits,
                                                     const uint32_t *slot, const uint32_t *emit_off, uint32_t *brick_words,
                                                     uint4 *sites) {
    const uint32_t b = blockIdx.x;
    const uint16_t *bid = ids + (size_t)b * 4096u;
    uint32_t s = slot[b];
    if (s != 0xFFFFFFFFu) {
        uint32_t *w = brick_words + (size_t)s * 2048u;
        for (uint32_t j = threadIdx.x; j < 2048u; j += blockDim.x) w[j] = (uint32_t)bid[2 * j] | ((uint32_t)bid[2 * j + 1] << 16);
    }
    // Emitting voxels: count per thread (16 consecutive voxels), scan across the block, write.
    __shared__ uint32_t scan[256];
    uint32_t cnt = 0u;
    for (uint32_t k = 0; k < 16; k++) cnt += model_emits[bid[threadIdx.x * 16u + k]];
    scan[threadIdx.x] = cnt;
    __syncthreads();
    for (uint32_t d = 1; d < 256u; d <<= 1) {
        uint32_t add = threadIdx.x >= d ? scan[threadIdx.x - d] : 0u;
        __syncthreads();
        scan[threadIdx.x] += add;
        __syncthreads();
    }
    uint32_t at = emit_off[b] + scan[threadIdx.x] - cnt;
    uint32_t dx = (uint32_t)v.sx / 16u, dz = (uint32_t)v.sz / 16u;
    uint32_t bx = b % dx, bz = (b / dx) % dz, by = b / (dx * dz);
    for (uint32_t k = 0; k < 16 && cnt; k++) {
        uint32_t local = threadIdx.x * 16u + k;
        uint32_t id = bid[local];
        if (model_emits[id]) {
            sites[at++] = make_uint4(bx * 16u + (local & 15u), by * 16u + (local >> 8), bz * 16u + ((local >> 4) & 15u), id);
        }
    }
}

}  // namespace

cudaError_t launch_keys_first(const BuildVol &bv, uint32_t *keys, uint32_t *first, cudaStream_t st) {
    Vol v{bv.blocks, (int)bv.size[0], (int)bv.size[1], (int)bv.size[2], bv.flags, bv.n_states, bv.error};
    size_t n = (size_t)bv.size[0] * bv.size[1] * bv.size[2];
    k_keys_first<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(v, keys, first);
    return cudaGetLastError();
}

cudaError_t launch_bricks_scan(const BuildVol &bv, const uint32_t *keys, const uint32_t *key_id, const uint8_t *model_emits,
                               uint16_t *ids, uint4 *cls, uint32_t nb, cudaStream_t st) {
    Vol v{bv.blocks, (int)bv.size[0], (int)bv.size[1], (int)bv.size[2], bv.flags, bv.n_states, bv.error};
    k_bricks_scan<<<nb, 256, 0, st>>>(v, keys, key_id, model_emits, ids, cls);
    return cudaGetLastError();
}

cudaError_t launch_bricks_pack(const BuildVol &bv, const uint16_t *ids, const uint8_t *model_emits, const uint32_t *slot,
                               const uint32_t *emit_off, uint32_t *brick_words, uint4 *sites, uint32_t nb, cudaStream_t st) {
    Vol v{bv.blocks, (int)bv.size[0], (int)bv.size[1], (int)bv.size[2], bv.flags, bv.n_states, bv.error};
    k_bricks_pack<<<nb, 256, 0, st>>>(v, ids, model_emits, slot, emit_off, brick_words, sites);
    return cudaGetLastError();
}

}  // namespace lw
