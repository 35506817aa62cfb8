// An allocation-free render entry point, for callers that must not allocate device memory once
// they are running: a renderer embedded in a host application that owns the GPU's memory budget
// (a game engine or an editor that hands out memory from its own pools), or a per-frame loop that
// must keep a steady state with no cudaMalloc/cudaFree (which synchronise the device and stall
// whatever else shares it). Such a caller sets up the context, the scene and the sky once, ahead
// of time (those calls allocate), and then renders frame after frame through this entry point,
// which allocates nothing: the render kernel's scratch memory (its work counter and the partial
// sums of its work items) lives in a fixed array compiled into the library, and the accumulator is
// the caller's own device buffer.
#include <cstring>
#include <mutex>

#include "../../include/lumenwright_b200.h"
#include "internal.h"

namespace lw {

// The scratch array: one 256-byte header (the work counter) and LW_NOALLOC_PARTIALS item sums.
// 32 MiB + 256 B, held by every GPU that loads the library until the process exits.
constexpr size_t LW_NOALLOC_PARTIALS = (size_t(32) << 20) / sizeof(float4);
static __device__ __align__(256) float4 g_noalloc_scratch[16 + LW_NOALLOC_PARTIALS];

const size_t kNoallocPartials = LW_NOALLOC_PARTIALS;

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
float4 *g_noalloc_ptr[kMaxDevices];  // the array's device address, per device (set up once)
}  // namespace

// The device address of the scratch array on the current device, looked up the first time a device
// is used. In host code `g_noalloc_scratch` names a host-side stand-in, not device memory, so the
// address must come from cudaGetSymbolAddress with that device current.
cudaError_t noalloc_scratch(int device, float4 **out) {
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_noalloc_ptr[device] = (float4 *)p;
    }
    *out = g_noalloc_ptr[device];
    return cudaSuccess;
}

}  // namespace lw
