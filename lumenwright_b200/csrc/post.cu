// The display pass on the device: the per-pixel mean of the accumulator (k_finalize's division)
// tone-mapped to packed RGBA8 in the same kernel, so a render's result leaves the GPU as 4 bytes
// per pixel instead of 12. The operators are the reference's `post::tonemap` and `tonemap_mix`
// (crates/lumenwright/src/render/post.rs:152-217): exposure, then clamp-and-gamma, the ACES fit,
// or a Hable curve (Chunky's FILMIC_WORLDS preset, or the game's curve: the preset brightened to
// hold mid-grey), then the display gamma v^(1/2.2) and the 8-bit rounding `(v * 255 + 0.5) as u32`.
// The Hable curve's parameter products are formed in f32 and the rest in f64, as the reference's
// `HableCurve::h` does; the curve constants come from the host (computed there as the reference
// does). The display gamma is evaluated in f64 and rounded to f32.
#include "device_math.cuh"
#include "internal.h"

namespace lw {
namespace {

enum : uint32_t { OP_GAMMA = 0, OP_ACES = 1, OP_FILMIC = 2, OP_FILMIC_MID_GREY = 3 };

// Rust's f32::clamp (a NaN passes through) and f32::max (a NaN gives the other operand).
LW_DI float clamp_rs(float x, float lo, float hi) { return x < lo ? lo : (x > hi ? hi : x); }
LW_DI float max_rs(float x, float y) { return x != x ? y : (x > y ? x : y); }

// aces (post.rs:23-26).
LW_DI float aces(float x) {
    const float a = 2.51f, b = 0.03f, c = 2.43f, d = 0.59f, e = 0.14f;
    return clamp_rs(__fdiv_rn(x * (a * x + b), x * (c * x + d) + e), 0.0f, 1.0f);
}

// HableCurve::h (post.rs:94-104) times the white scale, cast to f32.
LW_DI float hable(const ToneCurve &k, float v) {
    double y = 2.0 * (double)v;
    double h = __ddiv_rn(y * (k.a * y + k.cb) + k.de, y * (k.a * y + k.b) + k.df) - k.ef;
    return (float)(h * k.white);
}

// The value a channel shows before the 8-bit rounding (post.rs:189-201 `shown`, and `encode`).
LW_DI float shown(const TonemapDesc &t, uint32_t op, float v) {
    v = max_rs(v * t.exposure, 0.0f);
    if (op == OP_ACES) v = aces(v);
    else if (op == OP_FILMIC) v = hable(t.preset, v);
    else if (op == OP_FILMIC_MID_GREY) v = hable(t.game, v);
    float c = clamp_rs(v, 0.0f, 1.0f);
    return (float)pow((double)c, (double)t.inv_gamma);
}

LW_DI uint32_t to_byte(float d) { return __float2uint_rz(d * 255.0f + 0.5f); }

LW_DI uint32_t pack(const TonemapDesc &t, float r, float g, float b) {
    float c[3] = {r, g, b};
    uint32_t out = 0xFF000000u;
    for (int k = 0; k < 3; k++) {
        float d;
        if (!t.mix || t.weight >= 1.0f) d = shown(t, t.op_a, c[k]);
        else if (t.weight <= 0.0f) d = shown(t, t.op_b, c[k]);
        else d = t.weight * shown(t, t.op_a, c[k]) + (1.0f - t.weight) * shown(t, t.op_b, c[k]);
        out |= to_byte(d) << (8 * k);
    }
    return out;
}

// The mean of each pixel's accumulator (k_finalize) and its display bytes; the mean is written too
// when `hdr` is given.
__global__ void k_finalize_tonemap(const Accum *acc, uint32_t n, TonemapDesc t, uint32_t *rgba, float *hdr) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Accum a = acc[i];
    float cnt = fmax_r(a.sum.w, 1.0f);
    float r = __fdiv_rn(a.sum.x - a.comp.x, cnt);
    float g = __fdiv_rn(a.sum.y - a.comp.y, cnt);
    float b = __fdiv_rn(a.sum.z - a.comp.z, cnt);
    if (hdr) {
        hdr[3 * i] = r;
        hdr[3 * i + 1] = g;
        hdr[3 * i + 2] = b;
    }
    rgba[i] = pack(t, r, g, b);
}

// The display bytes of n linear RGB values.
__global__ void k_tonemap(const float *hdr, uint32_t n, TonemapDesc t, uint32_t *rgba) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    rgba[i] = pack(t, hdr[3 * i], hdr[3 * i + 1], hdr[3 * i + 2]);
}

}  // namespace

cudaError_t launch_finalize_tonemap(const Accum *acc, uint32_t n, const TonemapDesc &t, uint32_t *rgba, float *hdr,
                                    cudaStream_t st) {
    k_finalize_tonemap<<<(n + 255) / 256, 256, 0, st>>>(acc, n, t, rgba, hdr);
    return cudaGetLastError();
}

cudaError_t launch_tonemap(const float *hdr, uint32_t n, const TonemapDesc &t, uint32_t *rgba, cudaStream_t st) {
    k_tonemap<<<(n + 255) / 256, 256, 0, st>>>(hdr, n, t, rgba);
    return cudaGetLastError();
}

}  // namespace lw
