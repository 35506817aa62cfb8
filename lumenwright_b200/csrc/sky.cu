// Sky precompute on the device: Chunky's sky cache (`build_sky_cache`,
// crates/lumenwright-kernel/src/integrator.rs:133-148, which the reference evaluates on the host
// per frame) and the blend of Chunky's sky into the game sky's maps (`blend_chunky_sky`,
// crates/lumenwright/src/render/sky.rs:836-850). One thread per cache entry or map texel.
#include "device_integrator.cuh"
#include "internal.h"

namespace lw {

// preetham_radiance (integrator.rs:44-74). `expf` is CUDA's; the reference calls the platform's.
LW_DI V3 preetham_radiance(const DevParams &P, V3 d) {
    V3 sun = f4v(P.sky_sun);
    float cos_theta = fmax_r(d.y + P.sky_zenith.w, 0.0f);
    float cos_gamma = clamp_r(dot(d, sun), -1.0f, 1.0f);
    float gamma = acos_r(cos_gamma);
    float cos2_gamma = cos_gamma * cos_gamma;
    const float A[3] = {P.perez_a.x, P.perez_a.y, P.perez_a.z}, B[3] = {P.perez_b.x, P.perez_b.y, P.perez_b.z};
    const float Cc[3] = {P.perez_c.x, P.perez_c.y, P.perez_c.z}, D[3] = {P.perez_d.x, P.perez_d.y, P.perez_d.z};
    const float E[3] = {P.perez_e.x, P.perez_e.y, P.perez_e.z};
    float pz[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        float a = cos_theta > 0.0f ? A[k] * expf(__fdiv_rn(B[k], cos_theta)) : 0.0f;
        pz[k] = (1.0f + a) * (1.0f + Cc[k] * expf(D[k] * gamma) + E[k] * cos2_gamma);
    }
    float x = P.sky_zenith.x * pz[0];
    float y = P.sky_zenith.y * pz[1];
    float lum = P.sky_zenith.z * pz[2];
    if (y <= 5e-8f) return v3(0.0f, 0.0f, 0.0f);
    float f = __fdiv_rn(lum, y);
    float cx = x * f, cy = lum, cz = (1.0f - x - y) * f;
    return v3(2.3706743f * cx - 0.9000405f * cy - 0.4706338f * cz, -0.513885f * cx + 1.4253036f * cy + 0.0885814f * cz,
              0.0052982f * cx - 0.0146949f * cy + 1.0093968f * cz) *
           0.045f;
}

// rgb_to_hsl (integrator.rs:79-104).
LW_DI void rgb_to_hsl(V3 c, float &hue, float &sat, float &light) {
    float r = clamp_r(c.x, 0.0f, 1.0f), g = clamp_r(c.y, 0.0f, 1.0f), b = clamp_r(c.z, 0.0f, 1.0f);
    float cmax = fmax_r(fmax_r(r, g), b);
    float cmin = fmin_r(fmin_r(r, g), b);
    float delta = cmax - cmin;
    light = __fdiv_rn(cmax + cmin, 2.0f);
    if (delta == 0.0f) hue = 0.0f;
    else if (cmax == r) hue = __fdiv_rn(fmodf(__fdiv_rn(g - b, delta), 6.0f), 6.0f);
    else if (cmax == g) hue = __fdiv_rn(__fdiv_rn(b - r, delta) + 2.0f, 6.0f);
    else hue = __fdiv_rn(__fdiv_rn(r - g, delta) + 4.0f, 6.0f);
    sat = delta < 5e-8f ? 0.0f : __fdiv_rn(delta, 1.0f - fabs_r(2.0f * light - 1.0f));
}

__global__ void k_sky_cache(const DevParams P, uint32_t n, float *out) {
    uint32_t m = n + 1;
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m * m) return;
    uint32_t i = k / m, j = k - i * m;
    float sin_t, cos_t, sin_p, cos_p;
    sin_cos_turns(__fdiv_rn((float)i, (float)n), sin_t, cos_t);
    sin_cos_turns(__fdiv_rn((float)j, (float)(2 * n)) - 0.25f, sin_p, cos_p);
    float r = fabs_r(cos_p);
    float h, s, l;
    rgb_to_hsl(preetham_radiance(P, v3(cos_t * r, sin_p, sin_t * r)), h, s, l);
    out[3 * k] = h;
    out[3 * k + 1] = s;
    out[3 * k + 2] = l;
}

// map_direction (sky.rs:853-858) and the blend of sky_radiance into the map texel.
__global__ void k_blend_chunky(const DevScene S, const DevParams P, float *map, uint32_t w, uint32_t h, float weight) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= w * h) return;
    uint32_t i = k % w, j = k / w;
    float az = __fdiv_rn((float)i + 0.5f, (float)w) * (2.0f * kPI);
    float el = __fdiv_rn((float)j + 0.5f, (float)h) * kPI - kFRAC_PI_2;
    V3 d = v3(cosf(el) * cosf(az), sinf(el), cosf(el) * sinf(az));
    V3 c = sky_radiance(S, P, d);
    float *t = map + 3 * (size_t)k;
    t[0] = weight * c.x + (1.0f - weight) * t[0];
    t[1] = weight * c.y + (1.0f - weight) * t[1];
    t[2] = weight * c.z + (1.0f - weight) * t[2];
}

cudaError_t launch_sky_cache(const DevParams &P, uint32_t n, float *out, cudaStream_t st) {
    uint32_t cnt = (n + 1) * (n + 1);
    k_sky_cache<<<(cnt + 127) / 128, 128, 0, st>>>(P, n, out);
    return cudaGetLastError();
}

cudaError_t launch_blend_chunky(const DevScene &S, const DevParams &P, float *map, uint32_t w, uint32_t h, float weight,
                                cudaStream_t st) {
    k_blend_chunky<<<(w * h + 127) / 128, 128, 0, st>>>(S, P, map, w, h, weight);
    return cudaGetLastError();
}

}  // namespace lw
