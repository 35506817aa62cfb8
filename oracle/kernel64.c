/*
 * FP64 oracle: the reference kernel's algorithm and random draws in double precision with
 * libm's double functions (see lw_oracle.h). It is the converged-image reference the FP32
 * kernels are measured against. Test infrastructure only.
 */
#include <math.h>
#include <omp.h>

#define LWO_F64 1
#define REAL double
#define K(x) x
#define R_SQRT sqrt
#define R_FLOOR floor
#define R_EXP exp
#define R_TEXP exp
#define R_FMOD fmod
#define R_ACOS acos
#define R_ATAN2 atan2
#define R_GAMMA d_gamma_to_linear
#define R_SINCOS_TURNS d_sin_cos_turns

static inline double d_gamma_to_linear(double c) { return c <= 0.0 ? 0.0 : pow(c, 2.2); }
static inline void d_sin_cos_turns(double u, double *s, double *c) {
    double a = 6.283185307179586476925 * u;
    *s = sin(a);
    *c = cos(a);
}

#define lwo_bounds_error_count lwo_bounds_error_count
#include "kernel_impl.h"

static Cam cam64(const lwo_scene *s, const lwo_camera64 *c) {
    if (!c) {
        const lwo_params *p = s->params;
        Cam r = {v3f4(p->cam_pos), v3f4(p->cam_fwd), v3f4(p->cam_right), v3f4(p->cam_up), p->cam_pos[3], p->cam_fwd[3],
                 p->see_through[2], p->see_through[3]};
        return r;
    }
    /* the f64 camera's eye is relative to the grid origin: the grid's frame */
    Cam r = {v3(c->eye[0], c->eye[1], c->eye[2]), v3(c->fwd[0], c->fwd[1], c->fwd[2]),
             v3(c->right[0], c->right[1], c->right[2]), v3(c->up[0], c->up[1], c->up[2]), c->tan_half, c->aspect, 0u, 0u};
    return r;
}

void lwo64_render_sample(const lwo_scene *s, const lwo_camera64 *cam, uint32_t px, uint32_t py, uint32_t sample,
                         double out[3]) {
    Cam c = cam64(s, cam);
    V3 r = render_sample(s, &c, px, py, sample);
    out[0] = r.x;
    out[1] = r.y;
    out[2] = r.z;
}

void lwo64_render_samples(const lwo_scene *s, const lwo_camera64 *cam, uint32_t x0, uint32_t y0, uint32_t w, uint32_t h,
                          uint32_t sample_start, uint32_t count, double *out, int threads) {
    Cam c = cam64(s, cam);
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
    for (uint32_t py = 0; py < h; py++)
        for (uint32_t px = 0; px < w; px++)
            for (uint32_t k = 0; k < count; k++) {
                V3 r = render_sample(s, &c, x0 + px, y0 + py, sample_start + k);
                double *o = out + ((uint64_t)(py * w + px) * count + k) * 3u;
                o[0] = r.x;
                o[1] = r.y;
                o[2] = r.z;
            }
}

void lwo64_render_mean(const lwo_scene *s, const lwo_camera64 *cam, uint32_t x0, uint32_t y0, uint32_t w, uint32_t h,
                       uint32_t spp, double *out, int threads) {
    Cam c = cam64(s, cam);
    if (spp < 1) spp = 1;
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
    for (uint32_t py = 0; py < h; py++)
        for (uint32_t px = 0; px < w; px++) {
            double acc[3] = {0, 0, 0};
            for (uint32_t k = 0; k < spp; k++) {
                V3 r = render_sample(s, &c, x0 + px, y0 + py, k);
                if (isfinite(r.x) && isfinite(r.y) && isfinite(r.z)) {
                    acc[0] += r.x;
                    acc[1] += r.y;
                    acc[2] += r.z;
                }
            }
            double *o = out + (uint64_t)(py * w + px) * 3u;
            o[0] = acc[0] / (double)spp;
            o[1] = acc[1] / (double)spp;
            o[2] = acc[2] / (double)spp;
        }
}

__thread const lwo_theta *lwo_th;

void lwo64_render_mean_theta(const lwo_scene *s, const lwo_camera64 *cam, const lwo_theta *th, uint32_t x0,
                             uint32_t y0, uint32_t w, uint32_t h, uint32_t spp, double *out, int threads) {
    Cam c = cam64(s, cam);
    if (spp < 1) spp = 1;
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel num_threads(threads)
    {
        lwo_th = th;
#pragma omp for schedule(dynamic, 1)
        for (uint32_t py = 0; py < h; py++)
            for (uint32_t px = 0; px < w; px++) {
                double acc[3] = {0, 0, 0};
                for (uint32_t k = 0; k < spp; k++) {
                    V3 r = render_sample(s, &c, x0 + px, y0 + py, k);
                    if (isfinite(r.x) && isfinite(r.y) && isfinite(r.z)) {
                        acc[0] += r.x;
                        acc[1] += r.y;
                        acc[2] += r.z;
                    }
                }
                double *o = out + (uint64_t)(py * w + px) * 3u;
                for (int j = 0; j < 3; j++) o[j] = acc[j] / (double)spp;
            }
        lwo_th = NULL;
    }
}

void lwo64_render_fd_theta(const lwo_scene *s, const lwo_camera64 *cam, const lwo_theta *plus,
                           const lwo_theta *minus, uint32_t x0, uint32_t y0, uint32_t w, uint32_t h,
                           uint32_t spp, double *diff, double *mean, int threads) {
    Cam c = cam64(s, cam);
    if (spp < 1) spp = 1;
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel num_threads(threads)
    {
#pragma omp for schedule(dynamic, 1)
        for (uint32_t py = 0; py < h; py++)
            for (uint32_t px = 0; px < w; px++) {
                double dd[3] = {0, 0, 0}, mm[3] = {0, 0, 0};
                for (uint32_t k = 0; k < spp; k++) {
                    lwo_th = plus;
                    V3 a = render_sample(s, &c, x0 + px, y0 + py, k);
                    lwo_th = minus;
                    V3 b = render_sample(s, &c, x0 + px, y0 + py, k);
                    if (!(isfinite(a.x) && isfinite(a.y) && isfinite(a.z) && isfinite(b.x) && isfinite(b.y) && isfinite(b.z)))
                        continue;
                    dd[0] += a.x - b.x;
                    dd[1] += a.y - b.y;
                    dd[2] += a.z - b.z;
                    mm[0] += 0.5 * (a.x + b.x);
                    mm[1] += 0.5 * (a.y + b.y);
                    mm[2] += 0.5 * (a.z + b.z);
                }
                lwo_th = NULL;
                uint64_t i = (uint64_t)(py * w + px) * 3u;
                for (int j = 0; j < 3; j++) {
                    diff[i + j] = dd[j] / (double)spp;
                    mean[i + j] = mm[j] / (double)spp;
                }
            }
    }
}
