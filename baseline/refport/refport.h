/*
 * liblw_refport: the reference's CUDA backend ported to CUDA C++ as written, the comparison
 * baseline of the benchmark (not part of the product library). One call does what
 * `CudaBackend::render_hq` (crates/lumenwright/src/render/cuda.rs:77-184) does for one frame:
 * copies the scene and sky buffers to the device, runs `pt_render`
 * (crates/lumenwright-ptx/src/lib.rs:37-87) in batches of 1 to 64 spp towards 150 ms a launch with
 * a synchronize after each, reads the accumulator back, divides on the host and frees the
 * buffers. Same inputs and output as lw_render_hq. It also holds the benchmark's L2 read probe.
 */
#ifndef LW_REFPORT_H
#define LW_REFPORT_H

#include <stdint.h>

#include "lumenwright_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    double kernel_ms; /* CUDA-event time of the pt_render launches */
    double upload_ms; /* the buffers' allocation and copies */
    double total_ms;  /* the whole call, wall clock */
    uint32_t launches;
} lwr_timing;

/* 0 on success; otherwise an lw_status code (1 a null argument, 3 out of memory, 5 a CUDA
 * failure, 7 no such device). */
int lwr_render_hq(int device, const lw_scene_desc *scene, const lw_params *params, const float *sky, uint64_t sky_len,
                  uint32_t spp, float *out_rgb, lwr_timing *timing);

/* The L2 read bandwidth in GB/s: a buffer of `bytes` (small enough to stay in L2) read `passes`
 * times over by every SM after a warm-up pass, timed by CUDA events. */
int lwr_l2_read_gbs(int device, uint64_t bytes, uint32_t passes, double *gbs);

#ifdef __cplusplus
}
#endif
#endif
