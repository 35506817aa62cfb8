"""Benchmark of the hq path tracer on one node: Msamples/s at the drop-in configuration.

Workload (one step): the 12x12-chunk synthetic world (value-noise terrain, water to y = 63,
oak trees, lanterns and glowstone at 1 per 2000 solid blocks), 1280x720, 1024 spp, 8 bounces,
the game sky at dusk (tick 12800) blended with Chunky's sky by the day weight, the water plane
on, FP32 radiance. One step renders every sample of the frame.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line. ``value`` times the render kernels with the scene and sky resident on the
device (CUDA events on the library's stream, max over ranks); ``e2e`` times the public
``render_hq`` call with host buffers (scene and sky uploaded, image read back) every step. With
``--impl reference`` the reference's CPU path (the CPU oracle, a restatement of the reference's
kernel and CPU backend loop) is timed on the host cores on a bounded sample of the same frame.
Under ``torchrun`` (N > 1) the frame's spp is N x 1024 and each rank renders every sample of its
1/N of the frame's 8x4-pixel tiles (weak scaling); one NCCL reduce of the accumulators per step,
inside the timed region, gives rank 0 the frame bit for bit as one GPU renders it.

At N = 1 the line also carries the path's other forms, each on its own configuration and
timed the same way (unless --no-extras): ``reference_cuda_port`` (the reference's CUDA backend
ported as written, on the same frame), ``batched_c3`` (64 cameras in one CUDA graph against 64
separate renders), ``adjoint_c4`` (forward + backward), ``precision_c5`` (3840x2160 at --c5-spp
with chunk-origin rebasing and its FP64-oracle error, the grid's frame beside it), the drop-in
image's FP64-oracle error (``accuracy``) and the tracing
kernel against the L2 read bandwidth measured in the run (``roofline_l2``).
"""

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Msamples/s (hq, 8 bounces)"
WORKLOAD = "c2: 12x12-chunk synthetic world, 1280x720, 1024 spp, 8 bounces, game sky at dusk (t=12800), water plane"


def peaks():
    """The HBM copy bandwidth (GB/s) measured on this pool's B200s, else the pool's earlier
    measurement; a figure given per timing mode takes its burst value (kernels timed launch by
    launch)."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        v = d["hbm_gbs"]
        if isinstance(v, dict):
            v = v["burst"] if "burst" in v else next(x for x in v.values() if isinstance(x, (int, float)))
        return float(v), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def algorithmic_bytes(path):
    """Bytes per path sample the tracing and shading kernels must read, from the committed counts
    of the instrumented FP32 oracle on the c2 frame (tests/test_work_counts.py recounts them and
    holds the per-access byte sizes)."""
    with open(path) as f:
        return json.load(f)


def torch_sm_count(device):
    """The GPU's SM count (148 on a B200)."""
    try:
        import torch
        return torch.cuda.get_device_properties(device).multi_processor_count
    except Exception:
        return None


def cpu_baseline(frame, budget_s=12.0):
    """The CPU oracle (the reference's kernel and CPU backend loop, restated in C, f64 sums per
    pixel, OpenMP over rows) on all host cores, on full rows spread over the frame at the frame's
    spp cut to at most 64, with as many rows (at least 24) as fill about `budget_s` seconds."""
    from oracle import oracle as O
    v = O.OracleScene.from_frame(frame)
    w, h = int(frame.params["frame"][0]), int(frame.params["frame"][1])
    threads = os.cpu_count() or 1
    rows, spp = 2, 1
    t0 = time.perf_counter()
    v.render_mean(0, h // 2, w, rows, spp, threads)
    dt = max(time.perf_counter() - t0, 1e-6)
    rate = w * rows * spp / dt
    spp = int(max(1, min(64, rate * budget_s / (w * 24))))
    n_rows = int(max(24, min(h, rate * budget_s / (w * spp))))
    samples = 0
    t0 = time.perf_counter()
    for y in np.linspace(0, h - 1, n_rows).astype(int):
        v.render_mean(0, int(y), w, 1, spp, threads)
        samples += w * spp
    dt = time.perf_counter() - t0
    return {"value": samples / dt / 1e6, "unit": "Msamples/s", "cores": threads, "kind": "port",
            "sample": f"{n_rows} full rows spread over the frame at {spp} spp ({samples} samples, {dt:.1f} s)"}


def camera64(frame):
    """The frame's camera with its f64 eye (rebased to the grid in f64), for the FP64 oracle."""
    from oracle import oracle as O
    p = frame.params
    return O.Camera64(tuple(float(x) for x in frame.eye64), tuple(float(x) for x in p["cam_fwd"][:3]),
                      tuple(float(x) for x in p["cam_right"][:3]), tuple(float(x) for x in p["cam_up"][:3]),
                      float(p["cam_pos"][3]), float(p["cam_fwd"][3]))


def accuracy(frame, img, crop=64, ref=None):
    """The image's error against the FP64 oracle (FP64 throughout, camera rays from the f64 eye, the
    same random streams) on the crop x crop pixels at the frame's centre, relative to the crop's
    mean radiance. `ref`: the oracle's crop, when already rendered."""
    from oracle import oracle as O
    p = frame.params
    w, h = int(p["frame"][0]), int(p["frame"][1])
    x0, y0 = w // 2 - crop // 2, h // 2 - crop // 2
    t0 = time.perf_counter()
    if ref is None:
        ref = O.OracleScene.from_frame(frame).render_mean64(x0, y0, crop, crop, frame.spp, cam=camera64(frame))
    dt = time.perf_counter() - t0
    err = img[y0:y0 + crop, x0:x0 + crop].astype(np.float64) - ref
    mean = float(ref.mean())
    rmse = float(np.sqrt(np.mean(err ** 2)))
    return {"crop": [x0, y0, crop, crop], "spp": frame.spp, "rmse_rel_vs_fp64_oracle": rmse / mean,
            "max_abs_err": float(np.abs(err).max()), "crop_mean": mean, "oracle_s": round(dt, 1)}


def extra_reference_port(frame, device):
    """The reference's CUDA backend ported as written (one thread per pixel in 16x16 blocks, 1-64
    spp per launch towards 150 ms, a synchronize after each; its own library) on the same frame:
    `value` from its kernels' CUDA-event time, `e2e` from the whole call (the scene and sky copied
    in, the image read back and divided on the host), as CudaBackend::render_hq does."""
    from baseline.refport import port as RP
    RP.render_hq(device, frame, spp=8)  # warm-up: module load and first launches
    p = frame.params
    samples = int(p["frame"][0]) * int(p["frame"][1]) * frame.spp
    with ClockSampler(device) as clocks:
        img, t = RP.render_hq(device, frame)
    return img, {"value": samples / t["kernel_ms"] / 1e3, "unit": "Msamples/s",
                 "e2e": samples / t["total_ms"] / 1e3, "kernel_ms": t["kernel_ms"], "total_ms": t["total_ms"],
                 "launches": t["launches"], "spp": frame.spp, "clocks": clocks.summary(),
                 "what": "pt_render + CudaBackend::render_hq ported to CUDA C++ as written (baseline/refport), "
                         "nvcc for sm_100a; the reference's own Rust-to-PTX build needs a nightly Rust toolchain "
                         "that this box lacks"}


def extra_batched(device, scale=1.0):
    """The batched form at its configuration: 64 seeded cameras (320x180..1920x1080, spp from {16,
    64, 256, 1024}, 4-8 bounces, ticks 4000 and 12800) over the 12x12-chunk world in one CUDA graph,
    tuned by the autotuner (trial batches at 1/64 of each camera's spp), against the same cameras
    as 64 separate plain renders. One timed replay (the trials warmed the kernels)."""
    from lumenwright_b200 import batch as BT
    from lumenwright_b200.native import Context
    ctx = Context(device)
    hq, jobs = BT.c3_jobs(ctx, spp_scale=scale)
    ctx.upload_hq_scene(hq)
    samples = sum(int(p["frame"][0]) * int(p["frame"][1]) * spp for p, _, spp in jobs)
    t0 = time.perf_counter()
    tuning, entry = BT.Autotuner(ctx, trial_fraction=1 / 64).tune(jobs)
    tune_s = time.perf_counter() - t0
    ctx.batch_prepare(jobs)
    with ClockSampler(device) as clocks:
        ctx.mark(0)
        ctx.batch_run()
        ctx.mark(1)
        batched_ms = ctx.elapsed(0, 1)
    ctx.set_tuning(threads=128, budget=0, sub=0, engine=0, paths=0)
    sep_ms = 0.0
    last_sky = None
    for i in sorted(range(len(jobs)), key=lambda i: id(jobs[i][1])):
        p, sky, spp = jobs[i]
        if sky is not last_sky:
            ctx.upload_sky(sky)
            last_sky = sky
        ctx.clear_accumulator(int(p["frame"][0]), int(p["frame"][1]))
        ctx.mark(2)
        ctx.render_device(p, 0, spp)
        ctx.mark(3)
        sep_ms += ctx.elapsed(2, 3)
    ctx.close()
    return {"value": samples / batched_ms / 1e3, "unit": "Msamples/s", "ms": batched_ms, "samples": samples,
            "cameras": len(jobs), "spp_scale": scale, "tuning": tuning, "autotune_s": round(tune_s, 1),
            "separate_launches": {"value": samples / sep_ms / 1e3, "ms": sep_ms},
            "speedup_vs_separate": sep_ms / batched_ms, "clocks": clocks.summary()}


def extra_adjoint(device, steps=3):
    """The differentiable form: forward (FP64 image) + path-replay backward of the L2 image loss on
    the differentiation configuration (8x8 chunks, 512x288, 64 spp, 4 bounces, Chunky sky);
    `value` from the two kernels' CUDA-event time, `e2e` from DiffProblem.gradient (host set-up,
    copies and the sky cache's FP64 Jacobian included)."""
    from lumenwright_b200 import adjoint as A
    from lumenwright_b200.native import Context
    ctx = Context(device)
    prob = A.DiffProblem(ctx)
    a = prob._args(prob.theta0)
    samples = prob.width * prob.height * prob.spp
    img = ctx.adjoint_forward(*a, prob.spp)
    ctx.adjoint_backward(*a, prob.spp, 2.0 * (img - prob.target))
    fwd = bwd = 0.0
    with ClockSampler(device) as clocks:
        for _ in range(steps):
            img = ctx.adjoint_forward(*a, prob.spp)
            fwd += ctx.stats()["kernel_ms"]
            ctx.adjoint_backward(*a, prob.spp, 2.0 * (img - prob.target))
            bwd += ctx.stats()["kernel_ms"]
    t0 = time.perf_counter()
    for _ in range(steps):
        prob.gradient(prob.theta0)
    e2e_s = (time.perf_counter() - t0) / steps
    ctx.close()
    ms = (fwd + bwd) / steps
    return {"value": samples / ms / 1e3, "unit": "Msamples/s (forward + backward)", "forward_ms": fwd / steps,
            "backward_ms": bwd / steps, "e2e": samples / e2e_s / 1e6, "steps": steps, "parameters": A.N_THETA,
            "clocks": clocks.summary()}


def extra_precision(device, spp):
    """The precision configuration's frame (32x32 chunks translated to x = 1,000,000, 3840x2160, 8
    bounces) at `spp` (of its 4096): FP32 traversal with chunk-origin rebasing (every path origin
    held relative to its nearest chunk corner), Kahan FP32 sums; its error against the FP64 oracle
    on the 64x64 centre crop. The same frame in the grid's frame (positions relative to the grid
    origin, as the reference holds them) beside it, and, per sample on a 32x32 centre crop at 16
    spp, the paths that split from the FP64 twin in each frame."""
    from lumenwright_b200 import request as R
    from lumenwright_b200.native import Context
    from oracle import oracle as O
    ctx = Context(device)
    grid = R.make_frame(R.CONFIGS["c5"], sky_backend=ctx, spp=spp)
    chunk = R.with_chunk_frames(grid)
    p = grid.params
    w, h = int(p["frame"][0]), int(p["frame"][1])
    ctx.upload_hq_scene(grid.scene)
    ctx.upload_sky(grid.sky)
    view = O.OracleScene.from_frame(grid)
    crop = 64
    x0, y0 = w // 2 - crop // 2, h // 2 - crop // 2
    ref = view.render_mean64(x0, y0, crop, crop, spp, cam=camera64(grid))
    out = {}
    for name, frame in (("chunk", chunk), ("grid", grid)):
        ctx.clear_accumulator(w, h)
        ctx.render_device(frame.params, 0, 2)  # warm-up
        ctx.stats()
        ctx.clear_accumulator(w, h)
        with ClockSampler(device) as clocks:
            ctx.mark(0)
            ctx.render_device(frame.params, 0, spp)
            ctx.mark(1)
            ms = ctx.elapsed(0, 1)
        st = ctx.stats()
        img = ctx.read_accumulator(w, h)
        out[name] = {"value": w * h * spp / ms / 1e3, "unit": "Msamples/s", "ms": ms, "launches": st["launches"],
                     "trace_ms": st["trace_ms"], "shade_ms": st["shade_ms"], "accuracy": accuracy(frame, img, crop, ref),
                     "clocks": clocks.summary()}
    n, count = 32, 16
    sx, sy = w // 2 - n // 2, h // 2 - n // 2
    ref_s = view.render_samples64(sx, sy, n, n, 0, count, cam=camera64(grid))
    splits = {"crop": [sx, sy, n, n], "samples": n * n * count}
    for name, frame in (("chunk", chunk), ("grid", grid)):
        got = ctx.render_samples(frame.params, sx, sy, n, n, 0, count).astype(np.float64)
        err = np.abs(got - ref_s)
        split = np.any(err > 1e-3 * np.maximum(np.abs(ref_s), np.abs(got)) + 1e-5, axis=-1)
        splits[name] = int(split.sum())
    ctx.close()
    line = dict(out["chunk"])
    line.update({"frames": "chunk-origin rebasing", "width": w, "height": h, "spp": spp, "of_spp": R.CONFIGS["c5"].spp,
                 "grid_frame": out["grid"], "paths_split_from_fp64": splits})
    return line


def run_reference(args, rank, world):
    """--impl reference: the reference's CPU path (the oracle restatement) timed per step on a
    bounded sample of the workload, all host threads, rank 0 only."""
    if rank != 0:
        return
    from lumenwright_b200 import request as R
    from oracle import oracle as O
    frame = R.make_frame(R.CONFIGS["c2"], sky_backend=OracleSkyOnHost())
    v = O.OracleScene.from_frame(frame)
    w, h = int(frame.params["frame"][0]), int(frame.params["frame"][1])
    threads = os.cpu_count() or 1
    rows = np.linspace(0, h - 1, 8).astype(int)
    spp = 4

    def step():
        n = 0
        for y in rows:
            v.render_mean(0, int(y), w, 1, spp, threads)
            n += w * spp
        return n

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    n = 0
    for _ in range(args.steps):
        n += step()
    dt = time.perf_counter() - t0
    val = n / dt / 1e6
    sample = f"each step: 8 full rows spread over the frame at {spp} spp ({len(rows) * w * spp} samples)"
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": val, "unit": "Msamples/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "reference": "CPU path of the reference (kernel + CpuBackend loop) restated in C; "
                   "no Rust toolchain on this box to build the reference itself"},
        "cpu_baseline": {"value": val, "unit": "Msamples/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": val, "unit": "Msamples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


class OracleSkyOnHost:
    """Sky inputs built on the host by the oracle (for the CPU reference arm, which must not need
    a GPU): Chunky's sky cache, the game sky's maps, and the blend of Chunky's sky into them."""

    def build_sky_cache(self, params, n):
        from oracle import oracle as O
        v = O.OracleScene(params, None, None, None, None, None, None)
        return v.build_sky_cache(n)

    def draw_sky_map(self, quick_sky, stars, w, h, atlas, atlas_w):
        from oracle import oracle as O
        return O.draw_sky_map(quick_sky, stars, w, h, atlas, atlas_w)

    def blend_chunky_sky(self, params, cache, maps, sizes, weight):
        from lumenwright_b200 import sky as SK
        from oracle import oracle as O
        v = O.OracleScene(params, None, None, None, None, None, None, cache)
        out = maps.copy()
        off = 0
        w = np.float32(weight)
        for mw, mh in ((int(sizes[0]), int(sizes[1])), (int(sizes[2]), int(sizes[3]))):
            j, i = np.mgrid[0:mh, 0:mw]
            c = v.sky_radiance_many(SK.map_direction(i.ravel(), j.ravel(), mw, mh))
            seg = out[off:off + mw * mh * 3].reshape(-1, 3)
            seg[:] = w * c + (np.float32(1.0) - w) * seg
            off += mw * mh * 3
        return out


def run_batched(args):
    """The batched form: 64 seeded cameras (320x180..1920x1080, spp from {16, 64, 256, 1024} scaled
    by --c3-scale, 4-8 bounces, ticks 4000/12800) over the 12x12-chunk world in one CUDA graph (the
    wavefront engine's device-side iteration loop, or the persistent megakernel, as the autotuner
    picks), against the same cameras as 64 separate plain renders (`lw_render_device` with the
    default tuning, each with its own iterations and reduction)."""
    from lumenwright_b200 import batch as BT
    from lumenwright_b200.native import Context
    ctx = Context(0)
    hq, jobs = BT.c3_jobs(ctx, spp_scale=args.c3_scale)
    ctx.upload_hq_scene(hq)
    samples = sum(int(p["frame"][0]) * int(p["frame"][1]) * spp for p, _, spp in jobs)
    tuning, entry = BT.Autotuner(ctx).tune(jobs)
    ctx.batch_prepare(jobs)
    for _ in range(args.warmup):
        ctx.batch_run()
    ctx.stats()
    ctx.mark(0)
    for _ in range(args.steps):
        ctx.batch_run()
    ctx.mark(1)
    batched_ms = ctx.elapsed(0, 1) / args.steps
    # The same cameras as separate plain launches.
    ctx.set_tuning(threads=128, budget=0, sub=0, engine=0, paths=0)
    sep_ms = 0.0
    order = sorted(range(len(jobs)), key=lambda i: id(jobs[i][1]))
    last_sky = None
    for i in order:
        p, sky, spp = jobs[i]
        if sky is not last_sky:
            ctx.upload_sky(sky)
            last_sky = sky
        w, h = int(p["frame"][0]), int(p["frame"][1])
        ctx.clear_accumulator(w, h)
        ctx.mark(2)
        ctx.render_device(p, 0, spp)
        ctx.mark(3)
        sep_ms += ctx.elapsed(2, 3)
    print(json.dumps({
        "metric": "Msamples/s (hq batched, 64 cameras)", "value": samples / batched_ms / 1e3, "unit": "Msamples/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": batched_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"c3: 64 cameras over the 12x12-chunk world, spp x{args.c3_scale}",
                   "samples_per_step": samples, "tuning": tuning, "autotune_key": entry.get("key")},
        "separate_launches": {"value": samples / sep_ms / 1e3, "unit": "Msamples/s", "ms": sep_ms},
        "speedup_vs_separate": sep_ms / batched_ms,
    }), flush=True)
    ctx.close()


def run_adjoint(args):
    """The differentiable form: one gradient of the L2 image loss on the differentiation workload
    (8x8-chunk world with emitters, 512x288, 64 spp, 4 bounces, Chunky sky) per step: the FP64
    forward image then the two-replay backward. `value` counts the forward's samples per second of
    forward + backward kernel time; `e2e` times `DiffProblem.gradient` (host set-up, copies and the
    sky Jacobian included)."""
    from lumenwright_b200 import adjoint as A
    from lumenwright_b200.native import Context
    ctx = Context(0)
    prob = A.DiffProblem(ctx)
    theta = prob.theta0
    args_ = prob._args(theta)
    samples = prob.width * prob.height * prob.spp
    for _ in range(args.warmup):
        img = ctx.adjoint_forward(*args_, prob.spp)
        ctx.adjoint_backward(*args_, prob.spp, 2.0 * (img - prob.target))
    fwd_ms = bwd_ms = 0.0
    with ClockSampler(0) as clocks:
        for _ in range(args.steps):
            img = ctx.adjoint_forward(*args_, prob.spp)
            fwd_ms += ctx.stats()["kernel_ms"]
            ctx.adjoint_backward(*args_, prob.spp, 2.0 * (img - prob.target))
            bwd_ms += ctx.stats()["kernel_ms"]
    t0 = time.perf_counter()
    for _ in range(args.steps):
        prob.gradient(theta)
    e2e_s = (time.perf_counter() - t0) / args.steps
    ms = (fwd_ms + bwd_ms) / args.steps
    frame_in = args_[2].nbytes + args_[3].nbytes + args_[4].nbytes + args_[1].nbytes
    print(json.dumps({
        "metric": "Msamples/s (adjoint: forward + path-replay backward)", "value": samples / ms / 1e3,
        "unit": "Msamples/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 sums)",
        "data": "synthetic",
        "config": {"workload": "c4: 8x8-chunk world with emitters, 512x288, 64 spp, 4 bounces, Chunky sky",
                   "forward_ms": fwd_ms / args.steps, "backward_ms": bwd_ms / args.steps,
                   "parameters": A.N_THETA},
        "e2e": {"value": samples / e2e_s / 1e6, "unit": "Msamples/s",
                # forward and backward each upload theta, the texel map, the sky and the params;
                # the backward also the image gradient
                "h2d_bytes_per_step": int(2 * (frame_in + 432) + img.nbytes),
                # the sky cache built on the device, the image, the gradient
                "d2h_bytes_per_step": int(args_[1].nbytes + img.nbytes + (A.N_ALBEDO + A.GROUPS + args_[1].size + 3) * 8)},
        "gpu_launches": 2 * args.steps, "clocks": clocks.summary(),
    }), flush=True)
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--spp", type=int, default=1024)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="c2", choices=["c2", "c3", "c4"],
                    help="c2: the drop-in frame (default); c3: the batched form, 64 cameras; "
                         "c4: the differentiable form, one loss gradient")
    ap.add_argument("--c3-scale", type=float, default=0.25, help="spp scale of the 64 cameras (c3)")
    ap.add_argument("--no-extras", action="store_true",
                    help="leave out the other forms' lines (reference port, batched, adjoint, precision)")
    ap.add_argument("--c5-spp", type=int, default=1024, help="spp of the precision frame in the extras (each frame)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    from lumenwright_b200 import request as R
    from lumenwright_b200.native import Context

    if args.workload == "c3":
        run_batched(args)
        return
    if args.workload == "c4":
        run_adjoint(args)
        return

    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))

    ctx = Context(local)
    cfg = R.CONFIGS["c2"]
    frame = R.make_frame(cfg, sky_backend=ctx, spp=args.spp)
    p = frame.params
    w, h = int(p["frame"][0]), int(p["frame"][1])
    spp = frame.spp
    samples_per_step = w * h * spp
    ctx.upload_hq_scene(frame.scene)
    ctx.upload_sky(frame.sky)

    from lumenwright_b200 import shard

    # Under N ranks the frame's spp is N times the single GPU's and each rank renders every sample
    # of 1/N of the frame's tiles (weak scaling: each rank's work is one frame at `spp`); one NCCL
    # SUM reduce of the accumulator records per step, inside the timed region, gives rank 0 the
    # frame bit for bit as one GPU would render it.
    fspp = shard.frame_spp(spp, world)

    def device_step(i):
        ctx.clear_accumulator(w, h)
        if dist:
            ctx.render_device_shard(p, i * fspp, fspp, rank, world)
            shard.reduce_accumulator(ctx, dist)
        else:
            ctx.render_device(p, i * spp, spp)

    for i in range(args.warmup):
        device_step(i)
    ctx.stats()  # waits for the warm-up
    if dist:
        dist.barrier()
    ctx.mark(0)
    launches = 0
    trace_ms = shade_ms = kernel_ms = 0.0
    trace_launches = rays = 0
    with ClockSampler(local) as clocks:
        for i in range(args.steps):
            device_step(args.warmup + i)
            st = ctx.stats()
            launches += st["launches"]
            kernel_ms += st["kernel_ms"]
            trace_ms += st["trace_ms"]
            shade_ms += st["shade_ms"]
            trace_launches += st["trace_launches"]
            rays += st["rays"]
        ctx.mark(1)
        total_ms = ctx.elapsed(0, 1)
    if dist:
        import torch
        t = torch.tensor([total_ms], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = samples_per_step * args.steps * world / (total_ms / 1e3) / 1e6

    # End to end through the public render_hq with host buffers, every step.
    from lumenwright_b200.native import B200Backend
    be = B200Backend(local)
    h2d = frame.scene.memory_bytes() + frame.sky.nbytes + 432
    d2h = w * h * 3 * 4
    e2e_frame = frame
    # one GPU: the public render_hq; N ranks: the same calls with host buffers on each rank's tiles,
    # the accumulators reduced and read back on rank 0 (shard.render_hq_sharded)
    e2e_step = ((lambda: be.render_hq(e2e_frame).reshape(h, w, 3)) if not dist else
                (lambda: shard.render_hq_sharded(be.ctx, e2e_frame, dist, rank, world, spp=fspp)))
    e2e_img = e2e_step()  # warm-up (its image is checked below)
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for i in range(args.steps):
        e2e_step()
    e2e_s = time.perf_counter() - t0
    if dist:
        import torch
        t = torch.tensor([e2e_s], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = samples_per_step * args.steps * world / e2e_s / 1e6

    if rank == 0:
        peak, peak_kind = peaks()
        alg = algorithmic_bytes(os.path.join(ROOT, "profiles", "algorithmic_bytes_c2.json"))
        # The dominant kernel is the wavefront's tracing kernel: the scene bytes its traversals read
        # per launch over its average launch time (CUDA events around each launch).
        my_samples = samples_per_step * args.steps
        trace_bytes = alg["trace_bytes_per_sample"] * my_samples
        achieved = trace_bytes / (trace_ms / 1e3) / 1e9 if trace_ms > 0 else None
        # DRAM traffic per launch: the ncu capture's bytes per traced ray times this run's rays per
        # tracing launch.
        with open(os.path.join(ROOT, "profiles", "k_wf_trace_traffic_c2.json")) as f:
            capture = json.load(f)
        per_ray = capture["dram_bytes_per_ray"]
        traffic = per_ray * rays / max(1, trace_launches)
        # The bound the tracing kernel actually meets is instruction issue (the scene is L1/L2
        # resident): warp instructions per traced ray from the same capture, times this run's rays,
        # over the kernel's event time, against one instruction per scheduler per cycle (4 per SM)
        # at the SM clock sampled during the timed steps.
        clk = clocks.summary()
        sms = torch_sm_count(local)
        issue_peak = sms * 4 * (clk.get("sm_mhz") or 0) / 1e3 if clk and sms else None
        issue = (capture["warp_instructions_per_ray"] * rays / (trace_ms / 1e3) / 1e9
                 if trace_ms > 0 and "warp_instructions_per_ray" in capture else None)
        line = {
            "metric": METRIC, "value": value, "unit": "Msamples/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "width": w, "height": h, "spp": spp, "bounces": int(p["frame"][3]),
                       "parallelism": f"interleaved tiles x{world}, frame spp {fspp}" if world > 1 else "1 GPU",
                       "engine": "wavefront", "tuning": ctx.get_tuning(),
                       "l2": "the scene and sky maps (~30 MB) stay L2-resident by design; the path slots "
                             "(up to 2.7 GB) and the partial sums are larger than L2",
                       "emitters": cfg.notes.get("emitters"), "day_weight": cfg.notes.get("weight")},
            "e2e": {"value": e2e, "unit": "Msamples/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": launches,
            "kernels": {"trace_ms": trace_ms, "shade_ms": shade_ms, "other_ms": kernel_ms - trace_ms - shade_ms,
                        "trace_launches": trace_launches},
            "roofline": {"bound": "hbm", "kernel": "k_wf_trace", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak if achieved else None, "traffic": traffic, "peak_kind": peak_kind,
                         "traffic_unit": "bytes per launch (ncu DRAM bytes per ray x rays per launch)",
                         "rays_per_launch": rays / max(1, trace_launches),
                         "algorithmic_bytes_per_launch": trace_bytes / max(1, trace_launches),
                         "avg_launch_ms": trace_ms / max(1, trace_launches),
                         "trace_bytes_per_sample": alg["trace_bytes_per_sample"],
                         # the same accesses rounded up to the 32-byte sectors L2 and DRAM move
                         "trace_sector_bytes_per_sample": alg.get("trace_sector_bytes_per_sample"),
                         "achieved_sector_rounded": (alg["trace_sector_bytes_per_sample"] * my_samples / (trace_ms / 1e3) / 1e9
                                                     if trace_ms > 0 and "trace_sector_bytes_per_sample" in alg else None)},
            "roofline_issue": {"bound": "issue", "kernel": "k_wf_trace", "achieved": issue, "peak": issue_peak,
                               "unit": "G warp instructions/s",
                               "frac": issue / issue_peak if issue and issue_peak else None,
                               "peak_kind": f"nominal: {sms} SMs x 4 schedulers x the sampled SM clock",
                               "instructions": "ncu warp instructions per traced ray x rays"},
            "clocks": clk,
        }
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(frame)
        if world == 1 and not args.no_extras:
            # The other forms of the path (batched, adjoint, precision), each on its own configuration,
            # timed the same way.
            line["accuracy"] = accuracy(frame, e2e_img)
            port_img, port = extra_reference_port(frame, local)
            port["image_rel_rmse_vs_product"] = float(np.sqrt(np.mean((port_img - e2e_img) ** 2)) / e2e_img.mean())
            line["reference_cuda_port"] = port
            line["vs_reference_cuda_port"] = {"value": value / port["value"], "e2e": e2e / port["e2e"]}
            from baseline.refport import port as RP
            l2 = RP.l2_read_gbs(local)
            line["roofline_l2"] = {"bound": "l2", "kernel": "k_wf_trace", "achieved": achieved, "peak": l2,
                                   "unit": "GB/s", "frac": achieved / l2 if achieved and l2 else None,
                                   "peak_kind": "measured in this run: a 32 MB buffer read 200 times over by every "
                                                "SM (16-byte L2 loads), CUDA events",
                                   "warp_execution_efficiency": capture.get("active_lanes_per_instruction", 0) / 32.0}
            line["batched_c3"] = extra_batched(local, scale=1.0)
            line["adjoint_c4"] = extra_adjoint(local)
            line["precision_c5"] = extra_precision(local, args.c5_spp)
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
