"""Converged images against the FP64 oracle, per configuration and per origin frame: the GPU
renders the whole frame (FP32 DDA, Kahan-compensated FP32 sums) and the FP64 twin of the oracle
renders a 64x64 crop at the frame's centre with the same random streams, its camera rays starting
from the f64 eye (rebased to the grid in f64). "grid": the FP32 path holds its positions relative
to the grid origin, as the reference does; "chunk": with chunk-origin rebasing, relative to the
chunk corner nearest each origin. The per-pixel RMSE and maximum error, absolute and relative to
the crop's mean radiance, are checked against a bound and, with LW_REPORT_DIR set, written to
LW_REPORT_DIR/precision_<config>_<frames>.json.

A second test counts, per sample, the paths that split between the precisions (an FP32 sample
more than 1e-3 relative from its FP64 twin) on a 32x32 crop at the frame's centre, in both frames.

By default each configuration runs at a reduced spp (the full frame size); LW_PRECISION_FULL=1
runs the configurations' own spp (c5: 3840x2160 at 4096 spp)."""

import json
import os
import time

import numpy as np
import pytest

from lumenwright_b200 import request as R
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FULL = os.environ.get("LW_PRECISION_FULL") == "1"
SPP = {"c1": 16, "c2": 64, "c4": 64, "c5": 64}
CROP = 64


@pytest.fixture(scope="module")
def ctx():
    from lumenwright_b200.native import Context
    c = Context(0)
    yield c
    c.close()


_FRAMES = {}


def frame_of(ctx, name, spp, frames):
    """The configuration's frame (built once per spp), in the grid's or in chunk frames."""
    key = (name, spp)
    if key not in _FRAMES:
        _FRAMES.clear()  # one world resident at a time
        _FRAMES[key] = R.make_frame(R.CONFIGS[name], sky_backend=ctx, spp=spp)
    f = _FRAMES[key]
    return R.with_chunk_frames(f) if frames == "chunk" else f


def camera64(frame):
    p = frame.params
    return O.Camera64((frame.eye64[0], frame.eye64[1], frame.eye64[2]), tuple(float(x) for x in p["cam_fwd"][:3]),
                      tuple(float(x) for x in p["cam_right"][:3]), tuple(float(x) for x in p["cam_up"][:3]),
                      float(p["cam_pos"][3]), float(p["cam_fwd"][3]))


@pytest.mark.parametrize("name", ["c1", "c2", "c4", "c5"])
@pytest.mark.parametrize("frames", ["grid", "chunk"])
def test_converged_image_against_fp64_oracle(ctx, name, frames):
    cfg = R.CONFIGS[name]
    spp = cfg.spp if FULL else SPP[name]
    frame = frame_of(ctx, name, spp, frames)
    p = frame.params
    w, h = int(p["frame"][0]), int(p["frame"][1])
    ctx.upload_hq_scene(frame.scene)
    t0 = time.perf_counter()
    img = ctx.render_hq(p, frame.sky, spp)
    gpu_s = time.perf_counter() - t0
    x0, y0 = w // 2 - CROP // 2, h // 2 - CROP // 2
    view = O.OracleScene.from_frame(frame)
    t0 = time.perf_counter()
    ref = view.render_mean64(x0, y0, CROP, CROP, spp, cam=camera64(frame))
    cpu_s = time.perf_counter() - t0
    got = img[y0:y0 + CROP, x0:x0 + CROP].astype(np.float64)
    err = got - ref
    mean = float(ref.mean())
    rmse = float(np.sqrt(np.mean(err ** 2)))
    row = {"config": name, "frames": frames, "width": w, "height": h, "spp": spp, "bounces": int(p["frame"][3]),
           "crop": [x0, y0, CROP, CROP], "mean_radiance": mean, "rmse": rmse, "rmse_rel": rmse / mean,
           "max_abs": float(np.abs(err).max()), "max_rel_pixel": float((np.abs(err) / np.maximum(ref, 1e-3)).max()),
           "pixels_within_1e-3_rel": float(np.mean(np.abs(err) <= 1e-3 * np.maximum(ref, 1e-3))),
           "gpu_render_s": gpu_s, "gpu_msamples_per_s": w * h * spp / gpu_s / 1e6, "oracle_s": cpu_s,
           "eye64": list(frame.eye64)}
    out = os.environ.get("LW_REPORT_DIR")
    if out:
        os.makedirs(out, exist_ok=True)
        with open(os.path.join(out, f"precision_{name}_{frames}.json"), "w") as f:
            json.dump(row, f, indent=1)
    assert O.bounds_errors() == 0
    assert np.isfinite(img).all()
    assert row["rmse_rel"] < 2e-2, row


SPLIT_SPP = {"c1": 16, "c2": 16, "c4": 16, "c5": 16}


@pytest.mark.parametrize("name", ["c2", "c5"])
def test_paths_that_split_from_the_fp64_twin(ctx, name):
    # Per sample: the GPU's FP32 radiance (lw_render_samples) in each frame against the FP64 twin's
    # on the same streams; a sample more than 1e-3 relative (and 1e-5 absolute) away took another
    # path in one precision (an edge met, a roulette or Fresnel draw at its threshold).
    frame = frame_of(ctx, name, SPP[name], "grid")
    p = frame.params
    w, h = int(p["frame"][0]), int(p["frame"][1])
    n, count = 32, SPLIT_SPP[name]
    x0, y0 = w // 2 - n // 2, h // 2 - n // 2
    ref = O.OracleScene.from_frame(frame).render_samples64(x0, y0, n, n, 0, count, cam=camera64(frame))
    ctx.upload_hq_scene(frame.scene)
    ctx.upload_sky(frame.sky)
    row = {"config": name, "crop": [x0, y0, n, n], "samples": n * n * count}
    for frames in ("grid", "chunk"):
        f = frame_of(ctx, name, SPP[name], frames)
        got = ctx.render_samples(f.params, x0, y0, n, n, 0, count).astype(np.float64)
        err = np.abs(got - ref)
        split = np.any(err > 1e-3 * np.maximum(np.abs(ref), np.abs(got)) + 1e-5, axis=-1)
        row[frames] = {"split": int(split.sum()), "split_fraction": float(split.mean()),
                       "max_abs": float(err.max()), "median_rel": float(np.median(err / np.maximum(np.abs(ref), 1e-6)))}
    print(f"{name}: paths split from FP64, grid frame {row['grid']['split']} of {row['samples']}, chunk frames "
          f"{row['chunk']['split']}")
    out = os.environ.get("LW_REPORT_DIR")
    if out:
        os.makedirs(out, exist_ok=True)
        with open(os.path.join(out, f"splits_{name}.json"), "w") as f:
            json.dump(row, f, indent=1)
    assert row["grid"]["split_fraction"] < 0.05 and row["chunk"]["split_fraction"] < 0.05, row
