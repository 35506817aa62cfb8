"""Chunk-origin rebasing (the precision form's option, Params.see_through[2] = 1) on the GPU against
the FP32 oracle's restatement of it (oracle/kernel_impl.h), on the same inputs and seeded streams:

* per-sample radiance on crops of the C2 frame (emitters, water plane, game sky) and of the C5
  frame (32x32 chunks translated to x = 1,000,000, the camera at a fractional position): every
  sample within 1e-4 relative, the fraction bit-equal printed (the device and the oracle form the
  same frames by the same exact steps, so none is expected to differ);
* the wavefront engine's image equal bit for bit to the megakernel's in chunk frames;
* the forms that take the grid's frame only (the batched form) refuse chunk frames, and a frame
  flag other than 0 or 1 is refused.
"""

import numpy as np
import pytest

from lumenwright_b200 import request as R
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from lumenwright_b200.native import Context
    c = Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def c2(ctx):
    return R.with_chunk_frames(R.make_frame(R.CONFIGS["c2"], sky_backend=ctx, spp=4))


@pytest.fixture(scope="module")
def c5(ctx):
    return R.with_chunk_frames(R.make_frame(R.CONFIGS["c5"], sky_backend=ctx, spp=4))


def close(a, b, rel=1e-4, atol=1e-6):
    return np.abs(a - b) <= rel * np.maximum(np.abs(a), np.abs(b)) + atol


def per_sample(ctx, frame, x0, y0, w, h, count, start=0):
    ctx.upload_hq_scene(frame.scene)
    ctx.upload_sky(frame.sky)
    got = ctx.render_samples(frame.params, x0, y0, w, h, start, count)
    want = O.OracleScene.from_frame(frame).render_samples(x0, y0, w, h, start, count)
    ok = np.all(close(got, want), axis=-1)
    exact = np.all(got.view(np.uint32) == want.view(np.uint32), axis=-1)
    bad = np.argwhere(~ok)
    print(f"chunk frames {(x0, y0, w, h)} samples {start}..{start + count - 1}: {ok.mean():.6f} within 1e-4, "
          f"{exact.mean():.6f} bit-equal; first outside: {bad[:3].tolist()}")
    return ok.mean(), exact.mean()


def test_the_frames_start_at_the_cameras_chunk(c5):
    p = c5.params
    assert int(p["see_through"][2]) == 1
    assert all(abs(float(v)) <= 8.0 for v in p["cam_pos"][:3])


@pytest.mark.parametrize("rect", [(0, 0, 64, 32), (600, 300, 64, 32), (1200, 680, 64, 32), (320, 500, 64, 32)])
def test_c2_per_sample_radiance_in_chunk_frames(ctx, c2, rect):
    ok, exact = per_sample(ctx, c2, *rect, 2)
    assert ok == 1.0, ok


@pytest.mark.parametrize("rect", [(0, 0, 48, 24), (1896, 1068, 48, 24), (3792, 2136, 48, 24), (700, 1700, 48, 24),
                                  (3000, 400, 48, 24)])
def test_c5_per_sample_radiance_in_chunk_frames(ctx, c5, rect):
    ok, exact = per_sample(ctx, c5, *rect, 2)
    assert ok == 1.0, ok


def test_c5_per_sample_radiance_in_chunk_frames_far_into_the_stream(ctx, c5):
    ok, exact = per_sample(ctx, c5, 1896, 1068, 32, 16, 3, start=4093)
    assert ok == 1.0, ok


@pytest.mark.parametrize("paths", [0, 1 << 12])
def test_wavefront_and_megakernel_give_the_same_image_in_chunk_frames(ctx, c2, paths):
    from lumenwright_b200.native import ENGINE_MEGAKERNEL, ENGINE_WAVEFRONT
    p = c2.params
    ctx.upload_hq_scene(c2.scene)
    ctx.set_tuning(engine=ENGINE_MEGAKERNEL, sub=3)
    want = ctx.render_hq(p, c2.sky, 12)
    ctx.set_tuning(engine=ENGINE_WAVEFRONT, paths=paths)
    got = ctx.render_hq(p, c2.sky, 12)
    ctx.set_tuning(engine=ENGINE_WAVEFRONT, paths=0, sub=0)
    assert np.array_equal(got, want)


def test_the_grid_frame_only_forms_refuse_chunk_frames(ctx, c2):
    from lumenwright_b200.native import LwError
    ctx.upload_hq_scene(c2.scene)
    with pytest.raises(LwError) as e:
        ctx.batch_prepare([(c2.params, c2.sky, 1)])
    assert e.value.status == 1
    bad = c2.params.copy()
    bad["see_through"][2] = 2
    with pytest.raises(LwError) as e:
        ctx.render_hq(bad, c2.sky, 1)
    assert e.value.status == 1
