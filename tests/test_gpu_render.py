"""CUDA parity at the benchmark configurations (synthetic worlds): the device sky cache, per-sample
radiance on crops of the C1 and C2 frames, and the C1 frame's mean through `render_hq`, each
against the FP32 oracle on the same inputs and seeded RNG stream.

Tolerances: every sample within 1e-4 relative (the fraction bit-equal is printed; the kernels and
the oracle call the same correctly rounded exponential for the water, so none is expected to
differ), including samples far into the stream (indices 290-292, where the drop-in's launches of
the C2 frame meet, and 1000-1023); pixel means 1e-4 relative, on the C1 frame and on a 64x64 crop
of the C2 frame at its full 1024 spp (the render then runs in several launches).
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
def c1(ctx):
    return R.make_frame(R.CONFIGS["c1"], sky_backend=ctx)


@pytest.fixture(scope="module")
def c2(ctx):
    return R.make_frame(R.CONFIGS["c2"], sky_backend=ctx, spp=4)


def close(a, b, rel=1e-4, atol=1e-6):
    return np.abs(a - b) <= rel * np.maximum(np.abs(a), np.abs(b)) + atol


def test_device_sky_cache_matches_the_oracle(ctx, c1):
    p = c1.params
    got = ctx.build_sky_cache(p, 128)
    want = O.OracleScene(p, None, None, None, None, None, None).build_sky_cache(128)
    assert got.shape == want.shape
    np.testing.assert_allclose(got, want, rtol=2e-5, atol=2e-6)


def per_sample(ctx, frame, x0, y0, w, h, count, start=0):
    ctx.upload_hq_scene(frame.scene)
    ctx.upload_sky(frame.sky)
    got = ctx.render_samples(frame.params, x0, y0, w, h, start, count)
    want = O.OracleScene.from_frame(frame).render_samples(x0, y0, w, h, start, count)
    ok = np.all(close(got, want), axis=-1)
    exact = np.all(got.view(np.uint32) == want.view(np.uint32), axis=-1)
    return ok.mean(), exact.mean(), got, want


def report(name, rect, ok, exact, got, want):
    bad = np.argwhere(~np.all(close(got, want), axis=-1))
    print(f"{name} {rect}: {ok:.6f} of samples within 1e-4, {exact:.6f} bit-equal; first outside: {bad[:3].tolist()}")


@pytest.mark.parametrize("rect", [(0, 0, 64, 36), (96, 54, 64, 36), (192, 100, 64, 44)])
def test_c1_per_sample_radiance(ctx, c1, rect):
    ok, exact, got, want = per_sample(ctx, c1, *rect, 4)
    report("C1", rect, ok, exact, got, want)
    assert ok == 1.0, ok


@pytest.mark.parametrize("rect", [(0, 0, 64, 32), (600, 300, 64, 32), (1200, 680, 64, 32), (320, 500, 64, 32)])
def test_c2_per_sample_radiance(ctx, c2, rect):
    ok, exact, got, want = per_sample(ctx, c2, *rect, 2)
    report("C2", rect, ok, exact, got, want)
    assert ok == 1.0, ok


@pytest.mark.parametrize("start,count", [(290, 3), (1000, 4), (1020, 4)])
@pytest.mark.parametrize("rect", [(600, 300, 48, 24), (100, 600, 48, 24)])
def test_c2_per_sample_radiance_far_into_the_stream(ctx, c2, rect, start, count):
    # Samples 290-292 (where the drop-in's launches of the C2 frame met under a 4 GiB item-sum
    # cap) and 1000-1023, the frame's last samples at 1024 spp.
    ok, exact, got, want = per_sample(ctx, c2, *rect, count, start=start)
    report(f"C2 samples {start}..{start + count - 1}", rect, ok, exact, got, want)
    assert ok == 1.0, ok


@pytest.mark.parametrize("start", [500, 4093])
def test_c1_per_sample_radiance_far_into_the_stream(ctx, c1, start):
    ok, exact, got, want = per_sample(ctx, c1, 64, 40, 64, 36, 3, start=start)
    report(f"C1 samples {start}..{start + 2}", (64, 40, 64, 36), ok, exact, got, want)
    assert ok == 1.0, ok


def test_c2_full_spp_crop_matches_the_cpu_backend(ctx):
    # The drop-in at the C2 configuration's own 1024 spp (several launches of one-sample items,
    # Kahan sums) against the oracle's CPU-backend loop (f64 sums / spp) on a 64x64 crop at the
    # frame's centre: every pixel within 1e-4 relative.
    from lumenwright_b200.native import B200Backend
    frame = R.make_frame(R.CONFIGS["c2"], sky_backend=ctx)
    assert frame.spp == 1024
    be = B200Backend(0)
    img = be.render_hq(frame).reshape(720, 1280, 3)
    launches = be.ctx.stats()["launches"]
    x0, y0, n = 608, 328, 64
    want = O.OracleScene.from_frame(frame).render_mean(x0, y0, n, n, frame.spp)
    got = img[y0:y0 + n, x0:x0 + n]
    ok = np.all(close(got, want, 1e-4, 1e-6), axis=-1)
    rel = np.abs(got - want) / np.maximum(np.abs(want), 1e-6)
    print(f"C2 1024 spp crop: {ok.mean():.6f} of pixels within 1e-4, worst {rel.max():.2e}; "
          f"mean {got.mean():.6f} vs {want.mean():.6f}; {launches} kernel launches")
    assert ok.all(), np.argwhere(~ok)[:5]


def test_c1_render_hq_matches_the_cpu_backend(ctx, c1):
    from lumenwright_b200.native import B200Backend
    be = B200Backend(0)
    img = be.render_hq(c1).reshape(144, 256, 3)
    want = O.OracleScene.from_frame(c1).render_mean(0, 0, 256, 144, c1.spp)
    ok = np.all(close(img, want, 1e-4, 1e-6), axis=-1).mean()
    print(f"C1 mean: {ok:.5f} of pixels within 1e-4; mean {img.mean():.6f} vs {want.mean():.6f}")
    assert ok >= 0.99
    assert abs(img.mean() - want.mean()) <= 1e-4 * abs(want.mean())


@pytest.mark.parametrize("paths", [0, 1 << 12])
def test_wavefront_and_megakernel_give_the_same_image(ctx, c2, paths):
    # The wavefront engine (path slots, shade and trace iterations, rays carried across iterations)
    # and the persistent megakernel take the same items in the same order of Kahan additions: the
    # images are equal bit for bit, with the automatic pool and with a small one that carries many
    # rays over.
    # (The samples per item are set: by default each engine picks its own item size.)
    from lumenwright_b200.native import ENGINE_MEGAKERNEL, ENGINE_WAVEFRONT
    p = c2.params
    ctx.upload_hq_scene(c2.scene)
    ctx.set_tuning(engine=ENGINE_MEGAKERNEL, sub=3)
    want = ctx.render_hq(p, c2.sky, 12)
    ctx.set_tuning(engine=ENGINE_WAVEFRONT, paths=paths)
    got = ctx.render_hq(p, c2.sky, 12)
    ctx.set_tuning(engine=ENGINE_WAVEFRONT, paths=0, sub=0)
    assert np.array_equal(got, want)


def test_wavefront_default_items_are_one_sample(ctx, c2):
    # Left at 0, the wavefront's samples per item is one; the megakernel given one sample per item
    # takes the same items in the same order of additions, so the images are equal bit for bit.
    from lumenwright_b200.native import ENGINE_MEGAKERNEL, ENGINE_WAVEFRONT
    p = c2.params
    ctx.upload_hq_scene(c2.scene)
    ctx.set_tuning(engine=ENGINE_MEGAKERNEL, sub=1)
    want = ctx.render_hq(p, c2.sky, 6)
    ctx.set_tuning(engine=ENGINE_WAVEFRONT, sub=0, paths=0)
    got = ctx.render_hq(p, c2.sky, 6)
    assert np.array_equal(got, want)


def _same_hit(a, b):
    if a is None or b is None:
        return a is None and b is None
    f = lambda x: np.float32(x).tobytes()
    return a.quad == b.quad and a.texel == b.texel and f(a.t) == f(b.t) and f(a.s) == f(b.s) and f(a.tt) == f(b.tt)


def test_traversal_over_the_terrain_matches_the_oracle(ctx, c1):
    # Rays from points around the camera over the C1 terrain, in random directions and along the
    # axes (straight up and down, exactly level), through `lw_trace_rays` against the oracle's trace
    # of the reference algorithm: the hit (or its absence) is the same bit for bit. This covers
    # the early exit of rays above the last occupied brick row that do not go down, which the
    # reference reaches by skipping brick after brick.
    p = c1.params
    ctx.upload_hq_scene(c1.scene)
    rng = np.random.default_rng(7)
    eye = np.array(p["cam_pos"][:3], np.float32)
    n = 2048
    o = (eye + rng.uniform([-40, -45, -40], [40, 60, 40], (n, 3))).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    axes = np.array([[0, 1, 0], [0, -1, 0], [1, 0, 0], [-1, 0, 0], [0, 0, 1], [0, 0, -1]], np.float32)
    d[: 6 * 64] = np.repeat(axes, 64, axis=0)
    d[6 * 64: 8 * 64, 1] = 0.0  # level rays in random horizontal directions
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    d = d.astype(np.float32)
    got = ctx.trace_rays(p, o, d)
    v = O.OracleScene.from_frame(c1)
    want = [v.trace(oo, dd) for oo, dd in zip(o, d)]
    bad = [i for i, (g, w) in enumerate(zip(got, want)) if not _same_hit(g, w)]
    assert not bad, f"{len(bad)} of {n} rays differ from the oracle, first {bad[:5]}"
    hits = sum(g is not None for g in got)
    assert 0 < hits < n  # both hits and rays that leave the grid


@pytest.mark.parametrize("size", [(1, 1, 1), (3, 5, 7), (33, 9, 3)])
def test_small_and_ragged_frames_agree_between_engines(ctx, size):
    # Frames smaller than a tile, or not a multiple of it, and spp that do not fill an item
    # evenly: the wavefront (one-sample items, a pool of mostly idle slots) and the megakernel
    # given the same item size render the same image bit for bit.
    from lumenwright_b200.native import ENGINE_MEGAKERNEL, ENGINE_WAVEFRONT
    w, h, spp = size
    frame = R.make_frame(R.CONFIGS["c1"], sky_backend=ctx, width=w, height=h, spp=spp)
    ctx.upload_hq_scene(frame.scene)
    ctx.set_tuning(engine=ENGINE_MEGAKERNEL, sub=1)
    want = ctx.render_hq(frame.params, frame.sky, spp)
    ctx.set_tuning(engine=ENGINE_WAVEFRONT, sub=0, paths=0)
    got = ctx.render_hq(frame.params, frame.sky, spp)
    assert got.shape == (h, w, 3)
    assert np.array_equal(got, want)
    assert np.isfinite(got).all()


def test_renders_are_deterministic(ctx, c2):
    # render.rs:1015-1041 (byte-equal renders): the wavefront's rays go to whichever lane fetches
    # them first, but every sample's radiance and every addition's order are fixed, so two renders
    # of a frame are equal bit for bit, with the automatic pool and with a small one.
    from lumenwright_b200.native import ENGINE_WAVEFRONT
    p = c2.params
    ctx.upload_hq_scene(c2.scene)
    for paths in (0, 1 << 12):
        ctx.set_tuning(engine=ENGINE_WAVEFRONT, sub=0, paths=paths)
        a = ctx.render_hq(p, c2.sky, 8)
        b = ctx.render_hq(p, c2.sky, 8)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    ctx.set_tuning(engine=ENGINE_WAVEFRONT, sub=0, paths=0)



def test_a_scene_changed_in_place_is_drawn_as_it_now_is():
    # The backend copies the scene for every frame: the same HqScene object, changed in place
    # between two frames (its atlas recoloured), is drawn as it is now, as a fresh backend draws it.
    from lumenwright_b200.native import B200Backend
    import copy
    be = B200Backend(0)
    frame = R.make_frame(R.CONFIGS["c1"], sky_backend=be.ctx, spp=4)
    first = be.render_hq(frame)
    frame.scene.atlas[:] = (frame.scene.atlas & np.uint32(0xFF000000)) | (~frame.scene.atlas & np.uint32(0x00FFFFFF))
    second = be.render_hq(frame)
    fresh = B200Backend(0).render_hq(copy.deepcopy(frame))
    assert not np.array_equal(first, second)
    assert np.array_equal(second.view(np.uint32), fresh.view(np.uint32))


@pytest.mark.parametrize("shards", [2, 3])
def test_frame_shards_add_up_to_the_frame_bit_for_bit(ctx, c2, shards):
    # lw_render_device_shard: each shard renders its tiles (r, r + N, ...) into the accumulator and
    # leaves every other pixel's record as it is, so the shards rendered one after another into one
    # accumulator give the whole frame's render bit for bit; the records of one shard alone are zero
    # outside its tiles (what a SUM reduce over GPUs adds).
    from lumenwright_b200 import shard
    p = c2.params
    w, h = int(p["frame"][0]), int(p["frame"][1])
    ctx.upload_hq_scene(c2.scene)
    ctx.upload_sky(c2.sky)
    ctx.clear_accumulator(w, h)
    ctx.render_device(p, 0, 3)
    want = ctx.read_accumulator(w, h)
    ctx.clear_accumulator(w, h)
    for r in range(shards):
        ctx.render_device_shard(p, 0, 3, r, shards)
    got = ctx.read_accumulator(w, h)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    ctx.clear_accumulator(w, h)
    ctx.render_device_shard(p, 0, 3, 1, shards)
    one = ctx.read_accumulator(w, h)
    m = shard.tile_mask(w, h, 1, shards)
    assert not one[~m].any()
    assert np.array_equal(one[m].view(np.uint32), want[m].view(np.uint32))
