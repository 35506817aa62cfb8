"""CUDA parity on the reference kernel tests' fixtures (`crates/lumenwright-kernel/src/tests.rs`):
each query runs through the C ABI on the B200 and is checked against the FP32 oracle and against
the reference test's own known answer. Integer results (hit quad, texel, voxel id) must be equal;
floats must be bit-equal except where noted.
"""

import math

import numpy as np
import pytest

from kernel_fixtures import (INF, LAMP_EMITTANCE, LAMP_INTENSITY, SUN_ATLAS, basic_scene, hollow_scene, lamp_scene,
                             map_scene, norm, set_preetham_45, sun_atlas, sun_sprite_params, wall_rays, wall_scene)
from lumenwright_b200 import layout as L
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from lumenwright_b200.native import Context
    c = Context(0)
    yield c
    c.close()


def upload(ctx, ks):
    ctx.upload_buffers(ks.params, ks.grid, ks.models, ks.quads, ks.atlas, ks.emitters, ks.emitter_grid)
    ctx.upload_sky(ks.sky)


def same_hit(a, b):
    if a is None or b is None:
        return a is None and b is None
    return (a.quad == b.quad and a.texel == b.texel and np.float32(a.t).tobytes() == np.float32(b.t).tobytes()
            and np.float32(a.s).tobytes() == np.float32(b.s).tobytes())


def check_rays(ctx, ks, rays, tmin=0.0, tmax=INF):
    upload(ctx, ks)
    o = np.array([r[0] for r in rays], np.float32)
    d = np.array([r[1] for r in rays], np.float32)
    got = ctx.trace_rays(ks.params, o, d, tmin, tmax)
    v = O.OracleScene(*ks.buffers())
    want = [v.trace(oo, dd, tmin, tmax) for oo, dd in zip(o, d)]
    bad = [i for i, (g, w) in enumerate(zip(got, want)) if not same_hit(g, w)]
    assert not bad, f"{len(bad)} of {len(rays)} rays differ from the oracle, first {bad[:5]}"
    return got


def test_trace_known_answers(ctx):  # tests.rs:129-195
    ks = basic_scene(False)
    rays = [((0.5, 5.5, 5.5), (1, 0, 0)), ((-10.0, 5.5, 5.5), (1, 0, 0)), ((0.5, 9.5, 5.5), (1, 0, 0)),
            ((0.5, 5.5, 5.5), (0, 1, 0)), ((0.5, 5.5, 5.5), (-1, 0, 0))]
    o = np.array([18.0, 9.0, 3.0], np.float32)
    rays.append((o, norm(np.array([20.5, 6.0, 5.5], np.float32) - o)))
    got = check_rays(ctx, ks, rays)
    assert abs(got[0].t - 19.5) < 1e-3 and got[0].quad == 3
    assert abs(got[1].t - 30.0) < 1e-3
    assert abs(got[2].t - 31.5) < 1e-3
    assert got[3] is None and got[4] is None
    assert got[5].quad == 4
    assert check_rays(ctx, ks, [((0.5, 5.5, 5.5), (1, 0, 0))], 0.0, 10.0)[0] is None


def test_overlay_and_front_only(ctx):  # tests.rs:198-240
    ks = basic_scene(True)
    got = check_rays(ctx, ks, [((0.5, 5.5, 5.25), (1, 0, 0)), ((0.5, 5.5, 5.75), (1, 0, 0))])
    assert got[0].quad == 6 and abs(got[0].t - 8.0) < 1e-3 and abs(got[1].t - 19.5) < 1e-3
    L.quad_words(ks.quads)[6, 3] = L.ALPHA_CUTOUT | L.FLAG_FRONT_ONLY
    got = check_rays(ctx, ks, [((0.5, 5.5, 5.25), (1, 0, 0))], 0.0, 16.0)
    assert got[0].quad == 6
    assert check_rays(ctx, ks, [((12.0, 5.5, 5.25), (-1, 0, 0))])[0] is None


def test_front_face_far_along_the_ray(ctx):  # tests.rs:607-683
    ks = wall_scene()
    rays = wall_rays()
    got = check_rays(ctx, ks, rays)
    missed = sum(1 for (o, d), h in zip(rays, got)
                 if h is None or not (249.99 < float(o[0] + d[0] * np.float32(h.t)) < 250.01))
    assert missed == 0


def test_later_coplanar_quad(ctx):  # tests.rs:688-721
    ks = basic_scene(False)
    w = L.quad_words(ks.quads)
    ks.quads = L.quads_array([w[0], w[1], w[2], w[3], w[4], w[5], w[4], w[0]])
    ks.models[1]["quad_count"] = 8
    ks.params["off2"][3] = 8
    rays = []
    for i in range(16):
        f = np.float32(0.1) + np.float32(0.7) * (np.float32(i) + np.float32(0.5)) / np.float32(16.0)
        rays.append(((20.0 + f, 9.0, 5.0 + f), norm([0.01, -1.0, 0.02])))
        rays.append(((20.0 + f, 5.0 + f, 1.0), norm([0.02, 0.01, 1.0])))
    got = check_rays(ctx, ks, rays, 0.0, 100.0)
    assert [h.quad for h in got] == [6, 7] * 16


def test_voxel_lookup_is_bit_exact(ctx):  # scene.rs:271-284 on the uploaded reference grid
    for ks in (basic_scene(True), lamp_scene(L.EMITTER_SAMPLING_ONE, True), wall_scene()):
        upload(ctx, ks)
        dims = [int(v) for v in ks.params["grid_dims"][:3]]
        xs, ys, zs = np.meshgrid(np.arange(dims[0] * 16), np.arange(dims[1] * 16), np.arange(dims[2] * 16), indexing="ij")
        xyz = np.stack([xs.ravel(), ys.ravel(), zs.ravel()], 1).astype(np.int32)
        got = ctx.voxel_lookup(xyz)
        v = O.OracleScene(*ks.buffers())
        want = np.array([v.voxel(*map(int, p)) for p in xyz[:: max(1, len(xyz) // 20000)]], np.uint32)
        assert np.array_equal(got[:: max(1, len(xyz) // 20000)], want)


def test_cells_of_models_without_quads_are_traversed_as_the_reference_does(ctx):
    # The traversal's bricks hold a model without quads as air (and a uniform brick of it as a
    # uniform brick of air); the hits are the oracle's, on the reference's grid, bit for bit, and the
    # voxel lookup still gives the reference's ids.
    ks = hollow_scene()
    rng = np.random.default_rng(21)
    rays = [((0.5, 5.5, 5.5), (1, 0, 0)), ((0.5, 9.5, 9.5), (1, 0, 0)), ((-4.0, 5.2, 5.7), (1, 0.01, 0.0))]
    for _ in range(3000):
        o = rng.uniform((-8.0, -8.0, -8.0), (56.0, 24.0, 24.0)).astype(np.float32)
        tgt = rng.uniform((0.0, 0.0, 0.0), (48.0, 16.0, 16.0)).astype(np.float32)
        rays.append((o, norm(tgt - o)))
    got = check_rays(ctx, ks, rays)
    assert got[0] is not None and got[0].quad == 3 and abs(got[0].t - 23.5) < 1e-3  # the cube's face at x = 24
    assert sum(g is not None for g in got) > 1000
    xyz = np.array([(1, 1, 1), (20, 5, 5), (24, 5, 5), (19, 9, 9), (40, 3, 3)], np.int32)
    assert list(ctx.voxel_lookup(xyz)) == [2, 2, 1, 0, 1]


def test_water_exp_is_the_oracles_bit_for_bit(ctx):
    # The transmittance's exponential on the device against the oracle's build of the same source
    # (tests/test_water_exp.py holds that one against f64 exp and the platform expf): every 16th
    # float of [-104, 0], every float near 0 and the special values, bit for bit.
    lo, hi = np.array([-0.0, -104.0], np.float32).view(np.uint32)
    x = np.arange(lo, hi + 1, 16, dtype=np.uint64).astype(np.uint32).view(np.float32)
    tiny = np.arange(0x80000000, 0x80100000, dtype=np.uint64).astype(np.uint32).view(np.float32)
    special = np.array([0.0, np.inf, -np.inf, np.nan, -150.0, -200.0, 88.72284, 100.0, 1e30, 5.5], np.float32)
    x = np.concatenate([x, tiny, special])
    got = ctx.water_exp(x)
    want = O.water_exp(x)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), np.argwhere(got.view(np.uint32) != want.view(np.uint32))[:5]


def samples_match(ctx, ks, w, h, count, rel=0.0):
    upload(ctx, ks)
    got = ctx.render_samples(ks.params, 0, 0, w, h, 0, count)
    v = O.OracleScene(*ks.buffers())
    want = v.render_samples(0, 0, w, h, 0, count)
    if rel == 0.0:
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), np.argwhere(got != want)[:5]
    else:
        np.testing.assert_allclose(got, want, rtol=rel, atol=1e-7)
    return got


def test_empty_scene_shows_sky(ctx):  # tests.rs:262-291
    ks = basic_scene(False)
    p = ks.params
    p["frame"] = [4, 4, 0, 4]
    p["cam_pos"] = [0.5, 12.0, 0.5, 0.5]
    p["cam_fwd"] = [0.0, 1.0, 0.0, 1.0]
    p["cam_right"] = [1.0, 0.0, 0.0, 0.0]
    p["cam_up"] = [0.0, 0.0, -1.0, 0.0]
    set_preetham_45(p)
    p["sun_dir"] = [0.0, -1.0, 0.0, 1.0]
    p["misc_f"][2] = 128
    ks.sky = O.OracleScene(*ks.buffers()).build_sky_cache(128)
    got = samples_match(ctx, ks, 4, 4, 8)
    assert np.all(got[..., 2] > got[..., 0]) and np.all(got[..., 2] > 0.3)


def test_emitter_seen_from_the_camera(ctx):  # tests.rs:476-492
    ks = lamp_scene(L.EMITTER_SAMPLING_ONE, False)
    p = ks.params
    p["frame"] = [1, 1, 0, 1]
    p["cam_pos"] = [7.5, 2.0, 7.5, 0.01]
    p["cam_fwd"] = [0.0, 1.0, 0.0, 1.0]
    p["cam_right"] = [1.0, 0.0, 0.0, 0.0]
    p["cam_up"] = [0.0, 0.0, -1.0, 0.0]
    got = samples_match(ctx, ks, 1, 1, 16)
    want = LAMP_EMITTANCE * LAMP_INTENSITY
    assert np.all(np.abs(got[..., :2] - want) < 1e-4)


@pytest.mark.parametrize("strategy", [L.EMITTER_SAMPLING_NONE, L.EMITTER_SAMPLING_ONE,
                                      L.EMITTER_SAMPLING_ONE_BLOCK, L.EMITTER_SAMPLING_ALL])
@pytest.mark.parametrize("decoy", [False, True])
def test_lamp_room_per_sample(ctx, strategy, decoy):  # tests.rs:310-469 through render_sample
    ks = lamp_scene(strategy, decoy)
    p = ks.params
    p["frame"] = [8, 8, 0, 3]
    p["cam_pos"] = [8.0, 10.0, 8.0, 0.9]
    p["cam_fwd"] = [0.0, -1.0, 0.0, 1.0]
    p["cam_right"] = [1.0, 0.0, 0.0, 0.0]
    p["cam_up"] = [0.0, 0.0, -1.0, 0.0]
    p["sun_dir"] = [0.3, 0.9, 0.316, 0.9995]
    p["sun_color"] = [1.0, 0.9, 0.8, 0.03]
    got = samples_match(ctx, ks, 8, 8, 16)
    assert np.isfinite(got).all()


def test_the_camera_sees_the_sun_texture(ctx):  # integrator.rs:252-277, :617-621; sky.rs:1151-1253
    # Camera rays above the grid, aimed at a 45-degree sun, miss everything: each sample is the
    # sky through Chunky's cache plus the sun texture drawn from the 32x32 sprite of the
    # reference's sun-texture test, bit for bit the oracle's.
    from lumenwright_b200 import sky as SK
    ks = basic_scene(False)
    atlas = sun_atlas()
    atlas[0], atlas[1] = 0xFFFF_FFFF, 0  # the cube's texels (outside the sprite)
    ks.atlas = atlas
    p = ks.params
    p["off2"][1], p["off2"][2] = SUN_ATLAS
    sun = SK.sun_direction(45.0, 135.0)
    su, sv = sun_sprite_params(p, sun)
    pre = SK.Preetham(sun)
    p["sky_sun"] = [*pre.sun, 1.0]
    p["sky_zenith"] = [*pre.zenith, 0.0]
    for k, name in enumerate(("perez_a", "perez_b", "perez_c", "perez_d", "perez_e")):
        p[name] = [*pre.perez[k], 0.0]
    p["misc_f"][2] = 128
    p["frame"] = [24, 24, 0, 2]
    p["cam_pos"] = [24.0, 40.0, 8.0, 0.16]
    p["cam_fwd"] = [*sun, 1.0]
    p["cam_right"] = [*su, 0.0]
    p["cam_up"] = [*sv, 0.0]
    ks.sky = O.OracleScene(*ks.buffers()).build_sky_cache(128)
    got = samples_match(ctx, ks, 24, 24, 4)
    # the sprite (up to about 11 per channel) covers most of the view; the sky is below 1
    lit = got.max(-1) > 1.0
    assert 0.3 < lit.mean() < 0.95, lit.mean()


def test_sky_maps_lens_and_light(ctx):  # tests.rs:805-831
    ks = basic_scene(False)
    p = ks.params
    p["sky_map"] = [4.0, 2.0, 2.0, 2.0]
    ks.sky = np.concatenate([np.full(4 * 2 * 3, 5.0, np.float32), np.full(2 * 2 * 3, 0.3, np.float32)])
    p["frame"] = [1, 1, 0, 1]
    p["cam_pos"] = [40.25, 20.0, 8.25, 1e-3]
    p["cam_right"] = [1.0, 0.0, 0.0, 0.0]
    p["sun_dir"] = [0.0, 1.0, 0.0, 0.9995]
    p["cam_fwd"] = [0.0, -1.0, 0.0, 1.0]
    p["cam_up"] = [0.0, 0.0, -1.0, 0.0]
    got = samples_match(ctx, ks, 1, 1, 16)
    assert np.all(np.abs(got - 0.3) < 1e-4)
    p["sun_color"] = [1.0, 1.0, 1.0, 0.03]
    got = samples_match(ctx, ks, 1, 1, 4)
    assert got[0, 0, 0, 0] > 1.0
    ms = map_scene()
    ms.params["frame"] = [16, 8, 0, 2]
    ms.params["cam_pos"] = [24.0, 8.0, 8.0, 1.2]
    ms.params["cam_fwd"] = [0.0, 0.6, 0.8, 2.0]
    ms.params["cam_right"] = [1.0, 0.0, 0.0, 0.0]
    ms.params["cam_up"] = [0.0, 0.8, -0.6, 0.0]
    samples_match(ctx, ms, 16, 8, 4)


def test_render_hq_mean_matches_cpu_backend(ctx):  # cpu/mod.rs:39-87 against cuda.rs:77-184
    ks = lamp_scene(L.EMITTER_SAMPLING_ONE, True)
    p = ks.params
    p["frame"] = [32, 24, 0, 4]
    p["cam_pos"] = [8.0, 12.0, 8.0, 0.9]
    p["cam_fwd"] = [0.0, -1.0, 0.0, 1.3333]
    p["cam_right"] = [1.0, 0.0, 0.0, 0.0]
    p["cam_up"] = [0.0, 0.0, -1.0, 0.0]
    upload(ctx, ks)
    calls = []
    img = ctx.render_hq(p, ks.sky, 64, progress=lambda d, t: calls.append((d, t)))
    want = O.OracleScene(*ks.buffers()).render_mean(0, 0, 32, 24, 64)
    np.testing.assert_allclose(img, want, rtol=2e-6, atol=1e-6)
    assert calls and calls[-1] == (64, 64)


def quad_view(eye, at, overlay, see_through, chunk_frames):
    """basic_scene's cutout quad at x = 8.5 under a sky, seen from `eye`: as an overlay quad, or
    (with its overlay cell emptied) as the frame's see-through quad behind the cube at x = 20..21,
    in the grid's frame or in chunk frames."""
    from lumenwright_b200 import native as N
    ks = basic_scene(True)
    p = ks.params
    if not overlay:
        ks.grid = ks.grid.copy()
        ks.grid[int(p["off"][2])] = L.EMPTY
    p["see_through"] = [6, 1, 0, 0] if see_through else [0, 0, 0, 0]
    p["frame"] = [16, 16, 0, 2]
    f = norm(np.array(at, np.float32) - np.array(eye, np.float32))
    r = norm(np.cross(f, np.array([0, 1, 0], np.float32)).astype(np.float32))
    u = np.cross(r, f).astype(np.float32)
    p["cam_pos"] = [*eye, 0.12]
    p["cam_fwd"] = [*f, 1.0]
    p["cam_right"] = [*r, 0.0]
    p["cam_up"] = [*u, 0.0]
    set_preetham_45(p)
    p["sun_dir"] = [0.3, 0.9, 0.316, 0.9995]
    p["sun_color"] = [1.0, 0.9, 0.8, 0.03]
    p["misc_f"][2] = 128
    ks.sky = O.OracleScene(*ks.buffers()).build_sky_cache(128)
    if chunk_frames:
        ks.params = N.rebase_camera(p, eye)
    return ks


@pytest.mark.parametrize("view", ["overlay", "see-through"])
@pytest.mark.parametrize("chunk_frames", [False, True])
def test_overlay_and_see_through_quads_per_sample(ctx, view, chunk_frames):  # trace.rs:113-131 on the camera ray
    # The overlay traversal (quads tested relative to their cell) and the see-through test (quads
    # relative to the frame's corner) in both frames; the eyes sit in chunks 1 and 2 along x, so
    # chunk frames hold them relative to x = 16 and x = 32.
    eye, at = ((20.3, 7.6, 5.5), (8.5, 5.5, 5.5)) if view == "overlay" else ((24.3, 5.6, 5.4), (8.5, 5.5, 5.5))
    ks = quad_view(eye, at, view == "overlay", view == "see-through", chunk_frames)
    if chunk_frames:
        assert ks.params["see_through"][2] == 1 and ks.params["see_through"][3] == (1 if view == "overlay" else 2)
    got = samples_match(ctx, ks, 16, 16, 4)
    bare = O.OracleScene(*quad_view(eye, at, False, False, False).buffers()).render_samples(0, 0, 16, 16, 0, 4)
    assert (got != bare).any(-1).sum() >= 30  # the quad is in view in some samples


def test_bad_buffers_are_refused(ctx):  # the C ABI never traps on a malformed scene
    from lumenwright_b200.native import LwError
    ks = basic_scene(False)
    bad = ks.grid.copy()
    bad[1] = 7  # a top entry naming a brick that does not exist
    with pytest.raises(LwError) as e:
        ctx.upload_buffers(ks.params, bad, ks.models, ks.quads, ks.atlas, ks.emitters, ks.emitter_grid)
    assert e.value.status == 2
    m = ks.models.copy()
    m[1]["quad_count"] = 99
    with pytest.raises(LwError):
        ctx.upload_buffers(ks.params, ks.grid, m, ks.quads, ks.atlas, ks.emitters, ks.emitter_grid)
    upload(ctx, ks)
    p = ks.params.copy()
    p["misc_f"][2] = 128  # a sky cache that was not given
    p["frame"] = [4, 4, 0, 1]
    with pytest.raises(LwError) as e:
        ctx.render_samples(p, 0, 0, 4, 4, 0, 1)
    assert e.value.status == 2
