"""Pins the FP32 oracle to the reference kernel's own known-answer tests
(`crates/lumenwright-kernel/src/tests.rs`), case for case with the same fixtures, numbers and
tolerances. CPU only.
"""

import math

import numpy as np
import pytest

from kernel_fixtures import (INF, LAMP_EMITTANCE, LAMP_INTENSITY, basic_scene, lamp_scene, map_scene,
                             norm, set_preetham_45, sky_dir, wall_rays, wall_scene)
from lumenwright_b200 import layout as L
from oracle import oracle as O


def scene(ks):
    return O.OracleScene(*ks.buffers())


@pytest.fixture(autouse=True)
def _no_bounds_errors():
    O.reset_bounds_errors()
    yield
    assert O.bounds_errors() == 0


def test_ray_skips_empty_brick_and_hits_cube():  # tests.rs:129-136
    v = scene(basic_scene(False))
    h = v.trace((0.5, 5.5, 5.5), (1, 0, 0), 0.0, INF)
    assert h is not None and abs(h.t - 19.5) < 1e-3
    assert h.quad == 3, "west face"


def test_ray_from_outside_grid_enters_it():  # tests.rs:139-151
    v = scene(basic_scene(False))
    h = v.trace((-10.0, 5.5, 5.5), (1, 0, 0), 0.0, INF)
    assert h is not None and abs(h.t - 30.0) < 1e-3


def test_ray_reaches_uniform_brick():  # tests.rs:154-160
    v = scene(basic_scene(False))
    h = v.trace((0.5, 9.5, 5.5), (1, 0, 0), 0.0, INF)
    assert h is not None and abs(h.t - 31.5) < 1e-3


def test_ray_misses_everything():  # tests.rs:163-179
    v = scene(basic_scene(False))
    assert v.trace((0.5, 5.5, 5.5), (0, 1, 0), 0.0, INF) is None
    assert v.trace((0.5, 5.5, 5.5), (-1, 0, 0), 0.0, INF) is None
    assert v.trace((0.5, 5.5, 5.5), (1, 0, 0), 0.0, 10.0) is None


def test_oblique_rays_hit_cube_top():  # tests.rs:182-195
    v = scene(basic_scene(False))
    o = np.array([18.0, 9.0, 3.0], np.float32)
    d = norm(np.array([20.5, 6.0, 5.5], np.float32) - o)
    h = v.trace(o, d, 0.0, INF)
    p = o + d * np.float32(h.t)
    assert abs(p[1] - 6.0) < 1e-3 and h.quad == 4


def test_entity_overlay_quads_are_hit_and_alpha_tested():  # tests.rs:198-222
    v = scene(basic_scene(True))
    h = v.trace((0.5, 5.5, 5.25), (1, 0, 0), 0.0, INF)
    assert abs(h.t - 8.0) < 1e-3 and h.quad == 6
    h = v.trace((0.5, 5.5, 5.75), (1, 0, 0), 0.0, INF)
    assert abs(h.t - 19.5) < 1e-3


def test_front_only_quads_are_met_from_the_front_only():  # tests.rs:225-240
    ks = basic_scene(True)
    L.quad_words(ks.quads)[6, 3] = L.ALPHA_CUTOUT | L.FLAG_FRONT_ONLY
    v = scene(ks)
    front = v.trace((0.5, 5.5, 5.25), (1, 0, 0), 0.0, 16.0)
    assert front is not None and front.quad == 6
    assert v.trace((12.0, 5.5, 5.25), (-1, 0, 0), 0.0, INF) is None


def test_a_see_through_quad_is_found_behind_what_hides_it():  # tests.rs:243-259
    ks = basic_scene(True)
    ks.params["see_through"] = [6, 1, 0, 0]
    v = scene(ks)
    o, d = (25.5, 5.5, 5.25), (-1.0, 0.0, 0.0)
    h = v.trace(o, d, 0.0, INF)
    assert h.quad == 2
    st = v.see_through_hit(o, d, h.t)
    assert st is not None and st.quad == 6 and abs(st.t - 17.0) < 1e-3
    assert v.see_through_hit((25.5, 5.5, 5.75), d, h.t) is None
    ks.params["see_through"] = [0, 0, 0, 0]
    assert scene(ks).see_through_hit(o, d, h.t) is None


def test_empty_scene_shows_sky():  # tests.rs:262-291
    ks = basic_scene(False)
    p = ks.params
    p["frame"] = [4, 4, 0, 4]
    p["cam_pos"] = [0.5, 12.0, 0.5, 0.5]
    p["cam_fwd"] = [0.0, 1.0, 0.0, 1.0]
    p["cam_right"] = [1.0, 0.0, 0.0, 0.0]
    p["cam_up"] = [0.0, 0.0, -1.0, 0.0]
    set_preetham_45(p)
    p["sun_dir"] = [0.0, -1.0, 0.0, 1.0]
    n = 128
    p["misc_f"][2] = n
    v = scene(ks)
    v.set_sky(v.build_sky_cache(n))
    for y in range(4):
        for x in range(4):
            c = v.render_sample(x, y, 0)
            assert c[2] > c[0] and c[2] > 0.3, c


def test_rng_matches_reference_values():  # tests.rs:294-298
    assert O.pcg_hash(0) == 129708002
    assert O.pcg_hash(1) == 2831084092


def floor_emitter_light(ks, draws):  # tests.rs:400-411
    v = scene(ks)
    pos = np.array([7.3, 1.0, 7.6], np.float32)
    n = np.array([0.0, 1.0, 0.0], np.float32)
    origin = pos + n * np.float32(1e-3)
    st = O.rng_new(3, 0, 11)
    total = 0.0
    for _ in range(draws):
        c, st = v.sample_emitters(pos, origin, n, st)
        total += float(c[1])
    return total / draws


def floor_emitter_expectation():  # tests.rs:413-429
    px, py, pz = 7.3, 1.001, 7.6
    k = 400
    i = (np.arange(k) + 0.5) / k
    x, z = np.meshgrid(7.0 + i, 7.0 + i, indexing="ij")
    d0, d1, d2 = x - px, 4.0 - py, z - pz
    d2s = d0 * d0 + d1 * d1 + d2 * d2
    acc = np.sum((d1 / np.sqrt(d2s)) / np.maximum(d2s, 1.0) / (k * k))
    return math.pi * LAMP_INTENSITY * LAMP_EMITTANCE * acc


def test_emitter_sampling_is_chunkys_estimate():  # tests.rs:434-453
    want = floor_emitter_expectation()
    for strategy in (L.EMITTER_SAMPLING_ONE, L.EMITTER_SAMPLING_ONE_BLOCK, L.EMITTER_SAMPLING_ALL):
        got = floor_emitter_light(lamp_scene(strategy, False), 200_000)
        assert abs((got - want) / want) < 0.01, (strategy, got, want)
    assert floor_emitter_light(lamp_scene(L.EMITTER_SAMPLING_NONE, False), 1000) == 0.0


def test_an_unseen_emitter_in_the_cell_halves_the_sampled_light():  # tests.rs:458-469
    want = floor_emitter_expectation() / 2.0
    for strategy in (L.EMITTER_SAMPLING_ONE, L.EMITTER_SAMPLING_ALL):
        got = floor_emitter_light(lamp_scene(strategy, True), 200_000)
        assert abs((got - want) / want) < 0.02, (strategy, got, want)


def test_an_emitter_seen_from_the_camera_shows_its_emitted_light():  # tests.rs:476-492
    ks = lamp_scene(L.EMITTER_SAMPLING_ONE, False)
    p = ks.params
    p["frame"] = [1, 1, 0, 1]
    p["cam_pos"] = [7.5, 2.0, 7.5, 0.01]
    p["cam_fwd"] = [0.0, 1.0, 0.0, 1.0]
    p["cam_right"] = [1.0, 0.0, 0.0, 0.0]
    p["cam_up"] = [0.0, 0.0, -1.0, 0.0]
    v = scene(ks)
    want = LAMP_EMITTANCE * LAMP_INTENSITY
    for i in range(16):
        c = v.render_sample(0, 0, i)
        assert abs(c[0] - want) < 1e-4 and abs(c[1] - want) < 1e-4, c


def test_sin_cos_turns_is_within_its_bound_of_f64():  # tests.rs:495-520
    inside = np.arange(1 << 20, dtype=np.float32) / np.float32(1 << 20)
    outside = (np.arange(20_000, dtype=np.float32) - np.float32(10_000.0)) * np.float32(0.037)
    us = np.concatenate([inside[::64], outside[::4]])  # a strided subset keeps the CPU suite quick
    worst = 0.0
    for u in us:
        s, c = O.sin_cos_turns(float(u))
        a = 2.0 * math.pi * float(u)
        worst = max(worst, abs(s - math.sin(a)), abs(c - math.cos(a)))
    assert worst <= 1.5e-7, worst
    assert O.sin_cos_turns(0.0) == (0.0, 1.0)
    s, c = O.sin_cos_turns(0.25)
    assert s == 1.0 and c == 0.0 and math.copysign(1, c) < 0
    s, c = O.sin_cos_turns(0.5)
    assert s == 0.0 and math.copysign(1, s) < 0 and c == -1.0
    assert O.sin_cos_turns(0.75) == (-1.0, 0.0)


def test_ln_and_gamma_decoding_are_within_their_bounds_of_f64():  # tests.rs:523-548
    worst_ln = 0.0
    for i in range(0, 1 << 20, 97):
        x = float(np.float32(1.0 / 255.0) + np.float32(1.0 - 1.0 / 255.0) * np.float32(i) / np.float32((1 << 20) - 1))
        worst_ln = max(worst_ln, abs(O.ln(x) - math.log(x)))
    worst_gamma = 0.0
    for k in range(1, 256):
        c = float(np.float32(k) / np.float32(255.0))
        exact = c ** float(np.float32(2.2))
        worst_gamma = max(worst_gamma, abs((O.gamma_to_linear(c) - exact) / exact))
    assert worst_ln <= 5e-7, worst_ln
    assert worst_gamma <= 1e-6, worst_gamma
    assert O.gamma_to_linear(0.0) == 0.0
    assert O.gamma_to_linear(1.0) == 1.0


def test_acos_is_within_its_bound_of_f64():  # tests.rs:551-563
    worst = 0.0
    for i in range(0, (1 << 20) + 1, 61):
        x = float(np.float32(-1.0) + np.float32(2.0) * np.float32(i) / np.float32(1 << 20))
        worst = max(worst, abs(O.acos(x) - math.acos(x)))
    assert worst <= 1e-6, worst


def test_atan2_is_within_its_bound_of_f64():  # tests.rs:566-588
    worst = 0.0
    for i in range(0, 1 << 16, 7):
        a = np.float32(i) / np.float32(1 << 16) * np.float32(2 * math.pi)
        for r in (1e-3, 1.0, 250.0):
            y = float(np.float32(np.sin(a)) * np.float32(r))
            x = float(np.float32(np.cos(a)) * np.float32(r))
            worst = max(worst, abs(O.atan2(y, x) - math.atan2(y, x)))
    for y, x, want in ((0.0, 1.0, 0.0), (1.0, 0.0, math.pi / 2), (0.0, 0.0, 0.0)):
        assert abs(O.atan2(y, x) - want) < 1e-7
    assert worst <= 1e-6, worst


def test_a_front_face_far_along_the_ray_is_met():  # tests.rs:607-683
    v = scene(wall_scene())
    missed = 0
    for o, d in wall_rays():
        h = v.trace(o, d, 0.0, INF)
        if h is None:
            missed += 1
            continue
        x = float(o[0] + d[0] * np.float32(h.t))
        if not (249.99 < x < 250.01):
            missed += 1
    assert missed == 0


def test_a_later_coplanar_quad_is_met():  # tests.rs:688-721
    ks = basic_scene(False)
    w = L.quad_words(ks.quads)
    ks.quads = L.quads_array([w[0], w[1], w[2], w[3], w[4], w[5], w[4], w[0]])
    ks.models[1]["quad_count"] = 8
    ks.params["off2"][3] = 8
    v = scene(ks)
    for i in range(16):
        f = np.float32(0.1) + np.float32(0.7) * (np.float32(i) + np.float32(0.5)) / np.float32(16.0)
        down = v.trace((20.0 + f, 9.0, 5.0 + f), norm([0.01, -1.0, 0.02]), 0.0, 100.0)
        assert down is not None and down.quad == 6, f
        south = v.trace((20.0 + f, 5.0 + f, 1.0), norm([0.02, 0.01, 1.0]), 0.0, 100.0)
        assert south is not None and south.quad == 7, f


def near(a, b, tol):
    return all(abs(float(x) - float(y)) <= tol for x, y in zip(a, b))


def test_the_sky_maps_are_read_bilinearly():  # tests.rs:757-799
    v = scene(map_scene())
    for j in range(2):
        for i in range(4):
            d = sky_dir((i + 0.5) / 4.0, (j + 0.5) * (math.pi / 2) - math.pi / 2)
            assert near(v.sky_lens(d), (i, j, 1.0), 1e-3), (i, j)
    assert near(v.sky_lens(sky_dir(0.0, -math.pi / 4)), (1.5, 0.0, 1.0), 1e-3)
    assert near(v.sky_lens(sky_dir(0.125, 0.0)), (0.0, 0.5, 1.0), 1e-3)
    assert near(v.sky_lens((0.0, 1.0, 0.0)), (1.5, 1.0, 1.0), 1e-3)
    assert near(v.sky_lens((0.0, -1.0, 0.0)), (1.5, 0.0, 1.0), 1e-3)
    assert near(v.sky_light(sky_dir(0.25, math.pi / 4)), (10.0, 11.0, 2.0), 1e-3)
    assert near(v.sky_light(sky_dir(0.5, 0.0)), (10.5, 10.5, 2.0), 1e-3)


def test_the_lens_sees_one_map_and_a_bounce_is_lit_by_the_other():  # tests.rs:805-831
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
    v = scene(ks)
    for sample in range(16):
        assert near(v.render_sample(0, 0, sample), (0.3, 0.3, 0.3), 1e-4), sample
    p["cam_fwd"] = [0.0, 1.0, 0.0, 1.0]
    p["cam_up"] = [0.0, 0.0, 1.0, 0.0]
    assert near(scene(ks).render_sample(0, 0, 0), (5.0, 5.0, 5.0), 1e-4)
    p["cam_fwd"] = [0.0, -1.0, 0.0, 1.0]
    p["cam_up"] = [0.0, 0.0, -1.0, 0.0]
    p["sun_color"] = [1.0, 1.0, 1.0, 0.03]
    assert scene(ks).render_sample(0, 0, 0)[0] > 1.0
