"""Host side of the differentiable form, on the CPU: the FP64 sky cache the sky Jacobian is taken
from agrees with the oracle's f32 restatement of `build_sky_cache`
(crates/lumenwright-kernel/src/integrator.rs:133-148), the sun-direction Jacobian is the
direction's derivative, and every atlas texel of a texture maps to its slot with its decoded
colour as the nominal albedo."""

import math

import numpy as np

from lumenwright_b200 import adjoint as A
from lumenwright_b200 import layout as LY
from lumenwright_b200 import sky as SK
from lumenwright_b200 import synth as S
from lumenwright_b200.native import gamma_table
from oracle import oracle as O

F32 = np.float32


def oracle_cache(az, alt, tb):
    p = LY.new_params()
    pre = SK.Preetham(SK.normalize32(A.sun_vector(az, alt)), tb)
    p["sky_sun"] = [pre.sun[0], pre.sun[1], pre.sun[2], 1.0]
    p["sky_zenith"] = [pre.zenith[0], pre.zenith[1], pre.zenith[2], 0.0]
    for k, name in enumerate(("perez_a", "perez_b", "perez_c", "perez_d", "perez_e")):
        p[name] = [pre.perez[k][0], pre.perez[k][1], pre.perez[k][2], 0.0]
    return O.OracleScene(p, None, None, None, None, None, None).build_sky_cache(128).astype(np.float64)


def test_f64_sky_cache_matches_the_oracle():
    for az, alt, tb in ((0.3, 1.18, 2.5), (2.0, 0.4, 3.1), (-1.0, 0.9, 2.0)):
        got = A.sky_cache_f64(az, alt, tb).reshape(-1, 3)
        want = oracle_cache(az, alt, tb).reshape(-1, 3)
        # saturation and lightness to FP32 accuracy of the oracle's arithmetic; hue where the
        # colour is saturated enough to have one
        assert np.abs(got[:, 1:] - want[:, 1:]).max() < 2e-4
        sat = want[:, 1] > 0.02
        dh = np.abs(got[sat, 0] - want[sat, 0])
        assert np.minimum(dh, np.abs(dh - 1.0)).max() < 2e-3


def test_sky_cache_jacobian_follows_the_cache():
    x = (0.3, 1.18, 2.5)
    J = A.sky_cache_jacobian(*x)
    for k, h in enumerate((1e-3, 1e-3, 1e-2)):
        e = np.zeros(3)
        e[k] = h
        fd = (A.sky_cache_f64(*(np.array(x) + e)) - A.sky_cache_f64(*(np.array(x) - e))) / (2 * h)
        ok = np.abs(fd - J[:, k]) <= 1e-3 * np.abs(J[:, k]).max() + 1e-2 * np.abs(J[:, k])
        # the cache has kinks (|2l - 1| in the saturation, channels clamped to 1) that a step of
        # 1e-3..1e-2 crosses at a few entries in a thousand
        assert ok.mean() > 0.99


def test_sun_vector_jacobian():
    az, alt, h = 0.3, 1.1, 1e-6
    J = A.sun_vector_jacobian(az, alt)
    fa = (A.sun_vector(az + h, alt) - A.sun_vector(az - h, alt)) / (2 * h)
    fb = (A.sun_vector(az, alt + h) - A.sun_vector(az, alt - h)) / (2 * h)
    assert np.allclose(J[:, 0], fa, atol=1e-8) and np.allclose(J[:, 1], fb, atol=1e-8)
    assert abs(np.linalg.norm(A.sun_vector(az, alt)) - 1.0) < 1e-12


def test_texel_parameters_cover_the_textures():
    atlas = S.build_atlas(1)
    g = gamma_table()
    assert g[0] == 0.0 and g[255] == 1.0 and abs(g[128] - (128 / 255) ** 2.2) < 1e-3
    tp, alb = A.texel_parameters(atlas, g)
    h, w = atlas.pixels.shape
    tp2 = tp.reshape(h, w)
    for i, name in enumerate(S.TEXTURES):
        sp = atlas.sprites[name]
        block = tp2[sp.y - 1:sp.y + 17, sp.x - 1:sp.x + 17]
        assert block.min() == i * 256 and block.max() == i * 256 + 255
        # every mapped texel holds the bytes of its parameter's texel
        ys, xs = np.nonzero(block >= 0)
        px = atlas.pixels[sp.y - 1 + ys, sp.x - 1 + xs].astype(np.uint32)
        dec = np.stack([g[px & 0xFF], g[(px >> 8) & 0xFF], g[(px >> 16) & 0xFF]], -1)
        assert np.array_equal(dec, alb[block[ys, xs]])
    sun = atlas.sprites["sun"]
    assert (tp2[sun.y:sun.y + sun.h, sun.x:sun.x + sun.w] == -1).all()
    assert tp.max() < A.SLOTS * A.TEXELS and math.prod(atlas.pixels.shape) == tp.size


class OracleSky:
    """Sky set-up through the oracle's f32 cache builder (no device needed)."""

    def build_sky_cache(self, params, n):
        return O.OracleScene(params, None, None, None, None, None, None).build_sky_cache(n)


def test_fp64_oracle_theta_hooks_leave_the_nominal_render():
    # At albedos equal to the decoded texels, unit emitter groups, the frame's own sun and sky,
    # the FP64 oracle under a theta renders what it renders without one; freezing the roulette and
    # the shadow rays at that same theta changes nothing beyond rounding.
    from lumenwright_b200 import request as R
    cfg = R.Config("t", 2, 24, 14, 4, 4, 4000, "chunky", emitters=True)
    frame = R.make_frame(cfg, sky_backend=OracleSky())
    view = O.OracleScene.from_frame(frame)
    p = frame.params
    atlas = S.build_atlas(cfg.seed)
    tp, _ = A.texel_parameters(atlas, np.zeros(256, np.float32))
    alb = np.zeros((A.SLOTS * A.TEXELS, 3))
    px = atlas.pixels.ravel()
    m = tp >= 0
    for c in range(3):
        alb[tp[m], c] = (((px[m] >> (8 * c)) & 0xFF) / 255.0) ** 2.2
    sun = [float(x) for x in p["sun_dir"]]
    th, keep = O.make_theta(alb, alb, tp, np.ones(A.GROUPS), frame.sky.astype(np.float64), sun, sun, frozen=False)
    want = view.render_mean64(0, 0, 24, 14, 4)
    got = view.render_mean_theta(th, 0, 0, 24, 14, 4)
    assert np.allclose(got, want, rtol=1e-12, atol=1e-15)
    thf, keepf = O.make_theta(alb, alb, tp, np.ones(A.GROUPS), frame.sky.astype(np.float64), sun, sun, frozen=True)
    assert np.allclose(view.render_mean_theta(thf, 0, 0, 24, 14, 4), want, rtol=1e-9, atol=1e-12)
    # paired differences of a theta with itself vanish
    diff, mean = view.render_fd_theta(thf, thf, 0, 0, 24, 14, 4)
    assert not diff.any() and np.allclose(mean, want, rtol=1e-9, atol=1e-12)
    assert O.bounds_errors() == 0
