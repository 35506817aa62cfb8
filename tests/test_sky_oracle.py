"""The sky and the sun of the hq path against the reference's sky tests
(`crates/lumenwright/src/render/sky.rs:955-1585`) and its emitter default tests
(`crates/lumenwright/src/request.rs:1228-1260`): the host set-up in `lumenwright_b200.sky`, and
the oracle's `preetham_radiance` and `sun_texture` (`crates/lumenwright-kernel/src/integrator.rs`)
against FP64 restatements of Chunky's Preetham sky and sun, with the reference tests' cases,
counts and tolerances. CPU only.
"""

import math

import numpy as np
import pytest

from kernel_fixtures import SUN_ATLAS, SUN_SPRITE, sun_atlas, sun_sprite_params, sun_texel
from lumenwright_b200 import layout as L
from lumenwright_b200 import sky as SK
from oracle import oracle as O

F32 = np.float32


@pytest.fixture(autouse=True)
def _no_bounds_errors():
    O.reset_bounds_errors()
    yield
    assert O.bounds_errors() == 0


def test_sun_follows_the_vanilla_day_cycle():  # sky.rs:958-976 (the quick path's daylight left out)
    assert abs(SK.celestial_angle(6000)) < 1e-4
    noon = SK.sun_direction_from_angle(SK.celestial_angle(6000))
    assert noon[1] > 0.999
    morning = SK.sun_direction_from_angle(SK.celestial_angle(0))
    assert morning[0] > 0.95 and 0.1 < morning[1] < 0.3, morning
    evening = SK.sun_direction_from_angle(SK.celestial_angle(12000))
    assert evening[0] < -0.95 and evening[1] > 0.0, evening


def test_altitude_azimuth():  # sky.rs:1578-1583
    assert np.linalg.norm(SK.sun_direction(90.0, 0.0) - [0.0, 1.0, 0.0]) < 1e-5
    assert np.linalg.norm(SK.sun_direction(0.0, 90.0) - [1.0, 0.0, 0.0]) < 1e-5
    assert np.linalg.norm(SK.sun_direction(0.0, 0.0) + [0.0, 0.0, 1.0]) < 1e-5


def test_twilight_holds_chunkys_sky_until_the_disc_sets():  # sky.rs:1111-1131
    r = SK.SUN_RADIUS
    assert SK.twilight(0.5) == 1.0
    assert SK.twilight(0.0) == 1.0
    assert SK.twilight(-r) == 1.0
    assert SK.twilight(F32(-r - F32(1e-3))) < 1.0
    assert SK.twilight(SK.CIVIL_TWILIGHT_END) == SK.NIGHT_SKY_LIGHT
    assert SK.twilight(F32(-math.pi / 2)) == SK.NIGHT_SKY_LIGHT
    last = F32(1.0)
    for i in range(101):
        t = SK.twilight(F32(-r + F32(SK.CIVIL_TWILIGHT_END + r) * F32(i) / F32(100.0)))
        assert t <= last, "monotone"
        last = t
    # The dusk sun of tick 12800 sits at altitude -0.005091 rad, its disc still up.
    dusk = SK.hq_sky(SK.sun_direction(math.degrees(-0.005091), 270.0), F32(1.25), F32(1.0))
    assert dusk.sky_light == 1.0
    assert np.all(dusk.sun_color == np.power(F32(1.25), F32(2.2)))
    night = SK.hq_sky(np.array([0.0, -1.0, 0.0], F32), F32(1.25), F32(1.0))
    assert night.sky_light == SK.NIGHT_SKY_LIGHT


def test_the_day_weight_follows_the_sky_light_factor():  # sky.rs:1567-1576
    assert SK.day_weight(1.0, 0.24, 1.0) == 1.0
    assert SK.day_weight(0.24, 0.24, 1.0) == 0.0
    assert abs(SK.day_weight(0.62, 0.24, 1.0) - 0.5) < 1e-6
    assert abs(SK.day_weight(0.378182, 0.24, 1.0) - 0.181818) < 1e-5
    assert SK.day_weight(1.2, 0.24, 1.0) == 1.0
    assert SK.day_weight(0.1, 0.24, 1.0) == 0.0
    assert SK.day_weight(0.5, 0.5, 0.5) == 1.0


def test_the_lantern_default_is_the_fit_at_dusk():  # request.rs:1234-1245
    at = lambda w: SK.default_emitter_intensity(False, w)  # noqa: E731
    assert abs(at(0.181818) - 115.2423) < 1e-3
    assert at(1.0) == 13.0
    assert at(0.0) == SK.GAME_EMITTER_INTENSITY
    assert SK.default_emitter_intensity(True, 1.0) == 0.0
    assert SK.default_emitter_intensity(True, 0.0) == 0.0


def test_off_the_day_plateau_the_default_is_the_mix():  # request.rs:1247-1260
    w = (np.arange(1871, dtype=np.uint32).astype(F32) / F32(1870.0)).astype(F32)
    mix = w * SK.DEFAULT_EMITTER_INTENSITY + (F32(1.0) - w) * SK.GAME_EMITTER_INTENSITY
    got = np.array([SK.default_emitter_intensity(False, x) for x in w], F32)
    assert got.view(np.uint32).tolist() == mix.astype(F32).view(np.uint32).tolist()


def test_the_sun_texture_is_as_bright_as_chunkys():  # sky.rs:1133-1149
    assert abs(float(SK.SUN_TEXTURE_BRIGHTNESS) - 10.0 * 1.25 ** 2.2) < 1e-4
    su, sv = SK.sun_texture_axes(np.array([-0.999987, -0.005091, 0.0], F32))
    assert np.linalg.norm(su - [-0.005091, 0.999987, 0.0]) < 1e-5
    assert np.linalg.norm(sv - [0.0, 0.0, -1.0]) < 1e-5


# ---- FP64 restatements of Chunky's sky and sun ------------------------------------------------

# Preetham, Shirley and Smits, "A Practical Analytic Model for Daylight" (SIGGRAPH 1999),
# appendix A.2: the Perez coefficients A..E of Y, x and y as (slope, intercept) in the turbidity,
# and the zenith chromaticities as cubic polynomials in the sun's zenith angle whose coefficients
# are quadratics in the turbidity (rows: T^2, T, 1; columns: theta^3, theta^2, theta, 1).
PEREZ_LUMINANCE = np.array([[0.1787, -1.4630], [-0.3554, 0.4275], [-0.0227, 5.3251],
                            [0.1206, -2.5771], [-0.0670, 0.3703]])
PEREZ_X = np.array([[-0.0193, -0.2592], [-0.0665, 0.0008], [-0.0004, 0.2125],
                    [-0.0641, -0.8989], [-0.0033, 0.0452]])
PEREZ_Y = np.array([[-0.0167, -0.2608], [-0.0950, 0.0092], [-0.0079, 0.2102],
                    [-0.0441, -1.6537], [-0.0109, 0.0529]])
ZENITH_X = np.array([[0.00166, -0.00375, 0.00209, 0.0], [-0.02903, 0.06377, -0.03203, 0.00394],
                     [0.11693, -0.21196, 0.06052, 0.25886]])
ZENITH_Y = np.array([[0.00275, -0.00610, 0.00317, 0.0], [-0.04214, 0.08970, -0.04153, 0.00516],
                     [0.15346, -0.26756, 0.06670, 0.26688]])
# CIE XYZ to linear RGB and Chunky's exposure of the sky (`PreethamSky`).
XYZ_TO_RGB = np.array([[2.3706743, -0.9000405, -0.4706338], [-0.513885, 1.4253036, 0.0885814],
                       [0.0052982, -0.0146949, 1.0093968]])
SKY_SCALE = 0.045


def preetham64(alt, az, dirs, turbidity=2.5):
    """Chunky's Preetham sky radiance (linear RGB) for a sun at altitude `alt`, azimuth `az`
    (radians, the sun at (cos az cos alt, sin alt, sin az cos alt)), per direction of `dirs`
    (n x 3), in FP64."""
    T = turbidity

    def perez(cos_theta, gamma, coeff):
        # F(theta, gamma) with the horizon's 1/cos(theta) taken to +inf (the exponent's
        # coefficient is negative, so the term vanishes there)
        c = coeff[:, 0] * T + coeff[:, 1]
        with np.errstate(divide="ignore"):
            e = np.exp(c[1] / cos_theta) if np.ndim(cos_theta) == 0 else np.where(
                cos_theta > 0.0, np.exp(c[1] / np.where(cos_theta > 0.0, cos_theta, 1.0)), 0.0)
        return (1.0 + c[0] * e) * (1.0 + c[2] * np.exp(c[3] * gamma) + c[4] * np.cos(gamma) ** 2)

    def zenith_chroma(m, theta_s):
        poly = m @ np.array([theta_s ** 3, theta_s ** 2, theta_s, 1.0])
        return poly @ np.array([T * T, T, 1.0])

    theta_s = math.pi / 2 - alt
    chi = (4.0 / 9.0 - T / 120.0) * (math.pi - 2.0 * theta_s)
    y_zenith = abs((4.0453 * T - 4.9710) * math.tan(chi) - 0.2155 * T + 2.4192)
    sun = np.array([math.cos(az) * abs(math.cos(alt)), math.sin(alt), math.sin(az) * abs(math.cos(alt))])
    d = np.asarray(dirs, np.float64)
    cos_theta = np.maximum(d[:, 1], 0.0)
    gamma = np.arccos(np.clip(d @ sun, -1.0, 1.0))
    out = []
    for coeff, zenith in ((PEREZ_X, zenith_chroma(ZENITH_X, theta_s)), (PEREZ_Y, zenith_chroma(ZENITH_Y, theta_s)),
                          (PEREZ_LUMINANCE, y_zenith)):
        out.append(zenith * perez(cos_theta, gamma, coeff) / perez(1.0, theta_s, coeff))
    x, y, lum = out
    xyz = np.stack([x * lum / y, lum, (1.0 - x - y) * lum / y], -1)
    return xyz @ XYZ_TO_RGB.T * SKY_SCALE


def test_the_oracle_sky_is_chunkys_preetham_sky():  # sky.rs:1052-1109
    worst, n = 0.0, 0
    for alt_deg, az_deg in ((45.0, 45.0), (10.0, 200.0), (80.0, 300.0), (2.0, 90.0)):
        alt, az = math.radians(alt_deg), math.radians(az_deg)
        sun = np.array([math.cos(az) * math.cos(alt), math.sin(alt), math.sin(az) * math.cos(alt)], F32)
        pre = SK.Preetham(sun)
        p = L.new_params()
        p["sky_sun"] = [*pre.sun, 1.0]
        p["sky_zenith"] = [*pre.zenith, 0.0]
        for k, name in enumerate(("perez_a", "perez_b", "perez_c", "perez_d", "perez_e")):
            p[name] = [*pre.perez[k], 0.0]
        view = O.OracleScene(p, None, None, None, None, None, None)
        i, j = np.divmod(np.arange(64 * 17), 17)
        phi = i / 64.0 * 2.0 * math.pi
        h = j / 16.0 * 1.2 - 0.2  # a little below the horizon too
        r = np.sqrt(1.0 - h * h)
        dirs = np.stack([np.cos(phi) * r, h, np.sin(phi) * r], -1)
        want = preetham64(alt, az, dirs)
        got = np.array([view.preetham_radiance(dd.astype(F32)) for dd in dirs], np.float64)
        worst = max(worst, float((np.abs(got - want) / np.maximum(np.abs(want), 0.01)).max()))
        n += len(dirs)
    assert n == 4 * 64 * 17
    assert worst < 1e-4, worst


def chunky_sun_texel(sw, d):
    """Chunky's `Sun.intersect` and `Texture.getColor` in FP64, for a sun direction `sw` and
    directions `d` (n x 3): the (x, y) texel of a 32 x 32 sun texture each direction sees, or
    (-1, -1) where it sees none."""
    r = float(SK.SUN_RADIUS)
    su0 = np.array([0.0, 1.0, 0.0]) if abs(sw[0]) > 0.1 else np.array([1.0, 0.0, 0.0])
    sv = np.cross(sw, su0)
    sv /= np.linalg.norm(sv)
    su = np.cross(sv, sw)
    width, width2 = 4.0 * r, 8.0 * r
    a = math.pi / 2 - np.arccos(np.clip(d @ su, -1.0, 1.0)) + width
    b = math.pi / 2 - np.arccos(np.clip(d @ sv, -1.0, 1.0)) + width
    seen = (d @ sw >= 0.5) & (a >= 0.0) & (a < width2) & (b >= 0.0) & (b < width2)
    x = np.clip(np.trunc(a / width2 * 32.0 - 5e-8), 0, 31).astype(np.int64)
    y = np.clip(np.trunc((1.0 - b / width2) * 32.0 - 5e-8), 0, 31).astype(np.int64)
    return np.where(seen, x, -1), np.where(seen, y, -1)


def test_the_oracle_draws_chunkys_sun_texture():  # sky.rs:1151-1253
    atlas = sun_atlas()
    drawn = edge = checked = 0
    for sun in (np.array([-0.999987, -0.005091, 0.0], F32), SK.sun_direction(8.0, 330.0),
                SK.sun_direction(45.0, 135.0), SK.sun_direction(80.0, 3.0)):
        p = L.new_params()
        su, sv = sun_sprite_params(p, sun)
        p["off2"] = [0, SUN_ATLAS[0], SUN_ATLAS[1], 0]
        view = O.OracleScene(p, None, None, None, atlas, None, None)
        sw = sun.astype(np.float64)
        # directions over the square the texture covers and a little beyond
        da, db = np.meshgrid(np.arange(-60, 61) * 0.0025, np.arange(-60, 61) * 0.0025, indexing="ij")
        d = sw + su.astype(np.float64) * da.reshape(-1, 1) + sv.astype(np.float64) * db.reshape(-1, 1)
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        wx, wy = chunky_sun_texel(sw, d)
        for k in range(len(d)):
            got = view.sun_texture(d[k].astype(F32)).astype(np.float64)
            checked += 1
            if wx[k] < 0:
                edge += int(np.any(got != 0.0))
                continue
            c = sun_texel(int(wx[k]), int(wy[k]))
            want = np.array([((c >> s) & 0xFF) / 255.0 for s in (0, 8, 16)]) ** 2.2 * float(SK.SUN_TEXTURE_BRIGHTNESS)
            if np.all(np.abs(got - want) <= 1e-4 * np.maximum(want, 1.0)):
                drawn += 1
            else:
                edge += 1  # an f32 direction on a texel border may fall in the next texel
    assert checked == 4 * 121 * 121
    assert drawn > 4 * 90 * 90, drawn
    assert edge * 100 < checked, edge
    assert SUN_SPRITE[2] == 32 and SUN_SPRITE[3] == 32


def to_hsl64(c):
    """Chunky's `ColorUtil.RGBtoHSL` in FP64, per row of `c` (n x 3), the channels clamped to
    [0, 1]; the hue of a red maximum keeps the sign of its remainder, as Java's % does."""
    c = np.clip(c, 0.0, 1.0)
    r, g, b = c[:, 0], c[:, 1], c[:, 2]
    cmax, cmin = c.max(1), c.min(1)
    delta = cmax - cmin
    light = (cmax + cmin) / 2.0
    sd = np.where(delta == 0.0, 1.0, delta)
    hue = np.where(cmax == r, np.fmod((g - b) / sd, 6.0) / 6.0,
                   np.where(cmax == g, ((b - r) / sd + 2.0) / 6.0, ((r - g) / sd + 4.0) / 6.0))
    hue = np.where(delta == 0.0, 0.0, hue)
    den = 1.0 - np.abs(2.0 * light - 1.0)
    sat = np.where(delta < 5e-8, 0.0, delta / np.where(den == 0.0, 1.0, den))
    return np.stack([hue, sat, light], -1)


def from_hsl64(hsl):
    """Chunky's `ColorUtil.RGBfromHSL` in FP64, per row (n x 3)."""
    h, s, l = hsl[:, 0] * 6.0, hsl[:, 1], hsl[:, 2]
    c = np.minimum((1.0 - np.abs(2.0 * l - 1.0)) * s, 1.0)
    x = c * (1.0 - np.abs(np.fmod(h, 2.0) - 1.0))
    z = np.zeros_like(c)
    sector = np.select([h < 1.0, h < 2.0, h < 3.0, h < 4.0, h < 5.0], [0, 1, 2, 3, 4], 5)
    rgb = np.choose(sector[:, None], [np.stack(v, -1) for v in
                                      ((c, x, z), (x, c, z), (z, c, x), (z, x, c), (x, z, c), (c, z, x))])
    return rgb + np.maximum(l - 0.5 * c, 0.0)[:, None]


def test_the_oracle_reads_the_sky_through_chunkys_sky_cache():  # sky.rs:1255-1397
    n = SK.SKY_CACHE_RESOLUTION
    worst, count, saturated = 0.0, 0, 0
    for alt, az in ((-0.005091, math.pi), (0.1, 2.0), (0.8, 0.7)):
        # Chunky's `SkyCache.precalculateSky`: HSL of the sky at (n + 1)^2 directions, i over
        # the azimuth, j over the elevation.
        i, j = np.divmod(np.arange((n + 1) * (n + 1)), n + 1)
        theta = i / n * 2.0 * math.pi
        phi = j / n * math.pi - math.pi / 2
        table = to_hsl64(preetham64(max(alt, 0.0), az, np.stack(
            [np.cos(theta) * np.cos(phi), np.sin(phi), np.sin(theta) * np.cos(phi)], -1))).reshape(n + 1, n + 1, 3)
        sun = np.array([math.cos(az) * math.cos(alt), math.sin(alt), math.sin(az) * math.cos(alt)], F32)
        pre = SK.Preetham(sun)
        p = L.new_params()
        p["sky_sun"] = [*pre.sun, 1.0]
        p["sky_zenith"] = [*pre.zenith, 0.0]
        for k, name in enumerate(("perez_a", "perez_b", "perez_c", "perez_d", "perez_e")):
            p[name] = [*pre.perez[k], 0.0]
        p["misc_f"] = [0.0, 0.0, float(n), 0.0]
        view = O.OracleScene(p, None, None, None, None, None, None)
        cache = view.build_sky_cache(n)
        assert cache.size == (n + 1) * (n + 1) * 3
        view.set_sky(cache)
        a_i, h_j = np.divmod(np.arange(97 * 41), 41)
        a = a_i / 97.0 * 2.0 * math.pi + 0.013
        h = h_j / 40.0 * 1.9 - 0.95
        r = np.sqrt(1.0 - h * h)
        d = np.stack([np.cos(a) * r, h, np.sin(a) * r], -1)
        # `calcIncidentLight` and `getColorInterpolated`: bilinear in HSL between the cache's
        # entries around the direction's (azimuth, elevation)
        t = np.arctan2(d[:, 2], d[:, 0]) / (2.0 * math.pi)
        t = np.fmod(np.fmod(t, 1.0) + 1.0, 1.0)
        e = (np.arcsin(np.clip(d[:, 1], -1.0, 1.0)) + math.pi / 2) / math.pi
        x, y = t * n, e * n
        fx = np.clip(x, 0.0, n - 1.0).astype(np.int64)
        fy = np.clip(y, 0.0, n - 1.0).astype(np.int64)
        wx, wy = (x - fx)[:, None], (y - fy)[:, None]
        y0 = table[fx, fy] + wx * (table[fx + 1, fy] - table[fx, fy])
        y1 = table[fx, fy + 1] + wx * (table[fx + 1, fy + 1] - table[fx, fy + 1])
        want = from_hsl64(y0 + wy * (y1 - y0))
        got = view.sky_radiance_many(d.astype(F32)).astype(np.float64)
        worst = max(worst, float(np.abs(got - want).max()))
        bright = (preetham64(max(alt, 0.0), az, d) > 1.0).any(1)
        saturated += int(bright.sum())
        assert np.all(got[bright] <= 1.0 + 1e-5)
        count += len(d)
    assert count == 3 * 97 * 41
    assert saturated > 0, "no direction near a sun brighter than the cache's limit"
    assert worst < 1e-4, worst
