"""Host-side sun and sky set-up of an hq frame, restating the reference's
`crates/lumenwright/src/render/sky.rs` (sun position, Chunky's sun and Preetham sky parameters,
the sun texture axes, the game sky's map geometry) and the sky parts of
`crates/lumenwright/src/request.rs`. FP64 where the reference computes in f64.

The game sky's maps (the client's sky drawn per direction, sky.rs:855-952) are
``lumenwright_b200.gamesky``'s.
"""

import math

import numpy as np

F32 = np.float32

SUN_RADIUS = F32(0.03)                   # sky.rs:563
DEFAULT_SUN_INTENSITY = F32(1.25)        # sky.rs:559
SUN_TEXTURE_BRIGHTNESS = F32(16.338118)  # sky.rs:569
SKY_CACHE_RESOLUTION = 128               # sky.rs:588
CIVIL_TWILIGHT_END = F32(-6.0 * math.pi / 180.0)  # sky.rs:615
NIGHT_SKY_LIGHT = F32(0.03)              # sky.rs:618
LENS_MAP = (2048, 1024)                  # sky.rs:776
LIGHT_MAP = (360, 180)                   # sky.rs:781
MAX_SKY_LIGHT = F32(50.0)                # sky.rs:786
DEFAULT_EMITTER_INTENSITY = F32(13.0)    # request.rs:127
GAME_EMITTER_INTENSITY = F32(137.9628)   # request.rs:138
GAMMA = F32(2.2)


def celestial_angle(ticks: int) -> np.float32:
    """sky.rs:28-32."""
    f = ((ticks % 24000) / 24000.0 - 0.25) % 1.0
    g = 0.5 - math.cos(f * math.pi) / 2.0
    return F32((f * 2.0 + g) / 3.0)


def normalize32(v):
    v = np.asarray(v, F32)
    l = F32(np.sqrt(F32(F32(v[0] * v[0]) + F32(v[1] * v[1])) + F32(v[2] * v[2])))
    return (v * (F32(1.0) / l)).astype(F32)


def sun_direction_from_angle(angle) -> np.ndarray:
    """sky.rs:35-38 (f32)."""
    t = F32(angle) * F32(2 * math.pi)
    return normalize32([-np.sin(t, dtype=F32), np.cos(t, dtype=F32), F32(0.0)])


def sun_direction(altitude_deg, azimuth_deg) -> np.ndarray:
    """sky.rs:41-44 (f32): the sun at an altitude and azimuth in degrees, azimuth 0 north (-z),
    90 east (+x)."""
    alt = F32(F32(altitude_deg) * F32(math.pi / 180.0))
    az = F32(F32(azimuth_deg) * F32(math.pi / 180.0))
    ca = np.cos(alt, dtype=F32)
    return normalize32([np.sin(az, dtype=F32) * ca, np.sin(alt, dtype=F32), -np.cos(az, dtype=F32) * ca])


def day_weight(factor, night, day) -> np.float32:
    """sky.rs:824-829: where the sky light factor stands between its night and day values,
    clamped to [0, 1]; 1 for a timeline whose two values do not differ."""
    factor, night, day = F32(factor), F32(night), F32(day)
    if F32(day - night) <= np.finfo(F32).eps:
        return F32(1.0)
    return F32(min(max(F32((factor - night) / F32(day - night)), F32(0.0)), F32(1.0)))


def twilight(altitude) -> np.float32:
    """sky.rs:625-629: 1 while the sun's disc is up, falling linearly to the night's sky light
    at the end of civil twilight."""
    v = F32((F32(altitude) - CIVIL_TWILIGHT_END) / (-SUN_RADIUS - CIVIL_TWILIGHT_END))
    v = min(max(v, F32(0.0)), F32(1.0))
    return F32(max(v, NIGHT_SKY_LIGHT))


class HqSky:
    """`HqSky` (sky.rs:549-557)."""

    def __init__(self, sun_dir, sun_color, sky_light):
        self.sun_dir = np.asarray(sun_dir, F32)
        self.sun_color = np.asarray(sun_color, F32)
        self.sky_light = F32(sky_light)


def hq_sky(sun_dir, sun_intensity=DEFAULT_SUN_INTENSITY, sky_intensity=F32(1.0)) -> HqSky:
    """sky.rs:636-643."""
    altitude = F32(math.asin(max(-1.0, min(1.0, float(sun_dir[1])))))
    c = F32(float(sun_intensity) ** float(GAMMA))
    return HqSky(sun_dir, [c, c, c], F32(sky_intensity) * twilight(altitude))


class Preetham:
    """`Preetham::new` (sky.rs:666-742): Chunky's Preetham sky at turbidity 2.5, in f64."""

    X_ZENITH = [[0.00166, -0.00375, 0.00209, 0.0], [-0.02903, 0.06377, -0.03203, 0.00394],
                [0.11693, -0.21196, 0.06052, 0.25886]]
    Y_ZENITH = [[0.00275, -0.00610, 0.00317, 0.0], [-0.04214, 0.08970, -0.04153, 0.00516],
                [0.15346, -0.26756, 0.06670, 0.26688]]
    MDX = [[-0.0193, -0.2592], [-0.0665, 0.0008], [-0.0004, 0.2125], [-0.0641, -0.8989], [-0.0033, 0.0452]]
    MDY = [[-0.0167, -0.2608], [-0.0950, 0.0092], [-0.0079, 0.2102], [-0.0441, -1.6537], [-0.0109, 0.0529]]
    MD_LUM = [[0.1787, -1.4630], [-0.3554, 0.4275], [-0.0227, 5.3251], [0.1206, -2.5771], [-0.0670, 0.3703]]

    def __init__(self, sun_dir, turbidity=2.5):
        T = float(turbidity)
        d = np.asarray(sun_dir, np.float64)
        d = d / math.sqrt(float(d @ d))
        azimuth = math.atan2(d[2], d[0])
        alt = min(max(math.asin(max(-1.0, min(1.0, d[1]))), 0.0), math.pi)
        if alt > math.pi / 2:
            alt = math.pi - alt
        r = abs(math.cos(alt))
        sun = np.array([math.cos(azimuth) * r, math.sin(alt), math.sin(azimuth) * r])

        def coeff(m):
            return [m[i][0] * T + m[i][1] for i in range(5)]

        cx, cy, cl = coeff(self.MDX), coeff(self.MDY), coeff(self.MD_LUM)

        def perez_f(cos_theta, gamma, cos2_gamma, c):
            return (1.0 + c[0] * math.exp(c[1] / cos_theta)) * (1.0 + c[2] * math.exp(c[3] * gamma) + c[4] * cos2_gamma)

        def chroma(st, m):
            row = lambda r: r[0] * st ** 3 + r[1] * st * st + r[2] * st + r[3]  # noqa: E731
            return T * T * row(m[0]) + T * row(m[1]) + row(m[2])

        sun_theta = math.pi / 2 - alt
        cos2_theta = math.cos(sun_theta) ** 2
        chi = (4.0 / 9.0 - T / 120.0) * (math.pi - 2.0 * sun_theta)
        zenith_lum = abs((4.0453 * T - 4.9710) * math.tan(chi) - 0.2155 * T + 2.4192)
        zx, zy = chroma(sun_theta, self.X_ZENITH), chroma(sun_theta, self.Y_ZENITH)
        f0 = lambda c: 1.0 / perez_f(1.0, sun_theta, cos2_theta, c)  # noqa: E731
        # f64 values (the adjoint's sky Jacobian) and the f32 Params fields cast from them.
        self.sun64 = sun
        self.zenith64 = np.array([zx * f0(cx), zy * f0(cy), zenith_lum * f0(cl)])
        self.perez64 = np.array([[cx[i], cy[i], cl[i]] for i in range(5)])
        self.sun = sun.astype(F32)
        self.zenith = self.zenith64.astype(F32)
        self.perez = self.perez64.astype(F32)
        self.turbidity = T


def sun_texture_axes(sw):
    """sky.rs:574-585 (f64)."""
    s = np.asarray(sw, np.float64)
    su = np.array([0.0, 1.0, 0.0]) if abs(s[0]) > 0.1 else np.array([1.0, 0.0, 0.0])
    sv = np.cross(s, su)
    sv = sv / math.sqrt(float(sv @ sv))
    su = np.cross(sv, s)
    return su.astype(F32), sv.astype(F32)


def map_direction(i, j, w, h):
    """sky.rs:853-858 (f32), for arrays of texel indices."""
    az = (np.asarray(i, F32) + F32(0.5)) / F32(w) * F32(2 * math.pi)
    el = (np.asarray(j, F32) + F32(0.5)) / F32(h) * F32(math.pi) - F32(math.pi / 2)
    return np.stack([np.cos(el) * np.cos(az), np.sin(el), np.cos(el) * np.sin(az)], -1).astype(F32)


def default_emitter_intensity(on_day_plateau: bool, weight) -> np.float32:
    """request.rs:156-162."""
    if on_day_plateau:
        return F32(0.0)
    w = F32(weight)
    return F32(w * DEFAULT_EMITTER_INTENSITY + (F32(1.0) - w) * GAME_EMITTER_INTENSITY)


def dusk_day_weight(ticks: int) -> np.float32:
    """The day weight of the client's 1.21.11 day timeline at a tick (sky.rs:824-829 over the
    timeline `day_weight` describes): 1 on the day plateau 730..11270, falling linearly to 0 at
    13140, 0 on the night plateau to 22860, rising back by 730."""
    t = ticks % 24000
    if 730 <= t <= 11270:
        return F32(1.0)
    if 11270 < t < 13140:
        return F32((13140 - t) / 1870.0)
    if 13140 <= t <= 22860:
        return F32(0.0)
    return F32(((t - 22860) % 24000) / 1870.0) if t > 22860 else F32((t + 24000 - 22860) / 1870.0)
