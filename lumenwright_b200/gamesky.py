"""The game's sky as the hq kernel reads it under `SkyLook::Game` or a mixed day weight: the client's
sky drawn into two equirectangular maps (crates/lumenwright/src/render/sky.rs:855-952).

Host side, as the reference computes it, in f32 with the platform's f32 `sinf`, `cosf`, `atan2f`,
`asinf` and `powf` (what Rust's f32 methods call on Linux):
  * `SkyDescription` (sky.rs:225-252): what the sky passes draw at one tick;
  * `quick_sky` (`QuickSky::new`, sky.rs:321-375): the packed record the per-texel pass reads
    (the sun and moon quads, the star rotation, the sunrise fan);
  * `stars` / `star_table` (sky.rs:97-217): the client's 1500 star draws of `buildStars`
    (java.util.Random seeded with 10842) binned by direction;
  * `lightmap_sky` (sky.rs:798-811) and the light map's scale and veil (sky.rs:927-944).
On the device (``Context.draw_sky_map``, the library's `lw_draw_sky_map`): `QuickSky::background`
(sky.rs:509-530) for every texel of a map, decoded to linear (`draw_map`, sky.rs:861-878).

No client jar, and so no environment attributes or timeline, is available here: a frame's sky is
stated (`Sky::Stated` with a tick, request.rs:239-264) by a `SkyDescription`. `DUSK_12800` is the
client's dusk sky at tick 12800 as the reference's own test states it (sky.rs:1466-1481), the sky
of the dusk configurations.
"""

import ctypes as C
import math
from dataclasses import dataclass, replace
from typing import Optional, Tuple

import numpy as np

F32 = np.float32
LENS_MAP = (2048, 1024)   # sky.rs:776
LIGHT_MAP = (360, 180)    # sky.rs:781
MAX_SKY_LIGHT = F32(50.0)  # sky.rs:786
DEFAULT_BRIGHTNESS = F32(0.5)  # sky.rs:772
GAMMA = F32(2.2)
STAR_BINS_AZ, STAR_BINS_EL, STAR_WORDS = 128, 64, 9  # sky.rs:63-67

_libm = C.CDLL("libm.so.6")
for _n in ("sinf", "cosf", "atan2f", "asinf", "powf"):
    getattr(_libm, _n).restype = C.c_float
_libm.sinf.argtypes = _libm.cosf.argtypes = _libm.asinf.argtypes = [C.c_float]
_libm.atan2f.argtypes = _libm.powf.argtypes = [C.c_float, C.c_float]


def sinf(x):
    return F32(_libm.sinf(float(x)))


def cosf(x):
    return F32(_libm.cosf(float(x)))


def atan2f(y, x):
    return F32(_libm.atan2f(float(y), float(x)))


def asinf(x):
    return F32(_libm.asinf(float(x)))


def powf(x, y):
    return F32(_libm.powf(float(x), float(y)))


PI = F32(math.pi)
TAU = F32(2.0 * math.pi)
FRAC_PI_2 = F32(math.pi / 2.0)
RAD_PER_DEG = F32(PI / F32(180.0))  # f32::to_radians: PI / 180 in f32


def v3(x, y, z):
    return np.array([x, y, z], F32)


def length(v):
    return F32(np.sqrt(F32(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])))


def normalize(v):
    """glam `normalize`: times the reciprocal of the length."""
    return (v * F32(F32(1.0) / length(v))).astype(F32)


def cross(a, b):
    return v3(a[1] * b[2] - b[1] * a[2], a[2] * b[0] - b[2] * a[0], a[0] * b[1] - b[0] * a[1])


def dot(a, b):
    return F32(F32(a[0] * b[0] + a[1] * b[1]) + a[2] * b[2])


class Mat3:
    """glam's column-major `Mat3`, f32."""

    def __init__(self, x, y, z):
        self.c = [np.asarray(x, F32), np.asarray(y, F32), np.asarray(z, F32)]

    @staticmethod
    def rotation_x(a):
        s, c = sinf(a), cosf(a)
        return Mat3(v3(1, 0, 0), v3(0, c, s), v3(0, -s, c))

    @staticmethod
    def rotation_y(a):
        s, c = sinf(a), cosf(a)
        return Mat3(v3(c, 0, -s), v3(0, 1, 0), v3(s, 0, c))

    @staticmethod
    def rotation_z(a):
        s, c = sinf(a), cosf(a)
        return Mat3(v3(c, s, 0), v3(-s, c, 0), v3(0, 0, 1))

    @staticmethod
    def diagonal(d):
        return Mat3(v3(d[0], 0, 0), v3(0, d[1], 0), v3(0, 0, d[2]))

    def mul_vec(self, v):
        x, y, z = self.c
        return ((x * v[0] + y * v[1]).astype(F32) + z * v[2]).astype(F32)

    def __mul__(self, o):
        return Mat3(self.mul_vec(o.c[0]), self.mul_vec(o.c[1]), self.mul_vec(o.c[2]))

    def transpose(self):
        x, y, z = self.c
        return Mat3(v3(x[0], y[0], z[0]), v3(x[1], y[1], z[1]), v3(x[2], y[2], z[2]))

    def row(self, i):
        return v3(self.c[0][i], self.c[1][i], self.c[2][i])


def celestial_rotation(angle_deg):
    """sky.rs:55-58: `Axis.YP(-90 deg)` then `Axis.XP(angle)`."""
    return Mat3.rotation_y(-FRAC_PI_2) * Mat3.rotation_x(F32(angle_deg) * RAD_PER_DEG)


def celestial_direction(angle_deg):
    """sky.rs:62-64."""
    return celestial_rotation(angle_deg).mul_vec(v3(0, 1, 0))


@dataclass
class SkyDescription:
    """sky.rs:225-252 (colours sRGB 0..1)."""
    sky: tuple
    fog: tuple
    sky_fog_end: float
    render_fog: Tuple[float, float]
    env_fog: Tuple[float, float]
    sky_disc: bool
    sunrise: tuple  # rgb and alpha
    sun_angle: float
    sun: Optional[tuple]  # (direction, atlas rect x, y, w, h)
    moon: Optional[tuple]
    star_angle: float
    star_brightness: float


def dusk_12800(sun_rect):
    """The client's sky at tick 12800 (dusk) with its bodies, as the reference's test states it
    (sky.rs:1466-1481), the sun drawn from the atlas rectangle `sun_rect`."""
    return SkyDescription(sky=(0.18, 0.24, 0.37), fog=(0.62, 0.40, 0.33), sky_fog_end=192.0,
                          render_fog=(172.8, 192.0), env_fog=(0.0, 1024.0), sky_disc=True,
                          sunrise=(0.98, 0.57, 0.25, 0.62), sun_angle=90.29,
                          sun=(celestial_direction(90.29), tuple(float(v) for v in sun_rect)), moon=None,
                          star_angle=90.29, star_brightness=0.38)


# The lightmap's two attributes at tick 12800 (the same test, sky.rs:1505-1506).
DUSK_SKY_LIGHT_FACTOR = F32(0.378182)
DUSK_SKY_LIGHT_COLOR = (np.array([0x92, 0x92, 0xFF], F32) / F32(255.0)).astype(F32)


def stated_sky(ticks: int, sun_rect):
    """The stated game sky of a tick: (description, sky light factor, sky light colour). Only the
    dusk tick 12800 is stated (the reference's own dusk sky); any other tick is refused, as the
    reference refuses the game's sky without a jar's environment attributes (request.rs:765-771)."""
    if ticks % 24000 != 12800:
        raise ValueError(f"no stated game sky for tick {ticks}: only the dusk tick 12800 is stated "
                         "(the client's environment attributes, which give the others, need its jar)")
    return dusk_12800(sun_rect), DUSK_SKY_LIGHT_FACTOR, DUSK_SKY_LIGHT_COLOR


def bare(desc: SkyDescription) -> SkyDescription:
    """What the light's map draws: no sun, moon or stars (request.rs:850-855)."""
    return replace(desc, sun=None, moon=None, star_brightness=0.0)


# `QuickSky` (sky.rs:274-305): 38 vec4 = 608 bytes.
QUICK_SKY_DTYPE = np.dtype([
    ("sky_color", F32, 4), ("fog_color", F32, 4), ("fog_dist", F32, 4), ("sunrise", F32, 4), ("flags", F32, 4),
    ("sun", F32, (4, 4)), ("moon", F32, (4, 4)), ("star_rot", F32, (3, 4)), ("fan", F32, (18, 4)),
    ("cam_forward", F32, 4), ("cam_right", F32, 4), ("cam_up", F32, 4), ("cam_misc", F32, 4),
])
assert QUICK_SKY_DTYPE.itemsize == 608


def body_quad(d, size, rect, flip):
    """sky.rs:313-318: a sprite quad of half-size `size` at distance 100 towards `d`."""
    c = (d * F32(100.0)).astype(F32)
    ex = (v3(0, 0, 1) - d * d[2]).astype(F32)
    if dot(ex, ex) < F32(1e-8):
        ex = v3(1, 0, 0)
    ex = normalize(ex)
    ez = cross(ex, d)
    s = F32(-1.0) / F32(size) if flip else F32(1.0) / F32(size)
    return np.array([[c[0], c[1], c[2], 1.0], [*(ex * s), 0.0], [*(ez * s), 0.0], list(rect)], F32)


def quick_sky(desc: SkyDescription) -> np.ndarray:
    """`QuickSky::new` (sky.rs:321-375) without the camera fields (the maps do not use them)."""
    q = np.zeros((), QUICK_SKY_DTYPE)
    q["sky_color"] = [*desc.sky, desc.sky_fog_end]
    q["fog_color"] = [*desc.fog, desc.render_fog[0]]
    sb = F32(desc.star_brightness)
    q["fog_dist"] = [desc.render_fog[1], desc.env_fog[0], desc.env_fog[1], sb * sb]
    q["sunrise"] = list(desc.sunrise)
    q["flags"] = [float(desc.sky_disc), float(desc.sky_disc and desc.sunrise[3] > 0.001),
                  float(desc.sky_disc and desc.star_brightness > 0.0), 0.0]
    if desc.sky_disc:
        if desc.sun is not None:
            q["sun"] = body_quad(np.asarray(desc.sun[0], F32), 30.0, desc.sun[1], False)
        if desc.moon is not None:
            q["moon"] = body_quad(np.asarray(desc.moon[0], F32), 20.0, desc.moon[1], True)
    inv = celestial_rotation(desc.star_angle).transpose()
    for i in range(3):
        q["star_rot"][i] = [*inv.row(i), 0.0]
    flip = F32(180.0) if sinf(F32(desc.sun_angle) * RAD_PER_DEG) < 0.0 else F32(0.0)
    alpha = F32(desc.sunrise[3])
    m = Mat3.rotation_x(FRAC_PI_2) * Mat3.rotation_z(F32(flip + F32(90.0)) * RAD_PER_DEG) * Mat3.diagonal(v3(1, 1, alpha))
    q["fan"][0] = [*m.mul_vec(v3(0, 100, 0)), alpha]
    for k in range(17):
        t = F32(F32(k) * TAU) / F32(16.0)
        s, c = sinf(t), cosf(t)
        q["fan"][k + 1] = [*m.mul_vec(v3(s * F32(120.0), c * F32(120.0), -c * F32(40.0))), 0.0]
    return q


class _LegacyRandom:
    """java.util.Random's 48-bit LCG (sky.rs:70-95)."""

    MASK = (1 << 48) - 1

    def __init__(self, seed):
        self.s = (seed ^ 0x5DEECE66D) & self.MASK

    def next(self, bits):
        self.s = (self.s * 0x5DEECE66D + 0xB) & self.MASK
        v = self.s >> (48 - bits)
        return v - (1 << 32) if v >= (1 << 31) else v  # as i32

    def next_float(self):
        return F32(F32(self.next(24)) * F32(5.9604645e-8))

    def next_double(self):
        hi, lo = self.next(26), self.next(27)
        return float(F32(F32((hi << 27) + lo) * F32(1.110223e-16)))


_STARS = None


def stars():
    """`SkyRenderer.buildStars` (sky.rs:97-136): (centre, a1, a2) per star, star space."""
    global _STARS
    if _STARS is None:
        r = _LegacyRandom(10842)
        out = []
        for _ in range(1500):
            x = F32(r.next_float() * F32(2.0) - F32(1.0))
            y = F32(r.next_float() * F32(2.0) - F32(1.0))
            z = F32(r.next_float() * F32(2.0) - F32(1.0))
            size = F32(F32(0.15) + r.next_float() * F32(0.1))
            len2 = F32(F32(x * x + y * y) + z * z)
            if len2 <= F32(0.010000001) or len2 >= F32(1.0):
                continue
            v = v3(x, y, z)
            center = (v * F32(F32(100.0) / length(v))).astype(F32)
            theta = F32(r.next_double() * float(PI) * 2.0)
            ndir = normalize(-center)
            left = normalize(cross(v3(0, 1, 0), ndir))
            upn = cross(ndir, left)
            s, c = sinf(-theta), cosf(-theta)
            a1 = ((left * c + upn * s) * size).astype(F32)
            a2 = ((left * -s + upn * c) * size).astype(F32)
            out.append((center, a1, a2))
        _STARS = out
    return _STARS


_TABLE = None


def star_table() -> np.ndarray:
    """sky.rs:158-217: per (azimuth, elevation) bin the stars whose extent (with a margin) touches
    it, as u32 words: the bins' start indices and an end, then nine floats per entry (centre,
    a1 / |a1|^2, a2 / |a2|^2)."""
    global _TABLE
    if _TABLE is not None:
        return _TABLE
    nbins = STAR_BINS_AZ * STAR_BINS_EL
    bins = [[] for _ in range(nbins)]
    da, de = F32(TAU / F32(STAR_BINS_AZ)), F32(PI / F32(STAR_BINS_EL))
    for i, (center, a1, a2) in enumerate(stars()):
        d = (center / F32(100.0)).astype(F32)
        radius = F32(F32(F32(2.0) * F32(length(a1) + length(a2))) / F32(100.0))
        el = asinf(d[1])
        az = atan2f(d[2], d[0])
        el0, el1 = F32(el - radius), F32(el + radius)
        ie0 = max(int(math.floor(F32(F32(el0 + FRAC_PI_2) / de))), 0)
        ie1 = min(int(math.floor(F32(F32(el1 + FRAC_PI_2) / de))), STAR_BINS_EL - 1)
        cos_min = cosf(min(max(abs(el0), abs(el1)), FRAC_PI_2))
        half = PI if cos_min < F32(0.05) else F32(radius / cos_min)
        ia0 = int(math.floor(F32(F32(F32(az - half) + PI) / da)))
        ia1 = int(math.floor(F32(F32(F32(az + half) + PI) / da)))
        for ie in range(ie0, ie1 + 1):
            if half >= PI:
                for ia in range(STAR_BINS_AZ):
                    bins[ie * STAR_BINS_AZ + ia].append(i)
                continue
            for ia in range(ia0, ia1 + 1):
                b = ie * STAR_BINS_AZ + ia % STAR_BINS_AZ
                if i not in bins[b]:
                    bins[b].append(i)
    starts, n = [], 0
    for b in bins:
        starts.append(n)
        n += len(b)
    starts.append(n)
    words = [np.array(starts, np.uint32)]
    st = stars()
    for b in bins:
        for i in b:
            center, a1, a2 = st[i]
            e = np.concatenate([center, (a1 / dot(a1, a1)).astype(F32), (a2 / dot(a2, a2)).astype(F32)]).astype(F32)
            words.append(e.view(np.uint32))
    _TABLE = np.concatenate(words).astype(np.uint32)
    return _TABLE


def lightmap_sky(factor, colour, brightness=DEFAULT_BRIGHTNESS):
    """sky.rs:798-811: the lightmap's colour of a cell open to the sky, at its 8-bit level."""
    factor, brightness = F32(factor), F32(brightness)
    colour = np.asarray(colour, F32)
    mix75 = lambda c: (c * F32(0.96) + F32(F32(0.75) * F32(0.04))).astype(F32)  # noqa: E731
    c = np.clip(mix75((colour * factor).astype(F32)), F32(0.0), F32(1.0)).astype(F32)
    mx = F32(c.max())
    if mx > 0.0:
        inv = F32(F32(1.0) - mx)
        not_gamma = (c * F32(F32(F32(1.0) - inv * inv * inv * inv) / mx)).astype(F32)
    else:
        not_gamma = c
    c = mix75((c + (not_gamma - c) * brightness).astype(F32))
    level = np.floor((c * F32(255.0)).astype(F32).astype(np.float64) + 0.5).astype(F32)  # f32::round
    return (level / F32(255.0)).astype(F32)


def map_direction(i, j, w, h):
    """sky.rs:853-858 (f32) for arrays of texel indices."""
    from . import sky as SK
    return SK.map_direction(i, j, w, h)


def finish_maps(lens, game, factor, colour):
    """sky.rs:927-952: the light map scaled so a top face open to the whole sky takes the
    lightmap's light: mean = the cosine-weighted mean of `game` over the upper hemisphere (f64
    sums), target = lightmap_sky(...)^2.2, scale = min(50, target / mean per channel), veil =
    max(target / scale - mean, 0). Returns (buffer, sizes, info)."""
    gw, gh = LIGHT_MAP
    game = np.asarray(game, F32).reshape(gh, gw, 3)
    j, i = np.mgrid[0:gh, 0:gw]
    d = map_direction(i, j, gw, gh)
    y = d[..., 1]
    up = y > 0.0
    wgt = np.where(up, (y * np.sqrt(np.maximum(F32(1.0) - y * y, F32(0.0)))).astype(F32), F32(0.0)).astype(np.float64)
    acc = (game.astype(np.float64) * wgt[..., None])[up].sum(0)
    mean = (acc / wgt[up].sum()).astype(F32)
    target = np.array([powf(v, GAMMA) for v in lightmap_sky(factor, colour)], F32)
    scale = MAX_SKY_LIGHT
    for k in range(3):
        if mean[k] > 0.0:
            scale = min(scale, F32(target[k] / mean[k]))
    veil = np.maximum((target / scale - mean).astype(F32), F32(0.0)).astype(F32)
    light = ((game + veil) * scale).astype(F32)
    buf = np.concatenate([np.asarray(lens, F32).ravel(), light.ravel()]).astype(F32)
    sizes = np.array([LENS_MAP[0], LENS_MAP[1], LIGHT_MAP[0], LIGHT_MAP[1]], F32)
    return buf, sizes, {"light": target, "mean": mean, "scale": F32(scale), "veil": veil}


def game_sky_maps(backend, desc: SkyDescription, factor, colour, atlas, atlas_w):
    """`game_sky_maps` (sky.rs:909-952): the lens map of `desc` and the light map of its bare
    sky, drawn by ``backend.draw_sky_map(quick_sky, stars, w, h, atlas, atlas_w)`` (the device, or
    the oracle on the host), then the light map's scale and veil. Returns (buffer, sizes, info)."""
    table = star_table()
    lens = backend.draw_sky_map(quick_sky(desc), table, LENS_MAP[0], LENS_MAP[1], atlas, atlas_w)
    game = backend.draw_sky_map(quick_sky(bare(desc)), table, LIGHT_MAP[0], LIGHT_MAP[1], atlas, atlas_w)
    return finish_maps(lens, game, factor, colour)
