"""The game sky's maps on the host (`lumenwright_b200/gamesky.py`) and in the oracle
(`oracle/gamesky.c`), against the reference's own tests of them (crates/lumenwright/src/render/
sky.rs:1398-1460 and :1463-1565): the lightmap's colour is the client's lightmap shader at sky light
15 (restated here in f64) to within its 8-bit level; the maps of the client's dusk sky cast, on a
top face open to the whole sky, the lightmap's light to within 2e-3 (a second integration through
the kernel's own `sky_light` lookup); the veil is non-negative and zero in the channel that bounds
the scale; the sun is drawn in the lens's map and not in the light's. CPU only."""

import numpy as np
import pytest

from lumenwright_b200 import gamesky as G
from lumenwright_b200 import layout as L
from oracle import oracle as O

F32 = np.float32


def lightmap_fsh(sky_factor, sky_colour, brightness):
    """The client's lightmap.fsh at sky light 15 and block light 0, in f64 (the uniforms at their
    overworld values: no ambient light, darkening, night vision or darkness)."""
    get_brightness = lambda level: level / (4.0 - 3.0 * level)  # noqa: E731
    block = get_brightness(0.0) * 1.5
    sky = get_brightness(15.0 / 15.0) * sky_factor
    c = [block, block * ((block * 0.6 + 0.4) * 0.6 + 0.4), block * (block * block * 0.6 + 0.4)]
    for k in range(3):
        c[k] += sky_colour[k] * sky
        c[k] = min(max(c[k] * 0.96 + 0.75 * 0.04, 0.0), 1.0)
    mx = max(c)
    inv = 1.0 - mx
    scaled = 1.0 - inv ** 4
    out = []
    for k in range(3):
        ng = c[k] * (scaled / mx)
        v = c[k] + (ng - c[k]) * brightness
        out.append(v * 0.96 + 0.75 * 0.04)
    return out


def test_the_sky_light_is_the_clients_lightmap():  # sky.rs:1428-1460
    checked = 0
    for f in (0.0, 0.24, 0.385497, 0.62, 1.0):
        for col in ((1.0, 1.0, 1.0), (0x7A / 255.0, 0x7A / 255.0, 1.0)):
            for b in (0.0, 0.5, 1.0):
                col32 = np.array(col, F32)
                got = G.lightmap_sky(F32(f), col32, F32(b))
                want = lightmap_fsh(float(F32(f)), [float(v) for v in col32], float(F32(b)))
                for k in range(3):
                    assert abs(float(got[k]) - want[k]) <= 0.5 / 255.0 + 1e-6, (f, col, b, got, want)
                    assert float(got[k] * F32(255.0)) % 1.0 == 0.0
                checked += 1
    assert checked == 30
    c = 0x93 / 255.0
    light = np.power(G.lightmap_sky(F32(0.385497), np.array([c, c, 1.0], F32)).astype(np.float64), 2.2)
    engine = 0.374446
    level = round(engine ** (1.0 / 2.2) * 255.0) / 255.0
    assert abs(light[2] - level ** 2.2) < 2e-3


class OracleDraw:
    """The oracle as the maps' drawing backend."""

    def draw_sky_map(self, q, stars, w, h, atlas, atlas_w):
        return O.draw_sky_map(q, stars, w, h, atlas, atlas_w)


def dusk_maps(atlas, atlas_w, rect):
    desc = G.dusk_12800(rect)
    return G.game_sky_maps(OracleDraw(), desc, G.DUSK_SKY_LIGHT_FACTOR, G.DUSK_SKY_LIGHT_COLOR, atlas, atlas_w)


def sky_view(buf, sizes):
    p = L.new_params()
    p["sky_map"] = sizes
    z = np.zeros(1, np.uint32)
    return O.OracleScene(p, z, np.zeros(1, L.MODEL_DTYPE), np.zeros(1, L.QUAD_DTYPE), z, np.zeros(1, L.EMITTER_DTYPE), z,
                         buf)


def test_the_game_sky_casts_the_lightmaps_light():  # sky.rs:1497-1565
    atlas = np.full(4, 0xFFFFFFFF, np.uint32)
    buf, sizes, info = dusk_maps(atlas, 2, (0.0, 0.0, 2.0, 2.0))
    (lw, lh), (gw, gh) = G.LENS_MAP, G.LIGHT_MAP
    assert buf.size == (lw * lh + gw * gh) * 3
    veil, scale = info["veil"], info["scale"]
    assert veil.min() >= 0.0
    assert veil.min() == 0.0 or scale == G.MAX_SKY_LIGHT
    v = sky_view(buf, sizes)
    na, ne = 720, 180
    acc = np.zeros(3)
    wsum = 0.0
    for i in range(na):
        az = (i + 0.5) / na * 2.0 * np.pi
        for j in range(ne):
            el = (j + 0.5) / ne * np.pi / 2.0
            d = (F32(np.cos(el) * np.cos(az)), F32(np.sin(el)), F32(np.cos(el) * np.sin(az)))
            w = np.sin(el) * np.cos(el)
            acc += np.array(v.sky_light(d), np.float64) * w
            wsum += w
    cast = acc / wsum
    print(f"game sky at dusk: light {info['light']} cast {cast} (scale {scale}, mean {info['mean']}, veil {veil})")
    for k in range(3):
        assert abs(cast[k] - info["light"][k]) / info["light"][k] < 2e-3, (cast, info["light"])
    sun = G.celestial_direction(90.29)
    d = (float(sun[0]), max(float(sun[1]), 0.01), float(sun[2]))
    seen = np.array(v.sky_lens(d))
    lit = np.array(v.sky_light(d)) / scale
    assert seen[2] > 0.9 and seen[2] > lit[2] + 0.3, (seen, lit)


def test_stars_follow_build_stars():
    # The client's buildStars draws (sky.rs:97-136): every accepted star lies at distance 100 with
    # two perpendicular half-axes of length 0.15..0.25, and each is in the bin of its own direction.
    st = G.stars()
    assert 0 < len(st) < 1500
    table = G.star_table()
    nb = G.STAR_BINS_AZ * G.STAR_BINS_EL
    starts = table[:nb + 1]
    assert np.all(np.diff(starts.astype(np.int64)) >= 0) and starts[0] == 0
    assert table.size == nb + 1 + int(starts[-1]) * G.STAR_WORDS
    for c, a1, a2 in st:
        assert abs(float(np.linalg.norm(c)) - 100.0) < 1e-3
        for a in (a1, a2):
            assert 0.15 - 1e-5 <= float(np.linalg.norm(a)) <= 0.25 + 1e-5
        assert abs(float(a1 @ a2)) < 1e-6 and abs(float(a1 @ c)) < 1e-4
    # each star's own bin lists it (its centre, the table's first three words of an entry)
    entries = table[nb + 1:].view(np.float32).reshape(-1, G.STAR_WORDS)
    for c, _, _ in st[:200]:
        q = (c / F32(100.0)).astype(F32)
        ia = int(np.floor((G.atan2f(q[2], q[0]) + G.PI) / G.TAU * G.STAR_BINS_AZ))
        ie = int(np.floor((G.asinf(q[1]) + G.FRAC_PI_2) / G.PI * G.STAR_BINS_EL))
        b = min(ie, G.STAR_BINS_EL - 1) * G.STAR_BINS_AZ + min(ia, G.STAR_BINS_AZ - 1)
        assert any(np.array_equal(entries[e, :3], c) for e in range(starts[b], starts[b + 1]))


def test_the_light_map_draws_no_bodies_and_the_lens_map_its_stars():
    atlas = np.full(4, 0xFFFFFFFF, np.uint32)
    desc = G.dusk_12800((0.0, 0.0, 2.0, 2.0))
    table = G.star_table()
    lens = O.draw_sky_map(G.quick_sky(desc), table, 512, 256, atlas, 2)
    bare = O.draw_sky_map(G.quick_sky(G.bare(desc)), table, 512, 256, atlas, 2)
    diff = np.abs(lens - bare).max(-1)
    print(f"texels brightened by the sun or a star: {(diff > 1e-6).sum()} of {diff.size}")
    assert (diff > 1e-6).sum() > 0
    assert np.all(lens >= bare - 1e-7)  # bodies and stars only add light
    assert np.all((lens >= 0.0) & (lens <= 1.0))
