"""The game sky's maps on the device (`lw_draw_sky_map`) against the oracle's (`oracle/gamesky.c`,
pinned by the reference's own game-sky tests in tests/test_gamesky.py), for the client's dusk sky
with its sun and stars (the lens map, 2048x1024) and without them (the light map, 360x180), on
the synthetic atlas's sun sprite: every texel within 1e-5 relative but where a star's or the
sun's edge passes through the texel's direction (CUDA's sinf, cosf, atan2f and powf against the
platform's move a direction by an ulp, which can put it on the other side of an edge; those are
counted and bounded); and the finished maps (scale and veil) within 1e-5."""

import numpy as np
import pytest

from lumenwright_b200 import gamesky as G
from lumenwright_b200 import synth as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from lumenwright_b200.native import Context
    c = Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def atlas():
    a = S.build_atlas(1)
    sun = a.sprites["sun"]
    return np.ascontiguousarray(a.pixels, np.uint32).ravel(), a.pixels.shape[1], (sun.x, sun.y, sun.w, sun.h)


def close(a, b, rel=1e-5, atol=1e-7):
    return np.abs(a - b) <= rel * np.maximum(np.abs(a), np.abs(b)) + atol


@pytest.mark.parametrize("which", ["lens", "light"])
def test_device_map_matches_the_oracle(ctx, atlas, which):
    pix, aw, rect = atlas
    desc = G.dusk_12800(rect)
    if which == "light":
        desc = G.bare(desc)
    w, h = G.LENS_MAP if which == "lens" else G.LIGHT_MAP
    q = G.quick_sky(desc)
    got = ctx.draw_sky_map(q, G.star_table(), w, h, pix, aw)
    want = O.draw_sky_map(q, G.star_table(), w, h, pix, aw)
    ok = np.all(close(got, want), -1)
    bad = int((~ok).sum())
    print(f"{which} map {w}x{h}: {bad} of {ok.size} texels outside 1e-5 (an edge between the two "
          f"directions), worst {np.abs(got - want).max():.3g}")
    assert np.isfinite(got).all()
    assert bad <= 1e-4 * ok.size + 2


def test_finished_maps_match_the_oracle(ctx, atlas):
    pix, aw, rect = atlas

    class OracleDraw:
        def draw_sky_map(self, q, stars, w, h, a, a_w):
            return O.draw_sky_map(q, stars, w, h, a, a_w)

    desc = G.dusk_12800(rect)
    got, sizes, ginfo = G.game_sky_maps(ctx, desc, G.DUSK_SKY_LIGHT_FACTOR, G.DUSK_SKY_LIGHT_COLOR, pix, aw)
    want, _, winfo = G.game_sky_maps(OracleDraw(), desc, G.DUSK_SKY_LIGHT_FACTOR, G.DUSK_SKY_LIGHT_COLOR, pix, aw)
    assert np.allclose(ginfo["scale"], winfo["scale"], rtol=1e-5)
    assert np.allclose(ginfo["veil"], winfo["veil"], rtol=1e-5, atol=1e-7)
    n = G.LENS_MAP[0] * G.LENS_MAP[1] * 3
    light_ok = close(got[n:], want[n:])
    assert light_ok.all(), np.abs(got[n:] - want[n:]).max()


def test_a_sprite_outside_the_atlas_is_refused(ctx, atlas):
    from lumenwright_b200.native import LwError
    pix, aw, _ = atlas
    desc = G.dusk_12800((aw - 8, 0, 32, 32))  # reaches past the atlas's right edge
    with pytest.raises(LwError) as e:
        ctx.draw_sky_map(G.quick_sky(desc), G.star_table(), 64, 32, pix, aw)
    assert e.value.status == 2
    with pytest.raises(LwError):
        ctx.draw_sky_map(G.quick_sky(desc), G.star_table()[:100], 64, 32, pix, aw)
