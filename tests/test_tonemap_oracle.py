"""The oracle's restatement of the display pass (`post::tonemap`, `post::tonemap_mix`,
crates/lumenwright/src/render/post.rs:152-217) against the reference's own tests of it
(post.rs:253-310): the end points, mid-grey under the gamma filter, the game curve's gain and
parameters, the preset's mid-grey byte, white under both curves, and the mix at its ends."""

import numpy as np

from oracle import oracle as O

GAMMA, ACES, FILMIC, MID = 0, 1, 2, 3


def byte0(px):
    return int(px[0]) & 0xFF


def test_tonemap_endpoints():  # post.rs:257-266
    px = O.tonemap([[0.0] * 3, [1.0] * 3, [100.0] * 3], 1.0, GAMMA)
    assert px[0] == 0xFF000000 and px[1] == 0xFFFFFFFF and px[2] == 0xFFFFFFFF
    a = byte0(O.tonemap([[0.18] * 3], 1.0, ACES))
    assert 100 < a < 200
    assert byte0(O.tonemap([[0.18] * 3], 1.0, GAMMA)) == 117


def test_the_game_tone_curve_shows_mid_grey_as_the_game():  # post.rs:271-299
    k = O.lib().lwo_mid_grey_gain()
    assert abs(k - 1.463761) < 1e-6
    g = O.game_tone_curve()
    assert list(g) == list(np.array([0.32138956, 0.7318806, 0.1, 0.2, 0.02, 0.3, 7.651521], np.float32))
    assert abs(O.lib().lwo_game_before_gamma(0.18) - 0.18) < 1e-6
    assert byte0(O.tonemap([[0.18] * 3], 1.0, MID)) == byte0(O.tonemap([[0.18] * 3], 1.0, GAMMA))
    assert byte0(O.tonemap([[0.18] * 3], 1.0, FILMIC)) == int(np.float32(0.393285) * np.float32(255.0) + np.float32(0.5))
    assert O.tonemap([[g[6]] * 3], 1.0, MID)[0] == 0xFFFFFFFF


def test_the_tone_mix_is_each_curve_at_its_ends():  # post.rs:303-317
    hdr = np.array([[i * 0.05] * 3 for i in range(64)], np.float32)
    a, b = O.tonemap(hdr, 1.0, GAMMA), O.tonemap(hdr, 1.0, MID)
    assert np.array_equal(O.tonemap(hdr, 1.0, GAMMA, 1, MID, 1.0), a)
    assert np.array_equal(O.tonemap(hdr, 1.0, GAMMA, 1, MID, 0.0), b)
    m = O.tonemap(hdr, 1.0, GAMMA, 1, MID, 0.5)
    x, y, z = a & 0xFF, b & 0xFF, m & 0xFF
    assert np.all((z + 1 >= np.minimum(x, y)) & (z <= np.maximum(x, y) + 1))
