"""The seeded synthetic worlds that stand in for the reference's benchmark saves: the generator in
`lumenwright_b200/synth.py` keeps the terrain, water, tree and emitter rules of the benchmark
configurations (value-noise heights 64 + 24 n, stone / 3 dirt / grass, water up to y = 63, oak
trees with 4-6 block trunks, one lantern or glowstone per 2000 solid blocks on the land surface),
and the same seed gives the same world. CPU only."""

import numpy as np

from lumenwright_b200 import synth as S


def test_the_same_seed_gives_the_same_world():
    a = S.generate_world(2, seed=3, emitters=True)
    b = S.generate_world(2, seed=3, emitters=True)
    c = S.generate_world(2, seed=4, emitters=True)
    assert np.array_equal(a.blocks, b.blocks)
    assert not np.array_equal(a.blocks, c.blocks)


def test_heights_follow_the_value_noise():
    h = S.heightmap(96, 96, seed=1)
    assert h.min() >= 64 - 24 and h.max() <= 64 + 24
    assert h.max() - h.min() > 8  # the noise varies over a few lattice cells (pitch 32)
    # lattice points carry the hashed value exactly: smoothstep weights are 0 / 1 there
    lat = S.hash3(np.array([1]), np.array([2]), 1).astype(np.float64) / 4294967295.0 * 2.0 - 1.0
    assert h[2 * 32, 1 * 32] == int(np.floor(64 + 24 * lat[0]))


def test_columns_are_layered_and_flooded_to_sea_level():
    w = S.generate_world(2, seed=1)
    h = S.heightmap(32, 32, seed=1)
    b = w.blocks
    for z in range(0, 32, 3):
        for x in range(0, 32, 3):
            top = int(h[z, x])
            col = b[:, z, x]
            at = lambda y: int(col[y - w.min_y])  # noqa: E731
            assert at(top - 4) == S.STONE and at(w.min_y) == S.STONE
            assert all(at(y) == S.DIRT for y in range(top - 3, top))
            if top < 63:
                assert at(top) == S.DIRT and all(at(y) == S.WATER for y in range(top + 1, 64))
                assert at(64) == S.AIR
            else:
                assert at(top) == S.GRASS


def test_trees_and_emitters_stand_on_the_land():
    w = S.generate_world(4, seed=1, emitters=True)
    b = w.blocks
    h = S.heightmap(64, 64, seed=1)
    assert w.emitters_placed == max(1, w.solid_blocks // 2000)
    ys, zs, xs = np.nonzero((b == S.LANTERN) | (b == S.GLOWSTONE))
    assert len(ys) == w.emitters_placed
    for y, z, x in zip(ys, zs, xs):
        assert h[z, x] >= 63 and y + w.min_y == h[z, x] + 1
    logs = np.argwhere(b == S.LOG)
    assert len(logs)
    for z, x in {(int(z), int(x)) for _, z, x in logs}:
        trunk = np.nonzero(b[:, z, x] == S.LOG)[0] + w.min_y
        assert trunk.min() == h[z, x] + 1 and 4 <= len(trunk) <= 6
