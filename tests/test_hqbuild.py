"""The product's grid build (`lumenwright_b200.hqbuild`) against the plain restatement of
`voxel::build_hq` (oracle/build_hq_ref.py), word for word, and the reference's emitter-grid
property (crates/lumenwright/src/scene/voxel.rs:617-671). CPU only."""

import numpy as np
import pytest

from lumenwright_b200 import hqbuild as H
from lumenwright_b200 import layout as L
from lumenwright_b200 import synth as S
from oracle import oracle as O
from oracle.build_hq_ref import build_hq_ref, emitter_list_ref


@pytest.mark.parametrize("seed,emitters", [(1, True), (5, True), (9, False)])
def test_grid_build_is_word_for_word(seed, emitters):
    world = S.generate_world(2, seed, emitters=emitters, emitter_per_solid=300)
    atlas = S.build_atlas(seed)
    got = H.build_hq(world, atlas)
    want = build_hq_ref(world, atlas)
    assert tuple(got.offsets) == tuple(want["offsets"])
    assert np.array_equal(got.grid, want["grid"])
    assert [tuple(r) for r in got.models[["quad_offset", "quad_count"]].tolist()] == want["models"]
    assert np.array_equal(L.quad_words(got.quads), np.stack(want["quads"]))
    assert np.array_equal(got.emitter_grid, want["emitter_grid"])
    ew = got.emitters.view("<u4").reshape(-1, 8)
    if want["emitters"]:
        assert got.emitter_count == len(want["emitters"])
        for i, (c, fq, faces) in enumerate(want["emitters"]):
            assert np.array_equal(ew[i, 0:3].view("<f4"), np.array(c, np.float32))
            assert ew[i, 3] == fq and ew[i, 4] == faces
    assert got.stats.bricks + got.stats.uniform_bricks + got.stats.buried_bricks > 0


def test_every_voxel_reads_back_its_model():
    """SceneView::voxel over the built grid gives each voxel's instance (its state's quads)."""
    world = S.generate_world(2, 3, emitters=True, emitter_per_solid=300)
    atlas = S.build_atlas(3)
    hq = H.build_hq(world, atlas)
    p = L.new_params()
    p["grid_dims"] = [hq.dims[0], hq.dims[1], hq.dims[2], 0]
    p["off"] = list(hq.offsets[:4])
    v = O.OracleScene(p, hq.grid, hq.models, hq.quads, hq.atlas, hq.emitters, hq.emitter_grid)
    rng = np.random.default_rng(0)
    Y, Z, X = world.blocks.shape
    for _ in range(3000):
        x, y, z = int(rng.integers(X)), int(rng.integers(Y)), int(rng.integers(Z))
        m = v.voxel(x, y, z)
        sid = int(world.blocks[y, z, x])
        if sid == S.AIR:
            assert m == 0
        else:
            assert m != 0
            # Water inside water (every face hidden) is an instance with no quads.
            assert hq.models[m]["quad_count"] > 0 or sid == S.WATER


def test_the_emitter_grid_lists_every_emitter_within_a_cell():  # voxel.rs:617-671
    models = np.zeros(2, L.MODEL_DTYPE)
    models[1]["quad_offset"] = 3
    models[1]["quad_count"] = 2
    sites = [((25, 3, 0), 1), ((4, 40, 17), 1), ((26, 3, 1), 1)]
    emitters, grid = H.emitter_list(models, sites)
    assert emitters.size == 3
    ew = emitters.view("<u4").reshape(-1, 8)
    assert list(ew[1, 0:3].view("<f4")) == [4.0, 40.0, 17.0] and ew[1, 3] == 3 and ew[1, 4] == 2
    _, want = emitter_list_ref([(0, 0), (3, 2)], sites)
    assert np.array_equal(grid, np.array(want, np.uint32))
    v = O.OracleScene(L.new_params(), None, None, None, None, emitters, grid)
    cells = int(grid[1]) * int(grid[2]) * int(grid[3])
    lst = grid[L.EMITTER_GRID_HEADER + cells * 2:]
    checked = 0
    for x in range(-5, 50):
        for y in range(-5, 60):
            for z in range(-5, 40):
                start, count = v.emitter_cell((x + 0.5, y + 0.5, z + 0.5))
                found = set(lst[start:start + count].tolist())
                for i, (c, _) in enumerate(sites):
                    d = [abs(x - c[0]), abs(y - c[1]), abs(z - c[2])]
                    if all(a < H.EMITTER_CELL for a in d):
                        assert i in found, (i, x, y, z)
                    if any(a >= 2 * H.EMITTER_CELL for a in d):
                        assert i not in found, (i, x, y, z)
                    checked += 1
    assert checked == 55 * 65 * 45 * 3
