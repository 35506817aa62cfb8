"""The hq grid build on the device against the host build (`hqbuild.build_hq`, itself checked
word for word against a plain restatement of voxel.rs): the grid, models, quads, emitters and
emitter grid equal word for word on worlds with and without emitters, and a frame rendered on the
device-built scene equals the one rendered on the uploaded host build, bit for bit."""

import numpy as np
import pytest

from lumenwright_b200 import request as R
from lumenwright_b200 import synth as S
from lumenwright_b200.devbuild import build_hq_device
from lumenwright_b200.hqbuild import build_hq

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from lumenwright_b200.native import Context
    c = Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("chunks,emitters", [(2, True), (4, False), (12, True)])
def test_device_build_matches_the_host_build(ctx, chunks, emitters):
    world = S.generate_world(chunks, 1, emitters=emitters)
    atlas = S.build_atlas(1)
    want = build_hq(world, atlas)
    d = build_hq_device(ctx, world, atlas)
    got = d.read(ctx)
    assert got.dims == tuple(want.dims) and tuple(got.offsets) == tuple(want.offsets)
    assert np.array_equal(got.grid, want.grid)
    assert got.models.tobytes() == want.models.tobytes()
    assert got.quads.tobytes() == want.quads.tobytes()
    assert got.emitter_count == want.emitter_count
    assert got.emitters.tobytes() == want.emitters.tobytes()
    assert np.array_equal(got.emitter_grid, want.emitter_grid)
    assert tuple(got.see_through) == tuple(want.see_through)
    s, t = got.stats, want.stats
    assert (s.bricks, s.uniform_bricks, s.buried_bricks, s.instances, s.emitters) == \
        (t.bricks, t.uniform_bricks, t.buried_bricks, t.instances, t.emitters)


def test_render_on_the_device_built_scene(ctx):
    cfg = R.CONFIGS["c1"]
    frame = R.make_frame(cfg, sky_backend=ctx, width=96, height=54, spp=8)
    ctx.upload_hq_scene(frame.scene)
    want = ctx.render_hq(frame.params, frame.sky, 8)
    build_hq_device(ctx, S.generate_world(cfg.chunks, cfg.seed, emitters=cfg.emitters), S.build_atlas(cfg.seed))
    got = ctx.render_hq(frame.params, frame.sky, 8)
    assert np.array_equal(got, want)
