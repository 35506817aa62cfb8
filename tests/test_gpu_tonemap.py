"""The display pass on the GPU against the oracle's restatement of `post::tonemap` /
`post::tonemap_mix` (crates/lumenwright/src/render/post.rs:152-217), which the CPU tests pin to the
reference's own tests: byte for byte on the reference's test inputs and on a rendered frame; on
a million random values at most 1 channel in 100,000 may differ, by one step (the display gamma
is evaluated in f64 and rounded on the device, by the platform's `powf` in the oracle as in the
reference, and the two can round a value at a byte boundary differently)."""

import numpy as np
import pytest

from lumenwright_b200 import request as R
from oracle import oracle as O

pytestmark = pytest.mark.gpu
CASES = [(1.0, 0, 0, 0, 1.0), (1.0, 1, 0, 0, 1.0), (1.0, 2, 0, 0, 1.0), (1.0, 3, 0, 0, 1.0), (0.7, 0, 1, 3, 0.182),
         (2.5, 0, 1, 3, 0.5), (1.0, 1, 1, 2, 0.0), (1.3, 3, 1, 0, 1.0)]


@pytest.fixture(scope="module")
def ctx():
    from lumenwright_b200.native import Context
    c = Context(0)
    yield c
    c.close()


def test_reference_test_inputs(ctx):
    hdr = np.array([[0.0] * 3, [1.0] * 3, [100.0] * 3, [0.18] * 3, [7.651521] * 3] +
                   [[i * 0.05] * 3 for i in range(64)], np.float32)
    for e, op, mix, op_b, wgt in CASES:
        assert np.array_equal(ctx.tonemap_rgba(hdr, e, op, mix, op_b, wgt), O.tonemap(hdr, e, op, mix, op_b, wgt))


def test_random_values(ctx):
    rng = np.random.default_rng(4)
    hdr = np.exp(rng.uniform(np.log(1e-5), np.log(1e3), (1 << 20, 3))).astype(np.float32)
    hdr[:64] = [[0.0] * 3, [-1.0] * 3, [np.inf] * 3, [np.nan] * 3] * 16
    for e, op, mix, op_b, wgt in CASES:
        got = ctx.tonemap_rgba(hdr, e, op, mix, op_b, wgt)
        want = O.tonemap(hdr, e, op, mix, op_b, wgt)
        g = got.view(np.uint8).reshape(-1, 4).astype(int)
        w = want.view(np.uint8).reshape(-1, 4).astype(int)
        d = np.abs(g - w)
        assert d.max() <= 1 and np.count_nonzero(d) <= 1e-5 * d.size, (op, mix, np.count_nonzero(d))


def test_fused_display_pass_of_a_render(ctx):
    frame = R.make_frame(R.CONFIGS["c1"], sky_backend=ctx)
    p = frame.params
    w, h = int(p["frame"][0]), int(p["frame"][1])
    ctx.upload_hq_scene(frame.scene)
    want_hdr = ctx.render_hq(p, frame.sky, frame.spp)
    # the reference's default for an hq frame: gamma and the game curve mixed by the day weight
    rgba, hdr = ctx.read_accumulator_rgba(w, h, 1.0, 0, 1, 3, 0.4, with_hdr=True)
    assert np.array_equal(hdr, want_hdr)
    assert np.array_equal(rgba.ravel(), O.tonemap(hdr.reshape(-1, 3), 1.0, 0, 1, 3, 0.4))
