"""Cancelling a render on the GPU (`lw_cancel`): the cancelled call reports it, and the next
render on the context is whole. Kept in a file collected after the other render tests."""

import numpy as np
import pytest

from lumenwright_b200 import request as R

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from lumenwright_b200.native import Context
    c = Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def c1(ctx):
    return R.make_frame(R.CONFIGS["c1"], sky_backend=ctx)


def test_a_cancelled_render_reports_it_and_the_next_one_is_whole(ctx, c1):
    # lw_cancel from the progress callback (the calling thread, between launches): the render
    # returns LW_ERR_CANCELLED. The cancel's write to the device word lands before the next render
    # clears it, so the next render is the whole frame, bit for bit an uncancelled render's.
    from lumenwright_b200.native import LwError
    p = c1.params
    ctx.upload_hq_scene(c1.scene)
    want = ctx.render_hq(p, c1.sky, 4)
    with pytest.raises(LwError) as e:
        ctx.render_hq(p, c1.sky, 4, progress=lambda done, total: ctx.cancel())
    assert e.value.status == 6  # LW_ERR_CANCELLED
    got = ctx.render_hq(p, c1.sky, 4)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
