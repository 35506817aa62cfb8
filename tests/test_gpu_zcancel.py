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


def test_a_cancel_leaves_whole_launches_in_the_accumulator(ctx, c1):
    # lw_cancel right after an allocation-free render was queued (it returns before its kernels
    # run), while the render's kernels run: a launch the cancel reaches adds nothing, so every
    # pixel's record holds the whole launches done before it (none, usually), and its mean is the
    # mean of that many samples. The next call adds its samples in full.
    import torch
    p = c1.params
    w, h = int(p["frame"][0]), int(p["frame"][1])
    ctx.upload_hq_scene(c1.scene)
    ctx.upload_sky(c1.sky)
    spp = 2048
    acc = torch.zeros(w * h * 8, dtype=torch.float32, device="cuda:0")
    torch.cuda.synchronize()
    ctx.render_accumulate_noalloc(p, 0, spp, acc.data_ptr())
    ctx.cancel()
    torch.cuda.synchronize()
    a = acc.cpu().numpy().reshape(-1, 8).astype(np.float64)
    counts = np.unique(a[:, 3])
    print(f"sample counts per pixel after the cancel: {counts.tolist()}")
    for cnt in counts:
        sel = a[:, 3] == cnt
        if cnt == 0:
            assert not a[sel].any()  # untouched records
            continue
        assert cnt <= spp
        want = ctx.render_hq(p, c1.sky, int(cnt)).reshape(-1, 3)[sel]
        got = (a[sel, 0:3] - a[sel, 4:7]) / cnt
        assert np.all(np.abs(got - want) <= 1e-4 * np.maximum(np.abs(got), np.abs(want)) + 1e-6)
    # uncancelled again: 16 more samples in every record
    ctx.upload_sky(c1.sky)
    before = acc.cpu().numpy().reshape(-1, 8)[:, 3].copy()
    ctx.render_accumulate_noalloc(p, 0, 16, acc.data_ptr())
    torch.cuda.synchronize()
    after = acc.cpu().numpy().reshape(-1, 8)[:, 3]
    assert np.array_equal(after, before + 16)


def test_a_wait_past_its_deadline_returns_a_timeout_and_the_next_render_is_whole(ctx, c1):
    # A deadline far shorter than an ordinary C1 render at 256 spp: the call's wait runs out, the
    # render's kernels are stopped (no kernel is made to hang: they are cancelled as lw_cancel
    # cancels them) and the call returns LW_ERR_DEVICE_TIMEOUT; without the deadline the next
    # render of the frame is bit for bit an uninterrupted one.
    import time

    from lumenwright_b200.native import LwError
    p = c1.params
    ctx.upload_hq_scene(c1.scene)
    want = ctx.render_hq(p, c1.sky, 256)
    ctx.set_timeout(1e-4)
    t0 = time.perf_counter()
    with pytest.raises(LwError) as e:
        ctx.render_hq(p, c1.sky, 256)
    took = time.perf_counter() - t0
    assert e.value.status == 4, e.value  # LW_ERR_DEVICE_TIMEOUT
    assert "stopped" in str(e.value)
    print(f"timed out and drained in {took * 1e3:.1f} ms: {e.value}")
    ctx.set_timeout(0.0)
    got = ctx.render_hq(p, c1.sky, 256)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    # a generous deadline changes nothing
    ctx.set_timeout(60.0)
    again = ctx.render_hq(p, c1.sky, 256)
    ctx.set_timeout(0.0)
    assert np.array_equal(again.view(np.uint32), want.view(np.uint32))
