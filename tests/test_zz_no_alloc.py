"""The allocation-free entry point (`lw_render_accumulate_noalloc`), for callers that must not
allocate device memory while they render (an application that owns the GPU's memory, a per-frame
loop that must not stall on cudaMalloc): called through the C ABI into a device buffer the test
owns, twice in a row, and checked against `lw_render_hq`'s image within the per-pixel tolerance of
the other render tests (1e-4 relative). Collected last on purpose (the file name), so a run that
stops at the first failure has run every other test first."""

import numpy as np
import pytest

from lumenwright_b200 import request as R

pytestmark = pytest.mark.gpu


def mean_of(acc):
    a = acc.reshape(-1, 8).astype(np.float64)
    cnt = np.maximum(a[:, 3], 1.0)
    return ((a[:, 0:3] - a[:, 4:7]) / cnt[:, None]).astype(np.float32)


def close(a, b):
    return np.abs(a - b) <= 1e-4 * np.maximum(np.abs(a), np.abs(b)) + 1e-6


def test_no_alloc_render_matches_render_hq_on_two_calls():
    import torch

    from lumenwright_b200.native import Context, LwError

    ctx = Context(0)
    frame = R.make_frame(R.CONFIGS["c1"], sky_backend=ctx)
    p = frame.params
    w, h = int(p["frame"][0]), int(p["frame"][1])
    ctx.upload_hq_scene(frame.scene)
    want16 = ctx.render_hq(p, frame.sky, 16).reshape(-1, 3)
    want32 = ctx.render_hq(p, frame.sky, 32).reshape(-1, 3)
    ctx.upload_sky(frame.sky)

    # The caller's own accumulator: w*h records of 8 floats, zeroed before the first call.
    acc = torch.zeros(w * h * 8, dtype=torch.float32, device="cuda:0")
    ctx.render_accumulate_noalloc(p, 0, 16, acc.data_ptr())  # first call: samples 0..16
    torch.cuda.synchronize()
    got16 = mean_of(acc.cpu().numpy())
    ctx.render_accumulate_noalloc(p, 16, 16, acc.data_ptr())  # second call: samples 16..32 added
    torch.cuda.synchronize()
    got32 = mean_of(acc.cpu().numpy())

    assert np.all(close(got16, want16)), np.abs(got16 - want16).max()
    assert np.all(close(got32, want32)), np.abs(got32 - want32).max()

    # A frame larger than the fixed scratch array is refused, not rendered.
    big = p.copy()
    big["frame"] = [4096, 4096, 0, 4]
    with pytest.raises(LwError) as e:
        ctx.render_accumulate_noalloc(big, 0, 1, acc.data_ptr())
    assert e.value.status == 1
    ctx.close()
