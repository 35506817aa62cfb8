"""The allocation-free entry point (`lw_render_accumulate_noalloc`), for callers that must not
allocate device memory while they render (an application that owns the GPU's memory, a per-frame
loop that must not stall on cudaMalloc): called through the C ABI into a device buffer the test
owns, twice in a row, on a context that has had only its scene and sky uploaded (no render has
allocated its buffers), and checked against `lw_render_hq`'s image from a second context within
the per-pixel tolerance of the other render tests (1e-4 relative). The device's free memory is
the same before and after the calls that follow the first. Collected last on purpose (the file
name), so a run that stops at the first failure has run every other test first."""

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

    ref = Context(0)
    frame = R.make_frame(R.CONFIGS["c1"], sky_backend=ref)
    p = frame.params
    w, h = int(p["frame"][0]), int(p["frame"][1])
    ref.upload_hq_scene(frame.scene)
    want16 = ref.render_hq(p, frame.sky, 16).reshape(-1, 3)
    want32 = ref.render_hq(p, frame.sky, 32).reshape(-1, 3)
    want48 = ref.render_hq(p, frame.sky, 48).reshape(-1, 3)
    ref.close()

    # A fresh context: only the set-up calls (which allocate) before the allocation-free ones.
    ctx = Context(0)
    ctx.upload_hq_scene(frame.scene)
    ctx.upload_sky(frame.sky)

    # The caller's own accumulator: w*h records of 8 floats, zeroed before the first call.
    acc = torch.zeros(w * h * 8, dtype=torch.float32, device="cuda:0")
    torch.cuda.synchronize()
    ctx.render_accumulate_noalloc(p, 0, 16, acc.data_ptr())  # first call: samples 0..16
    torch.cuda.synchronize()
    got16 = mean_of(acc.cpu().numpy())
    free_before = torch.cuda.mem_get_info(0)[0]
    ctx.render_accumulate_noalloc(p, 16, 16, acc.data_ptr())  # second call: samples 16..32 added
    torch.cuda.synchronize()
    got32 = mean_of(acc.cpu().numpy())
    ctx.render_accumulate_noalloc(p, 32, 16, acc.data_ptr())  # a third: samples 32..48
    torch.cuda.synchronize()
    free_after = torch.cuda.mem_get_info(0)[0]
    got48 = mean_of(acc.cpu().numpy())

    assert np.all(close(got16, want16)), np.abs(got16 - want16).max()
    assert np.all(close(got32, want32)), np.abs(got32 - want32).max()
    assert np.all(close(got48, want48)), np.abs(got48 - want48).max()
    assert free_after == free_before, (free_before, free_after)

    # A frame larger than the fixed scratch array is refused, not rendered; so is a host pointer
    # in place of the device accumulator.
    big = p.copy()
    big["frame"] = [4096, 4096, 0, 4]
    with pytest.raises(LwError) as e:
        ctx.render_accumulate_noalloc(big, 0, 1, acc.data_ptr())
    assert e.value.status == 1
    host = np.zeros(w * h * 8, np.float32)
    with pytest.raises(LwError) as e:
        ctx.render_accumulate_noalloc(p, 0, 1, host.ctypes.data)
    assert e.value.status == 1
    ctx.close()
