"""The benchmark's comparison baseline (baseline/refport: the reference's CUDA backend ported as
written, in its own library): on the C1 frame its image equals `lw_render_hq`'s within 1e-4
relative per pixel (the same per-sample arithmetic; f32 sums against Kahan sums), its launches
follow CudaBackend::render_hq's batch schedule (1, 2, 4, ... spp per launch), and the L2 read
probe returns a bandwidth."""

import numpy as np
import pytest

from lumenwright_b200 import request as R

pytestmark = pytest.mark.gpu


def test_reference_port_matches_the_product_on_c1():
    from baseline.refport import port as RP
    from lumenwright_b200.native import B200Backend
    be = B200Backend(0)
    frame = R.make_frame(R.CONFIGS["c1"], sky_backend=be.ctx)
    want = be.render_hq(frame).reshape(144, 256, 3)
    got, t = RP.render_hq(0, frame)
    ok = np.abs(got - want) <= 1e-4 * np.maximum(np.abs(got), np.abs(want)) + 1e-6
    print(f"reference port: {ok.mean():.6f} of pixels within 1e-4, {t['launches']} launches, "
          f"{t['kernel_ms']:.1f} ms of kernels, {t['total_ms']:.1f} ms in all")
    assert ok.all()
    assert 1 <= t["launches"] <= frame.spp and t["kernel_ms"] > 0.0 and t["total_ms"] >= t["kernel_ms"]


def test_l2_read_probe():
    from baseline.refport import port as RP
    gbs = RP.l2_read_gbs(0)
    print(f"L2 read: {gbs:.0f} GB/s")
    assert gbs > 1000.0
