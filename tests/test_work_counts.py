"""The algorithmic work per path sample of the drop-in workload (c2), counted by the instrumented
FP32 oracle on 24 full rows spread over the frame at 1 spp, and the byte sizes per access that the
benchmark's roofline uses. The committed counts (profiles/algorithmic_bytes_c2.json, which
bench.py reads) must be what the oracle counts now; LW_WRITE_COUNTS=1 rewrites them.

Bytes per access: 8 B per DDA step (top + overlay entry), 2 B per non-uniform voxel id, 16 B per
model, 80 B per quad test, 4 B per texel, 8 B per overlay cell read (the tracing kernel's); 48 B
per sky-cache read, 96 B per map read (4 corners x 3 f32 x 2 rows), 8 B per emitter cell, 4 B per
emitter index, 32 B per emitter, 16 B per accumulated sample (the shading side's).

The same accesses rounded up to the 32-byte sectors that L2 and DRAM move: a DDA step's two words
lie in two regions (2 sectors), a voxel id, a model, a texel, an overlay cell, an emitter cell, an
index and an emitter are one sector each, an 80-byte quad record on a 16-byte boundary spans 3, a
sky-cache or map read's two runs of 24 bytes up to 2 each (4), an accumulated sample one."""

import json
import os

import numpy as np

from lumenwright_b200 import request as R
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PATH = os.path.join(ROOT, "profiles", "algorithmic_bytes_c2.json")
TRACE = {"dda_steps": 8, "voxel_lookups": 2, "model_fetches": 16, "quad_tests": 80, "texel_fetches": 4,
         "overlay_reads": 8}
SHADE = {"sky_reads": 48, "map_reads": 96, "emitter_cell_reads": 8, "emitter_index_reads": 4, "emitter_reads": 32}
TRACE_SECTORS = {"dda_steps": 64, "voxel_lookups": 32, "model_fetches": 32, "quad_tests": 96, "texel_fetches": 32,
                 "overlay_reads": 32}
SHADE_SECTORS = {"sky_reads": 128, "map_reads": 128, "emitter_cell_reads": 32, "emitter_index_reads": 32,
                 "emitter_reads": 32}


class OracleSky:
    """Sky inputs through the oracle (the counts do not depend on the sky's values: no decision
    along a path reads them)."""

    def build_sky_cache(self, params, n):
        return O.OracleScene(params, None, None, None, None, None, None).build_sky_cache(n)

    def blend_chunky_sky(self, params, cache, maps, sizes, weight):
        return maps

    def draw_sky_map(self, quick_sky, stars, w, h, atlas, atlas_w):
        return np.full((h, w, 3), 0.1, np.float32)


def count_c2():
    cfg = R.CONFIGS["c2"]
    frame = R.make_frame(cfg, sky_backend=OracleSky(), spp=1)
    v = O.OracleScene.from_frame(frame)
    w, h = int(frame.params["frame"][0]), int(frame.params["frame"][1])
    total = None
    for y in np.linspace(0, h - 1, 24).astype(int):
        c = v.count_work(0, int(y), w, 1, 1)
        total = c if total is None else {k: total[k] + c[k] for k in c}
    n = total["samples"]
    per = {k: total[k] / n for k in total}
    trace_b = sum(b * per[k] for k, b in TRACE.items())
    shade_b = sum(b * per[k] for k, b in SHADE.items()) + 16.0
    trace_s = sum(b * per[k] for k, b in TRACE_SECTORS.items())
    shade_s = sum(b * per[k] for k, b in SHADE_SECTORS.items()) + 32.0
    return {"workload": "c2", "command": "LW_WRITE_COUNTS=1 python -m pytest tests/test_work_counts.py -q",
            "sampled": n, "counts_per_sample": per, "trace_bytes_per_sample": trace_b,
            "shade_bytes_per_sample": shade_b, "bytes_per_sample": trace_b + shade_b,
            "bytes_per_access": {**TRACE, **SHADE, "accumulate": 16},
            "trace_sector_bytes_per_sample": trace_s, "shade_sector_bytes_per_sample": shade_s,
            "sector_bytes_per_sample": trace_s + shade_s,
            "sector_bytes_per_access": {**TRACE_SECTORS, **SHADE_SECTORS, "accumulate": 32}}


def test_committed_counts_are_current():
    got = count_c2()
    if os.environ.get("LW_WRITE_COUNTS") == "1":
        with open(PATH, "w") as f:
            json.dump(got, f, indent=1)
    with open(PATH) as f:
        want = json.load(f)
    assert want["sampled"] == got["sampled"]
    for k, v in got["counts_per_sample"].items():
        assert abs(want["counts_per_sample"][k] - v) <= 1e-9 * max(1.0, abs(v)), k
    assert abs(want["bytes_per_sample"] - got["bytes_per_sample"]) <= 1e-9 * got["bytes_per_sample"]
    assert abs(want["sector_bytes_per_sample"] - got["sector_bytes_per_sample"]) <= 1e-9 * got["sector_bytes_per_sample"]
    assert O.bounds_errors() == 0
