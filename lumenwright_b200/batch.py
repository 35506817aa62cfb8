"""The batched form's workload and its autotuner.

``c3_jobs`` builds the 64 seeded cameras of the batching configuration over the 12x12-chunk
world: resolutions drawn uniformly from 320x180 to 1920x1080 (16:9), spp from {16, 64, 256, 1024},
4 to 8 bounces, times of day 4000 (Chunky's sky) or 12800 (the game sky at dusk). ``Autotuner``
picks the launch tuning (engine, queue depth, visits between queue fetches or regrouping period,
threads per block, samples per work item) by timing short trial batches, and keeps the winner per
workload class in a JSON cache.
"""

import hashlib
import json
import math
import os
from dataclasses import dataclass

import numpy as np

from . import gamesky as G
from . import request as R
from . import sky as SK
from . import synth as S
from .hqbuild import build_hq

F32 = np.float32


@dataclass
class Camera3:
    eye: tuple
    target: tuple
    width: int
    height: int
    spp: int
    bounces: int
    time: int


def c3_cameras(n=64, seed=3, chunks=12, world_seed=1):
    """The batching configuration's cameras: seeded positions above the terrain of the world,
    looking at seeded points on it."""
    rng = np.random.default_rng(seed)
    size = chunks * 16
    h = S.heightmap(size, size, world_seed)
    cams = []
    for _ in range(n):
        w = int(rng.integers(320, 1921)) // 16 * 16
        w = max(320, min(1920, w))
        hh = w * 9 // 16
        ex, ez = rng.uniform(16, size - 16, 2)
        ey = float(max(h[int(ez), int(ex)], 63) + rng.uniform(8, 40))
        tx, tz = rng.uniform(0, size, 2)
        ty = float(max(h[int(tz) % size, int(tx) % size], 63))
        cams.append(Camera3((float(ex), ey, float(ez)), (float(tx), ty, float(tz)), w, hh,
                            int(rng.choice([16, 64, 256, 1024])), int(rng.integers(4, 9)),
                            int(rng.choice([4000, 12800]))))
    return cams


def c3_jobs(sky_backend, cams=None, spp_scale=1.0):
    """(scene, jobs): the world's HqScene and, per camera, (params, sky, spp). The two times of day
    share their sky buffers."""
    cams = cams or c3_cameras()
    cfg = R.CONFIGS["c2"]
    world = S.generate_world(cfg.chunks, cfg.seed, emitters=True)
    atlas = S.build_atlas(cfg.seed)
    hq = build_hq(world, atlas)
    origin = world.origin
    skies = {}
    jobs = []
    for c in cams:
        yaw, pitch = R.Camera.look_at(c.eye, c.target)
        cam = R.Camera(c.eye, float(yaw), float(pitch), 70.0)
        eye = [F32(c.eye[i] - origin[i]) for i in range(3)]
        sun_dir = SK.sun_direction_from_angle(SK.celestial_angle(c.time))
        weight = F32(1.0) if c.time == 4000 else SK.dusk_day_weight(c.time)
        intensity = SK.default_emitter_intensity(False, weight)
        p = R.hq_params(c.width, c.height, hq, eye, cam, SK.hq_sky(sun_dir), max_bounces=c.bounces,
                        emitter_intensity=intensity)
        p["water_plane"] = [F32(R.water_plane_height(63.0) - origin[1]), 1.0, 0.0, 0.0]
        if c.time not in skies:
            cache = sky_backend.build_sky_cache(p, int(p["misc_f"][2]))
            if weight >= 1.0:
                skies[c.time] = (cache, None)
            else:
                desc, factor, colour = G.stated_sky(c.time, hq.sun_sprite)
                maps, sizes, _ = G.game_sky_maps(sky_backend, desc, factor, colour, hq.atlas, hq.atlas_size[0])
                maps = sky_backend.blend_chunky_sky(p, cache, maps, sizes, weight)
                skies[c.time] = (maps, sizes)
        sky, sizes = skies[c.time]
        if sizes is not None:
            p["sun_color"][:3] = p["sun_color"][:3] * weight
            p["sun_su"][3] = p["sun_su"][3] * weight
            p["sky_map"] = sizes
            p["misc_f"][2] = 0.0
        spp = max(1, int(round(c.spp * spp_scale)))
        jobs.append((p, sky, spp))
    return hq, jobs


class Autotuner:
    """Picks the batched render's launch tuning for a workload by timing trial renders.

    Candidates: the wavefront engine with queue depth (path slots) {automatic, 2^22, 2^23, 2^24} x visits
    between queue fetches {4, 8}, and the persistent megakernel with threads per block {64, 128,
    256} x regrouping period {0 (whole traversals), 24}; each with samples per work item
    {automatic, 4}. A trial renders the workload with every camera's spp cut to
    ``trial_fraction`` of it (at least 1). The winner is cached per workload class (the rounded
    totals of pixels and samples and the bounce range) in ``$LUMENWRIGHT_CACHE/autotune.json``
    (default ``~/.cache/lumenwright_b200``)."""

    SUBS = (0, 4)

    @classmethod
    def candidates(cls):
        out = []
        for sub in cls.SUBS:
            for paths in (0, 1 << 22, 1 << 23, 1 << 24):
                for budget in (4, 8):
                    out.append({"engine": 0, "threads": 128, "budget": budget, "sub": sub, "paths": paths})
            for threads in (128, 64, 256):
                for budget in (0, 24):
                    out.append({"engine": 1, "threads": threads, "budget": budget, "sub": sub, "paths": 0})
        return out

    def __init__(self, ctx, cache_dir=None, trial_fraction=1 / 32):
        self.ctx = ctx
        self.trial_fraction = trial_fraction
        d = cache_dir or os.environ.get("LUMENWRIGHT_CACHE") or os.path.join(os.path.expanduser("~"), ".cache",
                                                                              "lumenwright_b200")
        self.path = os.path.join(d, "autotune.json")

    @staticmethod
    def workload_class(jobs):
        px = sum(int(p["frame"][0]) * int(p["frame"][1]) for p, _, _ in jobs)
        samples = sum(int(p["frame"][0]) * int(p["frame"][1]) * spp for p, _, spp in jobs)
        b = sorted({int(p["frame"][3]) for p, _, _ in jobs})
        key = f"n{len(jobs)}-px{round(math.log2(px), 1)}-s{round(math.log2(samples), 1)}-b{b[0]}-{b[-1]}"
        return hashlib.sha1(key.encode()).hexdigest()[:16], key

    def _load(self):
        try:
            with open(self.path) as f:
                return json.load(f)
        except Exception:
            return {}

    def _store(self, table):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        with open(self.path, "w") as f:
            json.dump(table, f, indent=1)

    def tune(self, jobs, force=False):
        """Sets and returns the best tuning for ``jobs`` (a list of (params, sky, spp))."""
        h, key = self.workload_class(jobs)
        table = self._load()
        if not force and h in table and set(table[h]["tuning"]) == set(self.candidates()[0]):
            t = table[h]["tuning"]
            self.ctx.set_tuning(**t)
            return t, table[h]
        trial = [(p, sky, max(1, int(round(spp * self.trial_fraction)))) for p, sky, spp in jobs]
        results = []
        for t in self.candidates():
            self.ctx.set_tuning(**t)
            self.ctx.batch_prepare(trial)
            self.ctx.batch_run()  # warm
            self.ctx.stats()
            self.ctx.batch_run()
            ms = self.ctx.stats()["kernel_ms"]
            results.append((t, ms))
        best = min(results, key=lambda r: r[1])
        entry = {"key": key, "tuning": best[0], "trial_ms": best[1],
                 "trials": [{"tuning": t, "ms": ms} for t, ms in results]}
        table[h] = entry
        self._store(table)
        self.ctx.set_tuning(**best[0])
        return best[0], entry
