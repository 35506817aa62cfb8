"""The hq grid build on the device (`voxel::build_hq`, crates/lumenwright/src/scene/voxel.rs:111-491),
host side: the block states' flags, and between the two device calls the models and quads of the
instances the device found (model generation depends on the assets, so it stays on the host, as
in the reference's phase 2, voxel.rs:274-343). The result is the context's resident scene; its
buffers are the host build's (`hqbuild.build_hq`) word for word."""

from dataclasses import dataclass, field
from typing import Optional, Tuple

import numpy as np

from . import layout as L
from . import synth as S
from .native import LwError  # noqa: F401  (raised by the calls below)
from .scene import HqScene, HqStats

STATE_OCCLUDES, STATE_INVISIBLE, STATE_FLUID = 1, 2, 4  # LW_STATE_*


def state_flags() -> np.ndarray:
    """LW_STATE_* bits per block state of the synthetic block set."""
    f = np.zeros(len(S.BLOCKS), np.uint8)
    for i, b in enumerate(S.BLOCKS):
        f[i] = (STATE_OCCLUDES if b.occludes else 0) | (STATE_INVISIBLE if b.invisible else 0) | \
               (STATE_FLUID if b.fluid else 0)
    return f


def instances(atlas: "S.Atlas", keys: np.ndarray):
    """(models, quads, model_emits) for the instance keys in interning order: model 0 is air, model
    i the instance of keys[i - 1]; quads laid out in that order, marked front-only except water's
    (voxel.rs:300-330)."""
    rows, quads, emits = [(0, 0)], [], [0]
    for k in keys.tolist():
        state, fm = k >> 8, k & 0xFF
        qs = S.block_quads(atlas, state, fm)
        off = len(quads)
        for q in qs:
            if not (int(q[3]) & L.FLAG_WATER):
                q = q.copy()
                q[3] |= L.FLAG_FRONT_ONLY
            quads.append(q)
        rows.append((off, len(qs)))
        emits.append(1 if (len(qs) > 0 and S.BLOCKS[state].emittance > 0.0) else 0)
    models = np.zeros(len(rows), L.MODEL_DTYPE)
    models["quad_offset"] = [r[0] for r in rows]
    models["quad_count"] = [r[1] for r in rows]
    quads_arr = L.quads_array(quads) if quads else L.quads_array([np.zeros(20, np.uint32)])
    return models, quads_arr, np.array(emits, np.uint8), len(quads)


@dataclass
class DeviceScene:
    """What a frame needs of a scene built on the device (the fields `hq_params` reads), and the
    host-side parts; ``read`` brings the device buffers back as an `HqScene`."""

    dims: Tuple[int, int, int]
    offsets: Tuple[int, int, int, int, int]
    atlas_size: Tuple[int, int]
    models: np.ndarray
    quads: np.ndarray
    atlas: np.ndarray
    see_through: Tuple[int, int]
    emitter_count: int
    sun_sprite: Optional[Tuple[int, int, int, int]]
    grid_len: int
    emitter_grid_len: int
    stats: HqStats = field(default_factory=HqStats)
    keys_ms: float = 0.0
    grid_ms: float = 0.0

    def read(self, ctx) -> HqScene:
        grid, em, eg = ctx.scene_read(self.grid_len, max(1, self.emitter_count), self.emitter_grid_len)
        return HqScene(grid=grid, models=self.models, quads=self.quads, atlas=self.atlas, atlas_size=self.atlas_size,
                       dims=self.dims, offsets=self.offsets, see_through=self.see_through, emitters=em,
                       emitter_count=self.emitter_count, emitter_grid=eg, sun_sprite=self.sun_sprite, stats=self.stats)


def build_hq_device(ctx, world: "S.World", atlas: "S.Atlas") -> DeviceScene:
    """`build_hq` for a synthetic world on the device of ``ctx``; the scene stays resident there."""
    flags = state_flags()
    keys = ctx.scene_build_keys(world.blocks, flags)
    models, quads, emits, n_real = instances(atlas, keys)
    info = ctx.scene_build_grid(world.blocks, flags, models, quads, emits, atlas.pixels.ravel(), atlas.size)
    stats = HqStats()
    stats.bricks, stats.uniform_bricks, stats.buried_bricks = info.bricks, info.uniform_bricks, info.buried_bricks
    stats.instances, stats.emitters = len(keys), info.emitters
    sun = atlas.sprites["sun"]
    return DeviceScene(dims=tuple(info.dims), offsets=tuple(info.offsets), atlas_size=atlas.size, models=models,
                       quads=quads, atlas=atlas.pixels.ravel(), see_through=(n_real, 0), emitter_count=info.emitters,
                       sun_sprite=(sun.x, sun.y, sun.w, sun.h), grid_len=int(info.grid_len),
                       emitter_grid_len=int(info.emitter_grid_len), stats=stats, keys_ms=info.keys_ms,
                       grid_ms=info.grid_ms)
