"""The host-side inputs of an hq render: `HqScene` and `HqFrame`, mirroring the reference's
(`crates/lumenwright/src/scene/voxel.rs:19-49`, `crates/lumenwright/src/render/mod.rs:80-89`).
"""

from dataclasses import dataclass, field
from typing import Optional, Tuple

import numpy as np

from .layout import EMITTER_DTYPE, MODEL_DTYPE, PARAMS_DTYPE, QUAD_DTYPE


@dataclass
class HqStats:
    """`HqStats` (voxel.rs:51-69): what the grid build put in the grid."""

    bricks: int = 0
    uniform_bricks: int = 0
    buried_bricks: int = 0
    instances: int = 0
    overlay_bricks: int = 0
    entity_quads: int = 0
    emitters: int = 0


@dataclass
class HqScene:
    """The hq buffers every path-tracing backend reads (voxel.rs:19-49)."""

    grid: np.ndarray                 # u32 words: top | bricks | ov_top | ov_cells | ov_quads | 0
    models: np.ndarray               # MODEL_DTYPE
    quads: np.ndarray                # QUAD_DTYPE
    atlas: np.ndarray                # u32 RGBA8 texels, row-major
    atlas_size: Tuple[int, int]
    dims: Tuple[int, int, int]       # grid size in bricks (x, y, z)
    offsets: Tuple[int, int, int, int, int]
    see_through: Tuple[int, int] = (0, 0)
    emitters: np.ndarray = field(default_factory=lambda: np.zeros(1, EMITTER_DTYPE))
    emitter_count: int = 0
    emitter_grid: np.ndarray = field(default_factory=lambda: np.zeros(8, np.uint32))
    sun_sprite: Optional[Tuple[int, int, int, int]] = None
    stats: HqStats = field(default_factory=HqStats)

    def __post_init__(self):
        self.grid = np.ascontiguousarray(self.grid, dtype=np.uint32)
        self.models = np.ascontiguousarray(self.models, dtype=MODEL_DTYPE)
        self.quads = np.ascontiguousarray(self.quads, dtype=QUAD_DTYPE)
        self.atlas = np.ascontiguousarray(self.atlas, dtype=np.uint32)
        self.emitters = np.ascontiguousarray(self.emitters, dtype=EMITTER_DTYPE)
        self.emitter_grid = np.ascontiguousarray(self.emitter_grid, dtype=np.uint32)

    def memory_bytes(self) -> int:
        """`HqScene::memory_bytes` (voxel.rs:91-98)."""
        return (self.grid.size * 4 + self.models.size * 16 + self.quads.size * 80 + self.atlas.size * 4
                + self.emitters.size * 32 + self.emitter_grid.size * 4)


@dataclass
class HqFrame:
    """`HqFrame` (render/mod.rs:80-89): the scene, the frame's `Params`, spp and the sky."""

    scene: HqScene
    params: np.ndarray  # PARAMS_DTYPE record
    spp: int
    sky: np.ndarray     # f32: the sky cache, or the lens map then the light map
    # The eye relative to the grid origin in f64 (the rebasing of request.rs:640-644 before its
    # cast to f32); FP64 references start their camera rays here.
    eye64: Optional[Tuple[float, float, float]] = None

    def __post_init__(self):
        self.params = np.array(self.params, dtype=PARAMS_DTYPE, order="C").reshape(())
        self.sky = np.ascontiguousarray(self.sky, dtype=np.float32)
