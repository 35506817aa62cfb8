"""Seeded synthetic inputs for the hq benchmarks: a block world and a block set.

The reference's benchmark frames need the Mojang client jar and a real save, neither of which
is available (nor reproduced here). This module writes new data of the same shapes instead:

* a world of ``chunks x chunks`` columns, 384 blocks tall (y -64..320, 24 sections), from a
  value-noise heightmap (base 64, amplitude 24, lattice pitch 32): stone below, dirt 3 deep,
  grass on top, water up to y = 63, oak trees at 1 in 400 columns, and optionally lanterns and
  glowstone at 1 per 2000 solid blocks on exposed ground;
* a block set ("synthetic jar"): 16x16 RGBA8 textures from a seeded per-texel hash and block
  models built from boxes, with the reference's quad conventions (`Quad::to_gpu`,
  crates/lumenwright/src/scene/mod.rs:105-129) and fluid faces (`fluid_quads`, :613-720).

Everything is a function of the seed, so every run builds the same bytes.
"""

from dataclasses import dataclass, field
from typing import Dict, List, Tuple

import numpy as np

from . import layout as L

# Block states of the synthetic set.
AIR, STONE, DIRT, GRASS, WATER, LOG, LEAVES, LANTERN, GLOWSTONE = range(9)
NAMES = ["air", "stone", "dirt", "grass_block", "water", "oak_log", "oak_leaves", "lantern", "glowstone"]

# Dir indices (crates/lumenwright/src/assets/model.rs:12-36).
DOWN, UP, NORTH, SOUTH, WEST, EAST = range(6)
DIR_OFFSET = {DOWN: (0, -1, 0), UP: (0, 1, 0), NORTH: (0, 0, -1), SOUTH: (0, 0, 1), WEST: (-1, 0, 0), EAST: (1, 0, 0)}

GRASS_TINT = (0x91, 0xBD, 0x59)    # plains grass colour
FOLIAGE_TINT = (0x77, 0xAB, 0x2F)  # plains foliage colour
WATER_TINT = (0x3F, 0x76, 0xE4)    # default water colour


def pcg(v):
    """The PCG-RXS-M-XS hash the kernel uses (crates/lumenwright-kernel/src/rng.rs:5-9), on
    numpy u32 arrays or ints."""
    v = np.asarray(v, dtype=np.uint32)
    with np.errstate(over="ignore"):
        state = v * np.uint32(747796405) + np.uint32(2891336453)
        word = ((state >> ((state >> np.uint32(28)) + np.uint32(4))) ^ state) * np.uint32(277803737)
        return (word >> np.uint32(22)) ^ word


def hash3(a, b, c):
    with np.errstate(over="ignore"):
        return pcg(pcg(pcg(np.asarray(c, np.uint32)) ^ np.asarray(a, np.uint32).astype(np.uint32)) ^ np.asarray(b, np.uint32).astype(np.uint32))


def rgba(r, g, b, a=255) -> int:
    return int(r) | (int(g) << 8) | (int(b) << 16) | (int(a) << 24)


# ---- textures -----------------------------------------------------------------------------

@dataclass
class Sprite:
    x: int
    y: int
    w: int
    h: int


@dataclass
class Atlas:
    pixels: np.ndarray  # u32 (h, w)
    sprites: Dict[str, Sprite]

    @property
    def size(self):
        return (self.pixels.shape[1], self.pixels.shape[0])


def _texture(name: str, seed: int, size: int = 16) -> np.ndarray:
    """A seeded 16x16 RGBA8 texture: a base colour varied per texel by a hash."""
    ys, xs = np.mgrid[0:size, 0:size]
    salt = int(pcg(np.uint32(seed) ^ np.uint32(sum(ord(c) * 131 ** i for i, c in enumerate(name)) & 0xFFFFFFFF)))
    h = hash3(xs, ys, salt)
    noise = ((h & 0xFF).astype(np.float64) / 255.0 - 0.5)
    base = {
        "stone": (125, 125, 125), "dirt": (134, 96, 67), "grass_top": (150, 150, 150),
        "grass_side": (134, 96, 67), "grass_side_overlay": (150, 150, 150), "oak_log": (109, 85, 50),
        "oak_log_top": (160, 130, 80), "oak_leaves": (140, 140, 140), "water_still": (180, 180, 180),
        "water_flow": (180, 180, 180), "lantern": (70, 60, 55), "glowstone": (250, 200, 110),
        "sun": (255, 240, 200),
    }[name]
    amp = {"glowstone": 60, "sun": 10, "water_still": 20, "water_flow": 20}.get(name, 40)
    rgb = np.clip(np.array(base)[None, None, :] + amp * noise[..., None] * np.array([1.0, 0.95, 0.9]), 0, 255)
    a = np.full((size, size), 255, np.int64)
    if name == "oak_leaves":
        a = np.where((h >> 8) % 4 == 0, 0, 255)
    elif name in ("water_still", "water_flow"):
        a = np.full((size, size), 170)
    elif name == "grass_side_overlay":
        drip = 3 + ((hash3(xs, 0, salt ^ 7) >> 4) % 3).astype(np.int64)
        a = np.where(ys < drip, 255, 0)
    elif name == "lantern":
        a = np.where((xs + ys) % 7 == 0, 0, 255)
        rgb = np.where(((xs % 5) == 2)[..., None], np.array([255, 200, 90]), rgb)
    elif name == "sun":
        r = np.hypot(xs - (size - 1) / 2, ys - (size - 1) / 2)
        a = np.where(r < size * 0.45, 255, 0)
        rgb = np.where((r < size * 0.45)[..., None], rgb, 0)
    rgb = rgb.astype(np.int64)
    return (rgb[..., 0] | (rgb[..., 1] << 8) | (rgb[..., 2] << 16) | (a << 24)).astype(np.uint32)


TEXTURES = ["stone", "dirt", "grass_top", "grass_side", "grass_side_overlay", "oak_log", "oak_log_top", "oak_leaves",
            "water_still", "water_flow", "lantern", "glowstone"]


def build_atlas(seed: int) -> Atlas:
    """Packs the textures on a grid of 18x18 cells (a 1-texel border copied from the edge, as the
    reference's packer leaves one, crates/lumenwright/src/assets/atlas.rs:302-420), with the
    32x32 sun texture after them."""
    cols = 8
    rows = (len(TEXTURES) + cols - 1) // cols
    w = cols * 18
    h = rows * 18 + 34
    pix = np.zeros((h, w), np.uint32)
    sprites = {}
    for i, name in enumerate(TEXTURES):
        cx, cy = (i % cols) * 18, (i // cols) * 18
        t = _texture(name, seed)
        pix[cy:cy + 18, cx:cx + 18] = np.pad(t, 1, mode="edge")
        sprites[name] = Sprite(cx + 1, cy + 1, 16, 16)
    sun = _texture("sun", seed, 32)
    pix[rows * 18 + 1:rows * 18 + 33, 1:33] = sun
    sprites["sun"] = Sprite(1, rows * 18 + 1, 32, 32)
    return Atlas(pix, sprites)


# ---- quads --------------------------------------------------------------------------------

def face(box, d):
    """(p0, eu, ev, uv rect in 16ths) of face ``d`` of the box ((x0,y0,z0), (x1,y1,z1)) in block
    units, with the vanilla winding (normal = ev x eu outward)."""
    (x0, y0, z0), (x1, y1, z1) = box
    w, h, dd = x1 - x0, y1 - y0, z1 - z0
    X = lambda v: v * 16.0  # noqa: E731
    if d == NORTH:
        return (x1, y1, z0), (-w, 0, 0), (0, -h, 0), (16 - X(x1), 16 - X(y1), 16 - X(x0), 16 - X(y0))
    if d == SOUTH:
        return (x0, y1, z1), (w, 0, 0), (0, -h, 0), (X(x0), 16 - X(y1), X(x1), 16 - X(y0))
    if d == EAST:
        return (x1, y1, z1), (0, 0, -dd), (0, -h, 0), (16 - X(z1), 16 - X(y1), 16 - X(z0), 16 - X(y0))
    if d == WEST:
        return (x0, y1, z0), (0, 0, dd), (0, -h, 0), (X(z0), 16 - X(y1), X(z1), 16 - X(y0))
    if d == UP:
        return (x0, y1, z0), (w, 0, 0), (0, 0, dd), (X(x0), X(z0), X(x1), X(z1))
    return (x0, y0, z1), (w, 0, 0), (0, 0, -dd), (X(x0), 16 - X(z1), X(x1), 16 - X(z0))


def resolve(atlas: Atlas, p0, eu, ev, tex, uv, flags, tint=None, emittance=0.0):
    """A quad with its model UVs (16ths of the sprite) resolved to atlas pixels and packed as
    `Quad::to_gpu` packs it."""
    s = atlas.sprites[tex]
    kx, ky = s.w / 16.0, s.h / 16.0
    u0, v0, u1, v1 = uv
    t = 0xFFFF_FFFF if tint is None else rgba(*tint)
    return L.make_quad(p0, eu, ev, flags=flags, tint=t, emittance=emittance,
                       uv=(s.x + u0 * kx, s.y + v0 * ky, (u1 - u0) * kx, 0.0), uvt=(0.0, (v1 - v0) * ky))


FULL = ((0.0, 0.0, 0.0), (1.0, 1.0, 1.0))
CUBE_ORDER = (NORTH, SOUTH, EAST, WEST, UP, DOWN)


@dataclass
class BlockInfo:
    """What the grid build needs of a block state (the reference's `BlockInfo`)."""

    occludes: bool
    simple: bool
    fluid: bool = False
    tinted: bool = False
    emittance: float = 0.0
    invisible: bool = False


BLOCKS = [
    BlockInfo(occludes=False, simple=True, invisible=True),            # air
    BlockInfo(occludes=True, simple=True),                             # stone
    BlockInfo(occludes=True, simple=True),                             # dirt
    BlockInfo(occludes=True, simple=False, tinted=True),               # grass_block
    BlockInfo(occludes=False, simple=False, fluid=True),               # water
    BlockInfo(occludes=True, simple=True),                             # oak_log
    BlockInfo(occludes=False, simple=False, tinted=True),              # oak_leaves
    BlockInfo(occludes=False, simple=True, emittance=1.0),             # lantern
    BlockInfo(occludes=True, simple=True, emittance=1.0),              # glowstone
]


def block_quads(atlas: Atlas, state: int, fluid_mask: int = 0) -> List[np.ndarray]:
    """The quads of one block instance in block-local coordinates (`Scene::block_quads`,
    crates/lumenwright/src/scene/mod.rs:525-582), before the grid build marks them front-only."""
    OPA, CUT, TRA = L.ALPHA_OPAQUE, L.ALPHA_CUTOUT, L.ALPHA_TRANSLUCENT
    sh = L.FLAG_SHADE
    em = BLOCKS[state].emittance
    out = []
    if state in (STONE, DIRT, GLOWSTONE, LEAVES):
        tex = {STONE: "stone", DIRT: "dirt", GLOWSTONE: "glowstone", LEAVES: "oak_leaves"}[state]
        mode = CUT if state == LEAVES else OPA
        tint = FOLIAGE_TINT if state == LEAVES else None
        for d in CUBE_ORDER:
            p0, eu, ev, uv = face(FULL, d)
            out.append(resolve(atlas, p0, eu, ev, tex, uv, mode | sh, tint, em))
    elif state == GRASS:
        for d in CUBE_ORDER:
            p0, eu, ev, uv = face(FULL, d)
            tex = "grass_top" if d == UP else ("dirt" if d == DOWN else "grass_side")
            out.append(resolve(atlas, p0, eu, ev, tex, uv, CUT | sh, GRASS_TINT if d == UP else None, em))
        for d in (NORTH, SOUTH, EAST, WEST):  # the tinted side overlay, drawn over the side
            p0, eu, ev, uv = face(FULL, d)
            out.append(resolve(atlas, p0, eu, ev, "grass_side_overlay", uv, CUT | sh, GRASS_TINT, em))
    elif state == LOG:
        for d in CUBE_ORDER:
            p0, eu, ev, uv = face(FULL, d)
            out.append(resolve(atlas, p0, eu, ev, "oak_log_top" if d in (UP, DOWN) else "oak_log", uv, OPA | sh, None, em))
    elif state == LANTERN:
        for box in (((5 / 16, 0.0, 5 / 16), (11 / 16, 7 / 16, 11 / 16)), ((6 / 16, 7 / 16, 6 / 16), (10 / 16, 9 / 16, 10 / 16))):
            for d in CUBE_ORDER:
                p0, eu, ev, uv = face(box, d)
                out.append(resolve(atlas, p0, eu, ev, "lantern", uv, CUT | sh, None, em))
    elif state == WATER:
        # fluid_quads (scene/mod.rs:613-720) for a source block.
        covered = fluid_mask & 0x80 != 0
        h = 1.0 if covered else 8.0 / 9.0
        shown = lambda d: fluid_mask & (1 << d) == 0  # noqa: E731
        fl = TRA | L.FLAG_WATER | sh
        if shown(UP):
            out.append(resolve(atlas, (0, h, 0), (1, 0, 0), (0, 0, 1), "water_still", (0, 0, 16, 16), fl, WATER_TINT))
        if shown(DOWN):
            out.append(resolve(atlas, (0, 0, 1), (1, 0, 0), (0, 0, -1), "water_still", (0, 0, 16, 16), fl, WATER_TINT))
        side = (0.0, (1.0 - h) * 8.0, 8.0, 8.0)
        dn = (0, -h, 0)
        if shown(NORTH):
            out.append(resolve(atlas, (1, h, 0), (-1, 0, 0), dn, "water_flow", side, fl, WATER_TINT))
        if shown(SOUTH):
            out.append(resolve(atlas, (0, h, 1), (1, 0, 0), dn, "water_flow", side, fl, WATER_TINT))
        if shown(EAST):
            out.append(resolve(atlas, (1, h, 1), (0, 0, -1), dn, "water_flow", side, fl, WATER_TINT))
        if shown(WEST):
            out.append(resolve(atlas, (0, h, 0), (0, 0, 1), dn, "water_flow", side, fl, WATER_TINT))
    return out


# ---- the world ----------------------------------------------------------------------------

@dataclass
class World:
    """A block volume: ``blocks[y, z, x]`` state ids, ``sections_y`` sections from ``min_y``."""

    blocks: np.ndarray
    chunks: Tuple[int, int]  # (x, z) chunks
    min_y: int = -64
    seed: int = 1
    origin: Tuple[int, int, int] = (0, -64, 0)  # world coordinates of grid (0, 0, 0)
    emitters_placed: int = 0
    solid_blocks: int = 0
    notes: Dict[str, float] = field(default_factory=dict)

    @property
    def size(self):
        return (self.blocks.shape[2], self.blocks.shape[0], self.blocks.shape[1])


def heightmap(nx: int, nz: int, seed: int, base=64, amplitude=24, pitch=32) -> np.ndarray:
    """h(x, z) = floor(base + amplitude * n(x, z)) from value noise: lattice values
    hash(ix, iz, seed) mapped to [-1, 1], smoothstep-bilinear between lattice points."""
    xs = np.arange(nx)
    zs = np.arange(nz)
    gx, gz = np.meshgrid(xs, zs, indexing="xy")  # (nz, nx)
    ix, iz = gx // pitch, gz // pitch
    fx, fz = (gx % pitch) / pitch, (gz % pitch) / pitch
    sx, sz = fx * fx * (3 - 2 * fx), fz * fz * (3 - 2 * fz)

    def lat(a, b):
        return hash3(a, b, seed).astype(np.float64) / 4294967295.0 * 2.0 - 1.0

    n00, n10, n01, n11 = lat(ix, iz), lat(ix + 1, iz), lat(ix, iz + 1), lat(ix + 1, iz + 1)
    n = (n00 * (1 - sx) + n10 * sx) * (1 - sz) + (n01 * (1 - sx) + n11 * sx) * sz
    return np.floor(base + amplitude * n).astype(np.int64)


def generate_world(chunks: int, seed: int = 1, emitters: bool = False, sea_level: int = 63,
                   tree_density: int = 400, emitter_per_solid: int = 2000) -> World:
    """The seeded world of the benchmark configs (see the module docstring)."""
    nx = nz = chunks * 16
    min_y, height = -64, 384
    b = np.zeros((height, nz, nx), np.uint16)
    h = heightmap(nx, nz, seed)
    y = np.arange(min_y, min_y + height)[:, None, None]
    hh = h[None]
    b[y <= hh - 4] = STONE
    b[(y > hh - 4) & (y < hh)] = DIRT
    b[y == hh] = GRASS
    b[(y > hh) & (y <= sea_level)] = WATER
    # Grass under water is dirt, as the game generates it.
    under = (y == hh) & (hh < sea_level)
    b[under] = DIRT
    # Trees: trunks 4-6 tall with a radius-2 leaf blob, on land columns.
    gx, gz = np.meshgrid(np.arange(nx), np.arange(nz), indexing="xy")
    th = hash3(gx, gz, seed ^ 0x7EE5)
    for z, x in zip(*np.nonzero((th % tree_density == 0) & (h >= sea_level))):
        top = int(h[z, x]) + 4 + int(th[z, x] >> 16) % 3
        for dy in range(-2, 3):
            for dz in range(-2, 3):
                for dx in range(-2, 3):
                    if dx * dx + dy * dy + dz * dz > 5:
                        continue
                    X, Y, Z = x + dx, top + dy, z + dz
                    if 0 <= X < nx and 0 <= Z < nz and b[Y - min_y, Z, X] == AIR:
                        b[Y - min_y, Z, X] = LEAVES
        b[int(h[z, x]) + 1 - min_y: top + 1 - min_y, z, x] = LOG
    w = World(b, (chunks, chunks), min_y, seed, (0, min_y, 0))
    solid = int(np.count_nonzero((b != AIR) & (b != WATER)))
    w.solid_blocks = solid
    if emitters:
        land = np.argwhere((h >= sea_level))
        want = max(1, solid // emitter_per_solid)
        eh = hash3(gx, gz, seed ^ 0xE417)
        order = np.argsort(eh[land[:, 0], land[:, 1]], kind="stable")
        placed = 0
        for k in order:
            z, x = land[k]
            yy = int(h[z, x]) + 1 - min_y
            if b[yy, z, x] != AIR:
                continue
            b[yy, z, x] = LANTERN if (int(eh[z, x]) >> 20) & 1 else GLOWSTONE
            placed += 1
            if placed >= want:
                break
        w.emitters_placed = placed
    return w
