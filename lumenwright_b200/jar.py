"""The synthetic block set as a resource jar, in the layout the reference's asset loader reads.

The jar is a zip of new data written by this module from `synth.py`'s block set, with no game
asset in it:

* ``assets/minecraft/blockstates/<block>.json``: one ``variants`` entry with the empty key, which
  matches every state (crates/lumenwright/src/assets/blockstate.rs:12-31, :103-113);
* ``assets/minecraft/models/block/<block>.json``: the block's cuboid elements in model units (16 to a
  block) with their faces' textures, cull faces and tint index, and no parent
  (crates/lumenwright/src/assets/model.rs:173-245): cubes for stone, dirt, glowstone and leaves
  (leaves tinted), grass as a cube plus a tinted side overlay, the log's end and side textures,
  the lantern's two boxes; water has no elements (fluid faces are generated, not modelled);
* ``assets/minecraft/textures/block/<texture>.png``: the seeded 16x16 RGBA8 textures, and the sun
  at ``textures/environment/celestial/sun.png`` (32x32; crates/lumenwright/src/scene/mod.rs:250-253);
* ``assets/minecraft/textures/colormap/grass.png`` and ``foliage.png``: 256x256 maps of one colour,
  the plains tints the synthetic set uses, so every climate samples them
  (crates/lumenwright/src/assets/biome.rs:118-151).

Like the save writer this is host code beside the hq path: the benchmark frames build their
scenes from `synth.py` directly.
"""

import json
import struct
import zipfile
import zlib
from typing import Dict, List

import numpy as np

from . import synth as S

NS = "minecraft"

# Face names of the model format by the synthetic set's direction index.
FACE_NAME = {S.DOWN: "down", S.UP: "up", S.NORTH: "north", S.SOUTH: "south", S.WEST: "west", S.EAST: "east"}
CUBE = ([0, 0, 0], [16, 16, 16])
LANTERN_BOXES = (([5, 0, 5], [11, 7, 11]), ([6, 7, 6], [10, 9, 10]))


# ---- PNG ----------------------------------------------------------------------------------

def _chunk(kind: bytes, data: bytes) -> bytes:
    return struct.pack(">I", len(data)) + kind + data + struct.pack(">I", zlib.crc32(kind + data) & 0xFFFFFFFF)


def png_rgba(pixels: np.ndarray) -> bytes:
    """An 8-bit RGBA PNG of u32 texels packed R | G << 8 | B << 16 | A << 24, rows top first."""
    px = np.ascontiguousarray(pixels, np.uint32)
    h, w = px.shape
    rgba = np.stack([(px >> s) & 0xFF for s in (0, 8, 16, 24)], -1).astype(np.uint8)
    raw = b"".join(b"\x00" + rgba[y].tobytes() for y in range(h))  # filter type 0 on every row
    return (b"\x89PNG\r\n\x1a\n" + _chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 6, 0, 0, 0))
            + _chunk(b"IDAT", zlib.compress(raw, 9)) + _chunk(b"IEND", b""))


# ---- models and blockstates ---------------------------------------------------------------

def _element(box, faces: Dict[int, dict]) -> dict:
    return {"from": list(box[0]), "to": list(box[1]), "faces": {FACE_NAME[d]: f for d, f in faces.items()}}


def _cube(textures: Dict[int, str], tint: bool = False) -> dict:
    faces = {}
    for d in S.CUBE_ORDER:
        f = {"texture": "#" + textures[d], "cullface": FACE_NAME[d]}
        if tint:
            f["tintindex"] = 0
        faces[d] = f
    return _element(CUBE, faces)


def block_models() -> Dict[str, dict]:
    """Model JSON per block name of the synthetic set."""
    tex = lambda **kw: {k: f"{NS}:block/{v}" for k, v in kw.items()}  # noqa: E731
    every = lambda name: {d: name for d in S.CUBE_ORDER}  # noqa: E731
    side = (S.NORTH, S.SOUTH, S.EAST, S.WEST)
    grass_faces = {d: ("top" if d == S.UP else "bottom" if d == S.DOWN else "side") for d in S.CUBE_ORDER}
    grass = _cube(grass_faces)
    grass["faces"]["up"]["tintindex"] = 0
    overlay = _element(CUBE, {d: {"texture": "#overlay", "cullface": FACE_NAME[d], "tintindex": 0} for d in side})
    log_faces = {d: ("end" if d in (S.UP, S.DOWN) else "side") for d in S.CUBE_ORDER}
    return {
        "stone": {"textures": tex(all="stone", particle="stone"), "elements": [_cube(every("all"))]},
        "dirt": {"textures": tex(all="dirt", particle="dirt"), "elements": [_cube(every("all"))]},
        "glowstone": {"textures": tex(all="glowstone", particle="glowstone"), "elements": [_cube(every("all"))]},
        "oak_leaves": {"textures": tex(all="oak_leaves", particle="oak_leaves"),
                       "elements": [_cube(every("all"), tint=True)]},
        "grass_block": {"textures": tex(top="grass_top", bottom="dirt", side="grass_side", overlay="grass_side_overlay",
                                        particle="dirt"),
                        "elements": [grass, overlay]},
        "oak_log": {"textures": tex(end="oak_log_top", side="oak_log", particle="oak_log"),
                    "elements": [_cube(log_faces)]},
        "lantern": {"textures": tex(all="lantern", particle="lantern"),
                    "elements": [_element(b, {d: {"texture": "#all"} for d in S.CUBE_ORDER}) for b in LANTERN_BOXES]},
        "water": {"textures": tex(particle="water_still")},
    }


def blockstates() -> Dict[str, dict]:
    """Blockstate JSON per block name: one variant for every state."""
    return {name: {"variants": {"": {"model": f"{NS}:block/{name}"}}} for name in block_models()}


# ---- the jar ------------------------------------------------------------------------------

def _uniform(rgb, size: int = 256) -> np.ndarray:
    r, g, b = rgb
    return np.full((size, size), r | (g << 8) | (b << 16) | (255 << 24), np.uint32)


def jar_entries(seed: int) -> Dict[str, bytes]:
    """Path -> bytes of every entry of the synthetic jar for `seed`."""
    out: Dict[str, bytes] = {}
    for name, bs in blockstates().items():
        out[f"assets/{NS}/blockstates/{name}.json"] = json.dumps(bs, indent=1).encode()
    for name, m in block_models().items():
        out[f"assets/{NS}/models/block/{name}.json"] = json.dumps(m, indent=1).encode()
    for name in S.TEXTURES:
        out[f"assets/{NS}/textures/block/{name}.png"] = png_rgba(S._texture(name, seed))
    out[f"assets/{NS}/textures/environment/celestial/sun.png"] = png_rgba(S._texture("sun", seed, 32))
    out[f"assets/{NS}/textures/colormap/grass.png"] = png_rgba(_uniform(S.GRASS_TINT))
    out[f"assets/{NS}/textures/colormap/foliage.png"] = png_rgba(_uniform(S.FOLIAGE_TINT))
    out["pack.mcmeta"] = json.dumps({"pack": {"description": f"Lumenwright synthetic block set, seed {seed}"}}).encode()
    return out


def write_jar(path: str, seed: int) -> List[str]:
    """Writes the synthetic jar for `seed` to `path` (entries in sorted order, fixed timestamps,
    so the same seed gives the same bytes) and returns its entry names."""
    entries = jar_entries(seed)
    names = sorted(entries)
    with zipfile.ZipFile(path, "w", zipfile.ZIP_DEFLATED) as z:
        for n in names:
            info = zipfile.ZipInfo(n, date_time=(2000, 1, 1, 0, 0, 0))
            info.compress_type = zipfile.ZIP_DEFLATED
            z.writestr(info, entries[n])
    return names


def read_texture(data: bytes) -> np.ndarray:
    """The u32 texels of a PNG this module wrote (8-bit RGBA, filter type 0 rows)."""
    if data[:8] != b"\x89PNG\r\n\x1a\n":
        raise ValueError("not a PNG")
    pos, idat, dims = 8, b"", None
    while pos < len(data):
        (n,) = struct.unpack(">I", data[pos:pos + 4])
        kind, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        if kind == b"IHDR":
            w, h, depth, ctype = struct.unpack(">IIBB", body[:10])
            if (depth, ctype) != (8, 6):
                raise ValueError("only 8-bit RGBA is read here")
            dims = (h, w)
        elif kind == b"IDAT":
            idat += body
        pos += 12 + n
    h, w = dims
    rows = np.frombuffer(zlib.decompress(idat), np.uint8).reshape(h, 1 + 4 * w)
    if rows[:, 0].any():
        raise ValueError("only filter type 0 is read here")
    c = rows[:, 1:].reshape(h, w, 4).astype(np.uint32)
    return c[..., 0] | (c[..., 1] << 8) | (c[..., 2] << 16) | (c[..., 3] << 24)
