"""Anvil saves of the synthetic worlds, in the layout the reference's world reader decodes.

A save is a folder holding ``level.dat`` (gzip-compressed NBT with a ``Data`` compound,
crates/lumenwright/src/world/level.rs:42-81) and ``region/r.<rx>.<rz>.mca`` files
(crates/lumenwright/src/world/region.rs:34-69): a header of 1024 big-endian location words
(sector offset << 8 | sector count, the chunk at local (lx, lz) in word lx + 32 lz) and 1024
timestamps, then one record per chunk on 4 KiB sectors (a 4-byte length that counts the
compression byte, the compression byte, the payload). Each chunk is 1.18+ chunk NBT
(crates/lumenwright/src/world/chunk.rs:101-151): ``DataVersion``, ``xPos``, ``zPos``, and a list of
``sections``, each with ``Y`` and a ``block_states`` palette whose indices are packed YZX into
64-bit words without spanning, at max(4, ceil(log2 n)) bits each (chunk.rs:154-179).

`write_world` writes a `synth.World` as such a save, every section of its 384-block column
included (so a reader's section range is the world's height); `read_world` reads one back into
a `synth.World` (1.18+ layout; gzip, zlib or uncompressed chunks) for the synthetic block set.
Both are host code beside the hq path: the benchmark frames build their scenes from the
in-memory world, and a save written here is the same world a reference run would load.
"""

import gzip
import os
import re
import struct
import zlib
from typing import Dict, Iterable, List, Optional, Tuple

import numpy as np

from . import synth as S

# NBT tag ids.
END, BYTE, SHORT, INT, LONG, FLOAT, DOUBLE, BYTE_ARRAY, STRING, LIST, COMPOUND, INT_ARRAY, LONG_ARRAY = range(13)

# The data version written into chunks and level.dat: a 1.21 save, whose chunks use the 1.18+
# layout (top-level ``sections`` with ``block_states`` and ``biomes``). The reference's own
# fixture writer stamps the same number (crates/lumenwright-cli/src/fixture.rs:17).
DATA_VERSION = 4671
VERSION_NAME = "1.21.11"
BIOME = "minecraft:plains"

# Block states of the synthetic set, as the game names them.
STATES: Dict[int, Tuple[str, Dict[str, str]]] = {
    S.AIR: ("minecraft:air", {}),
    S.STONE: ("minecraft:stone", {}),
    S.DIRT: ("minecraft:dirt", {}),
    S.GRASS: ("minecraft:grass_block", {"snowy": "false"}),
    S.WATER: ("minecraft:water", {"level": "0"}),
    S.LOG: ("minecraft:oak_log", {"axis": "y"}),
    S.LEAVES: ("minecraft:oak_leaves", {"distance": "1", "persistent": "true", "waterlogged": "false"}),
    S.LANTERN: ("minecraft:lantern", {"hanging": "false", "waterlogged": "false"}),
    S.GLOWSTONE: ("minecraft:glowstone", {}),
}
_BY_NAME = {name: sid for sid, (name, _) in STATES.items()}


# ---- NBT ----------------------------------------------------------------------------------

class Typed:
    """A value with an explicit NBT tag, for the integer widths and arrays plain Python types
    do not say (a bare ``int`` is written as TAG_Int, ``float`` as TAG_Double, ``str`` as
    TAG_String, ``dict`` as TAG_Compound, ``list`` as TAG_List)."""

    __slots__ = ("tag", "value")

    def __init__(self, tag: int, value):
        self.tag = tag
        self.value = value

    def __eq__(self, other):
        return isinstance(other, Typed) and self.tag == other.tag and np.array_equal(self.value, other.value)

    def __repr__(self):
        return f"Typed({self.tag}, {self.value!r})"


def Byte(v: int) -> Typed:
    return Typed(BYTE, int(v))


def Long(v: int) -> Typed:
    return Typed(LONG, int(v))


def LongArray(v) -> Typed:
    return Typed(LONG_ARRAY, np.asarray(v, np.int64))


def ByteArray(v) -> Typed:
    return Typed(BYTE_ARRAY, np.asarray(v, np.int8))


def _tag_of(v) -> int:
    if isinstance(v, Typed):
        return v.tag
    if isinstance(v, bool):
        return BYTE
    if isinstance(v, int):
        return INT
    if isinstance(v, float):
        return DOUBLE
    if isinstance(v, str):
        return STRING
    if isinstance(v, dict):
        return COMPOUND
    if isinstance(v, list):
        return LIST
    raise TypeError(f"no NBT tag for {type(v).__name__}")


def _put_string(out: bytearray, s: str) -> None:
    b = s.encode("utf-8")  # the game writes modified UTF-8; the two agree on every name used here
    if len(b) > 0xFFFF:
        raise ValueError("NBT string longer than 65535 bytes")
    out += struct.pack(">H", len(b))
    out += b


_SCALAR = {BYTE: ">b", SHORT: ">h", INT: ">i", LONG: ">q", FLOAT: ">f", DOUBLE: ">d"}
_ARRAY = {BYTE_ARRAY: ">i1", INT_ARRAY: ">i4", LONG_ARRAY: ">i8"}


def _put_payload(out: bytearray, tag: int, v) -> None:
    if isinstance(v, Typed):
        v = v.value
    if tag in _SCALAR:
        out += struct.pack(_SCALAR[tag], v)
    elif tag in _ARRAY:
        a = np.asarray(v)
        out += struct.pack(">i", a.size)
        out += a.astype(_ARRAY[tag]).tobytes()
    elif tag == STRING:
        _put_string(out, v)
    elif tag == LIST:
        et = _tag_of(v[0]) if v else END
        if any(_tag_of(e) != et for e in v):
            raise TypeError("an NBT list holds one tag type")
        out += struct.pack(">bi", et, len(v))
        for e in v:
            _put_payload(out, et, e)
    elif tag == COMPOUND:
        for k, e in v.items():
            et = _tag_of(e)
            out += struct.pack(">b", et)
            _put_string(out, k)
            _put_payload(out, et, e)
        out += b"\x00"
    else:
        raise ValueError(f"bad NBT tag {tag}")


def nbt_bytes(root: dict, name: str = "") -> bytes:
    """Uncompressed NBT of a named root compound."""
    out = bytearray(b"\x0a")
    _put_string(out, name)
    _put_payload(out, COMPOUND, root)
    return bytes(out)


def parse_nbt(data: bytes) -> Tuple[str, dict]:
    """(name, compound) of uncompressed NBT. Scalars come back as Python numbers, arrays as
    numpy arrays, lists as lists, compounds as dicts."""
    mv = memoryview(data)
    pos = 0

    def take(n):
        nonlocal pos
        if pos + n > len(mv):
            raise ValueError("truncated NBT")
        b = mv[pos:pos + n]
        pos += n
        return b

    def string():
        (n,) = struct.unpack(">H", take(2))
        return bytes(take(n)).decode("utf-8")

    def payload(tag):
        if tag in _SCALAR:
            fmt = _SCALAR[tag]
            return struct.unpack(fmt, take(struct.calcsize(fmt)))[0]
        if tag in _ARRAY:
            (n,) = struct.unpack(">i", take(4))
            dt = np.dtype(_ARRAY[tag])
            return np.frombuffer(bytes(take(n * dt.itemsize)), dt).astype(dt.newbyteorder("="))
        if tag == STRING:
            return string()
        if tag == LIST:
            et, n = struct.unpack(">bi", take(5))
            return [payload(et) for _ in range(max(n, 0))]
        if tag == COMPOUND:
            d = {}
            while True:
                (t,) = struct.unpack(">b", take(1))
                if t == END:
                    return d
                k = string()
                d[k] = payload(t)
        raise ValueError(f"bad NBT tag {tag}")

    (t,) = struct.unpack(">b", take(1))
    if t != COMPOUND:
        raise ValueError("NBT root is not a compound")
    name = string()
    return name, payload(COMPOUND)


# ---- packed palette indices ---------------------------------------------------------------

def bits_for(n: int) -> int:
    """Bits to index a palette of n entries (0 for one entry or none)."""
    return 0 if n <= 1 else int(n - 1).bit_length()


def block_bits(n: int) -> int:
    """Bits per block index: at least 4 (chunk.rs:168-171)."""
    return max(4, bits_for(n))


def pack_indices(ids: np.ndarray, bits: int) -> np.ndarray:
    """Indices packed into 64-bit words without spanning a word: entry i in word i // (64 // bits)
    at bit (i % (64 // bits)) * bits, the top bits of each word left zero."""
    per = 64 // bits
    ids = np.asarray(ids, np.uint64)
    if ids.size and int(ids.max()) >> bits:
        raise ValueError(f"an index does not fit {bits} bits")
    words = -(-ids.size // per)
    lanes = np.zeros(words * per, np.uint64)
    lanes[:ids.size] = ids
    fields = lanes.reshape(words, per) << (np.arange(per, dtype=np.uint64) * np.uint64(bits))
    return np.bitwise_or.reduce(fields, axis=1).view(np.int64) if words else np.zeros(0, np.int64)


def unpack_indices(data: np.ndarray, bits: int, count: int) -> np.ndarray:
    """The inverse of `pack_indices`; entries past the end of `data` read 0 (chunk.rs:154-165)."""
    per = 64 // bits
    i = np.arange(count)
    w = np.zeros(count, np.uint64)
    words = np.asarray(data, np.int64).view(np.uint64)
    have = i // per < words.size
    w[have] = words[i[have] // per]
    return ((w >> ((i % per).astype(np.uint64) * np.uint64(bits))) & np.uint64((1 << bits) - 1)).astype(np.uint16)


# ---- region files -------------------------------------------------------------------------

SECTOR = 4096
ZLIB, GZIP, NONE = 2, 1, 3


def region_name(rx: int, rz: int) -> str:
    return f"r.{rx}.{rz}.mca"


def parse_region_name(name: str) -> Optional[Tuple[int, int]]:
    """(rx, rz) of ``r.<rx>.<rz>.mca`` (region.rs:123-130), else None."""
    m = re.fullmatch(r"r\.(-?\d+)\.(-?\d+)\.mca", os.path.basename(name))
    return (int(m.group(1)), int(m.group(2))) if m else None


def write_region(chunks: Iterable[Tuple[int, int, bytes]]) -> bytes:
    """A region file holding ``(local x, local z, chunk NBT)`` records, zlib-compressed, each on
    whole sectors after the two header sectors, timestamps 0."""
    header = bytearray(2 * SECTOR)
    body = bytearray()
    seen = set()
    for lx, lz, nbt in chunks:
        if not (0 <= lx < 32 and 0 <= lz < 32) or (lx, lz) in seen:
            raise ValueError(f"bad or repeated local chunk ({lx}, {lz})")
        seen.add((lx, lz))
        comp = zlib.compress(nbt)
        rec = struct.pack(">IB", len(comp) + 1, ZLIB) + comp
        rec += bytes(-len(rec) % SECTOR)
        sectors = len(rec) // SECTOR
        if sectors > 255:
            raise ValueError("a chunk record over 255 sectors needs an external .mcc file")
        loc = ((2 + len(body) // SECTOR) << 8) | sectors
        header[4 * (lx + 32 * lz):4 * (lx + 32 * lz) + 4] = struct.pack(">I", loc)
        body += rec
    return bytes(header + body)


def decompress(kind: int, payload: bytes) -> bytes:
    if kind == ZLIB:
        return zlib.decompress(payload)
    if kind == GZIP:
        return gzip.decompress(payload)
    if kind == NONE:
        return bytes(payload)
    raise ValueError(f"unsupported chunk compression type {kind}")


def region_chunk(data: bytes, lx: int, lz: int) -> Optional[bytes]:
    """Decompressed NBT of the chunk at local (lx, lz) of a region file's bytes, or None when the
    region holds none there (region.rs:34-69; external ``.mcc`` chunks are not read here)."""
    if len(data) < 2 * SECTOR:
        return None
    idx = 4 * ((lx & 31) + (lz & 31) * 32)
    (loc,) = struct.unpack(">I", data[idx:idx + 4])
    offset, sectors = (loc >> 8) * SECTOR, loc & 0xFF
    if offset == 0 or sectors == 0:
        return None
    if offset + 5 > len(data):
        raise ValueError(f"chunk ({lx},{lz}) points past the end of the region")
    length, kind = struct.unpack(">IB", data[offset:offset + 5])
    if length == 0:
        return None
    if kind & 0x80:
        raise ValueError(f"chunk ({lx},{lz}) is stored in an external file")
    end = offset + 4 + length
    if end > len(data):
        raise ValueError(f"chunk ({lx},{lz}) is truncated")
    return decompress(kind & 0x7F, data[offset + 5:end])


# ---- chunks -------------------------------------------------------------------------------

def _state_nbt(sid: int) -> dict:
    name, props = STATES[int(sid)]
    d = {"Name": name}
    if props:
        d["Properties"] = dict(sorted(props.items()))
    return d


def section_nbt(blocks: np.ndarray, sy: int) -> dict:
    """One section's NBT from its 16x16x16 synthetic state ids ``blocks[y, z, x]``: the palette
    in increasing state id (air first where present), the indices packed YZX."""
    ids = np.ascontiguousarray(blocks).reshape(-1)
    pal, idx = np.unique(ids, return_inverse=True)
    states = {"palette": [_state_nbt(s) for s in pal]}
    if pal.size > 1:
        states["data"] = LongArray(pack_indices(idx, block_bits(pal.size)))
    return {"Y": Byte(sy), "block_states": states, "biomes": {"palette": [BIOME]}}


def chunk_nbt(world: "S.World", lcx: int, lcz: int, cx: int, cz: int) -> bytes:
    """The chunk NBT of the world's chunk column (lcx, lcz), placed at chunk (cx, cz)."""
    if world.min_y % 16 or world.blocks.shape[0] % 16:
        raise ValueError("the world's height is not whole sections")
    smin = world.min_y // 16
    col = world.blocks[:, lcz * 16:(lcz + 1) * 16, lcx * 16:(lcx + 1) * 16]
    sections = [section_nbt(col[k * 16:(k + 1) * 16], smin + k) for k in range(world.blocks.shape[0] // 16)]
    return nbt_bytes({"DataVersion": DATA_VERSION, "xPos": cx, "zPos": cz, "yPos": smin,
                      "Status": "minecraft:full", "sections": sections})


def origin_chunk(world: "S.World") -> Tuple[int, int]:
    """The chunk (x, z) of the world's first column; its origin must be chunk-aligned."""
    ox, oz = world.origin[0], world.origin[2]
    if float(ox) % 16 or float(oz) % 16:
        raise ValueError(f"world origin ({ox}, {oz}) is not on a chunk corner")
    return int(ox) // 16, int(oz) // 16


def write_world(world: "S.World", path: str, name: str = "Lumenwright synthetic",
                spawn: Optional[Tuple[int, int, int]] = None, day_time: int = 6000) -> List[str]:
    """Writes ``level.dat`` and ``region/`` of `world` into `path` (made if missing) and returns
    the region files written. The world's chunks sit at `origin_chunk`."""
    cx0, cz0 = origin_chunk(world)
    ncx, ncz = world.chunks
    os.makedirs(os.path.join(path, "region"), exist_ok=True)
    regions: Dict[Tuple[int, int], List[Tuple[int, int, bytes]]] = {}
    for lcz in range(ncz):
        for lcx in range(ncx):
            cx, cz = cx0 + lcx, cz0 + lcz
            regions.setdefault((cx >> 5, cz >> 5), []).append((cx & 31, cz & 31, chunk_nbt(world, lcx, lcz, cx, cz)))
    written = []
    for (rx, rz), chunks in sorted(regions.items()):
        f = os.path.join(path, "region", region_name(rx, rz))
        with open(f, "wb") as fh:
            fh.write(write_region(chunks))
        written.append(f)
    if spawn is None:
        spawn = (cx0 * 16 + ncx * 8, 64, cz0 * 16 + ncz * 8)
    data = {"LevelName": name, "DataVersion": DATA_VERSION,
            "Version": {"Name": VERSION_NAME, "Id": DATA_VERSION},
            "SpawnX": int(spawn[0]), "SpawnY": int(spawn[1]), "SpawnZ": int(spawn[2]),
            "DayTime": Long(day_time)}
    with open(os.path.join(path, "level.dat"), "wb") as fh:
        fh.write(gzip.compress(nbt_bytes({"Data": data}), mtime=0))
    return written


def read_level(path: str) -> dict:
    """The ``Data`` compound of a save's ``level.dat`` (gzip or plain NBT, level.rs:42-57)."""
    with open(os.path.join(path, "level.dat"), "rb") as fh:
        raw = fh.read()
    try:
        raw = gzip.decompress(raw)
    except OSError:
        pass
    _, root = parse_nbt(raw)
    if not isinstance(root.get("Data"), dict):
        raise ValueError("level.dat has no Data compound")
    return root["Data"]


def _state_id(state: dict) -> int:
    name = state.get("Name", "")
    if name in ("minecraft:cave_air", "minecraft:void_air"):
        return S.AIR
    if name not in _BY_NAME:
        raise ValueError(f"block {name} is not in the synthetic set")
    return _BY_NAME[name]


def read_world(path: str, min_chunk: Tuple[int, int], chunks: Tuple[int, int]) -> "S.World":
    """The chunks [min_chunk, min_chunk + chunks) of a save as a `synth.World`, the sections'
    range taken from the chunks read (as the reference's area loader does, mod.rs:406-414).
    Missing chunks and sections are air; a palette index past the palette's end reads its last
    entry."""
    read_level(path)
    parsed = []
    cache: Dict[Tuple[int, int], Optional[bytes]] = {}
    for cz in range(min_chunk[1], min_chunk[1] + chunks[1]):
        for cx in range(min_chunk[0], min_chunk[0] + chunks[0]):
            key = (cx >> 5, cz >> 5)
            if key not in cache:
                f = os.path.join(path, "region", region_name(*key))
                cache[key] = None
                if os.path.exists(f):
                    with open(f, "rb") as fh:
                        cache[key] = fh.read()
            if cache[key] is None:
                continue
            nbt = region_chunk(cache[key], cx & 31, cz & 31)
            if nbt is None:
                continue
            _, c = parse_nbt(nbt)
            if "sections" not in c:
                raise ValueError(f"chunk ({cx},{cz}) is not in the 1.18+ layout")
            parsed.append((c["xPos"], c["zPos"], c["sections"]))
    ys = [s["Y"] for _, _, secs in parsed for s in secs]
    smin, smax = (min(ys), max(ys)) if ys else (0, 0)
    blocks = np.zeros(((smax - smin + 1) * 16, chunks[1] * 16, chunks[0] * 16), np.uint16)
    for cx, cz, secs in parsed:
        lx, lz = cx - min_chunk[0], cz - min_chunk[1]
        if not (0 <= lx < chunks[0] and 0 <= lz < chunks[1]):
            continue
        for s in secs:
            bs = s.get("block_states") or {}
            pal = [_state_id(p) for p in bs.get("palette", [])]
            if not pal:
                continue
            if len(pal) > 1 and "data" in bs:
                idx = np.minimum(unpack_indices(bs["data"], block_bits(len(pal)), 4096), len(pal) - 1)
                vox = np.asarray(pal, np.uint16)[idx].reshape(16, 16, 16)
            else:
                vox = np.full((16, 16, 16), pal[0], np.uint16)
            y0 = (s["Y"] - smin) * 16
            blocks[y0:y0 + 16, lz * 16:(lz + 1) * 16, lx * 16:(lx + 1) * 16] = vox
    return S.World(blocks, chunks, smin * 16, origin=(min_chunk[0] * 16, smin * 16, min_chunk[1] * 16))
