"""Anvil saves of the synthetic worlds (`lumenwright_b200/anvil.py`): the known answers of the
reference's own world tests (crates/lumenwright/src/world/region.rs:158-196,
crates/lumenwright/src/world/chunk.rs:262-287), the byte layout its reader takes, and round trips
of the configs' worlds through a save.
"""

import gzip
import struct
import zlib

import numpy as np
import pytest

from lumenwright_b200 import anvil as A
from lumenwright_b200 import synth as S


def test_block_bits_known_answers():  # chunk.rs:266-274
    assert A.block_bits(1) == 4 and A.block_bits(16) == 4 and A.block_bits(17) == 5
    assert A.bits_for(2) == 1 and A.bits_for(3) == 2 and A.bits_for(64) == 6


def test_unpack_non_spanning_known_answer():  # chunk.rs:276-286
    # 5 bits per entry: 12 entries a word, the top 4 bits unused; 13 entries take two words.
    vals = np.arange(13, dtype=np.uint16) * 2
    words = [0, 0]
    for i, v in enumerate(vals):
        words[i // 12] |= int(v) << ((i % 12) * 5)
    words = np.array(words, np.uint64).view(np.int64)
    assert np.array_equal(A.unpack_indices(words, 5, 13), vals)
    assert np.array_equal(A.pack_indices(vals, 5), words)


@pytest.mark.parametrize("bits", [4, 5, 6, 7, 8, 12, 16])
def test_pack_and_unpack_are_inverse(bits):
    rng = np.random.default_rng(bits)
    ids = rng.integers(0, 1 << bits, 4096).astype(np.uint16)
    words = A.pack_indices(ids, bits)
    assert words.size == -(-4096 // (64 // bits))
    assert np.array_equal(A.unpack_indices(words, bits, 4096), ids)
    # a short array reads 0 past its end, as the reference's unpack does
    assert not A.unpack_indices(words[:1], bits, 4096)[64 // bits:].any()
    with pytest.raises(ValueError):
        A.pack_indices(np.array([1 << bits]), bits)


def test_region_round_trip_known_answer():  # region.rs:162-170
    data = A.write_region([(3, 7, b"hello"), (31, 31, bytes([9]) * 10_000)])
    assert A.region_chunk(data, 3, 7) == b"hello"
    assert A.region_chunk(data, 31, 31) == bytes([9]) * 10_000
    assert A.region_chunk(data, 0, 0) is None
    # the layout: the first record on sector 2, one sector each, zlib, length counting the type byte
    (loc,) = struct.unpack(">I", data[4 * (3 + 32 * 7):4 * (3 + 32 * 7) + 4])
    assert loc == (2 << 8) | 1
    length, kind = struct.unpack(">IB", data[2 * 4096:2 * 4096 + 5])
    assert kind == 2 and zlib.decompress(data[2 * 4096 + 5:2 * 4096 + 4 + length]) == b"hello"
    assert len(data) % 4096 == 0 and not any(data[4096:8192])  # timestamps 0


def test_region_reads_every_compression_the_reader_takes():
    nbt = b"\x0a\x00\x00\x00"
    for kind, payload in ((1, gzip.compress(nbt)), (2, zlib.compress(nbt)), (3, nbt)):
        rec = struct.pack(">IB", len(payload) + 1, kind) + payload
        data = bytearray(8192) + rec + bytes(-len(rec) % 4096)
        data[0:4] = struct.pack(">I", (2 << 8) | 1)
        assert A.region_chunk(bytes(data), 0, 0) == nbt
    with pytest.raises(ValueError):
        A.decompress(4, b"")  # LZ4 chunks are not read here


def test_region_name_known_answers():  # region.rs:172-179
    assert A.parse_region_name("/a/r.-1.12.mca") == (-1, 12)
    assert A.parse_region_name("/a/level.dat") is None
    assert A.region_name(-1, 12) == "r.-1.12.mca"


def test_nbt_round_trip_of_every_tag():
    root = {"b": A.Byte(-3), "i": 7, "l": A.Long(-(1 << 40)), "d": 0.25, "s": "minecraft:stone",
            "la": A.LongArray([1, -2, 1 << 62]), "ba": A.ByteArray([1, -1]), "list": [1, 2, 3],
            "empty": [], "nest": {"palette": [{"Name": "minecraft:air"}]}}
    name, back = A.parse_nbt(A.nbt_bytes(root, "root"))
    assert name == "root"
    assert back["b"] == -3 and back["i"] == 7 and back["l"] == -(1 << 40) and back["d"] == 0.25
    assert back["s"] == "minecraft:stone" and back["list"] == [1, 2, 3] and back["empty"] == []
    assert list(back["la"]) == [1, -2, 1 << 62] and list(back["ba"]) == [1, -1]
    assert back["nest"] == {"palette": [{"Name": "minecraft:air"}]}
    with pytest.raises(TypeError):
        A.nbt_bytes({"mixed": [1, "a"]})
    with pytest.raises(ValueError):
        A.parse_nbt(A.nbt_bytes(root)[:-3])


def test_section_layout_is_the_readers():
    # The tags the reference's serde structs name (chunk.rs:101-151): Y a TAG_Byte, block_states a
    # compound with a palette of {Name, Properties} and packed TAG_Long_Array data, biomes a
    # palette of strings; the indices YZX.
    blocks = np.zeros((16, 16, 16), np.uint16)
    blocks[0, :, :] = S.STONE
    blocks[3, 2, 1] = S.LOG
    raw = A.nbt_bytes({"s": A.section_nbt(blocks, -4)})
    assert b"\x01\x00\x01Y\xfc" in raw  # TAG_Byte "Y" = -4
    assert b"\x0c\x00\x04data" in raw and b"\x08\x00\x04Name" in raw and b"\x0a\x00\x0aProperties" in raw
    s = A.parse_nbt(raw)[1]["s"]
    names = [p["Name"] for p in s["block_states"]["palette"]]
    assert names == ["minecraft:air", "minecraft:stone", "minecraft:oak_log"]
    assert s["block_states"]["palette"][2]["Properties"] == {"axis": "y"}
    assert "Properties" not in s["block_states"]["palette"][1]
    idx = A.unpack_indices(s["block_states"]["data"], 4, 4096)
    assert idx[(3 * 16 + 2) * 16 + 1] == 2 and idx[5] == 1 and idx[16 * 16] == 0
    assert s["biomes"] == {"palette": ["minecraft:plains"]}
    uniform = A.section_nbt(np.full((16, 16, 16), S.WATER, np.uint16), 3)
    assert "data" not in uniform["block_states"] and len(uniform["block_states"]["palette"]) == 1


@pytest.mark.parametrize("origin_chunk", [(0, 0), (62_527, -3)])
def test_world_round_trip_through_a_save(tmp_path, origin_chunk):
    # The C2 world's generator at 2x2 chunks with emitters; the second origin puts the columns
    # across regions 1953 and 1954 in x (x = 1,000,432) and region -1 in z.
    w = S.generate_world(2, seed=5, emitters=True)
    w.origin = (origin_chunk[0] * 16, w.origin[1], origin_chunk[1] * 16)
    files = A.write_world(w, str(tmp_path), day_time=12800)
    regions = sorted(A.parse_region_name(f) for f in files)
    want = sorted({((origin_chunk[0] + i) >> 5, (origin_chunk[1] + j) >> 5) for i in range(2) for j in range(2)})
    assert regions == want
    level = A.read_level(str(tmp_path))
    assert level["DataVersion"] == A.DATA_VERSION and level["DayTime"] == 12800
    assert level["SpawnX"] == origin_chunk[0] * 16 + 16
    back = A.read_world(str(tmp_path), origin_chunk, (2, 2))
    assert back.min_y == -64 and back.blocks.shape == w.blocks.shape
    assert np.array_equal(back.blocks, w.blocks)
    assert back.origin == (origin_chunk[0] * 16, -64, origin_chunk[1] * 16)
    assert w.emitters_placed > 0 and np.count_nonzero((back.blocks == S.LANTERN) | (back.blocks == S.GLOWSTONE)) == w.emitters_placed
    # a chunk of the save holds every section of the column, -4..19
    with open(files[0], "rb") as fh:
        data = fh.read()
    c = A.parse_nbt(A.region_chunk(data, origin_chunk[0] & 31, origin_chunk[1] & 31))[1]
    assert [s["Y"] for s in c["sections"]] == list(range(-4, 20))
    assert c["xPos"] == origin_chunk[0] and c["zPos"] == origin_chunk[1] and c["Status"] == "minecraft:full"


def test_reading_past_the_save_is_air(tmp_path):
    w = S.generate_world(1, seed=2)
    A.write_world(w, str(tmp_path))
    back = A.read_world(str(tmp_path), (0, 0), (2, 1))
    assert np.array_equal(back.blocks[:, :, :16], w.blocks) and not back.blocks[:, :, 16:].any()
    with pytest.raises(FileNotFoundError):
        A.read_world(str(tmp_path / "none"), (0, 0), (1, 1))


def test_world_off_a_chunk_corner_is_refused(tmp_path):
    w = S.generate_world(1, seed=2)
    w.origin = (1_000_000.5, -64, 0)
    with pytest.raises(ValueError):
        A.write_world(w, str(tmp_path))


@pytest.mark.parametrize("name", ["c1", "c2", "c4", "c5"])
def test_config_saves_hold_the_frames_worlds(tmp_path, name):
    # Each benchmark configuration's world written as the save its frame would be loaded from:
    # read back at the frame's chunks, the same blocks at the same place (c5's columns start at
    # x = 1,000,000, chunk 62,500, and span regions 1953 and 1954).
    from lumenwright_b200 import request as R
    cfg = R.CONFIGS[name]
    files = R.write_save(cfg, str(tmp_path))
    cx0 = int(cfg.origin_x) // 16
    assert sorted(A.parse_region_name(f)[0] for f in files) == sorted({(cx0 + i) >> 5 for i in range(cfg.chunks)})
    want = R.config_world(cfg)
    back = A.read_world(str(tmp_path), (cx0, 0), (cfg.chunks, cfg.chunks))
    assert back.origin == tuple(float(v) for v in want.origin) and np.array_equal(back.blocks, want.blocks)
    assert A.read_level(str(tmp_path))["DayTime"] == cfg.time


def test_a_frame_built_from_its_save_is_the_frame(tmp_path):
    # make_frame on the save that write_save wrote: the same scene buffers, Params and sky as the
    # frame built from the generated world (the sky from a host stand-in, as no GPU is here).
    from lumenwright_b200 import request as R
    from test_frames import OracleSky
    cfg = R.CONFIGS["c1"]
    R.write_save(cfg, str(tmp_path))
    a = R.make_frame(cfg, sky_backend=OracleSky(), spp=4)
    b = R.make_frame(cfg, sky_backend=OracleSky(), spp=4, save=str(tmp_path))
    assert a.params.tobytes() == b.params.tobytes() and np.array_equal(a.sky, b.sky) and a.eye64 == b.eye64
    for name in ("grid", "models", "quads", "atlas", "emitters", "emitter_grid"):
        assert getattr(a.scene, name).tobytes() == getattr(b.scene, name).tobytes(), name  # bytes: tints are NaN patterns
