"""The synthetic block set as a resource jar (`lumenwright_b200/jar.py`): the entries the
reference's asset loader looks up, textures that decode (with PIL, a decoder of its own) to the
seeded texels, colormaps that sample to the set's tints by the reference's climate lookup
(crates/lumenwright/src/assets/biome.rs:141-151), and models whose elements give the quads the
synthetic set builds its scenes from.
"""

import io
import json
import zipfile

import numpy as np
import pytest

from lumenwright_b200 import anvil as AN
from lumenwright_b200 import jar as J
from lumenwright_b200 import layout as L
from lumenwright_b200 import synth as S

PIL = pytest.importorskip("PIL.Image")


@pytest.fixture(scope="module")
def jar(tmp_path_factory):
    path = tmp_path_factory.mktemp("jar") / "synthetic.jar"
    names = J.write_jar(str(path), seed=1)
    with zipfile.ZipFile(path) as z:
        yield {n: z.read(n) for n in names}, path


def test_same_seed_same_bytes(jar, tmp_path):
    _, path = jar
    again = tmp_path / "again.jar"
    J.write_jar(str(again), seed=1)
    assert again.read_bytes() == path.read_bytes()
    other = tmp_path / "other.jar"
    J.write_jar(str(other), seed=2)
    assert other.read_bytes() != path.read_bytes()


def test_textures_decode_to_the_seeded_texels(jar):
    entries, _ = jar
    for name in S.TEXTURES + ["sun"]:
        key = ("assets/minecraft/textures/environment/celestial/sun.png" if name == "sun"
               else f"assets/minecraft/textures/block/{name}.png")
        want = S._texture(name, 1, 32 if name == "sun" else 16)
        img = np.asarray(PIL.open(io.BytesIO(entries[key])).convert("RGBA")).astype(np.uint32)
        got = img[..., 0] | (img[..., 1] << 8) | (img[..., 2] << 16) | (img[..., 3] << 24)
        assert np.array_equal(got, want), name
        assert np.array_equal(J.read_texture(entries[key]), want), name


def colormap_sample(px, temperature, downfall):
    # biome.rs:141-151: x from the clamped temperature, y from downfall times temperature
    t = min(max(temperature, 0.0), 1.0)
    d = min(max(downfall, 0.0), 1.0) * t
    x, y = int((1.0 - t) * 255.0), int((1.0 - d) * 255.0)
    p = int(px[y, x])
    return ((p & 0xFF) << 16) | (((p >> 8) & 0xFF) << 8) | ((p >> 16) & 0xFF)


def test_colormaps_sample_to_the_sets_tints(jar):
    entries, _ = jar
    hexrgb = lambda c: (c[0] << 16) | (c[1] << 8) | c[2]  # noqa: E731
    for name, tint in (("grass", S.GRASS_TINT), ("foliage", S.FOLIAGE_TINT)):
        px = J.read_texture(entries[f"assets/minecraft/textures/colormap/{name}.png"])
        assert px.shape == (256, 256)
        for t, d in ((0.8, 0.4), (0.0, 0.0), (1.0, 1.0), (2.0, -1.0), (0.5, 0.9)):  # plains first
            assert colormap_sample(px, t, d) == hexrgb(tint)


def test_every_block_of_the_saves_has_a_blockstate_and_its_model_resolves(jar):
    entries, _ = jar
    for sid, (name, props) in AN.STATES.items():
        if sid == S.AIR:
            continue
        short = name.split(":")[1]
        bs = json.loads(entries[f"assets/minecraft/blockstates/{short}.json"])
        (key, variant), = bs["variants"].items()
        assert key == ""  # the empty key matches every state (blockstate.rs:103-113)
        loc = variant["model"].split(":")[1]
        model = json.loads(entries[f"assets/minecraft/models/{loc}.json"])
        for el in model.get("elements", []):
            for face in el["faces"].values():
                tex = model["textures"][face["texture"][1:]]
                assert f"assets/minecraft/textures/{tex.split(':')[1]}.png" in entries


MODEL_OF = {S.STONE: "stone", S.DIRT: "dirt", S.GRASS: "grass_block", S.LOG: "oak_log", S.LEAVES: "oak_leaves",
            S.LANTERN: "lantern", S.GLOWSTONE: "glowstone"}
DIR_OF = {v: k for k, v in J.FACE_NAME.items()}


@pytest.mark.parametrize("state", sorted(MODEL_OF))
def test_model_elements_give_the_sets_quads(state):
    # Each element face at its position (uv from the position where the model gives none), its
    # texture variable resolved and its tint index mapped to the block's tint, against the quads
    # `synth.block_quads` builds the scenes from: the same geometry, texture rectangle and tint,
    # in the same order (flags and emittance are the block's, not the model's).
    atlas = S.build_atlas(1)
    model = J.block_models()[MODEL_OF[state]]
    tint = {S.GRASS: S.GRASS_TINT, S.LEAVES: S.FOLIAGE_TINT}.get(state)
    got = []
    for el in model["elements"]:
        box = (tuple(v / 16.0 for v in el["from"]), tuple(v / 16.0 for v in el["to"]))
        for fname, face in el["faces"].items():
            p0, eu, ev, uv = S.face(box, DIR_OF[fname])
            tex = model["textures"][face["texture"][1:]].split("/")[-1]
            t = tint if face.get("tintindex", -1) == 0 else None
            got.append(S.resolve(atlas, p0, eu, ev, tex, uv, 0, t))
    want = S.block_quads(atlas, state)
    assert len(got) == len(want)
    keep = np.ones(20, bool)
    keep[[3, 11]] = False
    for g, w in zip(got, want):
        assert np.array_equal(np.asarray(g)[keep], np.asarray(w)[keep])
    assert L.quads_array(got).size == len(want)
