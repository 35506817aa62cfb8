"""Chunk-origin rebasing (the precision form's option: Params.see_through[2] = 1), on the CPU.

* `lw_rebase_camera` (the library's f64 camera set-up) against its statement: the chunk corner
  nearest the eye, 16 * rint(eye / 16) per axis with ties to even, the remainder rounded once to
  f32, the corner packed as see_through[3] says; refused for a non-finite eye or one outside the
  packed range.
* The oracle's rebase step (kernel_impl.h `rebase`, the kernels' `rebase` restated) against the
  same statement on seeded positions of every magnitude: the moved position is x - 16 k exactly
  (checked in f64), within 8 blocks of its corner unless the corner range is exhausted.
* Whole samples of the FP32 oracle in chunk frames against the grid's frame and the FP64 twin on a
  crop of the C1 frame: the camera moved into chunk frames changes no path there (coordinates below
  64 blocks), so the samples agree within 1e-4 relative, and sit as close to the FP64 samples.
"""

import numpy as np
import pytest

from lumenwright_b200 import layout as L
from lumenwright_b200 import native as N
from lumenwright_b200 import request as R
from oracle import oracle as O

F32 = np.float32
LIMITS = ((-1024, 1023), (-512, 511), (-1024, 1023))


def unpack(word):
    w = int(word)
    x = (w & 0x7FF) - ((w & 0x400) << 1)
    y = ((w >> 11) & 0x3FF) - (((w >> 11) & 0x200) << 1)
    z = ((w >> 21) & 0x7FF) - (((w >> 21) & 0x400) << 1)
    return x, y, z


def pack(k):
    return (k[0] & 0x7FF) | ((k[1] & 0x3FF) << 11) | ((k[2] & 0x7FF) << 21)


def test_rebase_camera_is_the_nearest_chunk_corner():
    rng = np.random.default_rng(5)
    eyes = [(256.37, 56.61, 256.29), (8.0, 24.0, -8.0), (-0.0, 0.0, 7.999999), (-16384.0, -8192.0, 16360.0)]
    eyes += [tuple(v) for v in rng.uniform(-4000.0, 4000.0, (200, 3))]
    eyes += [tuple(v) for v in rng.uniform(-2.0, 2.0, (50, 3))]
    for eye in eyes:
        p = N.rebase_camera(L.new_params(), eye)
        k = [int(np.rint(e / 16.0)) for e in eye]  # ties to even, as the library rounds
        want = [F32(e - 16.0 * c) for e, c in zip(eye, k)]
        assert list(p["cam_pos"][:3]) == want, (eye, p["cam_pos"])
        assert all(abs(float(v)) <= 8.0 for v in want)
        assert int(p["see_through"][2]) == 1
        assert unpack(p["see_through"][3]) == tuple(k)
        assert int(p["see_through"][3]) == pack(k)
    # ties go to the even chunk: 8 -> 0, 24 -> 2, -8 -> 0, -24 -> -2
    p = N.rebase_camera(L.new_params(), (8.0, 24.0, -24.0))
    assert unpack(p["see_through"][3]) == (0, 2, -2)
    assert list(p["cam_pos"][:3]) == [F32(8.0), F32(-8.0), F32(8.0)]


@pytest.mark.parametrize("eye", [(float("nan"), 0.0, 0.0), (0.0, float("inf"), 0.0), (16.0 * 1024 - 7.0, 0.0, 0.0),
                                 (0.0, -16.0 * 513, 0.0), (0.0, 0.0, 1e300)])
def test_rebase_camera_refuses_what_it_cannot_pack(eye):
    with pytest.raises(N.LwError) as e:
        N.rebase_camera(L.new_params(), eye)
    assert e.value.status == 1


def test_the_rebase_step_is_exact():
    rng = np.random.default_rng(11)
    checked = 0
    for scale in (1e-3, 1.0, 7.9, 8.0, 9.0, 100.0, 3000.0, 1e5, 1e7):
        xs = (rng.uniform(-1.0, 1.0, (300, 3)) * scale).astype(F32)
        words = [pack((int(a), int(b), int(c))) for a, b, c in
                 zip(rng.integers(-40, 40, 300), rng.integers(-20, 20, 300), rng.integers(-40, 40, 300))]
        for x, w in zip(xs, words):
            got, w2 = O.rebase(x, w)
            c0, c1 = np.array(unpack(w)), np.array(unpack(w2))
            for a in range(3):
                k = int(np.clip(np.rint(np.float64(F32(x[a] * F32(0.0625)))), -4096, 4096))
                lo, hi = LIMITS[a]
                assert c1[a] == min(max(c0[a] + k, lo), hi)
                # exact: the f32 result is the f64 difference
                assert np.float64(got[a]) == np.float64(x[a]) - 16.0 * float(c1[a] - c0[a]), (x, w, got)
                if c1[a] == c0[a] + k:
                    assert abs(float(got[a])) <= 8.0
            checked += 1
    assert checked == 2700
    # a non-finite coordinate leaves the frame at the bottom of the range on that axis
    got, w2 = O.rebase(np.array([np.nan, 0.0, np.inf], F32), 0)
    assert unpack(w2) == (-1024, 0, 1023) and np.isnan(got[0]) and got[2] == np.inf


class OracleSky:
    """Sky inputs through the oracle."""

    def build_sky_cache(self, params, n):
        return O.OracleScene(params, None, None, None, None, None, None).build_sky_cache(n)

    def blend_chunky_sky(self, params, cache, maps, sizes, weight):
        return maps

    def draw_sky_map(self, quick_sky, stars, w, h, atlas, atlas_w):
        return np.full((h, w, 3), 0.1, np.float32)


def test_oracle_samples_in_chunk_frames_follow_the_grid_frame():
    frame = R.make_frame(R.CONFIGS["c1"], sky_backend=OracleSky(), spp=4)
    framed = R.with_chunk_frames(frame)
    assert int(framed.params["see_through"][2]) == 1
    x0, y0, w, h, n = 96, 54, 32, 24, 4
    grid = O.OracleScene.from_frame(frame).render_samples(x0, y0, w, h, 0, n)
    chunk = O.OracleScene.from_frame(framed).render_samples(x0, y0, w, h, 0, n)
    v64 = O.OracleScene.from_frame(frame)
    cam = O.Camera64(tuple(frame.eye64), tuple(float(v) for v in frame.params["cam_fwd"][:3]),
                     tuple(float(v) for v in frame.params["cam_right"][:3]),
                     tuple(float(v) for v in frame.params["cam_up"][:3]), float(frame.params["cam_pos"][3]),
                     float(frame.params["cam_fwd"][3]))
    ref = np.array([[[v64.render_sample64(x0 + x, y0 + y, k, cam=cam) for k in range(n)] for x in range(w)]
                    for y in range(h)])

    def within(a, b, rel=1e-4):
        return np.all(np.abs(a - b) <= rel * np.maximum(np.abs(a), np.abs(b)) + 1e-6, axis=-1)

    same = within(chunk, grid).mean()
    near_grid, near_chunk = within(grid, ref).mean(), within(chunk, ref).mean()
    print(f"C1 crop: {same:.5f} of samples agree between the frames; within 1e-4 of FP64: grid {near_grid:.5f}, "
          f"chunk {near_chunk:.5f}")
    assert same >= 0.999
    assert near_chunk >= near_grid - 1e-3
    assert O.bounds_errors() == 0
