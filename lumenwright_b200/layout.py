"""The flat scene layout of the hq path tracer, as numpy dtypes.

Restates the `#[repr(C)]` records of the reference kernel crate
(`crates/lumenwright-kernel/src/scene.rs`), byte for byte: these are the C-ABI contract
between the host and `liblumenwright_b200.so` (`include/lumenwright_b200.h` declares the
same records as C structs).

Grid buffer (u32 words) at the word offsets in ``Params.off`` / ``off2``
(`scene.rs:1-9`): ``top[nb] | bricks[n*2048] | ov_top[nb] | ov_cells[n*8192] |
ov_quads[..] | 0``.
"""

import numpy as np

# scene.rs:16-37, 144-155
EMPTY = 0xFFFF_FFFF
UNIFORM = 0x8000_0000
BRICK_WORDS = 2048
OV_CELL_WORDS = 8192
ALPHA_OPAQUE = 0
ALPHA_CUTOUT = 1
ALPHA_TRANSLUCENT = 2
FLAG_ALPHA_MASK = 3
FLAG_WATER = 1 << 2
FLAG_SHADE = 1 << 3
FLAG_FRONT_ONLY = 1 << 4
EMITTER_SAMPLING_NONE = 0
EMITTER_SAMPLING_ONE = 1
EMITTER_SAMPLING_ONE_BLOCK = 2
EMITTER_SAMPLING_ALL = 3
EMITTER_GRID_HEADER = 8

# `GpuQuad` (scene.rs:46-57), 80 bytes.
QUAD_DTYPE = np.dtype(
    [("p0", "<f4", 4), ("eu", "<f4", 4), ("ev", "<f4", 4), ("uv", "<f4", 4), ("uvt", "<f4", 4)]
)
# `GpuModel` (scene.rs:103-112), 16 bytes.
MODEL_DTYPE = np.dtype(
    [("quad_offset", "<u4"), ("quad_count", "<u4"), ("flags", "<u4"), ("pad", "<u4")]
)
# `GpuEmitter` (scene.rs:119-124), 32 bytes.
EMITTER_DTYPE = np.dtype([("pos", "<f4", 4), ("faces", "<u4", 4)])

_F4 = ("<f4", 4)
_U4 = ("<u4", 4)
# `Params` (scene.rs:160-228), 27 x vec4 = 432 bytes.
PARAMS_DTYPE = np.dtype(
    [
        ("cam_pos", *_F4), ("cam_fwd", *_F4), ("cam_right", *_F4), ("cam_up", *_F4),
        ("sun_dir", *_F4), ("sun_color", *_F4), ("sky_sun", *_F4), ("sky_zenith", *_F4),
        ("perez_a", *_F4), ("perez_b", *_F4), ("perez_c", *_F4), ("perez_d", *_F4),
        ("perez_e", *_F4), ("water_color", *_F4), ("misc_f", *_F4),
        ("grid_dims", *_U4), ("off", *_U4), ("off2", *_U4), ("frame", *_U4),
        ("misc_u", *_U4), ("see_through", *_U4), ("emitter", *_U4),
        ("sun_su", *_F4), ("sun_sv", *_F4), ("sun_sprite", *_F4), ("sky_map", *_F4),
        ("water_plane", *_F4),
    ]
)

assert QUAD_DTYPE.itemsize == 80
assert MODEL_DTYPE.itemsize == 16
assert EMITTER_DTYPE.itemsize == 32
assert PARAMS_DTYPE.itemsize == 432  # trace.rs:327-333


def f32_bits(u: int) -> float:
    """`f32::from_bits`: the float whose bit pattern is the u32 ``u``."""
    return float(np.array([u], dtype="<u4").view("<f4")[0])


def bits_f32(f: float) -> int:
    """`f32::to_bits`."""
    return int(np.array([f], dtype="<f4").view("<u4")[0])


def new_params() -> np.ndarray:
    """A zeroed `Params` record (``Params::default()``)."""
    return np.zeros((), dtype=PARAMS_DTYPE)


def make_quad(p0, eu, ev, flags=0, tint=0xFFFF_FFFF, emittance=0.0, uv=(0, 0, 0, 0), uvt=(0, 0)):
    """One `GpuQuad` packed as `Quad::to_gpu` packs it (crates/lumenwright/src/scene/mod.rs:105-129):
    flags in ``p0.w``, the RGBA8 tint in ``eu.w``, the emittance in ``ev.w``. Returned as its
    20 little-endian words; ``quads_array`` stacks them into a `GpuQuad` array."""
    w = np.zeros(20, dtype="<u4")
    f = w.view("<f4")
    f[0:3] = p0
    f[4:7] = eu
    f[8:11] = ev
    f[11] = emittance
    f[12:16] = uv
    f[16:18] = uvt
    # Bit-cast lanes are written as words so NaN patterns (tint 0xFFFFFFFF) survive.
    w[3] = flags
    w[7] = tint
    return w


def quads_array(words) -> np.ndarray:
    """Stacks quads given as 20-word arrays into a contiguous `GpuQuad` array."""
    if len(words) == 0:
        return np.zeros(0, dtype=QUAD_DTYPE)
    return np.ascontiguousarray(np.stack([np.asarray(w, dtype="<u4") for w in words])).view(QUAD_DTYPE).reshape(-1)


def quad_words(quads: np.ndarray) -> np.ndarray:
    """The (n, 20) u32 word view of a `GpuQuad` array (flags at column 3, tint at 7)."""
    return quads.view("<u4").reshape(-1, 20)
