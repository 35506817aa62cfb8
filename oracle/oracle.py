"""ctypes bindings of the CPU oracle (oracle/_build/liblw_oracle.so).

TEST INFRASTRUCTURE: the tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg load this module, as the checker or as the timed CPU baseline. The product package
``lumenwright_b200`` never imports it.

The oracle restates the reference kernel crate (`crates/lumenwright-kernel/src/`) and the CPU
backend's per-pixel loop (`crates/lumenwright/src/render/cpu/mod.rs:39-87`); see
``oracle/lw_oracle.h``.
"""

import ctypes as C
import os
import subprocess

import numpy as np

from lumenwright_b200.layout import EMITTER_DTYPE, MODEL_DTYPE, PARAMS_DTYPE, QUAD_DTYPE

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liblw_oracle.so")


def build() -> str:
    """Compiles the oracle with its Makefile (gcc; no GPU needed)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = C.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


class Scene(C.Structure):
    """`lwo_scene`: borrowed pointers and lengths (the reference's `SceneView`)."""

    _fields_ = [
        ("params", C.c_void_p),
        ("grid", C.c_void_p), ("grid_len", C.c_uint64),
        ("models", C.c_void_p), ("models_len", C.c_uint64),
        ("quads", C.c_void_p), ("quads_len", C.c_uint64),
        ("atlas", C.c_void_p), ("atlas_len", C.c_uint64),
        ("emitters", C.c_void_p), ("emitters_len", C.c_uint64),
        ("emitter_grid", C.c_void_p), ("emitter_grid_len", C.c_uint64),
        ("sky", C.c_void_p), ("sky_len", C.c_uint64),
    ]


class Hit(C.Structure):
    _fields_ = [("t", C.c_float), ("quad", C.c_uint32), ("texel", C.c_uint32), ("s", C.c_float),
                ("tt", C.c_float), ("found", C.c_int32)]


class Camera64(C.Structure):
    _fields_ = [("eye", C.c_double * 3), ("fwd", C.c_double * 3), ("right", C.c_double * 3),
                ("up", C.c_double * 3), ("tan_half", C.c_double), ("aspect", C.c_double)]


class Theta(C.Structure):
    """`lwo_theta`: parameters of the differentiable form for the FP64 build."""
    _fields_ = [("albedo", C.c_void_p), ("albedo0", C.c_void_p), ("n_params", C.c_uint32), ("frozen", C.c_int32),
                ("texel_param", C.c_void_p), ("texel_param_len", C.c_uint64), ("emit_mult", C.c_void_p),
                ("sky64", C.c_void_p), ("sky64_len", C.c_uint64), ("sun", C.c_double * 4), ("sun0", C.c_double * 4)]


def make_theta(albedo, albedo0, texel_param, emit_mult, sky64, sun, sun0, frozen=True):
    """A `Theta` and the arrays it points to (keep both alive while it is used)."""
    keep = [np.ascontiguousarray(albedo, np.float64).reshape(-1, 3), np.ascontiguousarray(albedo0, np.float64).reshape(-1, 3),
            np.ascontiguousarray(texel_param, np.int32), np.ascontiguousarray(emit_mult, np.float64),
            None if sky64 is None else np.ascontiguousarray(sky64, np.float64)]
    t = Theta(keep[0].ctypes.data, keep[1].ctypes.data, keep[0].shape[0], int(frozen), keep[2].ctypes.data,
              keep[2].size, keep[3].ctypes.data, None if keep[4] is None else keep[4].ctypes.data,
              0 if keep[4] is None else keep[4].size, (C.c_double * 4)(*sun), (C.c_double * 4)(*sun0))
    return t, keep


class Counters(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in (
        "samples", "events", "traces", "dda_steps", "brick_skips", "voxel_lookups", "model_fetches",
        "quad_tests", "texel_fetches", "overlay_reads", "sky_reads", "map_reads", "emitter_cell_reads",
        "emitter_index_reads", "emitter_reads", "bounds_errors")]

    def as_dict(self):
        return {n: int(getattr(self, n)) for n, _ in self._fields_}


F3 = C.c_float * 3
D3 = C.c_double * 3
P = C.POINTER


def _declare(L):
    sp = P(Scene)
    L.lwo32_pcg_hash.restype = C.c_uint32
    L.lwo32_pcg_hash.argtypes = [C.c_uint32]
    L.lwo32_rng_new.restype = C.c_uint32
    L.lwo32_rng_new.argtypes = [C.c_uint32] * 3
    L.lwo32_rng_next.restype = C.c_float
    L.lwo32_rng_next.argtypes = [P(C.c_uint32)]
    L.lwo32_sin_cos_turns.argtypes = [C.c_float, P(C.c_float), P(C.c_float)]
    for n in ("lwo32_acos", "lwo32_ln", "lwo32_gamma_to_linear"):
        getattr(L, n).restype = C.c_float
        getattr(L, n).argtypes = [C.c_float]
    L.lwo32_atan2.restype = C.c_float
    L.lwo32_atan2.argtypes = [C.c_float, C.c_float]
    L.lwo32_voxel.restype = C.c_uint32
    L.lwo32_voxel.argtypes = [sp, C.c_int32, C.c_int32, C.c_int32]
    L.lwo32_trace.restype = Hit
    L.lwo32_trace.argtypes = [sp, F3, F3, C.c_float, C.c_float]
    L.lwo32_see_through_hit.restype = Hit
    L.lwo32_see_through_hit.argtypes = [sp, F3, F3, C.c_float]
    L.lwo32_render_sample.argtypes = [sp, C.c_uint32, C.c_uint32, C.c_uint32, F3]
    L.lwo32_sample_emitters.argtypes = [sp, F3, F3, F3, P(C.c_uint32), F3]
    L.lwo32_emitter_cell.argtypes = [sp, F3, P(C.c_uint32), P(C.c_uint32)]
    for n in ("lwo32_preetham_radiance", "lwo32_sky_radiance", "lwo32_sky_lens", "lwo32_sky_light",
              "lwo32_sun_texture"):
        getattr(L, n).argtypes = [sp, F3, F3]
    L.lwo32_build_sky_cache.argtypes = [sp, C.c_uint32, C.c_void_p]
    L.lwo32_sky_radiance_many.argtypes = [sp, C.c_uint64, C.c_void_p, C.c_void_p]
    L.lwo32_render_samples.argtypes = [sp] + [C.c_uint32] * 6 + [C.c_void_p, C.c_int]
    L.lwo32_render_mean.argtypes = [sp] + [C.c_uint32] * 5 + [C.c_void_p, C.c_int]
    L.lwo32_count_work.argtypes = [sp] + [C.c_uint32] * 5 + [P(Counters)]
    L.lwo_bounds_errors.restype = C.c_uint64
    L.lwo64_render_sample.argtypes = [sp, P(Camera64), C.c_uint32, C.c_uint32, C.c_uint32, D3]
    L.lwo64_render_mean.argtypes = [sp, P(Camera64)] + [C.c_uint32] * 5 + [C.c_void_p, C.c_int]
    L.lwo64_render_samples.argtypes = [sp, P(Camera64)] + [C.c_uint32] * 6 + [C.c_void_p, C.c_int]
    L.lwo_tonemap.argtypes = [C.c_void_p, C.c_uint64, C.c_float, C.c_uint32, C.c_uint32, C.c_uint32, C.c_float,
                              C.c_void_p]
    L.lwo_game_tone_curve.argtypes = [C.c_void_p]
    L.lwo_mid_grey_gain.restype = C.c_double
    L.lwo_game_before_gamma.restype = C.c_double
    L.lwo_game_before_gamma.argtypes = [C.c_double]
    L.lwo64_render_mean_theta.argtypes = [sp, P(Camera64), P(Theta)] + [C.c_uint32] * 5 + [C.c_void_p, C.c_int]
    L.lwo64_render_fd_theta.argtypes = [sp, P(Camera64), P(Theta), P(Theta)] + [C.c_uint32] * 5 + \
        [C.c_void_p, C.c_void_p, C.c_int]


def _arr(a, dtype):
    a = np.ascontiguousarray(a, dtype=dtype) if a is not None else np.zeros(0, dtype=dtype)
    return a


class OracleScene:
    """The buffers one frame reads, held alive for the oracle: a `SceneView`.

    ``params`` is a `Params` record (``layout.PARAMS_DTYPE``); the others are the flat buffers.
    """

    def __init__(self, params, grid, models, quads, atlas, emitters, emitter_grid, sky=None):
        self.params = np.array(params, dtype=PARAMS_DTYPE, order="C").reshape(())
        self.grid = _arr(grid, np.uint32)
        self.models = _arr(models, MODEL_DTYPE)
        self.quads = _arr(quads, QUAD_DTYPE)
        self.atlas = _arr(atlas, np.uint32)
        self.emitters = _arr(emitters, EMITTER_DTYPE)
        self.emitter_grid = _arr(emitter_grid, np.uint32)
        self.sky = _arr(sky, np.float32)
        self._refresh()

    @classmethod
    def from_frame(cls, frame):
        """From an ``lumenwright_b200.scene.HqFrame``."""
        s = frame.scene
        return cls(frame.params, s.grid, s.models, s.quads, s.atlas, s.emitters, s.emitter_grid, frame.sky)

    def _refresh(self):
        def ptr(a):
            return a.ctypes.data if a.size else None
        self._s = Scene(self.params.ctypes.data, ptr(self.grid), self.grid.size, ptr(self.models), self.models.size,
                        ptr(self.quads), self.quads.size, ptr(self.atlas), self.atlas.size, ptr(self.emitters),
                        self.emitters.size, ptr(self.emitter_grid), self.emitter_grid.size, ptr(self.sky),
                        self.sky.size)

    def set_sky(self, sky):
        self.sky = _arr(sky, np.float32)
        self._refresh()

    @property
    def ref(self):
        return C.byref(self._s)

    # ---- single calls -----------------------------------------------------------------
    def trace(self, o, d, tmin=0.0, tmax=float("inf")):
        h = lib().lwo32_trace(self.ref, F3(*o), F3(*d), tmin, tmax)
        return h if h.found else None

    def see_through_hit(self, o, d, tmin):
        h = lib().lwo32_see_through_hit(self.ref, F3(*o), F3(*d), tmin)
        return h if h.found else None

    def voxel(self, x, y, z):
        return lib().lwo32_voxel(self.ref, x, y, z)

    def render_sample(self, px, py, sample):
        out = F3()
        lib().lwo32_render_sample(self.ref, px, py, sample, out)
        return np.array(out[:], dtype=np.float32)

    def render_sample64(self, px, py, sample, cam=None):
        out = D3()
        lib().lwo64_render_sample(self.ref, C.byref(cam) if cam is not None else None, px, py, sample, out)
        return np.array(out[:], dtype=np.float64)

    def sample_emitters(self, pos, origin, n, rng_state):
        st = C.c_uint32(rng_state)
        out = F3()
        lib().lwo32_sample_emitters(self.ref, F3(*pos), F3(*origin), F3(*n), C.byref(st), out)
        return np.array(out[:], dtype=np.float32), st.value

    def emitter_cell(self, p):
        a, b = C.c_uint32(), C.c_uint32()
        lib().lwo32_emitter_cell(self.ref, F3(*p), C.byref(a), C.byref(b))
        return a.value, b.value

    def _v3(self, name, d):
        out = F3()
        getattr(lib(), name)(self.ref, F3(*d), out)
        return np.array(out[:], dtype=np.float32)

    def preetham_radiance(self, d):
        return self._v3("lwo32_preetham_radiance", d)

    def sky_radiance(self, d):
        return self._v3("lwo32_sky_radiance", d)

    def sky_radiance_many(self, dirs):
        d = np.ascontiguousarray(dirs, np.float32).reshape(-1, 3)
        out = np.zeros_like(d)
        lib().lwo32_sky_radiance_many(self.ref, d.shape[0], d.ctypes.data, out.ctypes.data)
        return out

    def sky_lens(self, d):
        return self._v3("lwo32_sky_lens", d)

    def sky_light(self, d):
        return self._v3("lwo32_sky_light", d)

    def sun_texture(self, d):
        return self._v3("lwo32_sun_texture", d)

    def build_sky_cache(self, n):
        out = np.zeros((n + 1) * (n + 1) * 3, dtype=np.float32)
        lib().lwo32_build_sky_cache(self.ref, n, out.ctypes.data)
        return out

    # ---- whole-rectangle calls ---------------------------------------------------------
    def render_samples(self, x0, y0, w, h, sample_start, count, threads=0):
        """Per-sample radiance, shape (h, w, count, 3)."""
        out = np.zeros((h, w, count, 3), dtype=np.float32)
        lib().lwo32_render_samples(self.ref, x0, y0, w, h, sample_start, count, out.ctypes.data, threads)
        return out

    def render_mean(self, x0, y0, w, h, spp, threads=0):
        """The CPU backend's mean radiance (f64 sums / spp), shape (h, w, 3), f32."""
        out = np.zeros((h, w, 3), dtype=np.float32)
        lib().lwo32_render_mean(self.ref, x0, y0, w, h, spp, out.ctypes.data, threads)
        return out

    def render_mean64(self, x0, y0, w, h, spp, cam=None, threads=0):
        """The FP64 oracle's mean radiance, shape (h, w, 3), f64."""
        out = np.zeros((h, w, 3), dtype=np.float64)
        lib().lwo64_render_mean(self.ref, C.byref(cam) if cam is not None else None, x0, y0, w, h, spp,
                                out.ctypes.data, threads)
        return out

    def render_samples64(self, x0, y0, w, h, sample_start, count, cam=None, threads=0):
        """The FP64 oracle's per-sample radiance, shape (h, w, count, 3), f64."""
        out = np.zeros((h, w, count, 3), dtype=np.float64)
        lib().lwo64_render_samples(self.ref, C.byref(cam) if cam is not None else None, x0, y0, w, h, sample_start,
                                   count, out.ctypes.data, threads)
        return out

    def render_mean_theta(self, theta, x0, y0, w, h, spp, cam=None, threads=0):
        """The FP64 mean radiance under a `Theta`, shape (h, w, 3)."""
        out = np.zeros((h, w, 3), dtype=np.float64)
        lib().lwo64_render_mean_theta(self.ref, C.byref(cam) if cam is not None else None, C.byref(theta), x0, y0, w,
                                      h, spp, out.ctypes.data, threads)
        return out

    def render_fd_theta(self, plus, minus, x0, y0, w, h, spp, cam=None, threads=0):
        """FP64 paired differences under two `Theta`s: (mean of plus - minus, mean of midpoints)."""
        diff = np.zeros((h, w, 3), dtype=np.float64)
        mean = np.zeros((h, w, 3), dtype=np.float64)
        lib().lwo64_render_fd_theta(self.ref, C.byref(cam) if cam is not None else None, C.byref(plus),
                                    C.byref(minus), x0, y0, w, h, spp, diff.ctypes.data, mean.ctypes.data, threads)
        return diff, mean

    def count_work(self, x0, y0, w, h, spp):
        c = Counters()
        lib().lwo32_count_work(self.ref, x0, y0, w, h, spp, C.byref(c))
        return c.as_dict()


def tonemap(hdr, exposure=1.0, op=0, mix=0, op_b=0, weight=1.0):
    """post::tonemap / tonemap_mix: (n, 3) linear values to n RGBA8 words (uint32)."""
    hdr = np.ascontiguousarray(hdr, np.float32).reshape(-1, 3)
    out = np.zeros(hdr.shape[0], np.uint32)
    lib().lwo_tonemap(hdr.ctypes.data, hdr.shape[0], exposure, op, mix, op_b, weight, out.ctypes.data)
    return out


def game_tone_curve():
    out = np.zeros(7, np.float32)
    lib().lwo_game_tone_curve(out.ctypes.data)
    return out


def pcg_hash(v):
    return lib().lwo32_pcg_hash(v)


def rng_new(pixel, sample, seed):
    return lib().lwo32_rng_new(pixel, sample, seed)


def rng_next(state):
    st = C.c_uint32(state)
    r = lib().lwo32_rng_next(C.byref(st))
    return r, st.value


def sin_cos_turns(u):
    s, c = C.c_float(), C.c_float()
    lib().lwo32_sin_cos_turns(u, C.byref(s), C.byref(c))
    return s.value, c.value


def acos(x):
    return lib().lwo32_acos(x)


def atan2(y, x):
    return lib().lwo32_atan2(y, x)


def ln(x):
    return lib().lwo32_ln(x)


def gamma_to_linear(c):
    return lib().lwo32_gamma_to_linear(c)


def water_exp(x):
    """The water transmittance's exponential (lumenwright_b200/csrc/water_exp.h, the oracle's build
    of it), elementwise over f32 arguments."""
    L = lib()
    L.lwo32_water_exp.argtypes = [C.c_uint64, C.c_void_p, C.c_void_p]
    L.lwo32_water_exp.restype = None
    x = np.ascontiguousarray(x, np.float32).ravel()
    out = np.zeros_like(x)
    L.lwo32_water_exp(x.size, x.ctypes.data, out.ctypes.data)
    return out


def rebase(x, word):
    """One step of chunk-origin rebasing (kernel_impl.h `rebase`): (x moved to the frame of the chunk
    corner nearest it, that corner's frame word), for x (3 f32) held in the frame of ``word``."""
    L = lib()
    L.lwo32_rebase.argtypes = [C.c_void_p, C.POINTER(C.c_uint32)]
    L.lwo32_rebase.restype = None
    v = np.ascontiguousarray(x, np.float32).copy()
    w = C.c_uint32(int(word))
    L.lwo32_rebase(v.ctypes.data, C.byref(w))
    return v, int(w.value)


def draw_sky_map(quick_sky, stars, w, h, atlas, atlas_w, threads=0):
    """`draw_map` (sky.rs:861-878) of a packed `QuickSky` (``lumenwright_b200.gamesky``) on the host:
    (h, w, 3) linear RGB, row 0 at the nadir."""
    L = lib()
    L.lwo_draw_sky_map.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p,
                                   C.c_int]
    L.lwo_draw_sky_map.restype = None
    q = np.ascontiguousarray(quick_sky)
    atlas = np.ascontiguousarray(atlas, np.uint32)
    stars = np.ascontiguousarray(stars, np.uint32)
    out = np.zeros((h, w, 3), np.float32)
    L.lwo_draw_sky_map(q.ctypes.data, atlas.ctypes.data, atlas_w, stars.ctypes.data, w, h, out.ctypes.data, threads)
    return out


def bounds_errors():
    return lib().lwo_bounds_errors()


def reset_bounds_errors():
    lib().lwo_reset_bounds_errors()
