"""ctypes bindings of ``liblumenwright_b200.so`` (the C ABI declared in
``include/lumenwright_b200.h``) and the Python mirror of the reference's backend interface.

The library is the product: every render and every parity query runs in its CUDA kernels. There
is no fallback: without the library or a B200 these calls raise.
"""

import ctypes as C
import os

import numpy as np

from .layout import EMITTER_DTYPE, MODEL_DTYPE, PARAMS_DTYPE, QUAD_DTYPE

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "liblumenwright_b200.so")

# lw_status (include/lumenwright_b200.h)
STATUS = {
    0: "LW_OK", 1: "LW_ERR_INVALID_ARGUMENT", 2: "LW_ERR_BUFFER_LENGTH", 3: "LW_ERR_OUT_OF_MEMORY",
    4: "LW_ERR_DEVICE_TIMEOUT", 5: "LW_ERR_LAUNCH", 6: "LW_ERR_CANCELLED", 7: "LW_ERR_NO_DEVICE",
    8: "LW_ERR_NO_SCENE",
}

# Every symbol the header declares, for the load check.
EXPORTS = (
    "lw_ctx_create", "lw_ctx_destroy", "lw_last_error", "lw_stream", "lw_get_stats", "lw_cancel", "lw_mark",
    "lw_elapsed_ms", "lw_set_tuning", "lw_get_tuning",
    "lw_scene_upload", "lw_render_hq", "lw_sky_upload", "lw_clear_accumulator", "lw_render_device",
    "lw_read_accumulator", "lw_render_samples", "lw_trace_rays", "lw_voxel_lookup", "lw_build_sky_cache",
    "lw_blend_chunky_sky", "lw_render_accumulate_noalloc", "lw_batch_prepare",
    "lw_batch_run", "lw_batch_read", "lw_render_batch", "lw_adjoint_forward", "lw_adjoint_backward", "lw_adjoint_fd",
    "lw_gamma_table", "lw_tonemap_rgba", "lw_read_accumulator_rgba", "lw_scene_build_keys", "lw_scene_build_grid",
    "lw_scene_read", "lw_water_exp", "lw_draw_sky_map", "lw_set_timeout", "lw_render_device_shard",
    "lw_accumulator_device", "lw_rebase_camera",
)

# lw_tonemap operators (post.rs `Tonemap`)
TONEMAP_GAMMA, TONEMAP_ACES, TONEMAP_FILMIC, TONEMAP_FILMIC_MID_GREY = 0, 1, 2, 3

EMITTER_GROUPS = 32  # LW_EMITTER_GROUPS


class LwError(RuntimeError):
    """A failed library call: ``status`` is the `lw_status` code."""

    def __init__(self, status, message):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


class SceneDesc(C.Structure):
    _fields_ = [
        ("grid", C.c_void_p), ("grid_len", C.c_uint64),
        ("models", C.c_void_p), ("models_len", C.c_uint64),
        ("quads", C.c_void_p), ("quads_len", C.c_uint64),
        ("atlas", C.c_void_p), ("atlas_len", C.c_uint64),
        ("emitters", C.c_void_p), ("emitters_len", C.c_uint64),
        ("emitter_grid", C.c_void_p), ("emitter_grid_len", C.c_uint64),
        ("dims", C.c_uint32 * 3), ("offsets", C.c_uint32 * 5), ("atlas_size", C.c_uint32 * 2),
    ]


class Stats(C.Structure):
    _fields_ = [("kernel_ms", C.c_double), ("upload_ms", C.c_double), ("launches", C.c_uint32),
                ("blocks", C.c_uint32), ("threads", C.c_uint32), ("samples", C.c_uint64),
                ("trace_ms", C.c_double), ("shade_ms", C.c_double), ("trace_launches", C.c_uint32),
                ("shade_launches", C.c_uint32), ("rays", C.c_uint64)]


class Tuning(C.Structure):
    _fields_ = [("threads", C.c_uint32), ("budget", C.c_uint32), ("sub", C.c_uint32), ("engine", C.c_uint32),
                ("paths", C.c_uint32)]


ENGINE_WAVEFRONT = 0  # LW_ENGINE_WAVEFRONT
ENGINE_MEGAKERNEL = 1  # LW_ENGINE_MEGAKERNEL


class CameraJob(C.Structure):
    """`lw_camera_job`: one camera of the batched form."""
    _fields_ = [("params", C.c_uint8 * 432), ("sky", C.c_void_p), ("sky_len", C.c_uint64), ("spp", C.c_uint32),
                ("sample_start", C.c_uint32), ("out_rgb", C.c_void_p)]


class AdjFrame(C.Structure):
    """`lw_adj_frame`: a frame of the differentiable form and its parameters theta."""
    _fields_ = [("params", C.c_void_p), ("sky", C.c_void_p), ("sky_len", C.c_uint64), ("albedo", C.c_void_p),
                ("n_params", C.c_uint32), ("texel_param", C.c_void_p), ("texel_param_len", C.c_uint64),
                ("emitter_scale", C.c_void_p)]


class WorldDesc(C.Structure):
    """`lw_world_desc`."""
    _fields_ = [("blocks", C.c_void_p), ("size", C.c_uint32 * 3), ("state_flags", C.c_void_p), ("n_states", C.c_uint32)]


class InstancesDesc(C.Structure):
    """`lw_instances_desc`."""
    _fields_ = [("models", C.c_void_p), ("models_len", C.c_uint64), ("quads", C.c_void_p), ("quads_len", C.c_uint64),
                ("model_emits", C.c_void_p), ("atlas", C.c_void_p), ("atlas_len", C.c_uint64),
                ("atlas_size", C.c_uint32 * 2)]


class BuildInfo(C.Structure):
    """`lw_build_info`."""
    _fields_ = [("dims", C.c_uint32 * 3), ("offsets", C.c_uint32 * 5), ("grid_len", C.c_uint64),
                ("emitter_grid_len", C.c_uint64), ("bricks", C.c_uint32), ("uniform_bricks", C.c_uint32),
                ("buried_bricks", C.c_uint32), ("emitters", C.c_uint32), ("keys_ms", C.c_double), ("grid_ms", C.c_double)]


class ToneMap(C.Structure):
    """`lw_tonemap`."""
    _fields_ = [("exposure", C.c_float), ("op", C.c_uint32), ("mix", C.c_uint32), ("op_b", C.c_uint32),
                ("weight", C.c_float)]


class Gradient(C.Structure):
    """`lw_gradient`."""
    _fields_ = [("albedo", C.c_void_p), ("emitter_scale", C.c_void_p), ("sky", C.c_void_p),
                ("sun_dir", C.c_double * 3)]


class HitRec(C.Structure):
    _fields_ = [("t", C.c_float), ("quad", C.c_uint32), ("texel", C.c_uint32), ("s", C.c_float),
                ("tt", C.c_float), ("found", C.c_int32)]


PROGRESS_FN = C.CFUNCTYPE(None, C.c_uint32, C.c_uint32, C.c_void_p)

_lib = None


def load(path: str = LIB_PATH):
    """Loads the library (once) and declares its functions."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: run `python -m lumenwright_b200.build` (nvcc, sm_100a)")
    L = C.CDLL(path)
    P = C.c_void_p
    L.lw_ctx_create.argtypes = [C.c_int, C.POINTER(P)]
    L.lw_ctx_destroy.argtypes = [P]
    L.lw_ctx_destroy.restype = None
    L.lw_last_error.argtypes = [P]
    L.lw_last_error.restype = C.c_char_p
    L.lw_stream.argtypes = [P]
    L.lw_stream.restype = P
    L.lw_get_stats.argtypes = [P, C.POINTER(Stats)]
    L.lw_cancel.argtypes = [P]
    L.lw_cancel.restype = None
    L.lw_scene_upload.argtypes = [P, C.POINTER(SceneDesc)]
    L.lw_mark.argtypes = [P, C.c_uint32]
    L.lw_set_tuning.argtypes = [P, C.POINTER(Tuning)]
    L.lw_get_tuning.argtypes = [P, C.POINTER(Tuning)]
    L.lw_elapsed_ms.argtypes = [P, C.c_uint32, C.c_uint32, C.POINTER(C.c_double)]
    L.lw_render_hq.argtypes = [P, P, P, C.c_uint64, C.c_uint32, PROGRESS_FN, P, P]
    L.lw_sky_upload.argtypes = [P, P, C.c_uint64]
    L.lw_clear_accumulator.argtypes = [P, C.c_uint32, C.c_uint32]
    L.lw_render_device.argtypes = [P, P, C.c_uint32, C.c_uint32]
    L.lw_read_accumulator.argtypes = [P, P]
    L.lw_render_samples.argtypes = [P, P] + [C.c_uint32] * 6 + [P]
    L.lw_trace_rays.argtypes = [P, P, C.c_uint32, P, P, C.c_float, C.c_float, P]
    L.lw_voxel_lookup.argtypes = [P, C.c_uint32, P, P]
    L.lw_water_exp.argtypes = [P, C.c_uint64, P, P]
    L.lw_set_timeout.argtypes = [P, C.c_double]
    L.lw_render_device_shard.argtypes = [P, P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32]
    L.lw_accumulator_device.argtypes = [P, C.POINTER(P), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
    L.lw_draw_sky_map.argtypes = [P, P, P, C.c_uint64, P, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, P]
    L.lw_build_sky_cache.argtypes = [P, P, C.c_uint32, P]
    L.lw_render_accumulate_noalloc.argtypes = [P, P, C.c_uint32, C.c_uint32, P]
    L.lw_batch_prepare.argtypes = [P, P, C.c_uint32]
    L.lw_batch_run.argtypes = [P]
    L.lw_batch_read.argtypes = [P]
    L.lw_render_batch.argtypes = [P, P, C.c_uint32]
    L.lw_blend_chunky_sky.argtypes = [P, P, P, C.c_uint64, P, P, C.c_float]
    L.lw_adjoint_forward.argtypes = [P, C.POINTER(AdjFrame), C.c_uint32, P]
    L.lw_adjoint_backward.argtypes = [P, C.POINTER(AdjFrame), C.c_uint32, P, C.POINTER(Gradient)]
    L.lw_adjoint_fd.argtypes = [P, C.POINTER(AdjFrame), C.POINTER(AdjFrame), C.POINTER(AdjFrame), C.c_uint32, P, P]
    L.lw_gamma_table.argtypes = [P]
    L.lw_rebase_camera.argtypes = [P, C.POINTER(C.c_double)]
    L.lw_tonemap_rgba.argtypes = [P, P, C.c_uint64, C.POINTER(ToneMap), P]
    L.lw_scene_build_keys.argtypes = [P, C.POINTER(WorldDesc), P, C.c_uint32, C.POINTER(C.c_uint32)]
    L.lw_scene_build_grid.argtypes = [P, C.POINTER(WorldDesc), C.POINTER(InstancesDesc), C.POINTER(BuildInfo)]
    L.lw_scene_read.argtypes = [P, P, C.c_uint64, P, C.c_uint64, P, C.c_uint64]
    L.lw_read_accumulator_rgba.argtypes = [P, C.POINTER(ToneMap), P, P]
    for name in EXPORTS:
        if name not in ("lw_ctx_destroy", "lw_last_error", "lw_stream", "lw_cancel"):
            getattr(L, name).restype = C.c_int
    _lib = L
    return L


def _ptr(a):
    return a.ctypes.data if a is not None and a.size else None


def gamma_table() -> np.ndarray:
    """The byte-to-linear table the kernels decode texels with (256 floats)."""
    out = np.zeros(256, np.float32)
    st = load().lw_gamma_table(out.ctypes.data)
    if st:
        raise LwError(st, "lw_gamma_table")
    return out


def rebase_camera(params: np.ndarray, eye64) -> np.ndarray:
    """Chunk-origin rebasing of a frame's camera (`lw_rebase_camera`, on the host in f64): a copy
    of ``params`` whose ``cam_pos.xyz`` is the eye relative to the chunk corner nearest it and whose
    ``see_through[2:4]`` switch the kernels to chunk frames from that corner. ``eye64`` is the eye
    relative to the grid origin, in f64 (request.rs:640-644 rebases it from the world)."""
    p = np.array(params, copy=True)
    e = (C.c_double * 3)(*[float(v) for v in eye64])
    st = load().lw_rebase_camera(p.ctypes.data, e)
    if st:
        raise LwError(st, f"lw_rebase_camera: eye {tuple(eye64)}")
    return p


class Context:
    """An `lw_ctx`: one CUDA device with its streams, its resident scene and its buffers."""

    def __init__(self, device: int = 0):
        self.L = load()
        h = C.c_void_p()
        st = self.L.lw_ctx_create(device, C.byref(h))
        if st != 0:
            raise LwError(st, self.L.lw_last_error(None).decode())
        self.h = h
        self.device = device
        self._keep = []

    def close(self):
        if getattr(self, "h", None):
            self.L.lw_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != 0:
            raise LwError(st, self.L.lw_last_error(self.h).decode())

    @property
    def stream(self) -> int:
        return self.L.lw_stream(self.h) or 0

    def stats(self) -> dict:
        s = Stats()
        self._check(self.L.lw_get_stats(self.h, C.byref(s)))
        return {n: getattr(s, n) for n, _ in Stats._fields_}

    def cancel(self):
        self.L.lw_cancel(self.h)

    def set_timeout(self, seconds: float):
        """A deadline for every wait on the GPU's work (0: none); past it a call returns
        LW_ERR_DEVICE_TIMEOUT after stopping its kernels."""
        self._check(self.L.lw_set_timeout(self.h, float(seconds)))

    def set_tuning(self, threads=None, budget=None, sub=None, engine=None, paths=None):
        """Launch tuning of the render (see `lw_tuning`); the knobs not given keep their values."""
        t = self.get_tuning()
        for k, v in (("threads", threads), ("budget", budget), ("sub", sub), ("engine", engine), ("paths", paths)):
            if v is not None:
                t[k] = int(v)
        self._check(self.L.lw_set_tuning(self.h, C.byref(Tuning(**t))))

    def get_tuning(self) -> dict:
        t = Tuning()
        self._check(self.L.lw_get_tuning(self.h, C.byref(t)))
        return {"threads": t.threads, "budget": t.budget, "sub": t.sub, "engine": t.engine, "paths": t.paths}

    def mark(self, slot: int):
        """Records a CUDA event on the context's stream."""
        self._check(self.L.lw_mark(self.h, slot))

    def elapsed(self, a: int, b: int) -> float:
        """Milliseconds between two marks, by the device's clock."""
        ms = C.c_double()
        self._check(self.L.lw_elapsed_ms(self.h, a, b, C.byref(ms)))
        return ms.value

    def upload_scene(self, grid, models, quads, atlas, emitters, emitter_grid, dims, offsets, atlas_size):
        grid = np.ascontiguousarray(grid, np.uint32)
        models = np.ascontiguousarray(models, MODEL_DTYPE)
        quads = np.ascontiguousarray(quads, QUAD_DTYPE)
        atlas = np.ascontiguousarray(atlas, np.uint32)
        emitters = np.ascontiguousarray(emitters, EMITTER_DTYPE)
        emitter_grid = np.ascontiguousarray(emitter_grid, np.uint32)
        d = SceneDesc(_ptr(grid), grid.size, _ptr(models), models.size, _ptr(quads), quads.size, _ptr(atlas),
                      atlas.size, _ptr(emitters), emitters.size, _ptr(emitter_grid), emitter_grid.size,
                      (C.c_uint32 * 3)(*dims), (C.c_uint32 * 5)(*offsets), (C.c_uint32 * 2)(*atlas_size))
        self._check(self.L.lw_scene_upload(self.h, C.byref(d)))

    def upload_buffers(self, params, grid, models, quads, atlas, emitters, emitter_grid):
        """Uploads a scene described by flat buffers and the offsets in its `Params`."""
        p = np.asarray(params, dtype=PARAMS_DTYPE).reshape(())
        dims = [int(v) for v in p["grid_dims"][:3]]
        off = [int(v) for v in p["off"]] + [int(p["off2"][0])]
        self.upload_scene(grid, models, quads, atlas, emitters, emitter_grid, dims, off,
                          (int(p["off2"][1]), int(p["off2"][2])))

    def upload_hq_scene(self, s):
        """Uploads an ``HqScene``."""
        self.upload_scene(s.grid, s.models, s.quads, s.atlas, s.emitters, s.emitter_grid, s.dims, s.offsets,
                          s.atlas_size)

    @staticmethod
    def _params(params):
        return np.array(params, dtype=PARAMS_DTYPE, order="C").reshape(())

    def render_hq(self, params, sky, spp, progress=None):
        """`Backend::render_hq` on the uploaded scene: mean linear radiance, shape (h, w, 3)."""
        p = self._params(params)
        sky = np.ascontiguousarray(sky if sky is not None else np.zeros(0), np.float32)
        w, h = int(p["frame"][0]), int(p["frame"][1])
        out = np.zeros((h, w, 3), np.float32)
        cb = PROGRESS_FN((lambda d, t, u: progress(d, t)) if progress else (lambda d, t, u: None))
        self._check(self.L.lw_render_hq(self.h, p.ctypes.data, _ptr(sky), sky.size, spp, cb, None, out.ctypes.data))
        return out

    def upload_sky(self, sky):
        sky = np.ascontiguousarray(sky if sky is not None else np.zeros(0), np.float32)
        self._check(self.L.lw_sky_upload(self.h, _ptr(sky), sky.size))

    def clear_accumulator(self, w, h):
        self._check(self.L.lw_clear_accumulator(self.h, w, h))

    def render_device(self, params, sample_start, spp):
        p = self._params(params)
        self._keep = [p]
        self._check(self.L.lw_render_device(self.h, p.ctypes.data, sample_start, spp))

    def render_device_shard(self, params, sample_start, spp, shard, shards):
        """Samples of the frame's tiles shard, shard + shards, ... added to the accumulator."""
        p = self._params(params)
        self._keep = [p]
        self._check(self.L.lw_render_device_shard(self.h, p.ctypes.data, sample_start, spp, shard, shards))

    def accumulator_device(self):
        """(device address, width, height) of the context's accumulator records (8 floats each)."""
        ptr, w, h = C.c_void_p(), C.c_uint32(), C.c_uint32()
        self._check(self.L.lw_accumulator_device(self.h, C.byref(ptr), C.byref(w), C.byref(h)))
        return ptr.value, w.value, h.value

    def render_accumulate_noalloc(self, params, sample_start, spp, accum_device_ptr: int):
        """Adds samples to a caller-owned device accumulator (w*h records of 8 floats) without
        allocating; queued on the context's stream."""
        p = self._params(params)
        self._keep = [p]
        self._check(self.L.lw_render_accumulate_noalloc(self.h, p.ctypes.data, sample_start, spp,
                                                         C.c_void_p(accum_device_ptr)))

    def batch_prepare(self, jobs):
        """The batched form: ``jobs`` is a list of (params, sky, spp[, sample_start]); returns the
        output images (h, w, 3) that lw_batch_read fills."""
        arr = (CameraJob * len(jobs))()
        keep, outs = [], []
        for i, jb in enumerate(jobs):
            params, sky, spp = jb[0], jb[1], jb[2]
            start = jb[3] if len(jb) > 3 else 0
            p = self._params(params)
            sky = np.ascontiguousarray(sky if sky is not None else np.zeros(0), np.float32)
            w, h = int(p["frame"][0]), int(p["frame"][1])
            out = np.zeros((h, w, 3), np.float32)
            C.memmove(arr[i].params, p.ctypes.data, 432)
            arr[i].sky = _ptr(sky)
            arr[i].sky_len = sky.size
            arr[i].spp = spp
            arr[i].sample_start = start
            arr[i].out_rgb = out.ctypes.data
            keep += [p, sky, out]
            outs.append(out)
        self._batch_keep = (arr, keep)
        self._check(self.L.lw_batch_prepare(self.h, C.cast(arr, C.c_void_p), len(jobs)))
        return outs

    def batch_run(self):
        self._check(self.L.lw_batch_run(self.h))

    def batch_read(self):
        self._check(self.L.lw_batch_read(self.h))

    def tonemap_rgba(self, hdr, exposure=1.0, op=TONEMAP_GAMMA, mix=0, op_b=TONEMAP_GAMMA, weight=1.0):
        """post::tonemap / tonemap_mix on the device: (n, 3) linear values to n RGBA8 words."""
        hdr = np.ascontiguousarray(hdr, np.float32).reshape(-1, 3)
        out = np.zeros(hdr.shape[0], np.uint32)
        tm = ToneMap(exposure, op, mix, op_b, weight)
        self._check(self.L.lw_tonemap_rgba(self.h, hdr.ctypes.data, hdr.shape[0], C.byref(tm), out.ctypes.data))
        return out

    def read_accumulator_rgba(self, w, h, exposure=1.0, op=TONEMAP_GAMMA, mix=0, op_b=TONEMAP_GAMMA, weight=1.0,
                              with_hdr=False):
        """The last render's image as RGBA8 words (h, w), tone-mapped on the device in the pass that
        divides the sums; with ``with_hdr`` also the linear means (h, w, 3)."""
        out = np.zeros((h, w), np.uint32)
        hdr = np.zeros((h, w, 3), np.float32) if with_hdr else None
        tm = ToneMap(exposure, op, mix, op_b, weight)
        self._check(self.L.lw_read_accumulator_rgba(self.h, C.byref(tm), out.ctypes.data,
                                                    hdr.ctypes.data if with_hdr else None))
        return (out, hdr) if with_hdr else out

    def read_accumulator(self, w, h):
        out = np.zeros((h, w, 3), np.float32)
        self._check(self.L.lw_read_accumulator(self.h, out.ctypes.data))
        return out

    def render_samples(self, params, x0, y0, w, h, sample_start, count):
        """Per-sample radiance, shape (h, w, count, 3)."""
        p = self._params(params)
        out = np.zeros((h, w, count, 3), np.float32)
        self._check(self.L.lw_render_samples(self.h, p.ctypes.data, x0, y0, w, h, sample_start, count,
                                             out.ctypes.data))
        return out

    def trace_rays(self, params, o, d, tmin=0.0, tmax=float("inf")):
        p = self._params(params)
        o = np.ascontiguousarray(o, np.float32).reshape(-1, 3)
        d = np.ascontiguousarray(d, np.float32).reshape(-1, 3)
        n = o.shape[0]
        out = (HitRec * n)()
        self._check(self.L.lw_trace_rays(self.h, p.ctypes.data, n, o.ctypes.data, d.ctypes.data, tmin, tmax,
                                         C.cast(out, C.c_void_p)))
        return [h if h.found else None for h in out]

    def build_sky_cache(self, params, n):
        """Chunky's sky cache at resolution n, built on the device."""
        p = self._params(params)
        out = np.zeros((n + 1) * (n + 1) * 3, np.float32)
        self._check(self.L.lw_build_sky_cache(self.h, p.ctypes.data, n, out.ctypes.data))
        return out

    def draw_sky_map(self, quick_sky, stars, w, h, atlas, atlas_w):
        """`draw_map` (sky.rs:861-878) of a packed `QuickSky` (``gamesky.QUICK_SKY_DTYPE``) on the
        device: (h, w, 3) linear RGB, row 0 at the nadir."""
        q = np.ascontiguousarray(quick_sky)
        stars = np.ascontiguousarray(stars, np.uint32)
        atlas = np.ascontiguousarray(atlas, np.uint32)
        out = np.zeros((h, w, 3), np.float32)
        self._check(self.L.lw_draw_sky_map(self.h, q.ctypes.data, stars.ctypes.data, stars.size, atlas.ctypes.data,
                                           atlas.size, atlas_w, w, h, out.ctypes.data))
        return out

    def blend_chunky_sky(self, params, cache, maps, sizes, weight):
        """Chunky's sky blended into the game sky's maps, on the device; returns the new maps."""
        p = self._params(params)
        cache = np.ascontiguousarray(cache, np.float32)
        out = np.ascontiguousarray(maps, np.float32).copy()
        sz = np.ascontiguousarray(sizes, np.float32)
        self._check(self.L.lw_blend_chunky_sky(self.h, p.ctypes.data, cache.ctypes.data, cache.size, out.ctypes.data,
                                               sz.ctypes.data, float(weight)))
        return out

    # ---- the differentiable form --------------------------------------------------------------
    def _adj_frame(self, params, sky, albedo, texel_param, emitter_scale):
        """An `lw_adj_frame` and the arrays it points to (kept alive by the caller)."""
        p = self._params(params)
        sky = np.ascontiguousarray(sky, np.float32)
        albedo = np.ascontiguousarray(albedo, np.float32).reshape(-1, 3)
        tp = np.ascontiguousarray(texel_param, np.int32)
        es = np.ascontiguousarray(emitter_scale, np.float32)
        if es.size != EMITTER_GROUPS:
            raise ValueError(f"{EMITTER_GROUPS} emitter group intensities expected, {es.size} given")
        f = AdjFrame(p.ctypes.data, _ptr(sky), sky.size, _ptr(albedo), albedo.shape[0], _ptr(tp), tp.size,
                     es.ctypes.data)
        return f, (p, sky, albedo, tp, es)

    def adjoint_forward(self, params, sky, albedo, texel_param, emitter_scale, spp):
        """The mean radiance under theta, FP64, shape (h, w, 3)."""
        f, keep = self._adj_frame(params, sky, albedo, texel_param, emitter_scale)
        w, h = int(keep[0]["frame"][0]), int(keep[0]["frame"][1])
        out = np.zeros((h, w, 3), np.float64)
        self._check(self.L.lw_adjoint_forward(self.h, C.byref(f), spp, out.ctypes.data))
        return out

    def adjoint_backward(self, params, sky, albedo, texel_param, emitter_scale, spp, d_rgb):
        """d loss / d theta for d loss / d image = ``d_rgb``: a dict with ``albedo`` (n, 3),
        ``emitter_scale`` (32), ``sky`` (per sky float) and ``sun_dir`` (3)."""
        f, keep = self._adj_frame(params, sky, albedo, texel_param, emitter_scale)
        d = np.ascontiguousarray(d_rgb, np.float64)
        ga = np.zeros((keep[2].shape[0], 3), np.float64)
        ge = np.zeros(EMITTER_GROUPS, np.float64)
        gs = np.zeros(keep[1].size, np.float64)
        g = Gradient(_ptr(ga), ge.ctypes.data, _ptr(gs))
        self._check(self.L.lw_adjoint_backward(self.h, C.byref(f), spp, d.ctypes.data, C.byref(g)))
        return {"albedo": ga, "emitter_scale": ge, "sky": gs, "sun_dir": np.array(list(g.sun_dir))}

    def adjoint_fd(self, plus, minus, nominal, spp):
        """Paired finite differences; ``plus``, ``minus``, ``nominal`` are (params, sky, albedo,
        texel_param, emitter_scale). Returns (mean of plus - minus, mean of the midpoints), each
        shape (h, w, 3), FP64."""
        fp, kp = self._adj_frame(*plus)
        fm, km = self._adj_frame(*minus)
        f0, k0 = self._adj_frame(*nominal)
        w, h = int(kp[0]["frame"][0]), int(kp[0]["frame"][1])
        diff = np.zeros((h, w, 3), np.float64)
        mean = np.zeros((h, w, 3), np.float64)
        self._check(self.L.lw_adjoint_fd(self.h, C.byref(fp), C.byref(fm), C.byref(f0), spp, diff.ctypes.data,
                                         mean.ctypes.data))
        return diff, mean

    # ---- the grid build on the device -------------------------------------------------------
    def _world(self, blocks, state_flags):
        blocks = np.ascontiguousarray(blocks, np.uint16)
        flags = np.ascontiguousarray(state_flags, np.uint8)
        Y, Z, X = blocks.shape
        return WorldDesc(blocks.ctypes.data, (C.c_uint32 * 3)(X, Y, Z), flags.ctypes.data, flags.size), (blocks, flags)

    def scene_build_keys(self, blocks, state_flags):
        """Phase 1 of the device grid build: the model-instance keys of ``blocks`` ((y, z, x) states)
        in the order the build interns them."""
        w, keep = self._world(blocks, state_flags)
        n = C.c_uint32()
        self._check(self.L.lw_scene_build_keys(self.h, C.byref(w), None, 0, C.byref(n)))
        out = np.zeros(max(1, n.value), np.uint32)
        self._check(self.L.lw_scene_build_keys(self.h, C.byref(w), out.ctypes.data, out.size, C.byref(n)))
        return out[:n.value]

    def scene_build_grid(self, blocks, state_flags, models, quads, model_emits, atlas, atlas_size):
        """Phase 2: the grid, emitters and emitter grid on the device, installed as the scene."""
        w, keep = self._world(blocks, state_flags)
        models = np.ascontiguousarray(models, MODEL_DTYPE)
        quads = np.ascontiguousarray(quads, QUAD_DTYPE)
        emits = np.ascontiguousarray(model_emits, np.uint8)
        atlas = np.ascontiguousarray(atlas, np.uint32)
        d = InstancesDesc(models.ctypes.data, models.size, quads.ctypes.data, quads.size, emits.ctypes.data,
                          atlas.ctypes.data, atlas.size, (C.c_uint32 * 2)(*atlas_size))
        info = BuildInfo()
        self._check(self.L.lw_scene_build_grid(self.h, C.byref(w), C.byref(d), C.byref(info)))
        return info

    def scene_read(self, grid_len, emitters_len, emitter_grid_len):
        """The context's scene buffers: (grid, emitters, emitter grid)."""
        from .layout import EMITTER_DTYPE
        grid = np.zeros(grid_len, np.uint32)
        em = np.zeros(emitters_len, EMITTER_DTYPE)
        eg = np.zeros(emitter_grid_len, np.uint32)
        self._check(self.L.lw_scene_read(self.h, grid.ctypes.data, grid.size, em.ctypes.data, em.size, eg.ctypes.data,
                                         eg.size))
        return grid, em, eg

    def water_exp(self, x):
        """The kernels' exponential of the water transmittance, exp(x) rounded to f32, per element."""
        x = np.ascontiguousarray(x, np.float32).ravel()
        out = np.zeros_like(x)
        self._check(self.L.lw_water_exp(self.h, x.size, x.ctypes.data, out.ctypes.data))
        return out

    def voxel_lookup(self, xyz):
        xyz = np.ascontiguousarray(xyz, np.int32).reshape(-1, 3)
        out = np.zeros(xyz.shape[0], np.uint32)
        self._check(self.L.lw_voxel_lookup(self.h, xyz.shape[0], xyz.ctypes.data, out.ctypes.data))
        return out


# ---- the reference's backend interface (crates/lumenwright/src/render/mod.rs:35-159) ----------

class BackendKind:
    """`BackendKind` (render/mod.rs:35-51) with the B200 backend added. Only `B200` is built
    here: the other kinds are the reference's own backends."""

    Auto = "auto"
    Cpu = "cpu"
    Cuda = "cuda"
    B200 = "b200"


class B200Backend:
    """A `Backend` (render/mod.rs:92-103) whose hq mode runs this library's kernels: the drop-in
    for `CudaBackend` (crates/lumenwright/src/render/cuda.rs)."""

    def __init__(self, device: int = 0):
        self.ctx = Context(device)

    def name(self) -> str:
        return f"b200 device {self.ctx.device} (cuda, sm_100a)"

    def render_quick(self, frame):
        raise NotImplementedError("quick mode is not part of this library; the reference's CPU rasterizer draws it")

    def render_hq(self, frame, progress=None) -> np.ndarray:
        """Mean linear radiance per pixel, row-major from the top row, as (w*h, 3) float32
        (the reference's `Vec<[f32; 3]>`). The scene is copied to the device for every frame, as
        `CudaBackend` copies it (cuda.rs:96-111): a cache keyed by the scene object's identity
        would draw a new scene at a reused address, or one changed in place, from stale buffers,
        and a content hash of the scene takes longer than its copy."""
        self.ctx.upload_hq_scene(frame.scene)
        img = self.ctx.render_hq(frame.params, frame.sky, max(int(frame.spp), 1), progress)
        return img.reshape(-1, 3)


def open_backend(kind=BackendKind.B200, device: int = 0):
    """`open_backend` (render/mod.rs:115-159) for the kind this library adds. A named backend
    that is unavailable is an error, as in the reference: nothing falls back to the CPU."""
    if kind in (BackendKind.B200, BackendKind.Cuda):
        return B200Backend(device)
    raise ValueError(f"backend {kind!r} is not provided by lumenwright_b200")
