"""ctypes bindings of the benchmark's comparison library (``liblw_refport.so``, refport.cu): the
reference's CUDA backend ported as written, and the L2 read probe. Benchmark only: the product
package never loads it."""

import ctypes as C
import os

import numpy as np

from . import build as B

_lib = None


class Timing(C.Structure):
    _fields_ = [("kernel_ms", C.c_double), ("upload_ms", C.c_double), ("total_ms", C.c_double),
                ("launches", C.c_uint32)]


def lib():
    global _lib
    if _lib is None:
        path = B.LIB_PATH if os.path.exists(B.LIB_PATH) else B.build()
        L = C.CDLL(path)
        L.lwr_render_hq.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint32, C.c_void_p,
                                    C.POINTER(Timing)]
        L.lwr_render_hq.restype = C.c_int
        L.lwr_l2_read_gbs.argtypes = [C.c_int, C.c_uint64, C.c_uint32, C.POINTER(C.c_double)]
        L.lwr_l2_read_gbs.restype = C.c_int
        _lib = L
    return _lib


def render_hq(device, frame, spp=None):
    """The frame (an ``HqFrame``) through the ported reference backend: (image (h, w, 3), timing)."""
    from lumenwright_b200 import native as N
    from lumenwright_b200.layout import EMITTER_DTYPE, MODEL_DTYPE, QUAD_DTYPE
    s = frame.scene
    keep = [np.ascontiguousarray(s.grid, np.uint32), np.ascontiguousarray(s.models, MODEL_DTYPE),
            np.ascontiguousarray(s.quads, QUAD_DTYPE), np.ascontiguousarray(s.atlas, np.uint32),
            np.ascontiguousarray(s.emitters, EMITTER_DTYPE), np.ascontiguousarray(s.emitter_grid, np.uint32)]
    d = N.SceneDesc(*[v for a in keep for v in (a.ctypes.data, a.size)], (C.c_uint32 * 3)(*s.dims),
                    (C.c_uint32 * 5)(*s.offsets), (C.c_uint32 * 2)(*s.atlas_size))
    p = N.Context._params(frame.params)
    sky = np.ascontiguousarray(frame.sky, np.float32)
    w, h = int(p["frame"][0]), int(p["frame"][1])
    out = np.zeros((h, w, 3), np.float32)
    t = Timing()
    rc = lib().lwr_render_hq(device, C.byref(d), p.ctypes.data, sky.ctypes.data, sky.size,
                             int(spp or frame.spp), out.ctypes.data, C.byref(t))
    if rc:
        raise RuntimeError(f"lwr_render_hq failed with status {rc}")
    return out, {n: getattr(t, n) for n, _ in Timing._fields_}


def l2_read_gbs(device=0, bytes_=32 << 20, passes=200):
    """The L2 read bandwidth (GB/s) of a 32 MB buffer read 200 times over."""
    g = C.c_double()
    rc = lib().lwr_l2_read_gbs(device, bytes_, passes, C.byref(g))
    if rc:
        raise RuntimeError(f"lwr_l2_read_gbs failed with status {rc}")
    return g.value
