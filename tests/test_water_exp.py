"""The exponential of the water transmittance (`lumenwright_b200/csrc/water_exp.h`), which the CUDA
kernels and the FP32 oracle both call: exp(x) rounded to the nearest f32, from Cody and Waite's
argument reduction and a degree-13 Taylor series in double.

Checked on the CPU (the oracle's build of the same source) over EVERY float in [-104, 0], the
range of the transmittance's argument -sigma * t (below -104 the rounded result is 0):
  * against exp in f64 rounded to f32 (numpy's libm `exp` through the oracle): equal on every input;
  * against the platform's f32 `expf` (the reference CPU build's `f32::exp`): at most one unit in
    the last place, on a small fraction of the inputs, where the platform's expf is not correctly
    rounded.
The device's results are held to these bits by tests/test_gpu_kernel.py."""

import ctypes as C
import struct

import numpy as np

from oracle import oracle as O


def bits(x):
    return struct.unpack("<I", struct.pack("<f", x))[0]


def sweep(lo, hi, stride):
    L = O.lib()
    L.lwo32_water_exp_sweep.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(C.c_uint64)]
    L.lwo32_water_exp_sweep.restype = None
    out = (C.c_uint64 * 5)()
    L.lwo32_water_exp_sweep(bits(lo), bits(hi), stride, out)
    n, diff_platform, ulp_platform, diff_f64, ulp_f64 = list(out)
    return n, diff_platform, ulp_platform, diff_f64, ulp_f64


def test_every_float_of_the_transmittance_range_is_correctly_rounded():
    # every float from -0.0 down to -104.0 (their bit patterns run upwards)
    n, diff_platform, ulp_platform, diff_f64, ulp_f64 = sweep(-0.0, -104.0, 1)
    print(f"{n} inputs: {diff_f64} differ from f64 exp rounded to f32; {diff_platform} "
          f"({diff_platform / n:.2e}) from the platform expf, by at most {ulp_platform} ulp")
    assert n == bits(-104.0) - bits(-0.0) + 1
    assert diff_f64 == 0 and ulp_f64 == 0
    assert ulp_platform <= 1
    assert diff_platform / n < 1e-3


def test_positive_arguments_sampled():
    # Not reached by the transmittance (sigma, t >= 0), checked on every 16th float up to 89.
    n, diff_platform, ulp_platform, diff_f64, ulp_f64 = sweep(0.0, 89.0, 16)
    assert diff_f64 == 0 and ulp_platform <= 1


def test_special_values():
    L = O.lib()
    L.lwo32_water_exp.argtypes = [C.c_uint64, C.c_void_p, C.c_void_p]
    L.lwo_platform_expf.argtypes = [C.c_uint64, C.c_void_p, C.c_void_p]
    x = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, -1e-30, 1e-30, -103.97, -104.0, -149.0, -150.0, -1e30,
                  88.7228, 88.72284, 100.0, 1e30, -1.0, 1.0, np.float32(-87.33655)], np.float32)
    got = np.zeros_like(x)
    plat = np.zeros_like(x)
    L.lwo32_water_exp(x.size, x.ctypes.data, got.ctypes.data)
    L.lwo_platform_expf(x.size, x.ctypes.data, plat.ctypes.data)
    assert np.isnan(got[4])
    fin = ~np.isnan(x)
    with np.errstate(over="ignore"):
        want = np.exp(x[fin].astype(np.float64)).astype(np.float32)
    assert np.array_equal(got[fin], want)
    assert np.array_equal(got[fin], plat[fin])  # these are all correctly rounded by the platform too
    assert got[0] == 1.0 and got[1] == 1.0 and got[3] == 0.0 and got[2] == np.inf
