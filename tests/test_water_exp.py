"""The exponential of the water transmittance (`lumenwright_b200/csrc/water_exp.h`), which the CUDA
kernels and the FP32 oracle both call: Cody and Waite's reduction and a degree-8 Taylor series in
f32 with fused multiply-adds.

Checked on the CPU (the oracle's build of the same source) over EVERY float of the range of the
transmittance's argument -sigma * t, [-104, 0] (below -104 the rounded result is 0):
  * against exp in f64 rounded to f32: within one unit in the last place on every argument, and
    equal on all but about half a percent of those with a normal result;
  * against the platform's f32 `expf` (the reference CPU build's `f32::exp`): within one unit in
    the last place on every argument.
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


def test_every_float_of_the_transmittance_range():
    # every float from -0.0 down to -104.0 (their bit patterns run upwards): the normal results
    # down to exp(-87.3365) = 2^-126, then the subnormal ones
    edge = float(np.float32(-87.33654022216797))
    n, diff_platform, ulp_platform, diff_f64, ulp_f64 = sweep(-0.0, edge, 1)
    print(f"normal results, {n} arguments: {diff_f64} ({diff_f64 / n:.1e}) differ from f64 exp rounded to f32 by at "
          f"most {ulp_f64} ulp; {diff_platform} ({diff_platform / n:.2e}) from the platform expf, by at most "
          f"{ulp_platform} ulp")
    assert diff_f64 / n < 1e-2 and ulp_f64 <= 1
    assert ulp_platform <= 1 and diff_platform / n < 1e-2
    n2, _, ulp_platform, diff_f64, ulp_f64 = sweep(edge, -104.0, 1)
    print(f"subnormal results, {n2} arguments: {diff_f64} one ulp off the rounded f64 exp")
    assert n + n2 - 1 == bits(-104.0) - bits(-0.0) + 1
    assert ulp_f64 <= 1 and ulp_platform <= 1


def test_positive_arguments_sampled():
    # Not reached by the transmittance (sigma, t >= 0), checked on every 16th float up to 88.72.
    n, diff_platform, ulp_platform, diff_f64, ulp_f64 = sweep(0.0, 88.72283172607421875, 16)
    assert diff_f64 / n < 1e-2 and ulp_f64 <= 1 and ulp_platform <= 1


def test_special_values():
    L = O.lib()
    L.lwo_platform_expf.argtypes = [C.c_uint64, C.c_void_p, C.c_void_p]
    x = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, -1e-30, 1e-30, -103.97, -104.0, -149.0, -150.0, -1e30,
                  88.7228, 88.72284, 100.0, 1e30, -1.0, 1.0, np.float32(-87.33655)], np.float32)
    got = O.water_exp(x)
    plat = np.zeros_like(x)
    L.lwo_platform_expf(x.size, x.ctypes.data, plat.ctypes.data)
    assert np.isnan(got[4])
    fin = ~np.isnan(x)
    with np.errstate(over="ignore"):
        want = np.exp(x[fin].astype(np.float64)).astype(np.float32)
    ulp = np.abs(got[fin].view(np.int32).astype(np.int64) - want.view(np.int32).astype(np.int64))
    assert ulp.max() <= 1
    assert got[0] == 1.0 and got[1] == 1.0 and got[3] == 0.0 and got[2] == np.inf and got[13] == np.inf
    assert got[9] == 0.0 and got[11] == 0.0 and got[8] == plat[8]
