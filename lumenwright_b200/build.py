"""Builds the CUDA library in-tree: ``lumenwright_b200/_lib/liblumenwright_b200.so``.

nvcc for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``). ``--fmad=false`` and the
default IEEE division and square root keep every float operation rounded as the reference
kernel's f32 code rounds it, so per-sample results match the reference's CPU path.
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "_lib")
LIB_PATH = os.path.join(LIB_DIR, "liblumenwright_b200.so")
SOURCES = ["render.cu", "batch.cu", "scene.cu", "sky.cu", "noalloc.cu", "adjoint.cu", "wavefront.cu", "post.cu", "build.cu", "capi.cu"]
HEADERS = ["water_exp.h", "device_math.cuh", "device_scene.cuh", "device_integrator.cuh", "device_path.cuh", "internal.h"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "--fmad=false", "-prec-div=true", "-prec-sqrt=true",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
    "-Xptxas", "-v",
    "-shared",
]


def _stale():
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "lumenwright_b200.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False) -> str:
    """Compiles the library when a source is newer than it; returns its path."""
    if not force and not _stale():
        return LIB_PATH
    os.makedirs(LIB_DIR, exist_ok=True)
    cmd = [NVCC, *FLAGS, "-o", LIB_PATH, *[os.path.join(CSRC, f) for f in SOURCES]]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stderr[-4000:])
    # The register and spill record, without ptxas's compile times, which differ on every build,
    # and with source paths relative to the package.
    with open(os.path.join(LIB_DIR, "ptxas.txt"), "w") as f:
        f.writelines(l.replace(HERE + os.sep, "") for l in r.stderr.splitlines(True)
                     if "Compile time" not in l)
    return LIB_PATH


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
