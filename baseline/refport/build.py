"""Builds the benchmark's comparison baseline, ``baseline/refport/_build/liblw_refport.so``: the
reference's CUDA backend ported as written (refport.cu), for sm_100a, with the product's build
flags (no contraction, IEEE division and square root). It is not part of the product library."""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
CSRC = os.path.join(ROOT, "lumenwright_b200", "csrc")
LIB_PATH = os.path.join(HERE, "_build", "liblw_refport.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def _stale():
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    deps = [os.path.join(HERE, f) for f in ("refport.cu", "refport.h", "build.py")]
    deps += [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False) -> str:
    if not force and not _stale():
        return LIB_PATH
    os.makedirs(os.path.dirname(LIB_PATH), exist_ok=True)
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17", "--fmad=false",
           "-prec-div=true", "-prec-sqrt=true", "-Xcompiler", "-fPIC,-ffp-contract=off,-O2", "-shared",
           "-I", CSRC, "-I", os.path.join(ROOT, "include"), "-o", LIB_PATH, os.path.join(HERE, "refport.cu")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stderr[-4000:])
    return LIB_PATH


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
