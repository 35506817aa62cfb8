"""The C-ABI library loads without a GPU and exports every function include/lumenwright_b200.h
declares; the records keep the reference's sizes. CPU only: nothing here calls into CUDA."""

import ctypes
import os
import re

from lumenwright_b200 import build, layout, native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "lumenwright_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lw_[a-z_]+)\s*\(", text)) - {"lw_progress_fn"})


def test_library_builds_and_exports_every_declared_function():
    path = build.build()
    lib = ctypes.CDLL(path)
    declared = header_functions()
    assert declared, "no declarations found"
    missing = [n for n in declared if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(native.EXPORTS) == declared


def test_records_keep_the_reference_sizes():
    assert layout.PARAMS_DTYPE.itemsize == 432
    assert layout.QUAD_DTYPE.itemsize == 80
    assert layout.MODEL_DTYPE.itemsize == 16
    assert layout.EMITTER_DTYPE.itemsize == 32
