"""The C-ABI library loads without a GPU and exports every function include/lumenwright_b200.h
declares; the records keep the reference's sizes, and the Python mirrors of the header's records
are laid out as the C compiler lays the header out. CPU only: nothing here calls into CUDA."""

import ctypes
import os
import re
import subprocess

from lumenwright_b200 import build, gamesky, layout, native

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


# The Python mirrors of the header's records: ctypes structures of the bindings and numpy dtypes
# of the scene records, each with the C struct it must match field for field.
MIRRORS = (
    ("lw_scene_desc", native.SceneDesc), ("lw_stats", native.Stats), ("lw_tuning", native.Tuning),
    ("lw_camera_job", native.CameraJob), ("lw_adj_frame", native.AdjFrame), ("lw_world_desc", native.WorldDesc),
    ("lw_instances_desc", native.InstancesDesc), ("lw_build_info", native.BuildInfo),
    ("lw_tonemap", native.ToneMap), ("lw_gradient", native.Gradient), ("lw_hit", native.HitRec),
    ("lw_params", layout.PARAMS_DTYPE), ("lw_quad", layout.QUAD_DTYPE), ("lw_model", layout.MODEL_DTYPE),
    ("lw_emitter", layout.EMITTER_DTYPE), ("lw_quick_sky", gamesky.QUICK_SKY_DTYPE),
)


def mirror_fields(m):
    """(size, [(field, offset, size)]) of a ctypes structure or a numpy record dtype."""
    if isinstance(m, type) and issubclass(m, ctypes.Structure):
        return ctypes.sizeof(m), [(f, getattr(m, f).offset, getattr(m, f).size) for f, *_ in m._fields_]
    return m.itemsize, [(f, m.fields[f][1], m.fields[f][0].itemsize) for f in m.names]


def check_layout(tmp_path, include_dir, header, mirrors):
    """Compiles a C program against `header` that prints each record's size and each field's
    offset and size as the C compiler lays them out, and compares the Python mirrors with it."""
    lines = ["#include <stddef.h>", "#include <stdio.h>", f'#include "{header}"', "int main(void) {"]
    for cname, m in mirrors:
        lines.append(f'printf("{cname} . 0 %zu\\n", sizeof({cname}));')
        for f, _, _ in mirror_fields(m)[1]:
            lines.append(f'printf("{cname} {f} %zu %zu\\n", offsetof({cname}, {f}), sizeof((({cname} *)0)->{f}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", include_dir, str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    c = {}
    for line in filter(None, out):
        name, field, a, b = line.split()
        c[(name, field)] = (int(a), int(b))
    for cname, m in mirrors:
        size, fields = mirror_fields(m)
        assert c[(cname, ".")][1] == size, (cname, size)
        for f, off, fsize in fields:
            assert c[(cname, f)] == (off, fsize), (cname, f, off, fsize, c[(cname, f)])


def test_python_mirrors_match_the_header_layout(tmp_path):
    check_layout(tmp_path, os.path.join(ROOT, "include"), "lumenwright_b200.h", MIRRORS)


def test_oracle_bindings_match_the_oracle_header_layout(tmp_path):
    # The oracle's ctypes records against oracle/lw_oracle.h, so the checker reads its inputs and
    # writes its answers where the C code does.
    from oracle import oracle as O
    check_layout(tmp_path, os.path.join(ROOT, "oracle"), "lw_oracle.h",
                 (("lwo_scene", O.Scene), ("lwo_hit", O.Hit), ("lwo_camera64", O.Camera64),
                  ("lwo_theta", O.Theta), ("lwo_counters", O.Counters), ("lwo_quick_sky", gamesky.QUICK_SKY_DTYPE)))


def test_the_header_compiles_strictly_as_c_and_cpp(tmp_path):
    # A binding generator or a C caller reads the header as C99, a C++ caller as C++11; both
    # with every warning an error.
    src = tmp_path / "h.c"
    src.write_text('#include "lumenwright_b200.h"\nint main(void) { return 0; }\n')
    inc = os.path.join(ROOT, "include")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I", inc, "-fsyntax-only",
                    str(src)], check=True)
    cpp = tmp_path / "h.cpp"
    cpp.write_text(src.read_text())
    subprocess.run(["g++", "-std=c++11", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I", inc, "-fsyntax-only",
                    str(cpp)], check=True)
