"""The C ABI on the CPU: the library loads, exports every function include/*.h
declares, and the ctypes mirror of the structs has the C layout. No GPU call."""
import ctypes as C
import os
import re
import shutil
import subprocess
import tempfile

import pytest

from meercadraytracer_b200 import abi
from meercadraytracer_b200._lib import LIB_PATH, SIGNATURES, mcrt_stats

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", h) for h in ("mcrt.h", "mcrt_types.h")]


def declared_functions():
    names = set()
    for h in HEADERS:
        text = open(h).read()
        names.update(re.findall(r"\b(mcrt_[a-z_0-9]+)\s*\(", text))
    return names


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB_PATH):
        from meercadraytracer_b200.build import build

        build()
    return C.CDLL(LIB_PATH)


def test_library_exports_every_declared_function(lib):
    declared = declared_functions()
    assert declared, "no declarations found"
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing
    # The Python binding covers the whole ABI, too.
    assert declared == set(SIGNATURES), declared ^ set(SIGNATURES)


def test_version_and_last_error_need_no_gpu(lib):
    lib.mcrt_version.restype = C.c_int32
    assert lib.mcrt_version() == 1
    lib.mcrt_last_error.restype = C.c_char_p
    assert isinstance(lib.mcrt_last_error(), bytes)


STRUCTS = {
    "mcrt_texture": abi.mcrt_texture, "mcrt_environment": abi.mcrt_environment, "mcrt_material": abi.mcrt_material,
    "mcrt_light": abi.mcrt_light, "mcrt_fog": abi.mcrt_fog, "mcrt_background": abi.mcrt_background,
    "mcrt_geometry": abi.mcrt_geometry, "mcrt_shading": abi.mcrt_shading, "mcrt_camera": abi.mcrt_camera,
    "mcrt_settings": abi.mcrt_settings, "mcrt_tile": abi.mcrt_tile, "mcrt_stats": mcrt_stats,
    "mcrt_request": abi.mcrt_request, "mcrt_batch_event": abi.mcrt_batch_event,
    "mcrt_batch_stats": abi.mcrt_batch_stats, "mcrt_mesh": abi.mcrt_mesh, "mcrt_instance": abi.mcrt_instance,
    "mcrt_build_info": abi.mcrt_build_info, "mcrt_compiled_out": abi.mcrt_compiled_out,
}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs a C compiler")
def test_ctypes_structs_match_c_layout():
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "mcrt.h"', "int main(void) {"]
    for name, cls in STRUCTS.items():
        lines.append(f'printf("{name} size %zu\\n", sizeof({name}));')
        for field, _ in cls._fields_:
            lines.append(f'printf("{name} {field} %zu\\n", offsetof({name}, {field}));')
    lines.append("return 0; }")
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "layout.c"), os.path.join(d, "layout")
        open(src, "w").write("\n".join(lines))
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split("\n")
    for line in filter(None, out):
        name, field, value = line.split()
        cls = STRUCTS[name]
        expect = C.sizeof(cls) if field == "size" else getattr(cls, field).offset
        assert int(value) == expect, (name, field, value, expect)
