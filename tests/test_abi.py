"""The C-ABI library loads on a CPU-only host, exports every entry point that
include/wmles_cuda.h declares, and the ctypes mirrors match the C struct layouts."""
import ctypes
import os
import re
import shutil
import subprocess

import pytest

from wmles_jax_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "wmles_cuda.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:int|void|const char\*)\s+(wm_\w+)\s*\(", text, re.M)))


def test_header_declares_what_the_binding_binds():
    assert declared_functions() == sorted(N.SIGNATURES)


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(N.LIB_PATH):
        from wmles_jax_b200.build import build
        build()
    return ctypes.CDLL(N.LIB_PATH)


def test_library_exports_every_declared_symbol(lib):
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_version_and_error_string_without_gpu(lib):
    lib.wm_version.restype = ctypes.c_int
    assert lib.wm_version() == N.ABI_VERSION
    lib.wm_last_error.restype = ctypes.c_char_p
    assert isinstance(lib.wm_last_error(), bytes)
    # argument validation runs before any device call
    lib.wm_case_create.restype = ctypes.c_int
    assert lib.wm_case_create(None, None) == -1
    lib.wm_batch_create.restype = ctypes.c_int
    out = ctypes.c_void_p()
    assert lib.wm_batch_create(0, None, ctypes.byref(out)) == -1
    assert lib.wm_batch_create(1, (ctypes.c_void_p * 1)(None), ctypes.byref(out)) == -1
    assert out.value is None


STRUCTS = {"wm_gas": N.WmGas, "wm_block": N.WmBlock, "wm_wall": N.WmWall,
           "wm_ghost_program": N.WmGhostProgram, "wm_inflow": N.WmInflow, "wm_sponge": N.WmSponge,
           "wm_case_desc": N.WmCaseDesc}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_struct_layouts_match_header(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){"]
    for cname, py in STRUCTS.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    for line in filter(None, out):
        cname, field, val = line.split()
        py = STRUCTS[cname]
        want = ctypes.sizeof(py) if field == "size" else getattr(py, field).offset
        assert int(val) == want, (cname, field, int(val), want)
