"""The ctypes mirrors of the C ABI's structs have the header's layout.

A C program compiled against include/fdtd.h prints the size of each struct and
the offset of each field; the ctypes classes the Python binding (and the
no-alloc test) pass across the ABI must agree field by field."""
import ctypes
import shutil
import subprocess
from pathlib import Path

import pytest

from rfnetwork_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]


def _c_layout(tmp_path, struct, fields):
    src = tmp_path / "layout.c"
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "fdtd.h"', "int main(void) {",
             f'  printf("%zu\\n", sizeof({struct}));']
    lines += [f'  printf("%zu\\n", offsetof({struct}, {f}));' for f in fields]
    lines += ["  return 0;", "}"]
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    return int(out[0]), [int(v) for v in out[1:]]


def _device_grid():
    import test_zz_no_alloc
    return test_zz_no_alloc.DeviceGrid


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
@pytest.mark.parametrize("struct,get_class", [("fdtd_stats", lambda: _lib.FdtdStats),
                                              ("fdtd_nf2ff_face", lambda: _lib.Nf2ffFace),
                                              ("fdtd_device_grid", _device_grid)])
def test_ctypes_structs_match_header(tmp_path, struct, get_class):
    klass = get_class()
    names = [f for f, _ in klass._fields_]
    size, offsets = _c_layout(tmp_path, struct, names)
    assert ctypes.sizeof(klass) == size, struct
    assert [getattr(klass, f).offset for f in names] == offsets, struct
