"""The ctypes mirror of the C ABI's structures (mlodsurfaces_b200/_capi.py)
against include/mlods.h: a small C program compiled with the host compiler
prints each structure's size and every field's offset, which must equal the
ctypes layout (a foreign binding reads the same bytes)."""
import ctypes as C
import shutil
import subprocess
from pathlib import Path

import pytest

from mlodsurfaces_b200 import _capi as capi

ROOT = Path(__file__).resolve().parents[1]
STRUCTS = [capi.mlods_kernel, capi.mlods_params, capi.mlods_scene_params, capi.mlods_server_config,
           capi.mlods_batch_schedule, capi.mlods_tree_info]


def _c_layout(tmp_path):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "mlods.h"', 'int main(void) {']
    for st in STRUCTS:
        name = st.__name__
        lines.append(f'  printf("{name} size %zu\\n", sizeof({name}));')
        for field, _ in st._fields_:
            lines.append(f'  printf("{name}.{field} %zu\\n", offsetof({name}, {field}));')
    lines += ['  return 0;', '}']
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c11", f"-I{ROOT / 'include'}", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return dict(line.rsplit(" ", 1) for line in out.strip().splitlines())


def test_struct_layouts_match_the_header(tmp_path):
    got = _c_layout(tmp_path)
    for st in STRUCTS:
        name = st.__name__
        assert int(got[f"{name} size"]) == C.sizeof(st), name
        for field, _ in st._fields_:
            assert int(got[f"{name}.{field}"]) == getattr(st, field).offset, f"{name}.{field}"
