"""The ctypes mirrors of the C ABI's structs (pyglu._capi) against the header.

A C program built from include/glu_b200.h reports each struct's size and the
offset of every field; the ctypes Structure must agree field by field, so a
field added to the header without its mirror (or the reverse) fails here
instead of silently shifting the fields read through ctypes.
"""
import ctypes
import json
import os
import shutil
import subprocess

import pytest

from pyglu import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

STRUCTS = {
    "glu_refine_stats": _capi.RefineStats,
    "glu_stats": _capi.Stats,
    "glu_tuning": _capi.Tuning,
}


def _c_layout(tmp_path):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "glu_b200.h"', "int main(void) {",
             '  printf("{");']
    first = True
    for cname, py in STRUCTS.items():
        sep = "" if first else ","
        first = False
        lines.append(f'  printf("{sep}\\"{cname}\\": {{\\"size\\": %zu, \\"fields\\": {{", sizeof({cname}));')
        for i, (f, _) in enumerate(py._fields_):
            fsep = "" if i == 0 else ","
            lines.append(f'  printf("{fsep}\\"{f}\\": %zu", offsetof({cname}, {f}));')
        lines.append('  printf("}}");')
    lines.append(f'  printf(", \\"kinds\\": %d", GLU_KERNEL_KINDS);')
    lines.append('  printf("}\\n");')
    lines.append("  return 0;\n}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    return json.loads(subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout)


def test_ctypes_structs_match_the_header(tmp_path):
    layout = _c_layout(tmp_path)
    for cname, py in STRUCTS.items():
        c = layout[cname]
        assert c["size"] == ctypes.sizeof(py), cname
        for f, _ in py._fields_:
            assert c["fields"][f] == getattr(py, f).offset, (cname, f)
    assert layout["kinds"] == _capi.GLU_KERNEL_KINDS
