"""The ctypes mirrors of the C-ABI structs match include/vsjoin.h field by
field: a small C program compiled against the header prints every field's
offset and size, and each ctypes Structure in vibespatial_b200/_abi.py must
agree (a field appended to the header and not to the mirror, or the other
way round, would make the library write past the caller's struct)."""
import ctypes
import shutil
import subprocess
from pathlib import Path

import pytest

from vibespatial_b200 import _abi

ROOT = Path(__file__).resolve().parents[1]

MIRRORS = {
    "vs_polygons": _abi.Polygons,
    "vs_points": _abi.Points,
    "vs_index_options": _abi.IndexOptions,
    "vs_join_stats": _abi.JoinStats,
    "vs_index_info": _abi.IndexInfo,
    "vs_batch_options": _abi.BatchOptions,
    "vs_wkb_sizes": _abi.WkbSizes,
    "vs_wkb_out": _abi.WkbOut,
}


def _c_layout(tmp_path):
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "vsjoin.h"', "int main(void) {"]
    for cname, py in MIRRORS.items():
        lines.append(f'printf("{cname} . %zu %zu\\n", (size_t)sizeof({cname}), (size_t)0);')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname} {fname} %zu %zu\\n", offsetof({cname}, {fname}), '
                         f'sizeof((({cname}*)0)->{fname}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True,
                   capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    layout = {}
    for line in out.splitlines():
        cname, fname, off, size = line.split()
        layout[(cname, fname)] = (int(off), int(size))
    return layout


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_ctypes_mirrors_match_the_header(tmp_path):
    layout = _c_layout(tmp_path)
    for cname, py in MIRRORS.items():
        assert layout[(cname, ".")][0] == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            field = getattr(py, fname)
            assert layout[(cname, fname)] == (field.offset, field.size), (cname, fname)
