"""The Python binding's ctypes structs (frep/_lib.py) against the C header
(include/frep.h): each struct's size and every field's offset, printed by a C
program compiled with gcc, must match. Guards the boundary when a struct
gains a field. No GPU."""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import pytest

from frep import _lib as L

REPO = Path(__file__).resolve().parents[1]

# ctypes struct -> (C type name, its fields in the header's names)
PAIRS = {
    "Dag": "frep_dag", "TapeOpts": "frep_tape_opts", "TapeInfo": "frep_tape_info", "Grid": "frep_grid",
    "BatchInfo": "frep_batch_info", "VoxelizeOpts": "frep_voxelize_opts", "TreeInfo": "frep_tree_info",
    "CameraStruct": "frep_camera", "ServerConfig": "frep_server_config", "RequestStruct": "frep_request",
    "RequestStatus": "frep_request_status", "ServerStats": "frep_server_stats", "LightsStruct": "frep_lights",
    "CompactInfo": "frep_compact_info", "AutotuneOpts": "frep_autotune_opts", "Image": "frep_image",
}


def _c_layouts(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "frep.h"', "int main(void) {"]
    for py, c in PAIRS.items():
        lines.append(f'    printf("{py} size %zu\\n", sizeof({c}));')
        for name, _ in getattr(L, py)._fields_:
            lines.append(f'    printf("{py} {name} %zu\\n", offsetof({c}, {name}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "layouts.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layouts"
    r = subprocess.run(["gcc", "-std=c11", "-I", str(REPO / "include"), str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    if r.returncode != 0:
        pytest.fail("a binding field is not a member of its C struct:\n" + r.stderr[-2000:])
    out = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        py, name, v = line.split()
        out[(py, name)] = int(v)
    return out


def test_binding_structs_match_the_header(tmp_path):
    c = _c_layouts(tmp_path)
    bad = []
    for py in PAIRS:
        st = getattr(L, py)
        if C.sizeof(st) != c[(py, "size")]:
            bad.append(f"{py}: size {C.sizeof(st)} != {c[(py, 'size')]}")
        for name, _ in st._fields_:
            off = getattr(st, name).offset
            if off != c[(py, name)]:
                bad.append(f"{py}.{name}: offset {off} != {c[(py, name)]}")
    assert bad == []
