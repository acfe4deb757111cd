"""The batch autotuner's host side (csrc/autotune.cpp) through the C-ABI, from
a C++ host (tests/cpp/autotune_host.cpp): tuning files load, look up and save
without a GPU; on a GPU, a tuning repeated with its own result as the
incumbent keeps every choice."""
from __future__ import annotations

import json
import subprocess
from pathlib import Path

import pytest

from frep import _lib
from frep.autotune import DEFAULT_TABLE, load_table

REPO = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def host(tmp_path_factory):
    exe = tmp_path_factory.mktemp("autotune") / "autotune_host"
    lib_dir = _lib.LIB_PATH.parent
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", str(REPO / "include"),
                    str(REPO / "tests" / "cpp" / "autotune_host.cpp"), "-L", str(lib_dir), "-lfrep",
                    f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], check=True)
    return exe


TABLE = {
    "NVIDIA B200": {
        "choices": {"64:0": {"dims": [16, 4], "point_cells_per_lane": 0, "ms_per_scene": 0.05},
                    "128:1": {"dims": [8, 4, 4], "point_cells_per_lane": 2, "ms_per_scene": 0.1},
                    "1024:3": {"dims": [32, 8, 4], "point_cells_per_lane": 0, "ms_per_scene": float("nan")}},
        "warps": [1, 4]},
    "Other GPU": {"choices": {"64:0": {"dims": [8, 8], "point_cells_per_lane": 4, "ms_per_scene": 1.0}},
                  "warps": [4, 4]},
}


def _lookups(text):
    out = {}
    for line in text.splitlines():
        p = line.split()
        if p and p[0] == "warps":
            out["warps"] = (int(p[1]), int(p[2]))
        elif len(p) >= 4:
            out[(int(p[0]), int(p[1]))] = tuple(p[2:])
    return out


def test_tuning_file_round_trip(host, tmp_path):
    src = tmp_path / "in.json"
    src.write_text(json.dumps(TABLE))
    out = tmp_path / "out.json"
    out.write_text(json.dumps({"Other GPU": TABLE["Other GPU"]}))  # save merges into what the file holds
    r1 = subprocess.run([str(host), "table", str(src), str(out)], check=True, capture_output=True, text=True).stdout
    got = _lookups(r1)
    assert got[(64, 100)] == ("2", "16", "4", "k0")
    assert got[(128, 500)] == ("3", "8", "4", "4", "k2")
    assert got[(1024, 9000)] == ("3", "32", "8", "4", "k0")
    assert got[(256, 100)] == ("0", "k0")          # no choice for the class
    assert got["warps"] == (1, 4)
    saved = json.loads(out.read_text().replace("NaN", "null"))
    assert set(saved) == {"NVIDIA B200", "Other GPU"}  # the other device's entry survives
    r2 = subprocess.run([str(host), "table", str(out), str(tmp_path / "again.json")], check=True,
                        capture_output=True, text=True).stdout
    assert r2 == r1
    table = load_table(str(out))  # the Python reader of the same file
    assert table["128:1"].dims == (8, 4, 4) and table["128:1"].point_cells_per_lane == 2


def test_committed_table_is_readable():
    if not Path(DEFAULT_TABLE).exists():
        pytest.skip("no committed tuning table")
    table = load_table(DEFAULT_TABLE)
    assert table and all(len(c.dims) >= 2 for c in table.values())


@pytest.mark.gpu
def test_repeated_tuning_keeps_its_choices(host, tmp_path):
    out = tmp_path / "tuned.json"
    r = subprocess.run([str(host), "tune", str(out)], check=True, capture_output=True, text=True).stdout
    first, second = r.split("tuning 1\n")
    a, b = _lookups(first.split("tuning 0\n")[1]), _lookups(second)
    assert a == b
    assert any(v[0] != "0" for k, v in a.items() if k != "warps")  # the sample's classes were tuned
