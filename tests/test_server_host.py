"""The serving loop's tree placement on the CPU: the arena's first fit and
coalescing, and least-recently-used eviction until a tree fits
(csrc/arena.h, compiled with g++ and run; no GPU)."""
from __future__ import annotations

import subprocess
from pathlib import Path

REPO = Path(__file__).resolve().parents[1]


def test_arena_and_lru_placement(tmp_path):
    exe = tmp_path / "arena_host"
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-I", str(REPO / "f-rep-voxel-rendering_b200" / "csrc"),
                    str(REPO / "tests" / "cpp" / "arena_host.cpp"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout
