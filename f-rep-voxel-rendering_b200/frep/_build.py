"""Build recipe of the native library (libfrep.so) for sm_100a.

Compiles csrc/*.cu and csrc/*.cpp with nvcc and links them into
frep/_native/libfrep.so, in-tree, so the built library travels with the source
tree. Objects are rebuilt only when a source or header is newer.
"""
from __future__ import annotations

import os
import subprocess
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent          # .../frep
ROOT = PKG_DIR.parent                               # f-rep-voxel-rendering_b200
REPO = ROOT.parent
CSRC = ROOT / "csrc"
BUILD = ROOT / "_build"
LIB = PKG_DIR / "_native" / "libfrep.so"
INCLUDE = REPO / "include"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

# -fmad=false: no multiply-add contraction, so every float operation rounds
# on its own exactly as the CPU oracle's (built with -ffp-contract=off).
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17", "-fmad=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O3",
    "-I", str(INCLUDE), "-I", str(CSRC),
]


def _sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def _headers():
    return list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.rglob("*.h"))


def _newest(paths):
    return max((p.stat().st_mtime for p in paths), default=0.0)


def _compile(src: Path, hdr_time: float, extra: list[str]) -> Path:
    obj = BUILD / (src.name + ".o")
    if obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, hdr_time):
        return obj
    cmd = [NVCC, *NVCC_FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cpp":
        cmd = [NVCC, "-x", "cu", *NVCC_FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    subprocess.run(cmd, check=True)
    return obj


def build(verbose_ptxas: bool = False) -> Path:
    """Builds libfrep.so if any input changed; returns its path."""
    BUILD.mkdir(exist_ok=True)
    LIB.parent.mkdir(exist_ok=True)
    hdr_time = _newest(_headers())
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, hdr_time, extra), _sources()))
    if not LIB.exists() or LIB.stat().st_mtime < _newest(objs):
        subprocess.run([NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a",
                        *map(str, objs), "-o", str(LIB)], check=True)
    return LIB


if __name__ == "__main__":
    print(build())
