"""The C++ host mirror (include/frep/csg.hpp): a C++ program written like the
reference's shapes.cpp compiles to the same tapes as the reference's own
compiler (golden vectors), through the C-ABI, without a GPU."""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np

from frep import _lib

REPO = Path(__file__).resolve().parents[1]
GOLDEN = np.load(REPO / "tests" / "golden" / "ref_tapes.npz")


def test_cpp_mirror_compiles_reference_shapes(tmp_path):
    exe = tmp_path / "mirror_shapes"
    lib_dir = _lib.LIB_PATH.parent
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", str(REPO / "include"), str(REPO / "tests" / "cpp" / "mirror_shapes.cpp"),
                    "-L", str(lib_dir), "-lfrep", f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    i = 0
    seen = 0
    while i < len(out) and out[i]:
        name, n, slots, nconst = out[i].split()
        n = int(n)
        words = np.array([int(w, 16) for w in out[i + 1: i + 1 + n]], np.uint32)
        np.testing.assert_array_equal(words, GOLDEN[f"{name}/ref_instrs"])
        assert int(slots) == int(GOLDEN[f"{name}/ref_slots"][0])
        assert int(nconst) == len(GOLDEN[f"{name}/ref_consts"])
        assert out[i + 1 + n].startswith("eval ")
        i += n + 2
        seen += 1
    assert seen == 2


def test_cpp_mirror_scene_builder_links(tmp_path):
    """SceneBuilder / Raytracer::Trace over a compact tree compile and link
    against libfrep.so (running them needs a GPU)."""
    src = tmp_path / "builder.cpp"
    src.write_text(
        '#include "frep/csg.hpp"\n'
        "int main(int argc, char**) {\n"
        "    if (argc < 2) return 0;  // linked, not run\n"
        "    frep_ctx* ctx = nullptr;\n"
        "    frep::check(frep_ctx_create(0, 0, &ctx));\n"
        "    frep::VoxelStorage voxels;\n"
        "    voxels.gridDims = {16, 4};\n"
        "    voxels.Init(ctx, frep::csg::Sphere({0, 0, 0}, 1.0f));\n"
        "    frep::Voxelizer vox; vox.Init(ctx, &voxels); vox.Voxelize(nullptr, 0.0f);\n"
        "    frep::SceneBuilder b; b.Init(ctx, &voxels); b.BuildScene(true);\n"
        "    std::vector<uint8_t> blob = b.Export();\n"
        "    frep::SceneBuilder c; c.Import(ctx, blob);\n"
        "    frep::Raytracer rt; rt.Init(ctx, &voxels);\n"
        "    rt.Trace(nullptr, c, frep::Camera{}, 0.0f, 64, 64, nullptr);\n"
        "    return (int)c.Info().levels;\n"
        "}\n")
    exe = tmp_path / "builder"
    lib_dir = _lib.LIB_PATH.parent
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", str(REPO / "include"), str(src), "-L", str(lib_dir), "-lfrep",
                    f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], check=True)
    assert subprocess.run([str(exe)]).returncode == 0
