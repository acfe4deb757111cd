"""Generates tests/golden/ref_tapes.npz from the REFERENCE's own code.

Run from the repository root, in a checkout where the reference tree is
present and oracle/_ref/libfrep_ref.so is built (``make -C oracle``):

    python tests/golden/make_golden.py

For each scene it records the flat DAG, the reference compiler's output
(csg::Tape instructions in the upload encoding, the constant pool and the slot
count; vulkan/src/csg/tape.cpp:14-228) and csg::Tape::Eval at 64 seeded points
(tape.cpp:274-302). Tests compare the library's compiler and the oracle's
point interpreter against these vectors, so they run without the reference.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(REPO / "f-rep-voxel-rendering_b200"))
sys.path.insert(0, str(REPO / "oracle"))

import oracle  # noqa: E402
from frep import scenes  # noqa: E402


def cases():
    yield "spheres_union_16", scenes.spheres_union(16, seed=1).shape.flatten()
    for n, seed in ((4, 11), (8, 12), (16, 13)):
        yield f"random_csg_{n}", scenes.random_csg(n, seed=seed).shape.flatten()
    for name in ("Screw", "ElasticCube", "TangleCube", "Morph", "OrganicBalls"):
        yield f"ref_{name}", oracle.ref_shape_dag(name, 0)
    yield "ref_MengerSponge_2", oracle.ref_shape_dag("MengerSponge", 2)
    yield "ref_TwistedTower_2", oracle.ref_shape_dag("TwistedTower", 2)


def main():
    out = {}
    rng = np.random.default_rng(2024)
    names = []
    for name, dag in cases():
        ops, in0, in1, consts, root = dag
        ref = oracle.RefTape(ops, in0, in1, consts, root)
        assert ref.fits, name
        # points in the scene's extent; the demo shapes live in a ~40-unit world
        scale = 20.0 if name.startswith("ref_") else 1.5
        pts = np.concatenate([rng.uniform(-scale, scale, (64, 3)), rng.uniform(0, 6.28, (64, 1))], 1)
        pts = pts.astype(np.float32)
        vals = ref.eval(pts)
        names.append(name)
        out[f"{name}/ops"] = ops
        out[f"{name}/in0"] = in0
        out[f"{name}/in1"] = in1
        out[f"{name}/consts"] = consts
        out[f"{name}/root"] = np.array([root], np.uint32)
        out[f"{name}/ref_instrs"] = ref.instrs
        out[f"{name}/ref_consts"] = ref.consts
        out[f"{name}/ref_slots"] = np.array([ref.n_slots], np.uint32)
        out[f"{name}/points"] = pts
        out[f"{name}/ref_eval"] = vals
    out["names"] = np.array(names)
    np.savez_compressed(REPO / "tests" / "golden" / "ref_tapes.npz", **out)
    print(f"wrote {len(names)} cases")


if __name__ == "__main__":
    main()
