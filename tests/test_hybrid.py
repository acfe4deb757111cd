"""The hybrid affine mode (FREP_ROUND_HYBRID) on the oracle: outward intervals
intersected with affine forms over the cell's axes.

* Sound: every hybrid interval of sampled cells of whole trees contains the
  tape's exact value (FP64 dense sampling with a rigorous error bound), and
  the trees' leaf / empty marks agree with the samples.
* Never looser than the outward mode: every cell the outward mode decides
  (leaf or empty) the hybrid mode decides the same way, so its trees hold a
  subset of the outward trees' ambiguous cells.
* Much tighter where intervals suffer from the dependency problem: the
  reference's polynomial demo shapes (TangleCube, Morph,
  vulkan/src/shapes.cpp:48-66) keep far fewer ambiguous cells.
The device's hybrid trees are compared with these bit for bit in
test_gpu_hybrid.py.
"""
from __future__ import annotations

import numpy as np
import pytest

import frep
import oracle
from containment import check_tree, oracle_intervals
from frep import scenes
from parity import oracle_tree


def _demo(name, level, dims=(16, 4, 4)):
    cam = frep.Camera(position=(0, 0, 40.0), forward=(0, 0, -1), initial_up=(0, 1, 0), fov_deg=45)
    return scenes.Scene(name, scenes.DEMO_SHAPES[name](level), list(dims), (-20, -20, -20), 40.0, cam, 64, 48)


CASES = [("spheres16", lambda: scenes.spheres_union(16), 0.0),
         ("csg24", lambda: scenes.random_csg(24, seed=5, grid_dims=[8, 8, 4]), 0.0),
         ("gyroid", lambda: scenes.stress_gyroid(n_spheres=8, grid_dims=(8, 8, 4)), 0.37),
         ("TangleCube", lambda: _demo("TangleCube", 0, (8, 8, 4)), 0.0),
         ("Morph", lambda: _demo("Morph", 0, (8, 8, 4)), 0.9),
         ("Screw", lambda: _demo("Screw", 0, (8, 4, 4)), 2.0),
         ("ElasticCube", lambda: _demo("ElasticCube", 0, (8, 4, 4)), 1.3)]


def _ambiguous(t):
    """Ambiguous cells per interval level (interior bits)."""
    out = []
    for lvl in range(t.levels - 1):
        dim = t.dims[lvl]
        W = dim ** 3 // 32
        n = 0
        for i in range(t.node_count[lvl]):
            rec = t.nodes[t.node_offset[lvl] + i * t.node_size[lvl]:][: 4 + 2 * W]
            n += int(np.bitwise_count(rec[4 + W:4 + 2 * W]).sum())
        out.append(n)
    return out


@pytest.mark.parametrize("name,make,t", CASES, ids=[c[0] for c in CASES])
def test_hybrid_tree_is_sound_and_never_looser(name, make, t):
    sc = make()
    tape = frep.Tape(sc.shape)
    hy = oracle_tree(sc, tape, rounding=frep.ROUND_HYBRID, tape_time=t)
    rep = check_tree(hy, tape.wide(), tape.n_slots, sc.low_vertex, sc.world_size, t,
                     lambda w, ns, b, tt: oracle_intervals(w, ns, b, tt, rounding=2),
                     nodes_per_level=6, cells_per_node=24)
    assert rep.ok(), rep.summary()
    out = oracle_tree(sc, tape, rounding=frep.ROUND_OUTWARD, tape_time=t)
    # the root level of both: the hybrid marks a subset of the outward ambiguous cells
    W = sc.grid_dims[0] ** 3 // 32
    h_int, o_int = hy.nodes[4 + W:4 + 2 * W], out.nodes[4 + W:4 + 2 * W]
    assert np.all((h_int & ~o_int) == 0)
    assert np.all((out.nodes[4:4 + W] & ~hy.nodes[4:4 + W]) == 0)  # outward leaves stay leaves
    assert _ambiguous(hy)[0] <= _ambiguous(out)[0]


def test_hybrid_interval_contains_outward_bounds():
    """Single boxes: the hybrid interval lies inside the outward one."""
    sc = _demo("TangleCube", 0)
    tape = frep.Tape(sc.shape)
    rng = np.random.default_rng(3)
    for _ in range(200):
        lo = rng.uniform(-20, 18, 3).astype(np.float32)
        hi = (lo + rng.uniform(0.01, 2.0, 3)).astype(np.float32)
        h, _ = oracle.eval_interval(tape.wide(), tape.n_slots, lo, hi, 0.0, 2)
        o, _ = oracle.eval_interval(tape.wide(), tape.n_slots, lo, hi, 0.0, 1)
        assert o[0] <= h[0] <= h[1] <= o[1]


@pytest.mark.parametrize("name", ["TangleCube", "Morph"])
def test_hybrid_cuts_ambiguous_cells_on_polynomial_shapes(name):
    sc = _demo(name, 0, (32, 4))
    t = 0.9 if name == "Morph" else 0.0
    tape = frep.Tape(sc.shape)
    hy = _ambiguous(oracle_tree(sc, tape, rounding=2, tape_time=t))[0]
    out = _ambiguous(oracle_tree(sc, tape, rounding=1, tape_time=t))[0]
    print(f"{name}: ambiguous cells of the 32^3 root level -- outward {out}, hybrid {hy}")
    assert hy < 0.5 * out
