"""The hybrid affine mode (FREP_ROUND_HYBRID) on the device against the oracle:
trees (masks, topology, shortened tapes) bit-exact in canonical form, hits and
pixels identical, intervals of single boxes bit-identical, and the device's
hybrid intervals sound against FP64 dense sampling. Also through a batch."""
from __future__ import annotations

import numpy as np
import pytest

import frep
import oracle
from containment import check_tree, oracle_intervals
from frep import scenes
from parity import compare_hits, compare_trees, device_tree, oracle_tree, render_both

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = frep.Context(0, hbm_budget_bytes=16 << 30)
    yield c
    c.close()


def _demo(name, level, dims=(16, 4, 4)):
    cam = frep.Camera(position=(0, 0, 40.0), forward=(0, 0, -1), initial_up=(0, 1, 0), fov_deg=45)
    return scenes.Scene(name, scenes.DEMO_SHAPES[name](level), list(dims), (-20, -20, -20), 40.0, cam, 96, 64)


CASES = [("spheres16", lambda: scenes.spheres_union(16, width=96, height=96), 0.0),
         ("csg64", lambda: scenes.random_csg(64, seed=7, grid_dims=[8, 8, 4], width=96, height=64), 0.0),
         ("gyroid", lambda: scenes.stress_gyroid(grid_dims=(8, 8, 4), width=96, height=64), 0.37),
         ("TangleCube", lambda: _demo("TangleCube", 0), 0.0),
         ("Morph", lambda: _demo("Morph", 0), 0.9),
         ("Screw", lambda: _demo("Screw", 0), 2.0),
         ("ElasticCube", lambda: _demo("ElasticCube", 0), 1.3)]


@pytest.mark.parametrize("name,make,t", CASES, ids=[c[0] for c in CASES])
def test_hybrid_tree_and_image_match_oracle(ctx, name, make, t):
    sc = make()
    vs = device_tree(ctx, sc, rounding=frep.ROUND_HYBRID, tape_time=t)
    exp = vs.export()
    orc = oracle_tree(sc, vs.tape, rounding=frep.ROUND_HYBRID, tape_time=t)
    assert compare_trees(exp, orc) == []
    lights = frep.Lights(shadow_mask=1)
    d_rgba, d_hits, o_rgba, o_hits = render_both(ctx, vs, orc, sc, lights, tape_time=t)
    assert compare_hits(d_hits, o_hits, exp, orc) == []
    np.testing.assert_array_equal(d_rgba, o_rgba)
    # the device's hybrid intervals: the oracle's bits, and sound
    compared = []

    def device_intervals(wide, ns, boxes, tt):
        iv = ctx.eval_intervals(frep.Tape.from_wide(wide), boxes, tt, frep.ROUND_HYBRID)
        if not compared:
            np.testing.assert_array_equal(iv, oracle_intervals(wide, ns, boxes, tt, rounding=2))
            compared.append(1)
        return iv

    rep = check_tree(exp, vs.tape.wide(), vs.tape.n_slots, sc.low_vertex, sc.world_size, t, device_intervals,
                     nodes_per_level=6, cells_per_node=24)
    assert rep.ok(), rep.summary()


def test_hybrid_batch_equals_alone(ctx):
    import torch
    scs = [_demo("TangleCube", 0, (8, 8, 4)), scenes.random_csg(24, seed=3, grid_dims=[16, 4], width=96, height=64)]
    want = []
    for sc in scs:
        vs = device_tree(ctx, sc, rounding=frep.ROUND_HYBRID)
        want.append(oracle.canonical_of_export(vs.export())[0])
    st = [frep.VoxelStorage(sc.grid_dims, sc.low_vertex, sc.world_size, rounding=frep.ROUND_HYBRID).init(ctx, sc.shape)
          for sc in scs]
    batch = frep.Batch(ctx, st)
    dev = torch.device("cuda", 0)
    rgba = [torch.zeros((sc.height, sc.width, 4), dtype=torch.uint8, device=dev) for sc in scs]
    batch.run([sc.camera for sc in scs], [(sc.width, sc.height) for sc in scs], rgba, lights=frep.Lights(),
              graph=True)
    torch.cuda.synchronize()
    for vs, w in zip(st, want):
        assert oracle.canonical_of_export(vs.export())[0] == w
    batch.close()
