"""GPU parity at the benchmarked configurations, against the oracle directly.

* The large scene exactly as the bench runs it: 256 random primitives
  (6,814-instruction tape), grid {16, 16, 8} = 2048^3, 1920x1080
  perspective with a shadow ray per hit.
* Scenes of the 512-scene batch workload, each voxelized and rendered by
  frep_batch_run under CUDA graph replay with one tape per block in the
  interval passes (the instantiation the bench's tuning picks): the longest
  tape of the batch (30,503 instructions), and one scene per grid of the
  kind the autotuner chooses (32,8,4 / 16,8,8 / 16,16 / 16,4,4 / 16,8,4 /
  16,8 / 16,4, with 2 or 4 cells per lane in the last level), 512x512 with
  shadow rays.
* The stress gyroid (SIN/COS, twist by T) on a {16, 16, 4} grid = 1024^3.
Trees are compared in canonical form (tests/parity.py compare_trees_fast:
node sets, masks, tapes by content, child links), hits cell for cell,
depths and normals within 1e-5 relative, rgba8 exactly.
"""
from __future__ import annotations

import numpy as np
import pytest

import frep
import oracle
from frep import scenes
from frep.autotune import fit_pools
from parity import compare_hits, compare_trees_fast, oracle_tree

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = frep.Context(0, hbm_budget_bytes=64 << 30)
    yield c
    c.close()


def _device(ctx, sc, t=0.0, k=0):
    tape = sc.shape if isinstance(sc.shape, frep.Tape) else frep.Tape(sc.shape)
    p = fit_pools(ctx, [tape], [sc.grid_dims], sc.low_vertex, sc.world_size, tape_times=[t])[0]
    vs = frep.VoxelStorage(sc.grid_dims, sc.low_vertex, sc.world_size, rounding=frep.ROUND_OUTWARD,
                           node_words=p.node_words, tape_words=p.tape_words, point_cells_per_lane=k)
    vs.init(ctx, tape)
    frep.Voxelizer(ctx, vs).voxelize(t)
    return vs


def _render_compare(ctx, vs, orc, sc, t=0.0):
    import torch
    rt = frep.Raytracer(ctx, vs)
    rt.lights = frep.Lights(shadow_mask=sc.shadow_mask)
    rgba, hits = rt.trace(sc.camera, t, sc.width, sc.height, hits=True)
    torch.cuda.synchronize()
    o_rgba, o_hits = orc.render(oracle.camera_vector(sc.camera, sc.width, sc.height),
                                frep.Lights(shadow_mask=sc.shadow_mask), t)
    d_hits = hits.cpu().numpy().view(np.uint32)
    assert compare_hits(d_hits, o_hits, vs.export(), orc) == []
    np.testing.assert_array_equal(rgba.cpu().numpy(), o_rgba)
    return int((o_hits[..., 4] != 0xFFFFFFFF).sum())


def test_large_scene_2048cube_1080p_matches_oracle(ctx):
    sc = scenes.random_csg(256, seed=2, grid_dims=[16, 16, 8], width=1920, height=1080, shadows=True)
    vs = _device(ctx, sc)
    assert vs.tape.n_instr > 6000
    exp = vs.export()
    orc = oracle_tree(sc, vs.tape, rounding=1)
    assert compare_trees_fast(exp, orc) == []
    assert _render_compare(ctx, vs, orc, sc) > 100_000


# (batch index, grid, last-level cells per lane): index 156 holds the longest
# tape of the 512-scene batch
BATCH_CASES = [
    (156, (16, 8), 4),
    (84, (32, 8, 4), 2),
    (185, (16, 8, 8), 4),
    (303, (16, 16), 4),
    (303, (16, 4, 4), 2),
    (489, (16, 8, 4), 2),
    (21, (16, 4), 2),
    (7, (16, 8), 2),
]


def test_batch_scenes_under_graph_replay_match_oracle(ctx):
    import torch
    jobs = scenes.batch_jobs()
    rng = np.random.default_rng(11)
    scs = []
    for idx, dims, k in BATCH_CASES:
        j = list(jobs[idx])
        j[4] = dims
        sc = scenes.batch_scene(tuple(j))
        sc.camera = scenes.orbit_camera(rng)
        sc.meta["k"] = k
        scs.append(sc)
    assert max(sc.shape.n_instr for sc in scs) == 30503
    pools = fit_pools(ctx, [sc.shape for sc in scs], [sc.grid_dims for sc in scs], scs[0].low_vertex,
                      scs[0].world_size)
    storages = []
    for sc, p in zip(scs, pools):
        vs = frep.VoxelStorage(sc.grid_dims, sc.low_vertex, sc.world_size, rounding=frep.ROUND_OUTWARD,
                               node_words=p.node_words, tape_words=p.tape_words,
                               point_cells_per_lane=sc.meta["k"])
        storages.append(vs.init(ctx, sc.shape))
    batch = frep.Batch(ctx, storages)
    batch.set_tuning(1, 4)  # one tape per block in the interval passes, four in the point passes
    dev = torch.device("cuda", 0)
    W = H = 512
    rgba = [torch.zeros((H, W, 4), dtype=torch.uint8, device=dev) for _ in scs]
    hits = [torch.zeros((H, W, 8), dtype=torch.int32, device=dev) for _ in scs]
    lights = frep.Lights(shadow_mask=1)
    for _ in range(2):  # the second run replays the captured graph
        for r in rgba:
            r.zero_()
        batch.run([sc.camera for sc in scs], [(W, H)] * len(scs), rgba, hits, lights=lights, graph=True)
        torch.cuda.synchronize()
    for i, (sc, vs) in enumerate(zip(scs, storages)):
        exp = vs.export()
        orc = oracle_tree(sc, vs.tape, rounding=1)
        assert compare_trees_fast(exp, orc) == [], (i, BATCH_CASES[i])
        o_rgba, o_hits = orc.render(oracle.camera_vector(sc.camera, W, H), lights, 0.0)
        d_hits = hits[i].cpu().numpy().view(np.uint32)
        assert compare_hits(d_hits, o_hits, exp, orc) == [], (i, BATCH_CASES[i])
        np.testing.assert_array_equal(rgba[i].cpu().numpy(), o_rgba)
    batch.close()


def test_stress_gyroid_1024cube_matches_oracle(ctx):
    t = 0.37
    sc = scenes.stress_gyroid(grid_dims=(16, 16, 4), width=480, height=270)
    vs = _device(ctx, sc, t)
    exp = vs.export()
    orc = oracle_tree(sc, vs.tape, rounding=1, tape_time=t)
    assert sum(exp.node_count) > 1_000_000
    assert compare_trees_fast(exp, orc) == []
    assert _render_compare(ctx, vs, orc, sc, t) > 10_000
