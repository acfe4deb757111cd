"""Batching: every scene voxelized and rendered in a batch (one launch per
level pass over all trees, one launch for all frames, with and without CUDA
graph replay) is bit-identical to the same scene run alone."""
from __future__ import annotations

import numpy as np
import pytest

import frep
import oracle
from frep import scenes

pytestmark = pytest.mark.gpu

GRIDS = [(16, 4), (8, 8, 4), (16, 8), (4, 16), (8, 12), (16, 4, 4)]


@pytest.fixture(scope="module")
def ctx():
    c = frep.Context(0, hbm_budget_bytes=16 << 30)
    yield c
    c.close()


def _scenes():
    out = []
    for i, dims in enumerate(GRIDS):
        sc = scenes.random_csg(6 + 9 * i, seed=40 + i, grid_dims=list(dims), width=96 + 16 * i, height=64 + 8 * i)
        out.append(sc)
    return out


def _alone(ctx, sc, t):
    import torch
    vs = frep.VoxelStorage(sc.grid_dims, sc.low_vertex, sc.world_size).init(ctx, sc.shape)
    frep.Voxelizer(ctx, vs).voxelize(t)
    rt = frep.Raytracer(ctx, vs)
    rt.lights = frep.Lights(shadow_mask=1)
    rgba, hits = rt.trace(sc.camera, t, sc.width, sc.height, hits=True)
    torch.cuda.synchronize()
    exp = vs.export()
    canon, prob = oracle.canonical_of_export(exp)
    assert prob == []
    cells = oracle.hit_cells(hits.cpu().numpy().view(np.uint32), exp.dims, exp.node_offset, exp.node_size, exp.nodes)
    return canon, rgba.cpu().numpy(), cells, hits.cpu().numpy()


@pytest.mark.parametrize("graph", [False, True])
def test_batch_equals_alone(ctx, graph):
    import torch
    scs = _scenes()
    times = [0.1 * i for i in range(len(scs))]
    want = [_alone(ctx, sc, t) for sc, t in zip(scs, times)]
    storages = [frep.VoxelStorage(sc.grid_dims, sc.low_vertex, sc.world_size).init(ctx, sc.shape) for sc in scs]
    batch = frep.Batch(ctx, storages)
    dev = torch.device("cuda", 0)
    rgba = [torch.zeros((sc.height, sc.width, 4), dtype=torch.uint8, device=dev) for sc in scs]
    hits = [torch.zeros((sc.height, sc.width, 8), dtype=torch.int32, device=dev) for sc in scs]
    sizes = [(sc.width, sc.height) for sc in scs]
    for rep in range(2):  # the second run replays the captured graph
        for r in rgba:
            r.zero_()
        batch.run([sc.camera for sc in scs], sizes, rgba, hits, lights=frep.Lights(shadow_mask=1),
                  tape_times=times, graph=graph)
        torch.cuda.synchronize()
        for i, vs in enumerate(storages):
            exp = vs.export()
            canon, prob = oracle.canonical_of_export(exp)
            assert prob == []
            assert canon == want[i][0], f"scene {i} tree differs (run {rep})"
            np.testing.assert_array_equal(rgba[i].cpu().numpy(), want[i][1])
            cells = oracle.hit_cells(hits[i].cpu().numpy().view(np.uint32), exp.dims, exp.node_offset,
                                     exp.node_size, exp.nodes)
            np.testing.assert_array_equal(cells, want[i][2])
    batch.close()


def test_batch_voxelize_then_render(ctx):
    import torch
    scs = _scenes()[:3]
    want = [_alone(ctx, sc, 0.0) for sc in scs]
    storages = [frep.VoxelStorage(sc.grid_dims, sc.low_vertex, sc.world_size).init(ctx, sc.shape) for sc in scs]
    batch = frep.Batch(ctx, storages)
    batch.voxelize()
    dev = torch.device("cuda", 0)
    rgba = [torch.zeros((sc.height, sc.width, 4), dtype=torch.uint8, device=dev) for sc in scs]
    batch.render([sc.camera for sc in scs], [(sc.width, sc.height) for sc in scs], rgba,
                 lights=frep.Lights(shadow_mask=1))
    torch.cuda.synchronize()
    for i, vs in enumerate(storages):
        assert oracle.canonical_of_export(vs.export())[0] == want[i][0]
        np.testing.assert_array_equal(rgba[i].cpu().numpy(), want[i][1])
    batch.close()


@pytest.mark.parametrize("dims", [(16, 8), (8, 8, 8)])
def test_point_cells_per_lane_override(ctx, dims):
    """The last-level tile (2 or 4 cells per lane) changes the schedule, not the tree."""
    import torch
    sc = scenes.random_csg(40, seed=71, grid_dims=list(dims), width=96, height=80)
    got = []
    for k in (2, 4):
        vs = frep.VoxelStorage(sc.grid_dims, sc.low_vertex, sc.world_size, point_cells_per_lane=k)
        vs.init(ctx, sc.shape)
        frep.Voxelizer(ctx, vs).voxelize(0.0)
        rt = frep.Raytracer(ctx, vs)
        rgba, _ = rt.trace(sc.camera, 0.0, sc.width, sc.height)
        torch.cuda.synchronize()
        canon, prob = oracle.canonical_of_export(vs.export())
        assert prob == []
        got.append((canon, rgba.cpu().numpy()))
        vs.cleanup()
    assert got[0][0] == got[1][0]
    np.testing.assert_array_equal(got[0][1], got[1][1])


def test_point_cells_per_lane_invalid(ctx):
    vs = frep.VoxelStorage((16, 4), point_cells_per_lane=4)  # 4^3 / 32 = 2 words: 4 cells per lane cannot tile
    with pytest.raises(frep.FrepError):
        vs.init(ctx, scenes.spheres_union(4).shape)


@pytest.mark.parametrize("warps", [(1, 1), (4, 4), (1, 4)])
def test_batch_tuning_same_result(ctx, warps):
    import torch
    scs = _scenes()[:4]
    want = [_alone(ctx, sc, 0.0) for sc in scs]
    storages = [frep.VoxelStorage(sc.grid_dims, sc.low_vertex, sc.world_size).init(ctx, sc.shape) for sc in scs]
    batch = frep.Batch(ctx, storages)
    batch.set_tuning(*warps)
    dev = torch.device("cuda", 0)
    rgba = [torch.zeros((sc.height, sc.width, 4), dtype=torch.uint8, device=dev) for sc in scs]
    batch.run([sc.camera for sc in scs], [(sc.width, sc.height) for sc in scs], rgba,
              lights=frep.Lights(shadow_mask=1), graph=True)
    torch.cuda.synchronize()
    info = batch.info()
    assert info.n_trees == len(scs) and info.voxelize_launches > 0
    for i, vs in enumerate(storages):
        assert oracle.canonical_of_export(vs.export())[0] == want[i][0]
        np.testing.assert_array_equal(rgba[i].cpu().numpy(), want[i][1])
    batch.close()


def test_cached_plans_of_many_trees(ctx):
    """Trees keep their level plans; planning a tree with a smaller shared-memory
    footprint must not break later launches of a tree planned earlier."""
    big = scenes.random_csg(300, seed=5, grid_dims=[16, 8], width=32, height=32)
    small = scenes.spheres_union(3)
    a = frep.VoxelStorage(big.grid_dims, big.low_vertex, big.world_size).init(ctx, big.shape)
    b = frep.VoxelStorage(small.grid_dims, small.low_vertex, small.world_size).init(ctx, small.shape)
    assert a.tape.n_slots > b.tape.n_slots
    frep.Voxelizer(ctx, a).voxelize(0.0)
    first = oracle.canonical_of_export(a.export())[0]
    frep.Voxelizer(ctx, b).voxelize(0.0)
    b.sync()
    frep.Voxelizer(ctx, a).voxelize(0.0)
    assert oracle.canonical_of_export(a.export())[0] == first
    a.cleanup()
    b.cleanup()


def test_set_trees_and_render_frames(ctx):
    """A batch object serves changing tree sets (one set per call, upload areas
    in rotation) and renders frames of any voxelized trees, repeats included."""
    import torch
    scs = _scenes()
    want = [_alone(ctx, sc, 0.05 * i) for i, sc in enumerate(scs)]
    storages = [frep.VoxelStorage(sc.grid_dims, sc.low_vertex, sc.world_size).init(ctx, sc.shape) for sc in scs]
    batch = frep.Batch(ctx, storages[:2])
    batch.voxelize(tape_times=[0.0, 0.05])
    batch.set_trees(storages[2:5])
    batch.voxelize(tape_times=[0.1, 0.15, 0.2])
    batch.set_trees(storages[5:])
    batch.voxelize(tape_times=[0.05 * i for i in range(5, len(scs))])
    order = [4, 0, 4, 2, 5, 1, 3, 0]
    dev = torch.device("cuda", 0)
    rgba = [torch.zeros((scs[i].height, scs[i].width, 4), dtype=torch.uint8, device=dev) for i in order]
    hits = [torch.zeros((scs[i].height, scs[i].width, 8), dtype=torch.int32, device=dev) for i in order]
    batch.render_frames([storages[i] for i in order], [scs[i].camera for i in order],
                        [(scs[i].width, scs[i].height) for i in order], rgba, hits, lights=frep.Lights(shadow_mask=1),
                        tape_times=[0.05 * i for i in order])
    torch.cuda.synchronize()
    for k, i in enumerate(order):
        exp = storages[i].export()
        assert oracle.canonical_of_export(exp)[0] == want[i][0]
        np.testing.assert_array_equal(rgba[k].cpu().numpy(), want[i][1])
        cells = oracle.hit_cells(hits[k].cpu().numpy().view(np.uint32), exp.dims, exp.node_offset, exp.node_size,
                                 exp.nodes)
        np.testing.assert_array_equal(cells, want[i][2])
    batch.close()


def test_root_level_of_a_large_batch(ctx):
    """A set whose root cells fill the grid (160 trees with 32^3 roots): the
    root level runs two cells per lane over 4x4x4 bricks (batch info), and
    every tree equals the same scene voxelized alone (one root: one cell per
    lane, 2x4x4 bricks) and, for two of them, the oracle's."""
    from parity import compare_trees_fast, oracle_tree
    scs = [scenes.random_csg(10 + 7 * (i % 6), seed=500 + i, grid_dims=[32, 4]) for i in range(160)]
    pools = dict(node_words=1 << 19, tape_words=1 << 21)  # 2 MB of nodes, 16 MB of tapes per tree
    alone = []
    for sc in scs:
        vs = frep.VoxelStorage(sc.grid_dims, sc.low_vertex, sc.world_size, **pools).init(ctx, sc.shape)
        frep.Voxelizer(ctx, vs).voxelize(0.0)
        alone.append(vs.export())
        vs.cleanup()
    storages = [frep.VoxelStorage(sc.grid_dims, sc.low_vertex, sc.world_size, **pools).init(ctx, sc.shape)
                for sc in scs]
    batch = frep.Batch(ctx, storages)
    for rep in range(2):  # the second run starts on the first one's scratch
        batch.voxelize()
        assert batch.info().root_cells_per_lane == 2
        for i, vs in enumerate(storages):
            assert compare_trees_fast(vs.export(), alone[i]) == [], f"tree {i} (run {rep})"
    for i in (0, 5):
        orc = oracle_tree(scs[i], frep.Tape(scs[i].shape))
        assert compare_trees_fast(storages[i].export(), orc) == [], f"tree {i}"
    batch.close()
    for vs in storages:
        vs.cleanup()
