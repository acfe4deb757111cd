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
