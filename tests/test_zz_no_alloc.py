"""frep_voxelize_static_scratch: voxelization that allocates no device memory.

For callers that cannot allocate when they voxelize (a budget reserved up
front, a frame loop that must avoid cudaMalloc's implicit synchronisation, an
application whose own allocator owns every buffer). The entry point takes the
interval pass's scratch from a fixed array in device memory instead of a
cudaMalloc'd buffer; its trees must be identical to frep_voxelize's.

This file is collected last on purpose, and it must pass both alone in a fresh
process and after every other test.
"""
from __future__ import annotations

import ctypes as C

import pytest

import frep
import oracle
from frep import scenes

pytestmark = pytest.mark.gpu


def _static_voxelize(ctx, vs, tape_time=0.0):
    lib = frep._lib.lib()
    st = lib.frep_voxelize_static_scratch(ctx._h, vs.tree, vs.tape.handle, C.c_float(tape_time), C.c_void_p(0))
    frep._lib.check(st)


@pytest.mark.parametrize("n,dims,rounding", [(16, (16, 4), 1), (48, (16, 8, 4), 1), (24, (8, 8), 0)])
def test_static_scratch_matches_frep_voxelize_twice(n, dims, rounding):
    ctx = frep.Context(0, hbm_budget_bytes=8 << 30)
    sc = scenes.random_csg(n, seed=21, grid_dims=list(dims))
    ref = frep.VoxelStorage(sc.grid_dims, sc.low_vertex, sc.world_size, rounding=rounding).init(ctx, sc.shape)
    frep.Voxelizer(ctx, ref).voxelize(0.0, stream=0)
    want, problems = oracle.canonical_of_export(ref.export())
    assert problems == []
    vs = frep.VoxelStorage(sc.grid_dims, sc.low_vertex, sc.world_size, rounding=rounding).init(ctx, sc.shape)
    for _ in range(2):  # the shared array keeps the previous call's contents
        _static_voxelize(ctx, vs)
        got, problems = oracle.canonical_of_export(vs.export())
        assert problems == []
        assert got == want
    vs.cleanup()
    ref.cleanup()
    ctx.close()
