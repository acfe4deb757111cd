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


def test_static_scratch_long_tape_runs_on_fewer_blocks():
    """The longest tape of the 512-scene batch (30,503 instructions): its
    per-block scratch is so large that the persistent grid is cut to what the
    array holds (fewer blocks than SMs even with one warp and one cell per
    lane), and the tree still equals frep_voxelize's."""
    from parity import compare_trees_fast
    ctx = frep.Context(0, hbm_budget_bytes=8 << 30)
    job = list(scenes.batch_jobs()[156])
    job[4] = (16, 8)
    sc = scenes.batch_scene(tuple(job))
    tape = sc.shape
    n, m = tape.n_instr, tape.n_minmax
    smallest_block = (n + 31) // 32 * 32 + (2 * m + 31) // 32 * 32  # 1 warp, 1 cell per lane
    import torch
    assert smallest_block * torch.cuda.get_device_properties(0).multi_processor_count > (2 << 20)
    ref = frep.VoxelStorage(sc.grid_dims, sc.low_vertex, sc.world_size).init(ctx, tape)
    frep.Voxelizer(ctx, ref).voxelize(0.0, stream=0)
    want = ref.export()
    vs = frep.VoxelStorage(sc.grid_dims, sc.low_vertex, sc.world_size).init(ctx, tape)
    for _ in range(2):
        _static_voxelize(ctx, vs)
        assert compare_trees_fast(vs.export(), want) == []
    vs.cleanup()
    ref.cleanup()
    ctx.close()


def test_static_scratch_refuses_a_tape_beyond_the_array():
    """A root tape whose scratch for one warp exceeds the array under any
    plan (n + 2m > 2^21 words): FREP_ERR_UNSUPPORTED before any work, and the
    tree stays usable."""
    import numpy as np
    ctx = frep.Context(0, hbm_budget_bytes=8 << 30)
    k = 540_000  # k pairs (CONST c -> slot 4; slot 0 = MIN(slot 0, slot 4)): n = 2k, m = k
    c = (np.float32(2.0) + np.arange(k, dtype=np.float32) * np.float32(1e-3)).view(np.uint32).astype(np.uint64)
    words = np.empty(2 * k, np.uint64)
    words[0::2] = np.uint64(0) | (np.uint64(4) << np.uint64(16)) | (c << np.uint64(32))
    words[1::2] = (np.uint64(7) | (np.uint64(0) << np.uint64(16)) | (np.uint64(0) << np.uint64(32))
                   | (np.uint64(4) << np.uint64(48)))
    long_tape = frep.Tape.from_wide(words)
    assert long_tape.n_instr + 2 * long_tape.n_minmax > (2 << 20)
    sc = scenes.random_csg(16, seed=21, grid_dims=[16, 4])
    small = frep.Tape(sc.shape)
    vs = frep.VoxelStorage(sc.grid_dims, sc.low_vertex, sc.world_size, tape_words=4 << 20).init(ctx, small)
    lib = frep._lib.lib()
    st = lib.frep_voxelize_static_scratch(ctx._h, vs.tree, long_tape.handle, C.c_float(0.0), C.c_void_p(0))
    assert st == frep._lib.ERR_UNSUPPORTED
    assert b"static scratch" in lib.frep_last_error()
    ref = frep.VoxelStorage(sc.grid_dims, sc.low_vertex, sc.world_size).init(ctx, small)
    frep.Voxelizer(ctx, ref).voxelize(0.0, stream=0)
    want, _ = oracle.canonical_of_export(ref.export())
    _static_voxelize(ctx, vs)
    got, problems = oracle.canonical_of_export(vs.export())
    assert problems == [] and got == want
    vs.cleanup()
    ref.cleanup()
    ctx.close()
