"""Re-voxelization with reuse (frep_voxelize_reuse): a tree built from the
previous frame's tree must equal, in canonical form, the oracle's full
voxelization at the new time — with the previous tree at another time, of
another tape, overflowed, or fully reusable — and render the same image as a
full voxelization. Reuse must actually skip work where the scene allows it."""
from __future__ import annotations

import numpy as np
import pytest

import frep
from frep import scenes
from parity import compare_hits, compare_trees, oracle_tree

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = frep.Context(0, hbm_budget_bytes=24 << 30)
    yield c
    c.close()


def _storage(sc, tape, ctx, rounding=1, **kw):
    vs = frep.VoxelStorage(sc.grid_dims, sc.low_vertex, sc.world_size, rounding=rounding, **kw)
    return vs.init(ctx, tape)


def _total_work(vs):
    vs.sync()
    return sum(vs.work())


@pytest.mark.parametrize("rounding", [0, 1])
def test_frames_equal_full_voxelizations(ctx, rounding):
    sc = scenes.animated_csg(60, 3, seed=11, grid_dims=[16, 8, 4], width=96, height=64)
    tape = frep.Tape(sc.shape)
    assert tape.uses_time
    anim = frep.AnimatedVoxelizer(ctx, lambda: frep.VoxelStorage(sc.grid_dims, sc.low_vertex, sc.world_size,
                                                                 rounding=rounding), tape)
    full = _storage(sc, tape, ctx, rounding)
    for t in (0.1, 0.13, 0.6, 0.61):
        vs = anim.voxelize(t)
        exp = vs.export()
        assert compare_trees(exp, oracle_tree(sc, tape, rounding=rounding, tape_time=t)) == [], t
        frep.Voxelizer(ctx, full).voxelize(t)
        if t != 0.1:  # frames after the first copy the static part (most of it after a small step)
            assert _total_work(vs) < (0.6 if t in (0.13, 0.61) else 0.95) * _total_work(full), t
    anim.cleanup()
    full.cleanup()


def test_image_equals_full_voxelization(ctx):
    import torch
    sc = scenes.animated_csg(60, 3, seed=12, grid_dims=[16, 8, 4], width=128, height=96)
    tape = frep.Tape(sc.shape)
    a, b, full = _storage(sc, tape, ctx), _storage(sc, tape, ctx), _storage(sc, tape, ctx)
    frep.Voxelizer(ctx, a).voxelize(0.25)
    frep.Voxelizer(ctx, b).voxelize(0.3, reuse=a)
    frep.Voxelizer(ctx, full).voxelize(0.3)
    lights = frep.Lights(shadow_mask=1)
    imgs = []
    for vs in (b, full):
        rt = frep.Raytracer(ctx, vs)
        rt.lights = lights
        rgba, hits = rt.trace(sc.camera, 0.3, sc.width, sc.height, hits=True)
        torch.cuda.synchronize()
        imgs.append((rgba.cpu().numpy(), hits.cpu().numpy().view(np.uint32)))
    np.testing.assert_array_equal(imgs[0][0], imgs[1][0])
    # hit records name nodes by id, which differ; the hit cells, depths and
    # normals are identical
    assert compare_hits(imgs[0][1], imgs[1][1], b.export(), full.export(), rtol=0.0) == []
    ib, ifull = b.sync(), full.sync()
    assert list(ib.node_count) == list(ifull.node_count)
    assert list(ib.tape_size_sum) == list(ifull.tape_size_sum)
    assert list(ib.tape_size_max) == list(ifull.tape_size_max)
    for s in (a, b, full):
        s.cleanup()


def test_time_free_scene_is_copied_whole(ctx):
    sc = scenes.random_csg(50, seed=21, grid_dims=[8, 8, 4], width=64, height=48)
    tape = frep.Tape(sc.shape)
    a, b = _storage(sc, tape, ctx), _storage(sc, tape, ctx)
    frep.Voxelizer(ctx, a).voxelize(0.0)
    frep.Voxelizer(ctx, b).voxelize(0.5, reuse=a)
    assert compare_trees(b.export(), oracle_tree(sc, tape, tape_time=0.5)) == []
    assert _total_work(b) == 0  # nothing evaluated, not even the root
    assert b.fp32_ops() == [0] * b.grid_levels
    assert a.fp32_ops() != [0] * a.grid_levels


def test_time_dependent_everywhere(ctx):
    """Morph rotates the whole shape with T: no tape is time-free below the
    root that could be copied; the result is still exact."""
    tape = frep.Tape(scenes.Morph())
    sc = scenes.Scene("morph", scenes.Morph(), [16, 4, 4], (-20.0, -20.0, -20.0), 40.0)
    a, b = _storage(sc, tape, ctx), _storage(sc, tape, ctx)
    frep.Voxelizer(ctx, a).voxelize(0.2)
    frep.Voxelizer(ctx, b).voxelize(0.9, reuse=a)
    assert compare_trees(b.export(), oracle_tree(sc, tape, tape_time=0.9)) == []


def test_prev_of_another_tape_or_overflowed(ctx):
    sc = scenes.animated_csg(40, 2, seed=13, grid_dims=[16, 8, 4], width=64, height=48)
    tape = frep.Tape(sc.shape)
    other = frep.Tape(scenes.animated_csg(40, 2, seed=14, grid_dims=[16, 8, 4]).shape)
    # prev of another scene: only exactly matching time-free tapes are copied
    a = _storage(sc, other, ctx)
    frep.Voxelizer(ctx, a).voxelize(0.4)
    b = _storage(sc, tape, ctx)
    frep.Voxelizer(ctx, b).voxelize(0.4, reuse=a)
    assert compare_trees(b.export(), oracle_tree(sc, tape, tape_time=0.4)) == []
    # prev whose node pool overflowed: not used
    small = _storage(sc, tape, ctx, node_words=8192)
    frep.Voxelizer(ctx, small).voxelize(0.4)
    with pytest.raises(frep.FrepError):
        small.sync()
    c = _storage(sc, tape, ctx)
    frep.Voxelizer(ctx, c).voxelize(0.45, reuse=small)
    assert compare_trees(c.export(), oracle_tree(sc, tape, tape_time=0.45)) == []
    # a reusing tree whose own pools are too small reports the overflow
    d = _storage(sc, tape, ctx, tape_words=4096)
    frep.Voxelizer(ctx, d).voxelize(0.45, reuse=c)
    with pytest.raises(frep.FrepError):
        d.sync()


def test_invalid_prev(ctx):
    sc = scenes.animated_csg(20, 1, seed=15, grid_dims=[8, 8, 4])
    tape = frep.Tape(sc.shape)
    a, b = _storage(sc, tape, ctx), _storage(sc, tape, ctx)
    with pytest.raises(frep.FrepError):  # prev not voxelized
        frep.Voxelizer(ctx, b).voxelize(0.1, reuse=a)
    frep.Voxelizer(ctx, a).voxelize(0.1)
    with pytest.raises(frep.FrepError):  # prev is the tree itself
        frep.Voxelizer(ctx, a).voxelize(0.2, reuse=a)
    g = frep.VoxelStorage([8, 4, 8], sc.low_vertex, sc.world_size).init(ctx, tape)
    with pytest.raises(frep.FrepError):  # another grid
        frep.Voxelizer(ctx, g).voxelize(0.2, reuse=a)
    r = frep.VoxelStorage(sc.grid_dims, sc.low_vertex, sc.world_size, rounding=0).init(ctx, tape)
    with pytest.raises(frep.FrepError):  # another rounding
        frep.Voxelizer(ctx, r).voxelize(0.2, reuse=a)
