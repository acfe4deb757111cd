"""GPU parity of compact trees (frep_tree_compact, frep_render_compact,
frep_compact_export / import) against the oracle's restatement of
SceneBuilder's compaction (scene_builder.cpp: BuildNode :91-156, LayoutNode
:199-238).

Compaction is integer work with a deterministic numbering (preorder), so the
device's compact tree must equal the oracle's node for node: coordinates,
masks and child links exactly, tapes by content. Renders through the compact
layout must hit the same nodes (by preorder index) and cells as the oracle's
render of its compact tree, with the same depths and normals."""
from __future__ import annotations

import numpy as np
import pytest

import frep
import oracle
from frep import compact, scenes
from parity import compare_hits, device_tree, oracle_tree

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = frep.Context(0, hbm_budget_bytes=24 << 30)
    yield c
    c.close()


def _records(t, l):
    return t.nodes[t.node_offset[l]: t.node_offset[l] + t.node_count[l] * t.node_size[l]].reshape(
        t.node_count[l], t.node_size[l])


def compare_compact(e, orc):
    """Differences between an expanded compact blob and the oracle's compact
    tree (same preorder numbering): empty = equal."""
    if list(e.node_count) != list(orc.node_count):
        return [f"node counts {e.node_count} != {orc.node_count}"]
    diffs = []
    for l in range(e.levels):
        a, b = _records(e, l), _records(orc, l)
        bad = np.nonzero((a[:, 1:] != b[:, 1:]).any(axis=1))[0]
        if len(bad):
            diffs.append(f"level {l}: {len(bad)} records differ (coords / masks / children), first {bad[0]}")
        nt = sum(oracle.tape_at(e.tapes, int(x)) != oracle.tape_at(orc.tapes, int(y)) for x, y in zip(a[:, 0], b[:, 0]))
        if nt:
            diffs.append(f"level {l}: {nt} tapes differ")
    return diffs


def _scenes():
    demo_cam = frep.Camera(position=(0, 0, 40.0), forward=(0, 0, -1), initial_up=(0, 1, 0), fov_deg=45)
    return {
        "spheres": (lambda: scenes.spheres_union(16, seed=1, width=128, height=128), 0.0),
        "random3": (lambda: scenes.random_csg(24, seed=5, grid_dims=[16, 4, 4], width=160, height=96), 0.0),
        "random8": (lambda: scenes.random_csg(64, seed=7, grid_dims=[8, 8, 4], width=160, height=96), 0.0),
        "organic": (lambda: scenes.Scene("OrganicBalls", scenes.DEMO_SHAPES["OrganicBalls"](0), [16, 4, 4],
                                         (-20, -20, -20), 40.0, demo_cam, 128, 96), 0.7),
        "menger": (lambda: scenes.Scene("MengerSponge", scenes.DEMO_SHAPES["MengerSponge"](2), [8, 4, 4],
                                        (-20, -20, -20), 40.0, demo_cam, 128, 96), 0.0),
    }


@pytest.mark.parametrize("prune", [False, True])
@pytest.mark.parametrize("name,rounding", [("spheres", 1), ("spheres", 0), ("random3", 1), ("random8", 1),
                                           ("organic", 0), ("menger", 1)])
def test_compact_tree_and_render_match_the_oracle(ctx, name, rounding, prune):
    make, t = _scenes()[name]
    sc = make()
    vs = device_tree(ctx, sc, rounding=rounding, tape_time=t)
    ct = frep.CompactTree.from_storage(ctx, vs, prune=prune)
    blob = ct.export()
    compact.check(blob)
    e = compact.expand(blob)
    assert e.mode == (1 if prune else 0)
    orc = oracle_tree(sc, vs.tape, rounding=rounding, tape_time=t).compact(prune)
    assert compare_compact(e, orc) == []

    import torch
    lights = frep.Lights(shadow_mask=1)
    ct.lights = lights
    rgba, hits = ct.trace(sc.camera, t, sc.width, sc.height, hits=True)
    torch.cuda.synchronize()
    d_rgba, d_hits = rgba.cpu().numpy(), hits.cpu().numpy().view(np.uint32)
    o_rgba, o_hits = orc.render(oracle.camera_vector(sc.camera, sc.width, sc.height), lights, t)
    np.testing.assert_array_equal(d_hits[..., 4:7], o_hits[..., 4:7])  # level, preorder node, cell
    assert compare_hits(d_hits, o_hits, e, orc) == []
    np.testing.assert_array_equal(d_rgba, o_rgba)
    assert (o_hits[..., 4] != 0xFFFFFFFF).sum() > 100


@pytest.mark.parametrize("name", ["spheres", "random3"])
def test_layout_mode_renders_exactly_like_the_source_tree(ctx, name):
    import torch
    make, t = _scenes()[name]
    sc = make()
    vs = device_tree(ctx, sc, rounding=1)
    ct = frep.CompactTree.from_storage(ctx, vs, prune=False)
    lights = frep.Lights(shadow_mask=1)
    rt = frep.Raytracer(ctx, vs)
    rt.lights = lights
    ct.lights = lights
    a_rgba, a_hits = rt.trace(sc.camera, t, sc.width, sc.height, hits=True)
    b_rgba, b_hits = ct.trace(sc.camera, t, sc.width, sc.height, hits=True)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(a_rgba.cpu().numpy(), b_rgba.cpu().numpy())
    ah, bh = a_hits.cpu().numpy().view(np.uint32), b_hits.cpu().numpy().view(np.uint32)
    for f in (0, 1, 2, 3, 4, 6, 7):  # t, normal, level, cell, steps: bit for bit
        np.testing.assert_array_equal(ah[..., f], bh[..., f])
    exp = vs.export()
    e = compact.expand(ct.export())
    ka = oracle.hit_cells(ah, exp.dims, exp.node_offset, exp.node_size, exp.nodes)
    kb = oracle.hit_cells(bh, e.dims, e.node_offset, e.node_size, e.nodes)
    np.testing.assert_array_equal(ka, kb)


def test_blob_import_round_trip(ctx):
    import torch
    make, _ = _scenes()["random3"]
    sc = make()
    vs = device_tree(ctx, sc, rounding=1)
    for prune in (False, True):
        ct = frep.CompactTree.from_storage(ctx, vs, prune=prune)
        blob = ct.export()
        ct2 = frep.CompactTree.from_blob(ctx, blob)
        np.testing.assert_array_equal(ct2.export(), blob)
        i1, i2 = ct.info(), ct2.info()
        assert list(i1.node_count) == list(i2.node_count) and i1.device_bytes == i2.device_bytes
        r1, h1 = ct.trace(sc.camera, 0.0, sc.width, sc.height, hits=True)
        r2, h2 = ct2.trace(sc.camera, 0.0, sc.width, sc.height, hits=True)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(r1.cpu().numpy(), r2.cpu().numpy())
        np.testing.assert_array_equal(h1.cpu().numpy(), h2.cpu().numpy())
        ct2.close()
        ct.close()
    # a damaged blob is refused before anything reaches the device
    bad = blob.copy()
    bad[120] ^= 0xFF  # the root's tape index
    with pytest.raises(frep.FrepError) as e:
        frep.CompactTree.from_blob(ctx, bad)
    assert e.value.status == frep._lib.ERR_INVALID_ARG


def test_compact_memory_and_shared_tapes(ctx):
    make, _ = _scenes()["random3"]
    sc = make()
    vs = device_tree(ctx, sc, rounding=1)
    info = vs.sync()
    full = info.node_words_used * 4 + info.tape_words_used * 8
    ct = frep.CompactTree.from_storage(ctx, vs, prune=False)
    ci = ct.info()
    assert ci.device_bytes == ci.node_words * 4 + ci.tape_words * 8
    assert ci.node_words * 4 < info.node_words_used * 4 / 4  # child lists dropped
    assert ci.tape_words <= info.tape_words_used
    assert ci.device_bytes < full
    # every distinct tape of the source is stored once in the compact pool
    exp = vs.export()
    src_tapes = {int(r[0]) for l in range(exp.levels) for r in _records(exp, l)}
    e = compact.expand(ct.export())
    dst_tapes = {int(r[0]) for l in range(e.levels) for r in _records(e, l)}
    assert len(dst_tapes) == len(src_tapes)
    assert sum((1 + int(e.tapes[i] & 0xFFFFFFFF) + 15) // 16 * 16 for i in dst_tapes) == ci.tape_words
    used, _ = ctx.memory()
    ct.close()
    assert ctx.memory()[0] == used - ci.device_bytes


def test_compact_refuses_unfinished_trees(ctx):
    sc = scenes.random_csg(32, seed=6, grid_dims=[16, 4], width=64, height=64)
    vs = frep.VoxelStorage(sc.grid_dims, sc.low_vertex, sc.world_size).init(ctx, sc.shape)
    with pytest.raises(frep.FrepError) as e:
        frep.CompactTree.from_storage(ctx, vs)
    assert e.value.status == frep._lib.ERR_INVALID_ARG
    vs2 = device_tree(ctx, sc, node_words=5000)  # overflows its node pool
    with pytest.raises(frep.FrepError) as e:
        frep.CompactTree.from_storage(ctx, vs2)
    assert e.value.status == frep._lib.ERR_CAPACITY


def test_compact_of_batched_and_reused_trees(ctx):
    """Trees voxelized by a batch (frep_batch_voxelize) and by reuse of a
    previous frame (frep_voxelize_reuse) compact to the oracle's compaction of
    the same tape, like trees voxelized alone."""
    scs = [scenes.random_csg(12 + 10 * i, seed=60 + i, grid_dims=list(d), width=64, height=48)
           for i, d in enumerate([(16, 4), (8, 8, 4), (16, 4, 4)])]
    storages = [frep.VoxelStorage(sc.grid_dims, sc.low_vertex, sc.world_size).init(ctx, sc.shape) for sc in scs]
    batch = frep.Batch(ctx, storages)
    times = [0.0, 0.2, 0.4]
    batch.voxelize(times)
    for sc, vs, t in zip(scs, storages, times):
        for prune in (False, True):
            e = compact.expand(frep.CompactTree.from_storage(ctx, vs, prune=prune).export())
            orc = oracle_tree(sc, vs.tape, rounding=1, tape_time=t).compact(prune)
            assert compare_compact(e, orc) == [], (sc.grid_dims, prune)
    batch.close()

    sc = scenes.animated_csg(40, 3, seed=13, grid_dims=[16, 8, 4], width=64, height=48)
    tape = frep.Tape(sc.shape)
    a = frep.VoxelStorage(sc.grid_dims, sc.low_vertex, sc.world_size).init(ctx, tape)
    b = frep.VoxelStorage(sc.grid_dims, sc.low_vertex, sc.world_size).init(ctx, tape)
    frep.Voxelizer(ctx, a).voxelize(0.25)
    frep.Voxelizer(ctx, b).voxelize(0.3, reuse=a)
    for prune in (False, True):
        e = compact.expand(frep.CompactTree.from_storage(ctx, b, prune=prune).export())
        orc = oracle_tree(sc, tape, rounding=1, tape_time=0.3).compact(prune)
        assert compare_compact(e, orc) == [], prune
