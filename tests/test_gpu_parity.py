"""GPU parity: the sm_100a voxelizer and raytracer against the CPU oracle.

Every case builds the tree on the device through the C-ABI (frep_voxelize /
frep_render via the Python mirror) and on the oracle from the same tape, then
requires
* tile classifications (leaf and interior masks), tree topology and shortened
  tapes to be bit-exact in canonical form (nodes keyed by coordinates);
* per-pixel hit cells to be identical and hit depth / normals to agree within
  1e-5 relative (they are computed with the same IEEE operations);
* rgba8 pixels to be identical.
"""
from __future__ import annotations

import numpy as np
import pytest

import frep
import oracle
from frep import scenes
from parity import compare_hits, compare_trees, device_tree, oracle_tree, render_both

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = frep.Context(0, hbm_budget_bytes=24 << 30)
    yield c
    c.close()


def _small_random(n, seed, dims):
    sc = scenes.random_csg(n, seed=seed, grid_dims=dims, width=160, height=96)
    return sc


@pytest.mark.parametrize("rounding", [0, 1])
def test_spheres_union_tree_and_image(ctx, rounding):
    sc = scenes.spheres_union()
    vs = device_tree(ctx, sc, rounding=rounding)
    exp = vs.export()
    orc = oracle_tree(sc, vs.tape, rounding=rounding)
    assert compare_trees(exp, orc) == []
    d_rgba, d_hits, o_rgba, o_hits = render_both(ctx, vs, orc, sc, frep.Lights())
    assert compare_hits(d_hits, o_hits, exp, orc) == []
    np.testing.assert_array_equal(d_rgba, o_rgba)
    assert (o_hits[..., 4] != 0xFFFFFFFF).sum() > 1000  # the image is not empty


@pytest.mark.parametrize("n,seed,dims", [(8, 3, (8, 4)), (24, 5, (16, 4, 4)), (64, 7, (8, 8, 4))])
def test_random_csg_perspective_with_shadows(ctx, n, seed, dims):
    sc = _small_random(n, seed, list(dims))
    vs = device_tree(ctx, sc, rounding=1)
    exp = vs.export()
    orc = oracle_tree(sc, vs.tape, rounding=1)
    assert compare_trees(exp, orc) == []
    lights = frep.Lights(shadow_mask=1)
    d_rgba, d_hits, o_rgba, o_hits = render_both(ctx, vs, orc, sc, lights)
    assert compare_hits(d_hits, o_hits, exp, orc) == []
    np.testing.assert_array_equal(d_rgba, o_rgba)


@pytest.mark.parametrize("dims", [(8, 12), (4, 16), (12, 8), (16, 32)])
def test_last_level_dims(ctx, dims):
    """Node sizes that select different cells-per-lane and mask layouts."""
    sc = _small_random(20, 8, list(dims))
    vs = device_tree(ctx, sc, rounding=1)
    exp = vs.export()
    orc = oracle_tree(sc, vs.tape, rounding=1)
    assert compare_trees(exp, orc) == []
    d_rgba, d_hits, o_rgba, o_hits = render_both(ctx, vs, orc, sc, frep.Lights())
    assert compare_hits(d_hits, o_hits, exp, orc) == []
    np.testing.assert_array_equal(d_rgba, o_rgba)


@pytest.mark.parametrize("dims,k", [((16, 8), 8), ((8, 16), 8), ((4, 4, 8), 8), ((8, 16), 2)])
def test_last_level_cells_per_lane_option(ctx, dims, k):
    """frep_voxelize_opts.point_cells_per_lane = 8 (and 2 where 4 is the
    default): the same tree and image."""
    sc = _small_random(28, 9, list(dims))
    vs = device_tree(ctx, sc, rounding=1, point_cells_per_lane=k)
    exp = vs.export()
    orc = oracle_tree(sc, vs.tape, rounding=1)
    assert compare_trees(exp, orc) == []
    d_rgba, d_hits, o_rgba, o_hits = render_both(ctx, vs, orc, sc, frep.Lights())
    assert compare_hits(d_hits, o_hits, exp, orc) == []
    np.testing.assert_array_equal(d_rgba, o_rgba)


def test_cells_per_lane_option_is_checked(ctx):
    sc = _small_random(8, 3, [8, 12])
    for k in (3, 4, 8):  # 54 mask words per last-level node: neither 4 nor 8 divides it
        with pytest.raises(frep.FrepError) as e:
            device_tree(ctx, sc, point_cells_per_lane=k)
        assert e.value.status == frep._lib.ERR_INVALID_ARG
    vs = frep.VoxelStorage([8, 16], sc.low_vertex, sc.world_size, point_cells_per_lane=8).init(ctx, sc.shape)
    with pytest.raises(frep.FrepError) as e:  # batches run 2 or 4 cells per lane
        frep.Batch(ctx, [vs])
    assert e.value.status == frep._lib.ERR_UNSUPPORTED


def test_wide_tape_scene(ctx):
    """More than 256 constants: only the wide encoding can hold this tape."""
    sc = _small_random(160, 9, [16, 8])
    vs = device_tree(ctx, sc, rounding=1)
    assert not vs.tape.fits_reference
    orc = oracle_tree(sc, vs.tape, rounding=1)
    assert compare_trees(vs.export(), orc) == []


@pytest.mark.parametrize("name,level,t", [("OrganicBalls", 0, 0.7), ("ElasticCube", 0, 1.3),
                                          ("Screw", 0, 2.0), ("MengerSponge", 2, 0.0)])
@pytest.mark.parametrize("rounding", [0, 1])
def test_reference_demo_shapes_animated(ctx, name, level, t, rounding):
    """The reference's own demo scenes (vulkan/src/shapes.cpp), with T != 0 and
    SIN/COS/EXP in the tapes, on the reference's 40-unit world."""
    shape = scenes.DEMO_SHAPES[name](level)
    cam = frep.Camera(position=(0, 0, 40.0), forward=(0, 0, -1), initial_up=(0, 1, 0), fov_deg=45)
    sc = scenes.Scene(name, shape, [16, 4, 4], (-20, -20, -20), 40.0, cam, 128, 96)
    vs = device_tree(ctx, sc, rounding=rounding, tape_time=t)
    exp = vs.export()
    orc = oracle_tree(sc, vs.tape, rounding=rounding, tape_time=t)
    assert compare_trees(exp, orc) == []
    d_rgba, d_hits, o_rgba, o_hits = render_both(ctx, vs, orc, sc, frep.Lights(), tape_time=t)
    assert compare_hits(d_hits, o_hits, exp, orc) == []
    np.testing.assert_array_equal(d_rgba, o_rgba)


def test_no_shortening_matches(ctx):
    sc = _small_random(16, 4, [8, 4])
    vs = device_tree(ctx, sc, rounding=0, shorten=False)
    orc = oracle_tree(sc, vs.tape, rounding=0, shorten=False)
    assert compare_trees(vs.export(), orc) == []


def test_voxelize_is_repeatable(ctx):
    sc = _small_random(32, 6, [16, 4])
    vs = device_tree(ctx, sc)
    a = oracle.canonical_of_export(vs.export())[0]
    frep.Voxelizer(ctx, vs).voxelize(0.0)
    b = oracle.canonical_of_export(vs.export())[0]
    assert a == b


def test_pool_overflow_reports_capacity_error(ctx):
    """A node pool too small for the tree: the voxelizer must stop writing and
    report FREP_ERR_CAPACITY instead of writing past the pool."""
    sc = _small_random(32, 6, [16, 4])
    vs = device_tree(ctx, sc, node_words=5000)
    with pytest.raises(frep.FrepError) as e:
        vs.sync()
    assert e.value.status == frep._lib.ERR_CAPACITY
    root_words = (1 + frep.Tape(sc.shape).n_instr + 15) // 16 * 16
    vs2 = device_tree(ctx, sc, tape_words=root_words + 64)
    with pytest.raises(frep.FrepError) as e:
        vs2.sync()
    assert e.value.status == frep._lib.ERR_CAPACITY


@pytest.mark.parametrize("rounding,t", [(1, 0.37), (0, 0.81)])
def test_stress_gyroid_small(ctx, rounding, t):
    """The stress scene (twisted gyroid lattice with SIN/COS in interval
    arithmetic, smooth-unioned with 64 spheres) on a reduced grid at a tape
    time T > 0: trees, hits and pixels as the oracle's."""
    sc = scenes.stress_gyroid(grid_dims=(8, 8), width=120, height=72)
    vs = device_tree(ctx, sc, rounding=rounding, tape_time=t)
    exp = vs.export()
    orc = oracle_tree(sc, vs.tape, rounding=rounding, tape_time=t)
    assert compare_trees(exp, orc) == []
    lights = frep.Lights(shadow_mask=1)
    d_rgba, d_hits, o_rgba, o_hits = render_both(ctx, vs, orc, sc, lights, tape_time=t)
    assert compare_hits(d_hits, o_hits, exp, orc) == []
    np.testing.assert_array_equal(d_rgba, o_rgba)
    assert sum(exp.node_count) > 100


@pytest.mark.parametrize("rounding", [0, 1])
def test_identical_child_tapes_are_stored_once(ctx, rounding):
    """Cells of a 32-cell group with identical shortened tapes share one copy:
    same canonical tree as the oracle (which stores every copy), a smaller
    pool, and leaf nodes that point at the same tape."""
    sc = scenes.random_csg(120, seed=31, grid_dims=[16, 8, 4], width=64, height=48)
    vs = device_tree(ctx, sc, rounding=rounding)
    exp = vs.export()
    orc = oracle_tree(sc, vs.tape, rounding=rounding)
    assert compare_trees(exp, orc) == []
    used = vs.sync().tape_words_used
    assert used < 0.6 * len(orc.tapes), (used, len(orc.tapes))
    last = exp.levels - 1
    base, size = exp.node_offset[last], exp.node_size[last]
    idx = exp.nodes[base: base + exp.node_count[last] * size: size]
    assert len(np.unique(idx)) < 0.5 * len(idx)
    # one copy per cell, as the reference (and the oracle) store them
    vs2 = frep.VoxelStorage(sc.grid_dims, sc.low_vertex, sc.world_size, rounding=rounding, separate_tapes=True)
    vs2.init(ctx, sc.shape)
    frep.Voxelizer(ctx, vs2).voxelize(0.0)
    exp2 = vs2.export()
    assert compare_trees(exp2, orc) == []
    idx2 = exp2.nodes[base: base + exp2.node_count[last] * size: size]
    assert vs2.sync().tape_words_used > used and len(np.unique(idx2)) > len(np.unique(idx))
