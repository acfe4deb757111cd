"""Exactness of item-level pruning, on the CPU oracle.

Below the root, the device's interval passes evaluate a node's tape once over
the bounding box of each work item (a 4x4x4 brick of the node's cells, 2x4x4
with one cell per lane)
and, when the tape is algebraic (no SIN / COS / EXP) and every interval of
that evaluation is finite, let the item's cells run the node tape shortened
over the item box; an item box that is empty or inside decides its cells
without evaluating them. The trees must not change. This test checks the
claims that rest on, cell by cell, with the oracle's own interval evaluator
and shortener (the reference's algorithm):
(a) a cell's interval from the item tape is bit-identical to its interval
    from the node tape, so its class (empty, leaf, ambiguous) is the same;
(b) an ambiguous cell's child tape from the item tape (kept when shorter
    than the node tape, else the node tape itself) equals its child tape from
    the node tape word for word;
(c) every cell of an empty (inside) item box is empty (a leaf).
Scenes: a sphere union, random CSG of spheres, boxes and capsules, a tape
with a division whose denominator stays positive and one whose denominator
changes sign (items there are left to the node tape); both roundings.
"""
from __future__ import annotations

import numpy as np
import pytest

import frep
import oracle
from containment import cell_sizes, n_slots_of, tape_of
from frep import csg, scenes
from parity import oracle_tree

OP_SIN, OP_COS, OP_EXP, OP_MIN, OP_MAX, OP_COPY = 1, 2, 9, 7, 8, 12
F32 = np.float32


def _scene(name):
    cam = frep.Camera(position=(0, 0, 40.0), forward=(0, 0, -1), initial_up=(0, 1, 0), fov_deg=45)
    if name == "spheres16":
        sc = scenes.spheres_union(16)
        sc.grid_dims = [8, 8, 4]
        return sc
    if name == "csg48":
        return scenes.random_csg(48, seed=3, grid_dims=[8, 8, 4])
    X, Y, Z = csg.X(), csg.Y(), csg.Z()
    if name == "div_positive":
        shape = csg.Min(csg.Sphere(csg.Vector3(0.3, -0.2, 0.1), 0.5),
                        (X * X + Y * Y + Z * Z) / (X + 3.0) - 0.2)
    else:  # div_sign_change: the denominator crosses zero inside the grid
        shape = csg.Min(csg.Sphere(csg.Vector3(-0.4, 0.3, 0.0), 0.4), X / (Y + 0.05) - 0.8)
    return scenes.Scene(name, shape, [8, 8, 4], (-1, -1, -1), 2.0, cam, 64, 48)


def _brick_cells(dim, item, xs=4):
    """The kernel's work item `item` of a node (bricks numbered z fastest,
    x extent xs): its cells' (x, y, z) in the node, brick cell order."""
    nb = dim // 4
    ox, oy, oz = item // (nb * nb) * xs, item // nb % nb * 4, item % nb * 4
    return [(ox + (i >> 4), oy + ((i >> 2) & 3), oz + (i & 3)) for i in range(16 * xs)]


def _item_box(low, cs, node_xyz, dim, cells):
    """The kernel's item box: the cells' own box formula at the brick's
    smallest and largest coordinates."""
    c = np.array(cells)
    g0 = np.array(node_xyz) * dim + c.min(axis=0)
    g1 = np.array(node_xyz) * dim + c.max(axis=0)
    lo = np.array([F32(F32(low[k]) + F32(F32(g0[k]) * cs)) for k in range(3)], F32)
    hi = np.array([F32(F32(F32(low[k]) + F32(F32(g1[k]) * cs)) + cs) for k in range(3)], F32)
    return lo, hi


def _cell_box(low, cs, g):
    lo = np.array([F32(F32(low[k]) + F32(F32(g[k]) * cs)) for k in range(3)], F32)
    return lo, (lo + cs).astype(F32)


def _kept_with_rewrites(tape, ns, choices):
    """The tape shortened by one evaluation's choices, without the "not
    shorter -> reuse" rule (the kernel keeps a cell's tape whenever it is
    shorter than the node's, even if no shorter than the item's)."""
    short = oracle.shorten(tape, ns, choices)
    if len(short) < len(tape):
        return short
    out = np.array(tape, np.uint64)
    op = out & np.uint64(0xFF)
    for j, i in enumerate(np.flatnonzero((op == OP_MIN) | (op == OP_MAX))):
        w = int(out[i])
        if choices[j] == 1:
            w = (w & ~0xFF) | OP_COPY
        elif choices[j] == 2:
            w = (w & ~0xFF & ~(0xFFFF << 32)) | OP_COPY | ((w >> 48) << 32)
        out[i] = np.uint64(w)
    return out


def _check_scene(sc, rounding, cells_per_item=64, nodes_per_level=6, items_per_node=4, seed=0):
    tape = frep.Tape(sc.shape)
    orc = oracle_tree(sc, tape, rounding=rounding)
    css = cell_sizes(sc.grid_dims, sc.world_size)
    rng = np.random.default_rng(seed)
    stats = dict(items=0, pruned=0, decided=0, skipped=0, cells=0)
    for lvl in range(orc.levels - 1):
        dim, cs = sc.grid_dims[lvl], F32(css[lvl])
        if dim ** 3 <= cells_per_item:
            continue
        n_items = dim ** 3 // cells_per_item
        nodes = orc.node_count[lvl]
        for ni in rng.choice(nodes, size=min(nodes, nodes_per_level), replace=False):
            rec = orc.nodes[orc.node_offset[lvl] + ni * orc.node_size[lvl]:][:4]
            node_tape = tape_of(orc.tapes, int(rec[0]))
            ns = n_slots_of(node_tape)
            n_node = len(node_tape)
            node_xyz = [int(v) for v in rec[1:4]]
            for item in rng.choice(n_items, size=min(n_items, items_per_node), replace=False):
                stats["items"] += 1
                cells = _brick_cells(dim, int(item), xs=cells_per_item // 16)
                lo, hi = _item_box(sc.low_vertex, cs, node_xyz, dim, cells)
                trace = oracle.eval_interval_trace(node_tape, ns, lo, hi, 0.0, rounding)
                ops = node_tape & np.uint64(0xFF)
                if np.isin(ops, (OP_SIN, OP_COS, OP_EXP)).any() or not np.isfinite(trace).all():
                    stats["skipped"] += 1
                    continue
                iv_item, ch_item = oracle.eval_interval(node_tape, ns, lo, hi, 0.0, rounding)
                item_tape = oracle.shorten(node_tape, ns, ch_item)
                decided = iv_item[0] > 0 or iv_item[1] < 0
                stats["decided"] += int(decided)
                stats["pruned"] += int(not decided and len(item_tape) < n_node)
                for c in cells:
                    g = np.array(node_xyz) * dim + np.array(c)
                    clo, chi = _cell_box(sc.low_vertex, cs, g)
                    iv_n, ch_n = oracle.eval_interval(node_tape, ns, clo, chi, 0.0, rounding)
                    stats["cells"] += 1
                    if iv_item[0] > 0:
                        assert iv_n[0] > 0, (lvl, int(ni), c)  # (c) empty item: empty cell
                        continue
                    if iv_item[1] < 0:
                        assert iv_n[1] < 0 and not iv_n[0] > 0, (lvl, int(ni), c)  # (c) inside: leaf
                        continue
                    iv_i, ch_i = oracle.eval_interval(item_tape, ns, clo, chi, 0.0, rounding)
                    # (a) the same interval, bit for bit
                    assert iv_i.view(np.uint32).tolist() == iv_n.view(np.uint32).tolist(), (lvl, int(ni), c)
                    if iv_n[0] > 0 or iv_n[1] < 0:
                        continue
                    # (b) the same child tape
                    child_n = oracle.shorten(node_tape, ns, ch_n)
                    kept = _kept_with_rewrites(item_tape, ns, ch_i)
                    child_i = kept if len(kept) < n_node else node_tape
                    assert np.array_equal(child_i, child_n), (lvl, int(ni), c, len(child_i), len(child_n))
    return stats


@pytest.mark.parametrize("rounding", [0, 1])
@pytest.mark.parametrize("name", ["spheres16", "csg48", "div_positive"])
def test_item_tapes_give_the_cells_their_node_tape_results(name, rounding):
    s = _check_scene(_scene(name), rounding)
    assert s["cells"] > 500, s
    assert s["pruned"] > 0, s  # item tapes shorter than the node's were exercised
    assert s["skipped"] == 0, s


def test_items_where_a_denominator_changes_sign_are_left_to_the_node_tape():
    s = _check_scene(_scene("div_sign_change"), 1, nodes_per_level=10, items_per_node=8)
    assert s["skipped"] > 0 and s["cells"] > 0, s


def test_decided_items_occur():
    s = _check_scene(_scene("csg48"), 1, nodes_per_level=12, items_per_node=8, seed=1)
    assert s["decided"] > 0, s
