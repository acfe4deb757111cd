"""Index arithmetic of the interval passes' brick work items, on the CPU.

The level passes (csrc/voxelizer.cu: brick_origin, brick_cell,
or_group_masks) give each work item a brick of a node: 4x4x4 cells with two
cells per lane, 2x4x4 with one; bricks are numbered z fastest; lane l's h-th
cell is brick cell i = 32h + l with z = i & 3, y = (i >> 2) & 3, x = i >> 4.
The node's leaf and interior masks keep the reference's layout (bit
z + dim*y + dim^2*x, voxelizer/main.comp:88-108, utils.comp:6), filled by
ORing each row of four lanes' bits into one mask word. This restates those
formulas and checks, for every node dim the grids allow (multiples of 4 up
to 32) and both cell counts per lane:
(a) the bricks of a node cover every cell exactly once;
(b) the four lanes 4r .. 4r+3 of a row are consecutive cells along z, their
    bits consecutive in one mask word, starting on a 4-bit boundary;
(c) the items per node equal the level scan's count, dim^3 / 32 / KI.
"""
from __future__ import annotations

import numpy as np
import pytest


def brick_origin(grp, dim, ki):
    xs = 2 * ki
    nb = dim // 4
    return grp // (nb * nb) * xs, grp // nb % nb * 4, grp % nb * 4


def brick_cell(origin, i, dim):
    x, y, z = origin[0] + (i >> 4), origin[1] + ((i >> 2) & 3), origin[2] + (i & 3)
    return (x * dim + y) * dim + z, (x, y, z)


@pytest.mark.parametrize("ki", [1, 2])
@pytest.mark.parametrize("dim", [4, 8, 12, 16, 20, 24, 28, 32])
def test_bricks_tile_the_node_and_rows_fill_whole_nibbles(dim, ki):
    items = dim ** 3 // 32 // ki  # level_items: words / cells per lane
    seen = np.zeros(dim ** 3, np.int32)
    for grp in range(items):
        o = brick_origin(grp, dim, ki)
        assert o[0] + 2 * ki <= dim and o[1] + 4 <= dim and o[2] + 4 <= dim
        for h in range(ki):
            cells = []
            for lane in range(32):
                c, xyz = brick_cell(o, 32 * h + lane, dim)
                assert all(0 <= v < dim for v in xyz)
                seen[c] += 1
                cells.append(c)
            for r in range(8):  # or_group_masks: lane 4r ORs the row's nibble at bit c & 31
                row = cells[4 * r:4 * r + 4]
                assert row == list(range(row[0], row[0] + 4))
                assert row[0] % 4 == 0 and (row[0] >> 5) == (row[3] >> 5)
    assert (seen == 1).all()


def test_two_cells_per_lane_split_a_brick_into_the_one_cell_bricks():
    """With two cells per lane, group h of brick g is the one-cell-per-lane
    brick at the same y, z and x offset 2h: the 32-cell groups within which
    shortened tapes are shared are the same whichever width a pass runs."""
    for dim in (8, 16, 32):
        nb = dim // 4
        for grp in range(dim ** 3 // 64):
            o2 = brick_origin(grp, dim, 2)
            for h in range(2):
                g1 = (o2[0] + 2 * h) // 2 * nb * nb + o2[1] // 4 * nb + o2[2] // 4
                o1 = brick_origin(g1, dim, 1)
                a = [brick_cell(o2, 32 * h + l, dim)[0] for l in range(32)]
                b = [brick_cell(o1, l, dim)[0] for l in range(32)]
                assert a == b
