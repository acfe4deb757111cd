"""NaN propagation through MIN / MAX in the level passes, against the oracle.

The reference's min / max are glm's selects, min(a, b) = (b < a) ? b : a and
max(a, b) = (a < b) ? b : a, so a NaN operand propagates from the first
argument of MIN but not from the second (and the other way round for MAX).
The square root of a negative product makes NaN cells in half of the grid;
each tape has the NaN operand first in one MIN / MAX and second in another,
with and without operand forwarding, and the leaf pass runs with 2, 4 and 8
cells per lane (each has its own dispatch).
"""
from __future__ import annotations

import pytest

import frep
from frep import csg, scenes
from parity import compare_trees_fast, device_tree, oracle_tree

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = frep.Context(0, hbm_budget_bytes=4 << 30)
    yield c
    c.close()


def _shapes():
    X, Y, Z = csg.X(), csg.Y(), csg.Z()
    ball = csg.Sphere(csg.Vector3(0.1, -0.2, 0.05), 0.6)
    nan_half = csg.Sqrt(X * Y) - 0.3  # NaN where x * y < 0
    return {
        "min_nan_first": csg.Min(nan_half, ball),
        "min_nan_second": csg.Min(ball, nan_half),
        "max_nan_first": csg.Max(nan_half, ball - 0.5),
        "max_nan_second": csg.Max(ball - 0.5, nan_half),
        "nested": csg.Min(csg.Max(nan_half, Z - 0.4), csg.Min(ball, csg.Sqrt(Y * Z) - 0.2)),
    }


@pytest.mark.parametrize("k", [2, 4, 8])
@pytest.mark.parametrize("name", list(_shapes()))
def test_nan_operands_of_min_max_match_the_oracle(ctx, name, k):
    cam = frep.Camera(position=(0, 0, 3.0), forward=(0, 0, -1), initial_up=(0, 1, 0), fov_deg=45)
    dims = [8, 8] if k != 8 else [8, 16]
    sc = scenes.Scene(name, _shapes()[name], dims, (-1, -1, -1), 2.0, cam, 64, 48)
    for rounding in (0, 1):
        vs = device_tree(ctx, sc, rounding=rounding, point_cells_per_lane=k)
        orc = oracle_tree(sc, vs.tape, rounding=rounding)
        assert compare_trees_fast(vs.export(), orc) == [], (name, k, rounding)
