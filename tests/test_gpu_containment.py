"""Soundness of the device's outward-rounding mode against FP64 dense sampling.

For trees the sm_100a level passes build (frep_voxelize, outward rounding),
on a sample of nodes at every interval level:
(a) the interval the device computes for each cell box
    (frep_tape_eval_intervals: the level passes' per-instruction functions)
    contains the tape's exact value at a 9^3 grid of points per cell,
    corners included, bounded by FP64 evaluation with a rigorous error bound
    (oracle/fp64.py);
(b) the level pass's own leaf / empty marks agree with those samples;
(c) each node's shortened tape has the root tape's exact value on the
    node's box.
The device's intervals for those boxes are also bit-identical to the
oracle's. Scenes: the 16-sphere union, a random CSG tree, the twisted gyroid
(SIN/COS), and the reference's demo shapes with EXP and time-driven rotations
(vulkan/src/shapes.cpp:5-117). Setting FREP_CONTAINMENT_REPORT=<path> writes
the per-scene figures (samples, largest FP64 excess, largest FP64 error
bound) there as JSON.

The directed-rounding operations themselves are pinned on the device too:
intervals of single operations over degenerate boxes [a, a], [b, b] are the
exact result rounded down and up (fractions.Fraction).
"""
from __future__ import annotations

import json
import os
from fractions import Fraction

import numpy as np
import pytest

import frep
from containment import check_tree, oracle_intervals
from frep import csg, scenes
from parity import device_tree

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = frep.Context(0, hbm_budget_bytes=16 << 30)
    yield c
    c.close()


_REPORT = {}


def _demo(name, level, dims=(16, 4, 4)):
    cam = frep.Camera(position=(0, 0, 40.0), forward=(0, 0, -1), initial_up=(0, 1, 0), fov_deg=45)
    return scenes.Scene(name, scenes.DEMO_SHAPES[name](level), list(dims), (-20, -20, -20), 40.0, cam, 64, 48)


CASES = [
    ("spheres16", lambda: scenes.spheres_union(16), 0.0),
    ("csg160", lambda: scenes.random_csg(160, seed=9, grid_dims=[16, 8, 4]), 0.0),
    ("gyroid64", lambda: scenes.stress_gyroid(grid_dims=(16, 16, 4)), 0.37),
    ("Screw", lambda: _demo("Screw", 0), 2.0),
    ("ElasticCube", lambda: _demo("ElasticCube", 0), 1.3),
    ("OrganicBalls", lambda: _demo("OrganicBalls", 0), 0.7),
    ("TwistedTower", lambda: _demo("TwistedTower", 4), 0.0),
    ("Morph", lambda: _demo("Morph", 0), 0.9),
]


@pytest.mark.parametrize("name,make,t", CASES, ids=[c[0] for c in CASES])
def test_device_outward_tree_is_sound(ctx, name, make, t):
    sc = make()
    vs = device_tree(ctx, sc, rounding=frep.ROUND_OUTWARD, tape_time=t)
    exp = vs.export()
    compared = []

    def device_intervals(wide, ns, boxes, tt):
        iv = ctx.eval_intervals(frep.Tape.from_wide(wide), boxes, tt, frep.ROUND_OUTWARD)
        if len(compared) < 3:  # the device's bits are the oracle's
            k = min(len(boxes), 16)
            np.testing.assert_array_equal(iv[:k], oracle_intervals(wide, ns, boxes[:k], tt))
            compared.append(k)
        return iv

    rep = check_tree(exp, vs.tape.wide(), vs.tape.n_slots, sc.low_vertex, sc.world_size, t, device_intervals,
                     nodes_per_level=12, cells_per_node=32, per_axis=9, seed=1, root_cells=64)
    s = rep.summary()
    s.update(tape_instructions=vs.tape.n_instr, grid=list(sc.grid_dims), tape_time=t)
    _REPORT[name] = s
    path = os.environ.get("FREP_CONTAINMENT_REPORT")
    if path:
        with open(path, "w") as f:
            json.dump(_REPORT, f, indent=1)
    assert rep.ok(), s
    assert s["samples"] >= 40_000, s
    assert s["max_fp64_excess"] <= s["max_fp64_error_bound"], s


def _round_dir(q: Fraction, up: bool) -> np.float32:
    """The float32 next to the exact value q in one direction (overflow to
    +-inf or +-FLT_MAX as directed rounding does)."""
    fmax = np.float32(np.finfo(np.float32).max)
    if q > Fraction(float(fmax)):
        return np.float32(np.inf) if up else fmax
    if q < -Fraction(float(fmax)):
        return -fmax if up else np.float32(-np.inf)
    c = np.float32(float(q))
    while (Fraction(float(c)) < q) if up else (Fraction(float(c)) > q):
        c = np.nextafter(c, np.float32(np.inf) if up else np.float32(-np.inf))
    while True:
        n = np.nextafter(c, np.float32(-np.inf) if up else np.float32(np.inf))
        if (Fraction(float(n)) >= q) if up else (Fraction(float(n)) <= q):
            c = n
        else:
            return c


def _operands(rng, n):
    mag = np.exp2(rng.uniform(-30, 30, (n, 2))).astype(np.float32)
    sgn = np.where(rng.random((n, 2)) < 0.5, -1, 1).astype(np.float32)
    v = (mag * sgn).astype(np.float32)
    v[:8] = np.array([[1.0, 3.0], [0.1, 0.2], [-7.0, 1e-7], [3.4e38, 3.4e38], [-3.4e38, 3.4e38],
                      [1e-30, 1e-30], [2.0, -0.0], [5.0, 5.0]], np.float32)
    return v


@pytest.mark.parametrize("opname", ["add", "sub", "mul", "sqrt"])
def test_device_directed_rounding_is_exact(ctx, opname):
    """ADD, SUB, MUL and SQRT over degenerate intervals: the device's bounds
    are the exact result rounded down and up."""
    X, Y = csg.X(), csg.Y()
    expr = {"add": X + Y, "sub": X - Y, "mul": X * Y, "sqrt": csg.Sqrt(X)}[opname]
    tape = frep.Tape(expr)
    rng = np.random.default_rng(11)
    v = _operands(rng, 600)
    if opname == "sqrt":
        v[:, 0] = np.abs(v[:, 0])
    boxes = np.stack([v[:, 0], v[:, 1], np.zeros(len(v), np.float32)] * 2, 1).astype(np.float32)
    iv = ctx.eval_intervals(tape, boxes, 0.0, frep.ROUND_OUTWARD)
    for i, (a, b) in enumerate(v):
        fa, fb = Fraction(float(a)), Fraction(float(b))
        if opname == "sqrt":
            lo, hi = iv[i]
            # lo^2 <= a < next_up(lo)^2 and next_down(hi)^2 < a <= hi^2
            assert Fraction(float(lo)) ** 2 <= fa < Fraction(float(np.nextafter(lo, np.float32(np.inf)))) ** 2
            assert fa <= Fraction(float(hi)) ** 2
            assert hi == 0 or Fraction(float(np.nextafter(hi, np.float32(-np.inf)))) ** 2 < fa
            continue
        q = {"add": fa + fb, "sub": fa - fb, "mul": fa * fb}[opname]
        assert iv[i, 0] == _round_dir(q, False) and iv[i, 1] == _round_dir(q, True), (a, b, iv[i])


def test_device_division_interval_contains_quotient(ctx):
    """DIV follows the reference's formula (multiply by the reciprocal's
    interval, interval.comp:79-92): not the tightest bound, but it contains
    the exact quotient."""
    tape = frep.Tape(csg.X() / csg.Y())
    rng = np.random.default_rng(12)
    v = _operands(rng, 600)
    v[np.abs(v[:, 1]) < 1e-30, 1] = 1.0
    boxes = np.stack([v[:, 0], v[:, 1], np.zeros(len(v), np.float32)] * 2, 1).astype(np.float32)
    iv = ctx.eval_intervals(tape, boxes, 0.0, frep.ROUND_OUTWARD)
    for i, (a, b) in enumerate(v):
        q = Fraction(float(a)) / Fraction(float(b))
        lo, hi = iv[i]
        assert (lo == -np.inf or Fraction(float(lo)) <= q) and (hi == np.inf or q <= Fraction(float(hi))), (a, b)
