"""Soundness of the outward-rounding mode, on the CPU oracle.

The oracle's outward intervals are the device's bit for bit (the GPU parity
tests compare whole trees); here they are checked against the tape's exact
value, bounded by FP64 dense sampling with a rigorous error bound
(oracle/fp64.py), on the scene kinds the path runs: a union of spheres, a
random CSG tree, the twisted gyroid with SIN/COS, and the reference's demo
shapes with EXP and rotations by the time input (vulkan/src/shapes.cpp:5-117).
The same checks run on the device's own trees in test_gpu_containment.py.
"""
from __future__ import annotations

import numpy as np
import pytest

import frep
from containment import Report, check_tree, oracle_intervals
from fp64 import Containment, box_samples, check_boxes, eval_f64
from frep import scenes
from parity import oracle_tree


def _scene_cases():
    yield "spheres16", scenes.spheres_union(16), 0.0
    yield "csg24", scenes.random_csg(24, seed=5, grid_dims=[8, 8, 4]), 0.0
    yield "gyroid", scenes.stress_gyroid(n_spheres=8, grid_dims=(8, 8, 4)), 0.37
    for name, level, t in (("Screw", 0, 2.0), ("OrganicBalls", 0, 0.7), ("TwistedTower", 3, 0.0)):
        cam = frep.Camera(position=(0, 0, 40.0), forward=(0, 0, -1), initial_up=(0, 1, 0), fov_deg=45)
        yield name, scenes.Scene(name, scenes.DEMO_SHAPES[name](level), [8, 4, 4], (-20, -20, -20), 40.0,
                                 cam, 64, 48), t


CASES = list(_scene_cases())


@pytest.mark.parametrize("name,sc,t", CASES, ids=[c[0] for c in CASES])
def test_oracle_outward_tree_is_sound(name, sc, t):
    tape = frep.Tape(sc.shape)
    orc = oracle_tree(sc, tape, rounding=1, tape_time=t)
    rep = check_tree(orc, tape.wide(), tape.n_slots, sc.low_vertex, sc.world_size, t,
                     oracle_intervals, nodes_per_level=6, cells_per_node=24, per_axis=9)
    s = rep.summary()
    assert rep.ok(), s
    assert s["samples"] > 1000 and s["classified_cells"] > 0, s
    # the check has teeth: the double value lies inside each interval
    assert s["max_fp64_excess"] <= 0.0, s


def test_checker_catches_a_narrowed_interval():
    """A mistake planted in the oracle's intervals (each bound moved inward
    by a tenth of the width) must be reported."""
    sc = scenes.spheres_union(16)
    tape = frep.Tape(sc.shape)
    orc = oracle_tree(sc, tape, rounding=1)

    def narrowed(wide, ns, boxes, t):
        iv = oracle_intervals(wide, ns, boxes, t).astype(np.float64)
        w = iv[:, 1] - iv[:, 0]
        return np.stack([iv[:, 0] + 0.1 * w, iv[:, 1] - 0.1 * w], 1)

    rep = check_tree(orc, tape.wide(), tape.n_slots, sc.low_vertex, sc.world_size, 0.0, narrowed,
                     nodes_per_level=4, cells_per_node=24)
    assert rep.containment.violations > 0


def test_round_to_nearest_is_not_always_sound():
    """The reference's round-to-nearest intervals can miss the exact value by
    an ulp; the outward ones never do. A product whose exact value is not a
    float: [a, a] * [b, b]."""
    x = frep.csg.X()
    tape = frep.Tape(x * x * 3.1)
    rng = np.random.default_rng(4)
    a = rng.uniform(0.1, 10.0, 200).astype(np.float32)
    boxes = np.stack([a, a, a, a, a, a], 1)
    rn = Containment()
    out = Containment()
    check_boxes(tape.wide(), tape.n_slots, boxes, oracle_intervals(tape.wide(), tape.n_slots, boxes, 0.0, 0),
                per_axis=2, summary=rn)
    check_boxes(tape.wide(), tape.n_slots, boxes, oracle_intervals(tape.wide(), tape.n_slots, boxes, 0.0, 1),
                per_axis=2, summary=out)
    assert out.violations == 0 and out.max_excess <= 0.0
    assert rn.max_excess > 0.0  # RN drops below / above the exact value somewhere


def test_fp64_error_bound_is_rigorous_on_a_cancellation():
    """(x - c)^2 - r^2 near the sphere surface: the FP64 value differs from an
    exact rational evaluation by no more than the stated bound."""
    from fractions import Fraction
    X = frep.csg.X()
    c, r = np.float32(0.3), np.float32(0.7)
    tape = frep.Tape(frep.csg.Square(X - float(c)) - float(np.float32(r * r)))
    pts = np.zeros((64, 4))
    pts[:, 0] = np.linspace(0.99, 1.01, 64)
    v, E = eval_f64(tape.wide(), tape.n_slots, pts)
    for i in range(64):
        xe = Fraction(float(pts[i, 0]))
        ex = (xe - Fraction(float(c))) ** 2 - Fraction(float(np.float32(r * r)))
        assert abs(Fraction(float(v[i])) - ex) <= Fraction(float(E[i]))


def test_box_samples_cover_corners():
    b = np.array([[0.0, 1.0, 2.0, 0.5, 1.5, 2.25]])
    p = box_samples(b, 9, 0.3)
    assert p.shape == (1, 729, 4)
    for corner in [(0.0, 1.0, 2.0), (0.5, 1.5, 2.25), (0.5, 1.0, 2.25)]:
        assert np.any(np.all(p[0, :, :3] == corner, axis=1))
    assert np.all(p[0, :, :3] >= b[0, :3]) and np.all(p[0, :, :3] <= b[0, 3:])
    assert np.all(p[0, :, 3] == 0.3)


def test_report_summary_keys():
    r = Report()
    s = r.summary()
    for k in ("samples", "max_fp64_excess", "max_fp64_error_bound", "violations", "leaf_violations",
              "shorten_violations"):
        assert k in s
