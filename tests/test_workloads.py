"""Host-side logic of the many-scene workload and the autotuner (no GPU)."""
from __future__ import annotations

import math

import numpy as np

from frep import scenes
from frep.autotune import BRANCHINGS, SIZE_CLASSES, Autotuner, Choice, size_class


def test_branching_candidates_valid():
    assert set(BRANCHINGS) == set(scenes.BATCH_RESOLUTIONS)
    for res, cands in BRANCHINGS.items():
        assert tuple(scenes.DEFAULT_BRANCHING[res]) in [tuple(c) for c in cands]
        for dims in cands:
            assert math.prod(dims) == res
            assert 2 <= len(dims) <= 4
            assert all(d % 4 == 0 and 4 <= d <= 32 for d in dims)


def test_size_classes():
    assert size_class(0) == 0
    assert size_class(SIZE_CLASSES[0] - 1) == 0
    assert size_class(SIZE_CLASSES[0]) == 1
    assert size_class(SIZE_CLASSES[-1]) == len(SIZE_CLASSES)


def test_batch_workload_distribution_and_determinism():
    a = scenes.batch_workload(24, seed=5, width=64, height=48)
    b = scenes.batch_workload(24, seed=5, width=64, height=48, processes=2)  # spawned workers
    assert [s.meta for s in a] == [s.meta for s in b]
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x.shape.wide(), y.shape.wide())
        assert x.grid_dims == list(scenes.DEFAULT_BRANCHING[x.meta["res"]])
        assert 4 <= x.meta["n"] <= 1024
        assert x.meta["res"] in scenes.BATCH_RESOLUTIONS
        assert (x.width, x.height) == (64, 48)
    # primitive count drives the tape length
    n = np.array([s.meta["n"] for s in a])
    instr = np.array([s.shape.n_instr for s in a])
    assert np.corrcoef(n, instr)[0, 1] > 0.9


def test_orbit_camera_looks_at_origin():
    rng = np.random.default_rng(0)
    for _ in range(10):
        cam = scenes.orbit_camera(rng)
        p = np.array(cam.position)
        f = np.array(cam.forward)
        assert abs(np.linalg.norm(p) - 4.1) < 1e-9
        np.testing.assert_allclose(f, -p)


def test_autotuner_cache_round_trip(tmp_path):
    """The Python wrapper reads and writes the C++ tuner's cache file."""
    import json
    path = tmp_path / "tune.json"
    path.write_text(json.dumps({"NVIDIA B200": {"choices": {"256:2": {"dims": [16, 4, 4], "point_cells_per_lane": 2,
                                                                      "ms_per_scene": 0.5}},
                                                "warps": [1, 4]}}))
    t = Autotuner(ctx=None, cache_path=str(path))
    copy = str(tmp_path / "copy.json")
    t.save(copy)
    u = Autotuner(ctx=None, cache_path=copy)
    assert u.choice_for(256, 1500).dims == (16, 4, 4)
    assert u.choice_for(256, 1500).point_cells_per_lane == 2
    assert u.warps == (1, 4)

    class S:
        pass
    s = S()
    s.meta = {"res": 256}
    s.grid_dims = [16, 16]
    s.shape = type("T", (), {"n_instr": 1500})()
    assert u.apply(s) == ((16, 4, 4), 2)
    s.meta = {"res": 64}
    assert u.apply(s) == ((16, 16), 0)  # no tuned choice: the scene's own grid
