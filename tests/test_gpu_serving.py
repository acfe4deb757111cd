"""Serving (frep_server): every request's image is the same alone and in a
mix of concurrent requests — with re-renders of resident trees, evictions
under a small arena, re-voxelization at new tape times, pool overflow retries
and requests that cannot be admitted."""
from __future__ import annotations

import numpy as np
import pytest

import frep
from frep import scenes
from frep.autotune import fit_pools

pytestmark = pytest.mark.gpu

W, H = 96, 72
LIGHTS = frep.Lights(shadow_mask=1)


@pytest.fixture(scope="module")
def ctx():
    c = frep.Context(0, hbm_budget_bytes=24 << 30)
    yield c
    c.close()


@pytest.fixture(scope="module")
def world(ctx):
    """Scenes (5 static random CSGs of several grids + the time-dependent
    Morph), fitted pools, cameras and the expected image of every (scene,
    camera, time) rendered alone through the plain API."""
    rng = np.random.default_rng(9)
    scs = []
    for i, dims in enumerate([(16, 4), (8, 8, 4), (16, 8), (4, 16), (8, 12)]):
        sc = scenes.random_csg(8 + 11 * i, seed=300 + i, grid_dims=list(dims), width=W, height=H)
        scs.append((sc.shape if isinstance(sc.shape, frep.Tape) else frep.Tape(sc.shape), sc.grid_dims,
                    sc.low_vertex, sc.world_size))
    scs.append((frep.Tape(scenes.Morph()), [16, 4, 4], (-20.0, -20.0, -20.0), 40.0))
    cams = [scenes.orbit_camera(rng) for _ in range(3)]
    morph_cams = [frep.Camera(position=(0, 0, 40.0), forward=(0, 0, -1), initial_up=(0, 1, 0), fov_deg=45),
                  frep.Camera(position=(30, 10, 30.0), forward=(-30, -10, -30), initial_up=(0, 1, 0), fov_deg=45)]
    times = [0.0, 0.7]
    pools = []
    for tape, dims, low, ws in scs:
        p = [fit_pools(ctx, [tape], [dims], low, ws, tape_times=[t])[0] for t in times]
        pools.append(frep.autotune.Pool(max(q.node_words for q in p), max(q.tape_words for q in p)))
    import torch
    expected = {}
    for si, (tape, dims, low, ws) in enumerate(scs):
        cam_list = morph_cams if si == len(scs) - 1 else cams
        for t in (times if tape.uses_time else [0.0]):
            vs = frep.VoxelStorage(dims, low, ws).init(ctx, tape)
            frep.Voxelizer(ctx, vs).voxelize(t)
            rt = frep.Raytracer(ctx, vs)
            rt.lights = LIGHTS
            for ci, cam in enumerate(cam_list):
                rgba, _ = rt.trace(cam, t, W, H)
                torch.cuda.synchronize()
                expected[(si, ci, t)] = rgba.cpu().numpy()
            vs.cleanup()
    return {"scenes": scs, "pools": pools, "cams": cams, "morph_cams": morph_cams, "times": times,
            "expected": expected}


def _cam(w, si, ci):
    return (w["morph_cams"] if si == len(w["scenes"]) - 1 else w["cams"])[ci]


def _server(ctx, w, budget, sized=True, max_batch=0):
    import torch
    srv = frep.Server(ctx, hbm_budget_bytes=budget, max_batch=max_batch, lights=LIGHTS)
    ids = []
    for (tape, dims, low, ws), p in zip(w["scenes"], w["pools"]):
        ids.append(srv.add_scene(tape, dims, low, ws, node_words=p.node_words if sized else 0,
                                 tape_words=p.tape_words if sized else 0))
    return srv, ids


def _pinned():
    import torch
    return torch.empty((H, W, 4), dtype=torch.uint8, pin_memory=True)


def test_alone_then_in_the_mix(ctx, world):
    w = world
    tree_bytes = sorted(p.bytes + 4096 for p in w["pools"])
    budget = tree_bytes[-1] + tree_bytes[-2] + (64 << 10)  # two trees at most: evictions
    srv, ids = _server(ctx, w, budget)
    # alone
    out = _pinned()
    rid = srv.submit(ids[1], _cam(w, 1, 2), 0.0, W, H, out)
    st = srv.wait(rid, 120000)
    assert st.state == frep.REQ_DONE and st.voxelized == 1
    np.testing.assert_array_equal(out.numpy(), w["expected"][(1, 2, 0.0)])
    # the same request again: a re-render of the resident tree
    out2 = _pinned()
    st = srv.wait(srv.submit(ids[1], _cam(w, 1, 2), 0.0, W, H, out2), 120000)
    assert st.state == frep.REQ_DONE and st.voxelized == 0
    np.testing.assert_array_equal(out2.numpy(), w["expected"][(1, 2, 0.0)])
    # a mix, submitted as fast as possible: repeats, all scenes, the animated
    # scene at two tape times
    rng = np.random.default_rng(4)
    jobs = []
    for _ in range(60):
        si = int(rng.integers(0, len(ids)))
        tape = w["scenes"][si][0]
        ci = int(rng.integers(0, 2 if si == len(ids) - 1 else 3))
        t = float(w["times"][int(rng.integers(0, 2))]) if tape.uses_time else 0.0
        buf = _pinned()
        jobs.append((srv.submit(ids[si], _cam(w, si, ci), t, W, H, buf), si, ci, t, buf))
    srv.drain(300000)
    for rid, si, ci, t, buf in jobs:
        st = srv.poll(rid)
        assert st.state == frep.REQ_DONE, (si, st.status)
        np.testing.assert_array_equal(buf.numpy(), w["expected"][(si, ci, t)], err_msg=f"scene {si} cam {ci} t {t}")
    s = srv.stats()
    assert s["completed"] == s["submitted"] == 62 and s["failed"] == 0
    assert s["evictions"] > 0 and s["rerendered"] > 0 and s["voxelized"] > 0, (s, tree_bytes)
    assert 0 < s["p50_ms"] <= s["p99_ms"] <= s["max_ms"]
    assert s["resident_bytes"] <= s["arena_bytes"]
    srv.close()


def test_unsized_pools_grow_and_refit(ctx, world):
    """Scenes registered without pool sizes: the estimate may overflow; the
    voxelization is retried with doubled pools and the image is unchanged."""
    w = world
    srv, ids = _server(ctx, w, 6 << 30, sized=False, max_batch=4)
    jobs = []
    for si in range(len(ids)):
        for t in (w["times"] if w["scenes"][si][0].uses_time else [0.0]):
            buf = _pinned()
            jobs.append((srv.submit(ids[si], _cam(w, si, 0), t, W, H, buf), si, t, buf))
    srv.drain(300000)
    for rid, si, t, buf in jobs:
        st = srv.poll(rid)
        assert st.state == frep.REQ_DONE, (si, st.status)
        np.testing.assert_array_equal(buf.numpy(), w["expected"][(si, 0, t)])
    srv.close()


def test_overflow_retry(ctx, world):
    w = world
    srv = frep.Server(ctx, hbm_budget_bytes=2 << 30, lights=LIGHTS)
    tape, dims, low, ws = w["scenes"][2]
    p = w["pools"][2]
    sid = srv.add_scene(tape, dims, low, ws, node_words=max(4096, p.node_words // 8),
                        tape_words=max(tape.n_instr + 64, p.tape_words // 8))
    buf = _pinned()
    st = srv.wait(srv.submit(sid, _cam(w, 2, 1), 0.0, W, H, buf), 120000)
    assert st.state == frep.REQ_DONE and st.retries > 0
    np.testing.assert_array_equal(buf.numpy(), w["expected"][(2, 1, 0.0)])
    rid = srv.submit(sid, _cam(w, 2, 0), 0.0, W, H, _pinned())
    srv.wait(rid, 60000)
    srv.release(rid)
    with pytest.raises(frep.FrepError):
        srv.poll(rid)
    srv.close()


def test_request_larger_than_the_arena_fails_cleanly(ctx, world):
    w = world
    srv = frep.Server(ctx, hbm_budget_bytes=64 << 20, lights=LIGHTS)
    tape, dims, low, ws = w["scenes"][0]
    big = srv.add_scene(tape, dims, low, ws, node_words=64 << 20, tape_words=64 << 20)  # > 64 MB
    ok = srv.add_scene(tape, dims, low, ws, node_words=w["pools"][0].node_words, tape_words=w["pools"][0].tape_words)
    b1, b2 = _pinned(), _pinned()
    r1 = srv.submit(big, _cam(w, 0, 0), 0.0, W, H, b1)
    r2 = srv.submit(ok, _cam(w, 0, 0), 0.0, W, H, b2)
    st1 = srv.wait(r1, 60000)
    st2 = srv.wait(r2, 60000)
    assert st1.state == frep.REQ_FAILED and st1.status == frep.L.ERR_OOM
    assert st2.state == frep.REQ_DONE
    np.testing.assert_array_equal(b2.numpy(), w["expected"][(0, 0, 0.0)])
    srv.close()
