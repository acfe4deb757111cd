"""Helpers shared by the GPU parity tests: run a scene on the device and on the
oracle, and compare canonical trees and per-pixel hits."""
from __future__ import annotations

import numpy as np

import frep
import oracle


def device_tree(ctx, scene, rounding=1, tape_time=0.0, shorten=True, node_words=0, tape_words=0,
                point_cells_per_lane=0):
    vs = frep.VoxelStorage(scene.grid_dims, scene.low_vertex, scene.world_size, rounding=rounding,
                           shorten=shorten, node_words=node_words, tape_words=tape_words,
                           point_cells_per_lane=point_cells_per_lane)
    vs.init(ctx, scene.shape)
    frep.Voxelizer(ctx, vs).voxelize(tape_time)
    return vs


def oracle_tree(scene, tape: frep.Tape, rounding=1, tape_time=0.0, shorten=True):
    return oracle.OracleTree(tape.wide(), tape.n_slots, scene.grid_dims, scene.low_vertex,
                             scene.world_size, tape_time=tape_time, rounding=rounding, shorten=shorten)


def compare_trees(dev_export, orc: oracle.OracleTree):
    """Returns a list of differences between the canonical forms (empty = equal)."""
    dc, dprob = oracle.canonical_of_export(dev_export)
    oc, oprob = oracle.canonical_of_oracle(orc)
    diffs = [f"device: {p}" for p in dprob[:5]] + [f"oracle: {p}" for p in oprob[:5]]
    if dev_export.node_count != orc.node_count:
        diffs.append(f"node counts {dev_export.node_count} != {orc.node_count}")
    for lvl, (d, o) in enumerate(zip(dc, oc)):
        if d.keys() != o.keys():
            only_d = sorted(set(d) - set(o))[:3]
            only_o = sorted(set(o) - set(d))[:3]
            diffs.append(f"level {lvl}: node sets differ (device-only {only_d}, oracle-only {only_o})")
            continue
        n_bad = 0
        for k in d:
            if d[k] != o[k]:
                if n_bad < 3:
                    what = [name for name, a, b in zip(("leaf", "interior", "tape"), d[k], o[k]) if a != b]
                    diffs.append(f"level {lvl} node {k}: {what} differ")
                n_bad += 1
        if n_bad:
            diffs.append(f"level {lvl}: {n_bad} nodes differ")
    return diffs


def render_both(ctx, vs, orc, scene, lights, tape_time=0.0, width=None, height=None):
    import torch
    W = width or scene.width
    H = height or scene.height
    rt = frep.Raytracer(ctx, vs)
    rt.lights = lights
    rgba, hits = rt.trace(scene.camera, tape_time, W, H, hits=True)
    torch.cuda.synchronize()
    d_rgba = rgba.cpu().numpy()
    d_hits = hits.cpu().numpy().view(np.uint32)
    o_rgba, o_hits = orc.render(oracle.camera_vector(scene.camera, W, H), lights, tape_time)
    return d_rgba, d_hits, o_rgba, o_hits


def compare_hits(d_hits, o_hits, dev_export, orc, rtol=1e-5):
    """Hit cells must be identical; t and normals within rtol (relative)."""
    dk = oracle.hit_cells(d_hits, dev_export.dims, dev_export.node_offset, dev_export.node_size,
                          dev_export.nodes)
    ok = oracle.hit_cells(o_hits, orc.dims, orc.node_offset, orc.node_size, orc.nodes)
    diffs = []
    bad = np.any(dk != ok, axis=-1)
    if bad.any():
        ys, xs = np.nonzero(bad)
        diffs.append(f"{int(bad.sum())} pixels hit different cells, e.g. ({ys[0]}, {xs[0]}): "
                     f"{dk[ys[0], xs[0]].tolist()} vs {ok[ys[0], xs[0]].tolist()}")
    hit = ok[..., 0] >= 0
    dt = d_hits[..., 0].view(np.float32)[hit]
    ot = o_hits[..., 0].view(np.float32)[hit]
    if not np.allclose(dt, ot, rtol=rtol, atol=0):
        diffs.append(f"hit depth differs: max rel {np.max(np.abs(dt - ot) / np.maximum(np.abs(ot), 1e-30)):.3g}")
    dn = d_hits[..., 1:4].view(np.float32)[hit]
    on = o_hits[..., 1:4].view(np.float32)[hit]
    finite = np.isfinite(on).all(-1)
    if not np.allclose(dn[finite], on[finite], rtol=rtol, atol=rtol):
        diffs.append(f"normals differ: max abs {np.max(np.abs(dn[finite] - on[finite])):.3g}")
    return diffs
