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


# ---- vectorised canonical comparison, for trees of millions of nodes ----------

def _tape_hashes(tapes: np.ndarray, idx: np.ndarray, chunk: int = 200_000):
    """(length, content hash) of the tape record at each index in idx."""
    tapes = np.asarray(tapes, np.uint64)
    idx = np.asarray(idx, np.int64)
    lens = (tapes[idx] & np.uint64(0xFFFFFFFF)).astype(np.int64)
    out = np.zeros(len(idx), np.uint64)
    mul = np.uint64(0x9E3779B97F4A7C15)
    for s in range(0, len(idx), chunk):
        li = lens[s:s + chunk]
        ii = idx[s:s + chunk]
        tot = int(li.sum())
        if tot == 0:
            continue
        starts = np.cumsum(li) - li
        pos = np.arange(tot) - np.repeat(starts, li)
        w = tapes[np.repeat(ii + 1, li) + pos]
        with np.errstate(over="ignore"):
            mixed = (w ^ (pos.astype(np.uint64) * mul)) * np.uint64(0xBF58476D1CE4E5B9)
            mixed ^= mixed >> np.uint64(31)
        h = np.zeros(len(li), np.uint64)
        nz = li > 0
        h[nz] = np.add.reduceat(mixed, starts[nz])
        out[s:s + chunk] = h
    return lens, out


def _level_arrays(t, lvl):
    dim = t.dims[lvl]
    c3 = dim ** 3
    W = c3 // 32
    last = lvl == t.levels - 1
    cnt = t.node_count[lvl]
    size = t.node_size[lvl]
    rec = np.asarray(t.nodes[t.node_offset[lvl]: t.node_offset[lvl] + cnt * size], np.uint32).reshape(cnt, size)
    coords = rec[:, 1:4].astype(np.int64)
    leaf = rec[:, 4:4 + W]
    inter = None if last else rec[:, 4 + W:4 + 2 * W]
    clist = None if last else rec[:, 4 + 2 * W:4 + 2 * W + c3]
    return rec[:, 0].astype(np.int64), coords, leaf, inter, clist


def compare_trees_fast(a, b, max_report: int = 3):
    """compare_trees for large trees, vectorised: per level the node sets
    keyed by coordinates, leaf / interior words bit for bit, tapes by
    (length, content hash), and in both trees every interior bit's child id
    in range with the child's coordinates. a, b: TreeExport or OracleTree."""
    diffs = []
    if list(a.node_count) != list(b.node_count):
        diffs.append(f"node counts {list(a.node_count)} != {list(b.node_count)}")
        return diffs
    for lvl in range(a.levels):
        span = 1
        for d in a.dims[:lvl]:
            span *= d
        per = []
        for t in (a, b):
            tidx, coords, leaf, inter, clist = _level_arrays(t, lvl)
            key = (coords[:, 0] * span + coords[:, 1]) * span + coords[:, 2]
            o = np.argsort(key, kind="stable")
            if len(key) and np.any(np.diff(key[o]) == 0):
                diffs.append(f"level {lvl}: duplicate node coordinates")
            lens, hs = _tape_hashes(t.tapes, tidx[o])
            per.append((key[o], leaf[o], None if inter is None else inter[o], lens, hs))
            if inter is not None and len(key):  # child links
                dim = t.dims[lvl]
                bits = np.unpackbits(inter.astype("<u4").view(np.uint8), axis=1, bitorder="little").astype(bool)
                ni, cell = np.nonzero(bits)
                child = clist[ni, cell].astype(np.int64)
                if np.any(child >= t.node_count[lvl + 1]):
                    diffs.append(f"level {lvl}: child id out of range")
                    continue
                crec = t.node_offset[lvl + 1] + child * t.node_size[lvl + 1]
                got = np.stack([t.nodes[crec + 1], t.nodes[crec + 2], t.nodes[crec + 3]], 1).astype(np.int64)
                want = coords[ni] * dim + np.stack([cell // (dim * dim), (cell // dim) % dim, cell % dim], 1)
                nbad = int(np.any(got != want, axis=1).sum())
                if nbad:
                    diffs.append(f"level {lvl}: {nbad} child links point at wrong coordinates")
        (ka, la, ia, na, ha), (kb, lb, ib, nb, hb) = per
        if not np.array_equal(ka, kb):
            diffs.append(f"level {lvl}: node sets differ")
            continue
        for name, x, y in (("leaf", la, lb), ("interior", ia, ib), ("tape length", na, nb), ("tape", ha, hb)):
            if x is None or len(x) == 0:  # (a level without nodes: nothing to compare)
                continue
            bad = np.nonzero(np.any((x != y).reshape(len(x), -1), axis=1))[0]
            if len(bad):
                diffs.append(f"level {lvl}: {name} differs at {len(bad)} nodes, e.g. key {ka[bad[:max_report]].tolist()}")
    return diffs
