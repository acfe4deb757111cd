"""Soundness checks of outward-rounded voxelizations against FP64 dense
sampling (shared by the CPU and GPU containment tests).

For a voxelized tree (the device's export or the oracle's), a sample of its
nodes at every level is checked three ways, each at a 9^3 grid of points per
cell that includes the cell's corners, with fp64.eval_f64's rigorous FP64
error bound E:

(a) containment: the interval of the node's tape over each cell box, as the
    level pass computes it (interval.comp:8-160 over [lo, lo + cell],
    voxelizer/main.comp:113-126), contains the tape's exact value at every
    sample (lo <= v + E and v - E <= hi);
(b) classification: a cell the level pass marked as a leaf has no sample
    with v - E >= 0 (the function is negative on the whole cell), an empty
    cell none with v + E <= 0 (main.comp:88-108);
(c) shortening: on the node's box, the node's shortened tape and the root
    tape have the same exact value (|v_node - v_root| <= E_node + E_root):
    a pruned MIN/MAX branch (shorten.comp:148-186) was never the result.
"""
from __future__ import annotations

import numpy as np

import oracle
from fp64 import Containment, box_samples, eval_f64


def cell_sizes(dims, world_size):
    """Per-level cell size as the voxelizer computes it (successive float32
    divisions, voxelizer.cpp:209-220)."""
    cs = np.float32(world_size)
    out = []
    for d in dims:
        cs = np.float32(cs / np.float32(d))
        out.append(cs)
    return out


def cell_boxes(low, cs, gxyz):
    """Float32 boxes [low + g*cs, that + cs] of global cells g (M, 3)."""
    low = np.asarray(low, np.float32)
    lo = (low[None, :] + (np.asarray(gxyz, np.float64).astype(np.float32) * np.float32(cs))).astype(np.float32)
    hi = (lo + np.float32(cs)).astype(np.float32)
    return np.concatenate([lo, hi], 1)


def tape_of(tapes, idx):
    n = int(tapes[idx] & 0xFFFFFFFF)
    return np.ascontiguousarray(tapes[idx + 1: idx + 1 + n], np.uint64)


def n_slots_of(wide):
    w = np.asarray(wide, np.uint64)
    op = w & np.uint64(0xFF)
    out = (w >> np.uint64(16)) & np.uint64(0xFFFF)
    a = (w >> np.uint64(32)) & np.uint64(0xFFFF)
    b = w >> np.uint64(48)
    m = int(out.max(initial=0))
    m = max(m, int(a[op != 0].max(initial=0)))
    binop = np.isin(op, (3, 4, 5, 6, 7, 8))
    m = max(m, int(b[binop].max(initial=0)))
    return max(4, m + 1)


class Report:
    def __init__(self):
        self.containment = Containment()
        self.leaf_violations = 0
        self.empty_violations = 0
        self.classified_cells = 0
        self.shorten_violations = 0
        self.shorten_samples = 0
        self.shorten_max_diff = 0.0
        self.nodes_checked = [0] * 8
        self.cells_checked = 0

    def ok(self):
        return (self.containment.violations == 0 and self.leaf_violations == 0 and self.empty_violations == 0
                and self.shorten_violations == 0)

    def summary(self):
        d = self.containment.summary()
        d.update(leaf_violations=self.leaf_violations, empty_violations=self.empty_violations,
                 classified_cells=self.classified_cells, shorten_violations=self.shorten_violations,
                 shorten_samples=self.shorten_samples, shorten_max_abs_diff=self.shorten_max_diff,
                 cells_checked=self.cells_checked, nodes_checked=[n for n in self.nodes_checked if n])
        return d


def check_tree(export, root_wide, root_slots, low, world_size, tape_time, interval_fn, *, nodes_per_level=24,
               cells_per_node=48, per_axis=9, seed=0, report=None, root_cells=None):
    """Runs checks (a)-(c) on a sample of `export`'s nodes (a frep TreeExport
    or an oracle.OracleTree: levels, dims, node_count, node_offset,
    node_size, nodes, tapes). interval_fn(wide, n_slots, boxes (M, 6), t)
    returns the (M, 2) intervals to check (the device's or the oracle's).
    Ambiguous and classified cells are preferred: they carry the tight bounds.
    root_cells: cells sampled in the root node (default cells_per_node)."""
    rng = np.random.default_rng(seed)
    rep = report or Report()
    dims = list(export.dims)
    css = cell_sizes(dims, world_size)
    for lvl in range(export.levels - 1):  # the last level is point-evaluated
        dim = dims[lvl]
        c3 = dim ** 3
        W = c3 // 32
        cnt = export.node_count[lvl]
        if cnt == 0:
            continue
        pick = rng.choice(cnt, size=min(cnt, nodes_per_level), replace=False)
        for i in sorted(int(p) for p in pick):
            rec = export.nodes[export.node_offset[lvl] + i * export.node_size[lvl]:][: 4 + 2 * W]
            wide = tape_of(export.tapes, int(rec[0]))
            ns = n_slots_of(wide)
            coords = np.array([int(rec[1]), int(rec[2]), int(rec[3])], np.int64)
            leaf = np.unpackbits(rec[4:4 + W].astype("<u4").view(np.uint8), bitorder="little").astype(bool)
            inter = np.unpackbits(rec[4 + W:4 + 2 * W].astype("<u4").view(np.uint8), bitorder="little").astype(bool)
            marked = np.nonzero(leaf | inter)[0]
            rest = np.nonzero(~(leaf | inter))[0]
            want = root_cells if (lvl == 0 and root_cells) else cells_per_node
            k1 = min(len(marked), want * 3 // 4)
            sel = list(rng.choice(marked, size=k1, replace=False)) if k1 else []
            k2 = min(len(rest), want - k1)
            sel += list(rng.choice(rest, size=k2, replace=False)) if k2 else []
            cells = np.array(sorted(sel), np.int64)
            if len(cells) == 0:
                continue
            cz, cy, cx = cells % dim, (cells // dim) % dim, cells // (dim * dim)
            g = coords[None, :] * dim + np.stack([cx, cy, cz], 1)
            boxes = cell_boxes(low, css[lvl], g)
            iv = np.asarray(interval_fn(wide, ns, boxes, tape_time), np.float64).reshape(-1, 2)
            pts = box_samples(boxes, per_axis, tape_time)
            M, P = pts.shape[:2]
            v, E = eval_f64(wide, ns, pts.reshape(-1, 4))
            v, E = v.reshape(M, P), E.reshape(M, P)
            rep.containment.add(iv, v, E)  # (a)
            fin = np.isfinite(v) & np.isfinite(E)
            lf, em = leaf[cells], ~(leaf | inter)[cells]
            rep.leaf_violations += int(np.sum(lf[:, None] & fin & (v - E >= 0)))   # (b)
            rep.empty_violations += int(np.sum(em[:, None] & fin & (v + E <= 0)))
            rep.classified_cells += int(lf.sum() + em.sum())
            rep.cells_checked += M
            rep.nodes_checked[lvl] += 1
            if lvl > 0:  # (c) on the node's own box, as its parent's cell
                pbox = cell_boxes(low, css[lvl - 1], coords[None, :])
                pp = box_samples(pbox, 5, tape_time).reshape(-1, 4)
                vn, en = eval_f64(wide, ns, pp)
                vr, er = eval_f64(root_wide, root_slots, pp)
                ok = np.isfinite(vn) & np.isfinite(vr) & np.isfinite(en) & np.isfinite(er)
                d = np.abs(vn - vr)
                rep.shorten_samples += int(ok.sum())
                if ok.any():
                    rep.shorten_max_diff = max(rep.shorten_max_diff, float(d[ok].max()))
                rep.shorten_violations += int(np.sum(ok & (d > en + er)))
    return rep


def oracle_intervals(wide, n_slots, boxes, t, rounding=1):
    out = np.zeros((len(boxes), 2), np.float32)
    for i, b in enumerate(np.asarray(boxes, np.float32)):
        out[i], _ = oracle.eval_interval(wide, n_slots, b[:3], b[3:], t, rounding)
    return out
