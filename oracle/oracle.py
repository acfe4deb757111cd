"""Python access to the CPU oracle and the reference bridge — TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
arm use this module, and only as the checker. It wraps:

* lib/liboracle.so   — the C++ restatement of the reference's shader semantics
                       (frep_oracle.h lists the reference file:line for each);
* _ref/libfrep_ref.so — the reference's own CSG front end (csg::Tape,
                       csg::Tape::Eval, the demo shapes), compiled from the
                       reference tree by oracle/Makefile.

It also holds the canonical form used for parity: nodes keyed by (level,
coords), masks bit for bit, tapes by content, child links resolved to coords.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
ORACLE_LIB = ORACLE_DIR / "lib" / "liboracle.so"
REF_LIB = ORACLE_DIR / "_ref" / "libfrep_ref.so"

_P = C.c_void_p


def build(quiet: bool = True) -> None:
    """Runs oracle/Makefile (the reference bridge only where its sources exist)."""
    out = subprocess.DEVNULL if quiet else None
    subprocess.run(["make", "-C", str(ORACLE_DIR)], check=True, stdout=out)


_oracle = None
_ref = None


def oracle_lib() -> C.CDLL:
    global _oracle
    if _oracle is None:
        if not ORACLE_LIB.exists():
            build()
        lib = C.CDLL(str(ORACLE_LIB))
        lib.oracle_eval_interval.argtypes = [_P, C.c_uint32, C.c_uint32, _P, _P, C.c_float, C.c_int, _P, _P]
        lib.oracle_eval_interval_trace.argtypes = [_P, C.c_uint32, C.c_uint32, _P, _P, C.c_float, C.c_int, _P]
        lib.oracle_eval_point.argtypes = [_P, C.c_uint32, C.c_uint32, C.c_float, C.c_float, C.c_float, C.c_float]
        lib.oracle_eval_point.restype = C.c_float
        lib.oracle_eval_gradient.argtypes = [_P, C.c_uint32, C.c_uint32, C.c_float, C.c_float, C.c_float,
                                             C.c_float, _P]
        lib.oracle_shorten.argtypes = [_P, C.c_uint32, C.c_uint32, _P, C.c_uint32, _P]
        lib.oracle_shorten.restype = C.c_uint32
        lib.oracle_directed.argtypes = [C.c_int, C.c_int, C.c_float, C.c_float]
        lib.oracle_directed.restype = C.c_float
        lib.oracle_voxelize.argtypes = [_P, C.c_uint32, C.c_uint32, _P, C.c_uint32, _P, C.c_float,
                                        C.c_float, C.c_int, C.c_int, C.c_int]
        lib.oracle_voxelize.restype = _P
        lib.oracle_tree_free.argtypes = [_P]
        lib.oracle_tree_info.argtypes = [_P, _P]
        lib.oracle_tree_nodes.argtypes = [_P, _P]
        lib.oracle_tree_tapes.argtypes = [_P, _P]
        lib.oracle_tree_work.argtypes = [_P, _P]
        lib.oracle_compact.argtypes = [_P, C.c_int]
        lib.oracle_compact.restype = _P
        lib.oracle_render.argtypes = [_P, _P, C.c_uint32, _P, _P, _P, _P, C.c_uint32, C.c_float, _P, _P,
                                      C.c_int]
        _oracle = lib
    return _oracle


def ref_available() -> bool:
    return REF_LIB.exists()


def ref_lib() -> C.CDLL:
    global _ref
    if _ref is None:
        lib = C.CDLL(str(REF_LIB))
        lib.ref_tape_new.argtypes = [C.c_uint32, _P, _P, _P, _P, C.c_uint32]
        lib.ref_tape_new.restype = _P
        lib.ref_tape_free.argtypes = [_P]
        lib.ref_tape_info.argtypes = [_P, _P]
        lib.ref_tape_info.restype = C.c_int
        lib.ref_tape_instrs.argtypes = [_P, _P]
        lib.ref_tape_consts.argtypes = [_P, _P]
        lib.ref_tape_eval.argtypes = [_P, _P, C.c_uint32, _P]
        lib.ref_dag_eval.argtypes = [C.c_uint32, _P, _P, _P, _P, C.c_uint32, _P, C.c_uint32, _P]
        lib.ref_shape_new.argtypes = [C.c_char_p, C.c_int]
        lib.ref_shape_new.restype = _P
        lib.ref_expr_free.argtypes = [_P]
        lib.ref_expr_flatten.argtypes = [_P, C.c_uint32, _P, _P, _P, _P, _P]
        lib.ref_expr_flatten.restype = C.c_uint32
        _ref = lib
    return _ref


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


# ---- reference bridge --------------------------------------------------------

class RefTape:
    """csg::Tape built by the reference's own compiler."""

    def __init__(self, ops, in0, in1, consts, root):
        self.dag = tuple(np.ascontiguousarray(a, t) for a, t in
                         ((ops, np.uint8), (in0, np.uint32), (in1, np.uint32), (consts, np.float32)))
        self.root = int(root)
        lib = ref_lib()
        self.h = lib.ref_tape_new(len(self.dag[0]), *map(_p, self.dag), self.root)
        if not self.h:
            raise ValueError("the reference compiler rejected the expression")
        counts = np.zeros(3, np.uint32)
        self.fits = lib.ref_tape_info(self.h, _p(counts)) == 0
        self.n_instr, self.n_consts, self.n_slots = (int(c) for c in counts)
        self.instrs = np.zeros(self.n_instr, np.uint32)
        lib.ref_tape_instrs(self.h, _p(self.instrs))
        self.consts = np.zeros(max(self.n_consts, 1), np.float32)
        lib.ref_tape_consts(self.h, _p(self.consts))
        self.consts = self.consts[: self.n_consts]

    def eval(self, xyzt) -> np.ndarray:
        xyzt = np.ascontiguousarray(xyzt, np.float32).reshape(-1, 4)
        out = np.zeros(len(xyzt), np.float32)
        ref_lib().ref_tape_eval(self.h, _p(xyzt), len(xyzt), _p(out))
        return out

    def __del__(self):
        if getattr(self, "h", None):
            ref_lib().ref_tape_free(self.h)
            self.h = None


def ref_dag_eval(ops, in0, in1, consts, root, xyzt) -> np.ndarray:
    arrs = [np.ascontiguousarray(a, t) for a, t in
            ((ops, np.uint8), (in0, np.uint32), (in1, np.uint32), (consts, np.float32))]
    xyzt = np.ascontiguousarray(xyzt, np.float32).reshape(-1, 4)
    out = np.zeros(len(xyzt), np.float32)
    ref_lib().ref_dag_eval(len(arrs[0]), *map(_p, arrs), int(root), _p(xyzt), len(xyzt), _p(out))
    return out


def ref_shape_dag(name: str, level: int = 0):
    """Flat DAG of a reference demo shape (vulkan/src/shapes.cpp)."""
    lib = ref_lib()
    h = lib.ref_shape_new(name.encode(), level)
    if not h:
        raise ValueError(name)
    try:
        n = lib.ref_expr_flatten(h, 0, None, None, None, None, None)
        ops = np.zeros(n, np.uint8)
        in0 = np.zeros(n, np.uint32)
        in1 = np.zeros(n, np.uint32)
        consts = np.zeros(n, np.float32)
        root = np.zeros(1, np.uint32)
        lib.ref_expr_flatten(h, n, _p(ops), _p(in0), _p(in1), _p(consts), _p(root))
        return ops, in0, in1, consts, int(root[0])
    finally:
        lib.ref_expr_free(h)


# ---- oracle: single tapes ------------------------------------------------------

def eval_interval(wide, n_slots, lo, hi, t=0.0, rounding=0):
    wide = np.ascontiguousarray(wide, np.uint64)
    n_mm = int(np.sum(np.isin(wide & 0xFF, (7, 8))))
    lo = np.ascontiguousarray(lo, np.float32)
    hi = np.ascontiguousarray(hi, np.float32)
    out = np.zeros(2, np.float32)
    ch = np.zeros(max(n_mm, 1), np.uint8)
    oracle_lib().oracle_eval_interval(_p(wide), len(wide), n_slots, _p(lo), _p(hi), t, rounding, _p(out), _p(ch))
    return out, ch[:n_mm]


def eval_interval_trace(wide, n_slots, lo, hi, t=0.0, rounding=0) -> np.ndarray:
    """Every instruction's result interval, (n, 2) float32."""
    wide = np.ascontiguousarray(wide, np.uint64)
    lo = np.ascontiguousarray(lo, np.float32)
    hi = np.ascontiguousarray(hi, np.float32)
    out = np.zeros((len(wide), 2), np.float32)
    oracle_lib().oracle_eval_interval_trace(_p(wide), len(wide), n_slots, _p(lo), _p(hi), t, rounding, _p(out))
    return out


def eval_point(wide, n_slots, x, y, z, t=0.0) -> float:
    wide = np.ascontiguousarray(wide, np.uint64)
    return oracle_lib().oracle_eval_point(_p(wide), len(wide), n_slots, x, y, z, t)


def eval_gradient(wide, n_slots, x, y, z, t=0.0):
    wide = np.ascontiguousarray(wide, np.uint64)
    g = np.zeros(3, np.float32)
    oracle_lib().oracle_eval_gradient(_p(wide), len(wide), n_slots, x, y, z, t, _p(g))
    return g


def shorten(wide, n_slots, choices):
    wide = np.ascontiguousarray(wide, np.uint64)
    choices = np.ascontiguousarray(choices, np.uint8)
    out = np.zeros(len(wide), np.uint64)
    k = oracle_lib().oracle_shorten(_p(wide), len(wide), n_slots, _p(choices), len(choices), _p(out))
    return out[:k] if k < len(wide) else wide.copy()


def directed(op: int, direction: int, a: float, b: float = 0.0) -> float:
    return oracle_lib().oracle_directed(op, direction, a, b)


# ---- oracle: whole tree and render ----------------------------------------------

class OracleTree:
    """The oracle's tree for a tape and grid, in the reference's node layout."""

    def __init__(self, wide, n_slots, dims, low_vertex, world_size, tape_time=0.0, rounding=1,
                 shorten=True, threads=None):
        wide = np.ascontiguousarray(wide, np.uint64)
        d = np.zeros(8, np.uint32)
        d[: len(dims)] = dims
        low = np.ascontiguousarray(low_vertex, np.float32)
        threads = threads or os.cpu_count() or 1
        self.dims = list(dims)
        self.low_vertex = tuple(float(v) for v in low)
        self.world_size = float(world_size)
        self.n_slots = n_slots
        self.h = oracle_lib().oracle_voxelize(_p(wide), len(wide), n_slots, _p(d), len(dims), _p(low),
                                              world_size, tape_time, rounding, 1 if shorten else 0, threads)
        if not self.h:
            raise ValueError("oracle_voxelize rejected its arguments")
        self._read()

    def _read(self):
        info = np.zeros(27, np.uint64)
        oracle_lib().oracle_tree_info(self.h, _p(info))
        self.levels = int(info[0])
        self.node_count = [int(v) for v in info[1:1 + self.levels]]
        self.node_size = [int(v) for v in info[9:9 + self.levels]]
        self.node_offset = [int(v) for v in info[17:17 + self.levels]]
        self.nodes = np.zeros(int(info[25]), np.uint32)
        self.tapes = np.zeros(int(info[26]), np.uint64)
        oracle_lib().oracle_tree_nodes(self.h, _p(self.nodes))
        oracle_lib().oracle_tree_tapes(self.h, _p(self.tapes))
        w = np.zeros(8, np.uint64)
        oracle_lib().oracle_tree_work(self.h, _p(w))
        self.work = [int(v) for v in w[: self.levels]]

    def compact(self, prune: bool) -> "OracleTree":
        """The tree compacted as SceneBuilder does (oracle_compact): levels in
        depth-first preorder; with prune, empty children dropped and all-leaf
        children turned into leaf cells."""
        t = OracleTree.__new__(OracleTree)
        t.dims, t.low_vertex, t.world_size, t.n_slots = list(self.dims), self.low_vertex, self.world_size, self.n_slots
        t.h = oracle_lib().oracle_compact(self.h, 1 if prune else 0)
        t._read()
        return t

    def render(self, camera_vec, lights, tape_time=0.0, threads=None):
        """camera_vec: 16 floats (see frep_oracle.h); lights: a frep.Lights."""
        cam = np.ascontiguousarray(camera_vec, np.float32)
        W, H = int(cam[12]), int(cam[13])
        n = len(lights.directions)
        ldir = np.zeros((8, 3), np.float32)
        lcol = np.zeros((8, 4), np.float32)
        ldir[:n] = lights.directions
        lcol[:n] = lights.colors
        amb = np.asarray(lights.ambient, np.float32)
        bg = np.asarray(lights.background, np.float32)
        rgba = np.zeros((H, W, 4), np.uint8)
        hits = np.zeros((H, W, 8), np.uint32)
        oracle_lib().oracle_render(self.h, _p(cam), n, _p(ldir), _p(lcol), _p(amb), _p(bg),
                                   int(lights.shadow_mask), tape_time, _p(rgba), _p(hits),
                                   threads or os.cpu_count() or 1)
        return rgba, hits

    def __del__(self):
        if getattr(self, "h", None):
            oracle_lib().oracle_tree_free(self.h)
            self.h = None


def camera_vector(cam, width: int, height: int) -> np.ndarray:
    """A frep.Camera as the 16-float vector oracle_render takes."""
    v = np.zeros(16, np.float32)
    v[0:3] = cam.position
    v[3:6] = cam.forward
    v[6:9] = cam.initial_up
    v[9] = cam.fov_deg
    v[10] = cam.ortho_width
    v[11] = 1 if cam.orthographic else 0
    v[12], v[13] = width, height
    v[14] = 1 if cam.jitter else 0
    v[15] = cam.jitter_seed
    return v


# ---- canonical form ------------------------------------------------------------

def tape_at(tapes: np.ndarray, idx: int) -> tuple:
    n = int(tapes[idx] & 0xFFFFFFFF)
    return tuple(int(w) for w in tapes[idx + 1: idx + 1 + n])


def canonical(levels, dims, node_count, node_offset, node_size, nodes, tapes):
    """Per level: {coords: (leaf words, interior words, tape)}; checks that every
    interior bit points at a child with the right coords and that child ids are
    in range. Returns (canon, problems)."""
    canon, problems = [], []
    for lvl in range(levels):
        dim = dims[lvl]
        c3 = dim ** 3
        last = lvl == levels - 1
        per = {}
        base = node_offset[lvl]
        size = node_size[lvl]
        for i in range(node_count[lvl]):
            rec = nodes[base + i * size: base + (i + 1) * size]
            coords = (int(rec[1]), int(rec[2]), int(rec[3]))
            leaf = tuple(int(v) for v in rec[4:4 + c3 // 32])
            inter = () if last else tuple(int(v) for v in rec[4 + c3 // 32: 4 + c3 // 16])
            if coords in per:
                problems.append(f"level {lvl}: duplicate node at {coords}")
            per[coords] = (leaf, inter, tape_at(tapes, int(rec[0])))
            if not last:
                clist = rec[4 + c3 // 16: 4 + c3 // 16 + c3]
                nbase, nsize = node_offset[lvl + 1], node_size[lvl + 1]
                for w, word in enumerate(inter):
                    bits = word
                    while bits:
                        b = (bits & -bits).bit_length() - 1
                        bits &= bits - 1
                        cell = w * 32 + b
                        child = int(clist[cell])
                        if child >= node_count[lvl + 1]:
                            problems.append(f"level {lvl}: child id {child} out of range")
                            continue
                        crec = nodes[nbase + child * nsize: nbase + child * nsize + 4]
                        cz, cy, cx = cell % dim, (cell // dim) % dim, cell // (dim * dim)
                        want = (coords[0] * dim + cx, coords[1] * dim + cy, coords[2] * dim + cz)
                        got = (int(crec[1]), int(crec[2]), int(crec[3]))
                        if want != got:
                            problems.append(f"level {lvl}: child of {coords} cell {cell} has coords {got}")
        canon.append(per)
    return canon, problems


def canonical_of_oracle(t: OracleTree):
    return canonical(t.levels, t.dims, t.node_count, t.node_offset, t.node_size, t.nodes, t.tapes)


def canonical_of_export(e):
    return canonical(e.levels, e.dims, e.node_count, e.node_offset, e.node_size, e.nodes, e.tapes)


def hit_cells(hits: np.ndarray, dims, node_offset, node_size, nodes) -> np.ndarray:
    """Per-pixel canonical hit id = (level, global cell x, y, z at that level);
    -1 everywhere for a miss. hits: (H, W, 8) uint32 records (frep_hit)."""
    hits = hits.view(np.uint32)
    lvl, node, cell = hits[..., 4], hits[..., 5].astype(np.int64), hits[..., 6].astype(np.int64)
    out = np.full(hits.shape[:-1] + (4,), -1, np.int64)
    for l, dim in enumerate(dims):
        m = lvl == l
        if not m.any():
            continue
        rec = node_offset[l] + node[m] * node_size[l]
        c = cell[m]
        out[m, 0] = l
        out[m, 1] = nodes[rec + 1].astype(np.int64) * dim + c // (dim * dim)
        out[m, 2] = nodes[rec + 2].astype(np.int64) * dim + (c // dim) % dim
        out[m, 3] = nodes[rec + 3].astype(np.int64) * dim + c % dim
    return out


def resolve_layers(layers: np.ndarray) -> np.ndarray:
    """Temporal resolve (renderer/triangle.frag:14-23): the mean of the layers'
    rgb with alpha 1. layers: (n, H, W, 4) uint8. The mean is taken exactly
    and rounded to nearest, ties up, as the library defines it (the
    reference's float -> unorm rounding is the driver's)."""
    n = layers.shape[0]
    s = layers[..., :3].astype(np.int64).sum(axis=0)
    out = np.empty(layers.shape[1:], np.uint8)
    out[..., :3] = (2 * s + n) // (2 * n)
    out[..., 3] = 255
    return out
