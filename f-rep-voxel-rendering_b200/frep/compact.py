"""Host-side access to the compact tree format (include/frep.h, "Compact trees").

A compact tree blob is a ``frep_compact_header`` (120 bytes), the node pool
(u32 words) and the tape pool (u64 words), each section on an 8-byte boundary.
Every level is numbered in depth-first preorder with children in ascending
cell order, as SceneBuilder::LayoutNode lays out its node buffer
(vulkan/src/engine/scene_builder.cpp:199-238). A non-last node is
``[tapeIdx, leaf[W], interior[W], prefix[W], base]`` (W = dim^3 / 32), a
last-level node ``[tapeIdx, leaf[W]]``.

* :func:`parse` / :func:`build` — blob <-> arrays;
* :func:`pack` — a tree in the reference's node layout (voxel_storage.h:57-88,
  node.comp; e.g. ``VoxelStorage.export()``) to a blob, renumbered in preorder
  with every node and mask kept (``FREP_COMPACT_LAYOUT``);
* :func:`expand` — a blob back to the reference's layout (coordinates and full
  child lists restored);
* :func:`check` — the library's own validation (``frep_compact_check``; host
  only, no device needed); :func:`save` / :func:`load` — a blob to and from a
  file (checked on load).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L

COMPACT_LAYOUT = 0
COMPACT_PRUNE = 1
MAGIC = b"FREPCT01"

HEADER = np.dtype([("magic", "S8"), ("version", "<u4"), ("levels", "<u4"), ("dims", "<u4", (8,)),
                   ("low_vertex", "<f4", (3,)), ("world_size", "<f4"), ("mode", "<u4"), ("n_slots", "<u4"),
                   ("node_count", "<u4", (8,)), ("node_words", "<u8"), ("tape_words", "<u8")])
assert HEADER.itemsize == 120


def record_words(dim: int, last: bool) -> int:
    w = dim ** 3 // 32
    return 1 + w if last else 2 + 3 * w


def reference_words(dim: int, last: bool) -> int:
    """Node size of the reference's layout (node.comp:4-15)."""
    c3 = dim ** 3
    return 4 + c3 // 16 if last else 4 + 17 * c3 // 16


def _align8(n: int) -> int:
    return (n + 7) // 8 * 8


@dataclass
class Blob:
    levels: int
    dims: list
    low_vertex: tuple
    world_size: float
    mode: int
    n_slots: int
    node_count: list
    nodes: np.ndarray   # u32
    tapes: np.ndarray   # u64

    @property
    def node_size(self) -> list:
        return [record_words(d, l == self.levels - 1) for l, d in enumerate(self.dims)]

    @property
    def node_offset(self) -> list:
        ofs, at = [], 0
        for n, s in zip(self.node_count, self.node_size):
            ofs.append(at)
            at += n * s
        return ofs


def parse(blob) -> Blob:
    raw = np.frombuffer(bytes(blob) if not isinstance(blob, np.ndarray) else blob.tobytes(), np.uint8)
    h = raw[:HEADER.itemsize].view(HEADER)[0]
    if bytes(h["magic"]) != MAGIC:
        raise ValueError("not a compact tree blob")
    levels = int(h["levels"])
    nw, tw = int(h["node_words"]), int(h["tape_words"])
    at = _align8(HEADER.itemsize)
    nodes = raw[at:at + 4 * nw].view(np.uint32).copy()
    at = _align8(at + 4 * nw)
    tapes = raw[at:at + 8 * tw].view(np.uint64).copy()
    return Blob(levels, [int(d) for d in h["dims"][:levels]], tuple(float(v) for v in h["low_vertex"]),
                float(h["world_size"]), int(h["mode"]), int(h["n_slots"]),
                [int(c) for c in h["node_count"][:levels]], nodes, tapes)


def build(b: Blob) -> np.ndarray:
    """The blob bytes (uint8 array) of ``b``."""
    h = np.zeros(1, HEADER)
    h["magic"] = MAGIC
    h["version"] = 1
    h["levels"] = b.levels
    h["dims"][0, :b.levels] = b.dims
    h["low_vertex"] = b.low_vertex
    h["world_size"] = b.world_size
    h["mode"] = b.mode
    h["n_slots"] = b.n_slots
    h["node_count"][0, :b.levels] = b.node_count
    h["node_words"] = len(b.nodes)
    h["tape_words"] = len(b.tapes)
    n_at = _align8(HEADER.itemsize)
    t_at = _align8(n_at + 4 * len(b.nodes))
    out = np.zeros(t_at + 8 * len(b.tapes), np.uint8)
    out[:HEADER.itemsize] = h.view(np.uint8)
    out[n_at:n_at + 4 * len(b.nodes)] = np.ascontiguousarray(b.nodes, np.uint32).view(np.uint8)
    out[t_at:] = np.ascontiguousarray(b.tapes, np.uint64).view(np.uint8)
    return out


def _cells(words: np.ndarray) -> np.ndarray:
    """Set bit indices of a mask (u32 words, bit i of word w = cell 32 w + i), ascending."""
    bits = np.unpackbits(np.ascontiguousarray(words, "<u4").view(np.uint8), bitorder="little")
    return np.nonzero(bits)[0]


def pack(levels, dims, node_count, node_offset, node_size, nodes, tapes, low_vertex, world_size,
         n_slots) -> np.ndarray:
    """A tree in the reference's node layout -> blob (FREP_COMPACT_LAYOUT):
    the nodes reachable from the root, every level renumbered in preorder
    (children in (parent, cell) order), masks and tape indices unchanged (the
    tape pool is copied as is)."""
    nodes = np.asarray(nodes, np.uint32)
    order = np.array([0], np.int64)          # source ids of this level, in preorder
    counts, records = [], []
    for l in range(levels):
        dim = dims[l]
        c3 = dim ** 3
        w = c3 // 32
        last = l == levels - 1
        rec = nodes[node_offset[l] + order[:, None] * node_size[l] + np.arange(node_size[l])[None, :]]
        d = np.zeros((len(order), record_words(dim, last)), np.uint32)
        d[:, 0] = rec[:, 0]
        d[:, 1:1 + w] = rec[:, 4:4 + w]
        counts.append(len(order))
        if not last:
            inter = np.ascontiguousarray(rec[:, 4 + w:4 + 2 * w])
            pc = np.bitwise_count(inter).astype(np.int64)
            d[:, 1 + w:1 + 2 * w] = inter
            d[:, 1 + 2 * w:1 + 3 * w] = np.cumsum(pc, axis=1) - pc
            per = pc.sum(axis=1)
            d[:, 1 + 3 * w] = np.cumsum(per) - per
            bits = np.unpackbits(inter.astype("<u4").view(np.uint8), axis=1, bitorder="little")[:, :c3]
            parent, cell = np.nonzero(bits)
            order = rec[parent, 4 + c3 // 16 + cell].astype(np.int64)
        records.append(d.reshape(-1))
    out = np.concatenate(records) if records else np.zeros(0, np.uint32)
    return build(Blob(levels, list(dims), tuple(low_vertex), float(world_size), COMPACT_LAYOUT, int(n_slots),
                      counts, out, np.ascontiguousarray(tapes, np.uint64)))


@dataclass
class ReferenceLayout:
    """A tree in the reference's node layout (what ``VoxelStorage.export()``
    and the oracle hold), node ids = preorder indices."""
    levels: int
    dims: list
    node_count: list
    node_offset: list
    node_size: list
    nodes: np.ndarray
    tapes: np.ndarray
    low_vertex: tuple
    world_size: float
    n_slots: int
    mode: int


def expand(blob) -> ReferenceLayout:
    """A blob -> the reference's layout, with node coordinates (in units of
    the level's node size) and full child lists (0xFFFFFFFF = no child).
    Vectorized per level: children are numbered in (parent, cell) order, which
    is the blob's preorder."""
    b = blob if isinstance(blob, Blob) else parse(blob)
    sizes = [reference_words(d, l == b.levels - 1) for l, d in enumerate(b.dims)]
    offs, at = [], 0
    for n, s in zip(b.node_count, sizes):
        offs.append(at)
        at += n * s
    out = np.zeros(at, np.uint32)
    csz, cofs = b.node_size, b.node_offset
    coords = np.zeros((1, 3), np.int64)
    for l in range(b.levels):
        dim, n = b.dims[l], b.node_count[l]
        c3 = dim ** 3
        w = c3 // 32
        last = l == b.levels - 1
        src = b.nodes[cofs[l]: cofs[l] + n * csz[l]].reshape(n, csz[l])
        dst = out[offs[l]: offs[l] + n * sizes[l]].reshape(n, sizes[l])
        dst[:, 0] = src[:, 0]
        dst[:, 1:4] = coords
        dst[:, 4:4 + w] = src[:, 1:1 + w]
        if last:
            break
        inter = np.ascontiguousarray(src[:, 1 + w:1 + 2 * w])
        dst[:, 4 + w:4 + 2 * w] = inter
        bits = np.unpackbits(inter.astype("<u4").view(np.uint8), axis=1, bitorder="little")[:, :c3]
        parent, cell = np.nonzero(bits)                    # row-major: (parent, cell) order
        ids = np.arange(len(cell), dtype=np.int64)
        # each node's base must be the number of children of the nodes before it
        per = bits.sum(axis=1, dtype=np.int64)
        starts = np.cumsum(per) - per
        has = per > 0
        if len(ids) != b.node_count[l + 1] or not np.array_equal(src[has, 1 + 3 * w].astype(np.int64), starts[has]):
            raise ValueError(f"level {l}: children are not numbered in preorder")
        lst = dst[:, 4 + 2 * w:4 + 2 * w + c3]
        lst[:] = 0xFFFFFFFF
        lst[parent, cell] = ids
        cxyz = np.stack([cell // (dim * dim), (cell // dim) % dim, cell % dim], 1)
        coords = coords[parent] * dim + cxyz
    return ReferenceLayout(b.levels, list(b.dims), list(b.node_count), offs, sizes, out, b.tapes, b.low_vertex,
                           b.world_size, b.n_slots, b.mode)


def as_bytes(blob) -> np.ndarray:
    """The blob's bytes as a contiguous uint8 array: an ndarray of any dtype
    (e.g. a blob held as u32 or u64 words) is reinterpreted, not converted
    value by value; anything else goes through bytes()."""
    if isinstance(blob, np.ndarray):
        return np.ascontiguousarray(blob).view(np.uint8).ravel()
    return np.frombuffer(bytes(blob), np.uint8)


def save(blob, path) -> None:
    """Writes a blob to a file (the bytes as they are: the format is position
    independent and little endian)."""
    as_bytes(blob).tofile(str(path))


def load(path) -> np.ndarray:
    """Reads a blob from a file and checks it (frep_compact_check)."""
    blob = np.fromfile(str(path), np.uint8)
    check(blob)
    return blob


def check(blob) -> None:
    """frep_compact_check on a host blob; raises FrepError with the first problem."""
    arr = as_bytes(blob)
    L.check(L.lib().frep_compact_check(arr.ctypes.data_as(C.c_void_p), arr.nbytes))
