"""frep — B200-native F-rep voxelize-and-raytrace (host-side Python mirror).

The classes follow the reference's host interface for this path so that code
written against it reads the same:

* ``csg`` (``frep.csg``)       — ``csg::Expr`` / ``csg::lib`` scene construction
* ``Tape``                     — ``csg::Tape`` (vulkan/include/csg/tape.h:12-83)
* ``VoxelStorage``             — ``VoxelStorage`` (vulkan/include/engine/voxel_storage.h:9-89)
* ``Voxelizer.voxelize``       — ``Voxelizer::Voxelize`` (vulkan/src/engine/voxelizer.cpp:429-440)
* ``Camera`` / ``Raytracer.trace`` — ``Camera`` (camera.h) / ``Raytracer::Trace`` (raytracer.cpp:243-272)

Everything below calls the C-ABI in include/frep.h (libfrep.so); the compute
runs in the sm_100a kernels. Device buffers and streams are torch's.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import csg
from . import _lib as L
from ._lib import FrepError

__all__ = ["csg", "Tape", "Context", "VoxelStorage", "Voxelizer", "Camera", "Lights", "Raytracer",
           "FrepError", "ROUND_NEAREST", "ROUND_OUTWARD", "ROUND_HYBRID", "TreeExport", "CompactTree"]

ROUND_NEAREST = 0
ROUND_OUTWARD = 1
ROUND_HYBRID = 2   # outward intervals intersected with affine forms (include/frep.h)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _dag_struct(expr: csg.Expr):
    ops, in0, in1, consts, root = expr.flatten()
    d = L.Dag(len(ops), ops.ctypes.data_as(C.POINTER(C.c_uint8)), in0.ctypes.data_as(C.POINTER(C.c_uint32)),
              in1.ctypes.data_as(C.POINTER(C.c_uint32)), consts.ctypes.data_as(C.POINTER(C.c_float)), root)
    return d, (ops, in0, in1, consts)


class Tape:
    """A compiled tape (csg::Tape). ``Tape(expr)`` runs the library's compiler
    (simplify, topological sort, constant pool, slot allocation)."""

    def __init__(self, expr: csg.Expr | None = None, *, _handle=None, const_reload: int = 0):
        """const_reload: frep_tape_opts.const_reload_distance (0 = default,
        0xFFFFFFFF = keep the reference's slot allocation everywhere)."""
        self._h = C.c_void_p()
        if _handle is not None:
            self._h = _handle
        elif expr is not None:
            d, keep = _dag_struct(expr)
            opts = L.TapeOpts(const_reload)
            L.check(L.lib().frep_tape_compile_opts(C.byref(d), C.byref(opts), C.byref(self._h)))
        else:
            raise ValueError("Tape needs an expression")
        info = L.TapeInfo()
        L.check(L.lib().frep_tape_get_info(self._h, C.byref(info)))
        self.n_instr = info.n_instr
        self.n_slots = info.n_slots
        self.n_consts = info.n_consts
        self.n_minmax = info.n_minmax
        self.fits_reference = bool(info.fits_reference)
        self.uses_time = bool(info.uses_time)

    @classmethod
    def from_reference(cls, instrs, consts) -> "Tape":
        """Imports a tape in the reference's 8-bit upload format + constant pool."""
        instrs = np.ascontiguousarray(instrs, np.uint32)
        consts = np.ascontiguousarray(consts, np.float32)
        h = C.c_void_p()
        L.check(L.lib().frep_tape_from_reference(_ptr(instrs), len(instrs), _ptr(consts), len(consts), C.byref(h)))
        return cls(_handle=h)

    @classmethod
    def from_wide(cls, instrs) -> "Tape":
        """A tape in the wide encoding (Tape.wide())."""
        instrs = np.ascontiguousarray(instrs, np.uint64)
        h = C.c_void_p()
        L.check(L.lib().frep_tape_from_wide(_ptr(instrs), len(instrs), C.byref(h)))
        return cls(_handle=h)

    @classmethod
    def from_dag(cls, ops, in0, in1, consts, root) -> "Tape":
        ops = np.ascontiguousarray(ops, np.uint8)
        in0 = np.ascontiguousarray(in0, np.uint32)
        in1 = np.ascontiguousarray(in1, np.uint32)
        consts = np.ascontiguousarray(consts, np.float32)
        d = L.Dag(len(ops), ops.ctypes.data_as(C.POINTER(C.c_uint8)), in0.ctypes.data_as(C.POINTER(C.c_uint32)),
                  in1.ctypes.data_as(C.POINTER(C.c_uint32)), consts.ctypes.data_as(C.POINTER(C.c_float)), int(root))
        h = C.c_void_p()
        L.check(L.lib().frep_tape_compile(C.byref(d), C.byref(h)))
        return cls(_handle=h)

    def __del__(self):
        # at interpreter exit the module globals may already be gone
        if L is not None and C is not None and L._lib is not None and getattr(self, "_h", None) and self._h.value:
            L.lib().frep_tape_destroy(self._h)
            self._h = C.c_void_p()

    @property
    def handle(self):
        return self._h

    def wide(self) -> np.ndarray:
        """Instruction words of the library's wide encoding (include/frep.h)."""
        out = np.zeros(self.n_instr, np.uint64)
        L.check(L.lib().frep_tape_get_instrs(self._h, _ptr(out), self.n_instr))
        return out

    @property
    def instructions(self) -> np.ndarray:
        """csg::Tape::instructions packed as the reference uploads them."""
        instrs = np.zeros(self.n_instr, np.uint32)
        consts = np.zeros(max(self.n_consts, 1), np.float32)
        L.check(L.lib().frep_tape_get_reference(self._h, _ptr(instrs), _ptr(consts)))
        return instrs

    @property
    def constant_pool(self) -> np.ndarray:
        instrs = np.zeros(self.n_instr, np.uint32)
        consts = np.zeros(max(self.n_consts, 1), np.float32)
        L.check(L.lib().frep_tape_get_reference(self._h, _ptr(instrs), _ptr(consts)))
        return consts[: self.n_consts]

    def slot_count(self) -> int:
        return self.n_slots

    def eval_points(self, xyzt) -> np.ndarray:
        xyzt = np.ascontiguousarray(xyzt, np.float32).reshape(-1, 4)
        out = np.zeros(len(xyzt), np.float32)
        L.check(L.lib().frep_tape_eval(self._h, _ptr(xyzt), len(xyzt), _ptr(out)))
        return out

    def eval(self, x, y, z, t=0.0) -> float:
        return float(self.eval_points(np.array([[x, y, z, t]], np.float32))[0])


class Context:
    """One device and its HBM budget (frep_ctx)."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0):
        self._h = C.c_void_p()
        L.check(L.lib().frep_ctx_create(device, hbm_budget_bytes, C.byref(self._h)))
        self.device = device

    def memory(self):
        used, budget = C.c_uint64(), C.c_uint64()
        L.check(L.lib().frep_ctx_memory(self._h, C.byref(used), C.byref(budget)))
        return used.value, budget.value

    def eval_points(self, tape: "Tape", xyzt) -> np.ndarray:
        """Tape values at n points (x, y, z, t) on the device, with the point
        pass's operations (frep_tape_eval_device)."""
        xyzt = np.ascontiguousarray(xyzt, np.float32).reshape(-1, 4)
        out = np.zeros(len(xyzt), np.float32)
        L.check(L.lib().frep_tape_eval_device(self._h, tape.handle, _ptr(xyzt), len(xyzt), _ptr(out)))
        return out

    def eval_intervals(self, tape: "Tape", boxes, tape_time: float = 0.0,
                       rounding: int = ROUND_OUTWARD) -> np.ndarray:
        """Interval bounds of the tape over n boxes (low xyz, high xyz) on the
        device, with the level passes' operations (frep_tape_eval_intervals).
        Returns an (n, 2) array of (low, high)."""
        boxes = np.ascontiguousarray(boxes, np.float32).reshape(-1, 6)
        out = np.zeros((len(boxes), 2), np.float32)
        L.check(L.lib().frep_tape_eval_intervals(self._h, tape.handle, _ptr(boxes), len(boxes),
                                                 float(tape_time), int(rounding), _ptr(out)))
        return out

    def close(self):
        if self._h is not None and self._h.value and L is not None and L._lib is not None:
            L.lib().frep_ctx_destroy(self._h)
        self._h = C.c_void_p()

    def __del__(self):
        if L is not None and C is not None:
            self.close()


@dataclass
class TreeExport:
    """A tree copied to the host: its header (frep_tree_info fields), the node
    pool (reference layout, u32) and the tape pool (u64)."""

    levels: int
    dims: list
    node_count: list
    node_offset: list
    node_size: list
    tape_size_sum: list
    tape_size_max: list
    tape_words_used: int
    nodes: np.ndarray
    tapes: np.ndarray


class VoxelStorage:
    """Grid description + device tree (VoxelStorage, voxel_storage.h:9-89).
    Fill grid_dims / low_vertex / world_size, then call init(ctx, shape)."""

    def __init__(self, grid_dims=(16, 4), low_vertex=(-1.5, -1.5, -1.5), world_size=3.0,
                 rounding: int = ROUND_OUTWARD, shorten: bool = True, node_words: int = 0,
                 tape_words: int = 0, point_cells_per_lane: int = 0, separate_tapes: bool = False):
        self.grid_dims = list(grid_dims)
        self.low_vertex = tuple(float(v) for v in low_vertex)
        self.world_size = float(world_size)
        self.rounding = rounding
        self.shorten = shorten
        self.node_words = node_words
        self.tape_words = tape_words
        self.point_cells_per_lane = point_cells_per_lane
        self.separate_tapes = separate_tapes
        self.tape: Tape | None = None
        self.ctx: Context | None = None
        self._tree = C.c_void_p()
        self.interior_node_count: list[int] = []

    @property
    def grid_levels(self) -> int:
        return len(self.grid_dims)

    @property
    def fine_grid_dim(self) -> int:
        return int(np.prod(self.grid_dims))

    def grid_struct(self) -> L.Grid:
        g = L.Grid()
        g.levels = len(self.grid_dims)
        for i, d in enumerate(self.grid_dims):
            g.dims[i] = d
        for i in range(3):
            g.low_vertex[i] = self.low_vertex[i]
        g.world_size = self.world_size
        return g

    def init(self, ctx: Context, shape) -> "VoxelStorage":
        self.ctx = ctx
        self.tape = shape if isinstance(shape, Tape) else Tape(shape)
        opts = L.VoxelizeOpts(self.rounding, 1 if self.shorten else 0, self.node_words, self.tape_words,
                              self.point_cells_per_lane, 1 if self.separate_tapes else 0)
        g = self.grid_struct()
        L.check(L.lib().frep_tree_create(ctx._h, C.byref(g), C.byref(opts), C.byref(self._tree)))
        self.interior_node_count = [0] * self.grid_levels
        return self

    @property
    def tree(self):
        return self._tree

    def cleanup(self):
        if self._tree.value and L._lib is not None:
            L.lib().frep_tree_destroy(self._tree)
            self._tree = C.c_void_p()

    def __del__(self):
        if L is not None and C is not None:
            self.cleanup()

    def sync(self, raise_on_overflow: bool = True) -> L.TreeInfo:
        info = L.TreeInfo()
        st = L.lib().frep_tree_sync(self._tree, C.byref(info))
        if st != L.OK and (raise_on_overflow or st != L.ERR_CAPACITY):
            L.check(st)
        self.interior_node_count = list(info.node_count[: self.grid_levels])
        return info

    def work(self) -> list[int]:
        arr = (C.c_uint64 * L.MAX_LEVELS)()
        L.check(L.lib().frep_tree_work(self._tree, arr))
        return list(arr[: self.grid_levels])

    def fp32_ops(self) -> list[int]:
        arr = (C.c_uint64 * L.MAX_LEVELS)()
        L.check(L.lib().frep_tree_fp32_ops(self._tree, arr))
        return list(arr[: self.grid_levels])

    def set_profiling(self, enable: bool = True) -> None:
        L.check(L.lib().frep_tree_set_profiling(self._tree, 1 if enable else 0))

    def level_timings(self) -> list[float]:
        """Device milliseconds of each level pass of the last voxelization."""
        arr = (C.c_float * L.MAX_LEVELS)()
        L.check(L.lib().frep_tree_timings(self._tree, arr))
        return list(arr[: self.grid_levels])

    def export(self) -> TreeExport:
        info = self.sync()
        nodes = np.zeros(max(info.node_words_used, 1), np.uint32)
        tapes = np.zeros(max(info.tape_words_used, 1), np.uint64)
        L.check(L.lib().frep_tree_copy_nodes(self._tree, _ptr(nodes), info.node_words_used))
        L.check(L.lib().frep_tree_copy_tapes(self._tree, _ptr(tapes), info.tape_words_used))
        n = self.grid_levels
        return TreeExport(n, list(info.dims[:n]), list(info.node_count[:n]), list(info.node_offset[:n]),
                          list(info.node_size[:n]), list(info.tape_size_sum[:n]),
                          list(info.tape_size_max[:n]), info.tape_words_used, nodes, tapes)


def _stream_ptr(stream):
    if stream is None:
        try:
            import torch
            return C.c_void_p(torch.cuda.current_stream().cuda_stream)
        except Exception:
            return C.c_void_p(0)
    if hasattr(stream, "cuda_stream"):
        return C.c_void_p(stream.cuda_stream)
    return C.c_void_p(int(stream))


class Voxelizer:
    """Builds the sparse tree on the device (Voxelizer, voxelizer.h:12-113)."""

    def __init__(self, ctx: Context, voxels: VoxelStorage):
        self.ctx = ctx
        self.voxels = voxels

    def voxelize(self, tape_time: float = 0.0, stream=None, reuse: "VoxelStorage | None" = None) -> None:
        """Enqueues every level pass on `stream`; no host round trip per level.
        reuse: a VoxelStorage of the same grid voxelized earlier (the previous
        frame); subtrees whose tape does not read the time and matches it are
        copied from it instead of evaluated (frep_voxelize_reuse)."""
        if reuse is None:
            L.check(L.lib().frep_voxelize(self.ctx._h, self.voxels.tree, self.voxels.tape.handle,
                                          float(tape_time), _stream_ptr(stream)))
        else:
            L.check(L.lib().frep_voxelize_reuse(self.ctx._h, self.voxels.tree, reuse.tree, self.voxels.tape.handle,
                                                float(tape_time), _stream_ptr(stream)))

    def print_stats(self) -> None:
        info = self.voxels.sync()
        total = sum(info.node_count[: self.voxels.grid_levels])
        print(f"[+] Total interior nodes :\n\tcount={total}\tnode buf words={info.node_words_used}")
        print(f"[+] Total tapes :\n\ttape buf bytes={8 * info.tape_words_used}")
        for i in range(self.voxels.grid_levels):
            cnt = max(info.node_count[i], 1)
            print(f"\t{i}: nodes={info.node_count[i]}  avg tape={info.tape_size_sum[i] / cnt:.1f}"
                  f"  max tape={info.tape_size_max[i]}")


class AnimatedVoxelizer:
    """Re-voxelizes a time-dependent shape every frame (the reference's
    real-time mode, application.cpp:68-79) into two alternating trees, each
    frame reusing the time-independent subtrees of the previous one.
    `voxelize(t)` returns the VoxelStorage holding frame t; a Raytracer follows
    it through `raytracer.voxels = ...`."""

    def __init__(self, ctx: Context, make_storage, shape):
        """make_storage: a callable returning a new (un-initialised) VoxelStorage."""
        self.ctx = ctx
        tape = shape if isinstance(shape, Tape) else Tape(shape)
        self.storages = [make_storage().init(ctx, tape), make_storage().init(ctx, tape)]
        self.frame = 0

    @property
    def current(self) -> VoxelStorage:
        return self.storages[(self.frame - 1) % 2]

    def voxelize(self, tape_time: float, stream=None) -> VoxelStorage:
        vs = self.storages[self.frame % 2]
        prev = self.storages[(self.frame - 1) % 2] if self.frame > 0 else None
        Voxelizer(self.ctx, vs).voxelize(tape_time, stream=stream, reuse=prev)
        self.frame += 1
        return vs

    def cleanup(self) -> None:
        for s in self.storages:
            s.cleanup()


@dataclass
class Camera:
    """Camera (camera.h:6-41). forward / initial_up are normalised by the
    library; fov_deg is the horizontal field of view."""

    position: tuple = (0.0, 0.0, 40.0)
    forward: tuple = (0.0, 0.0, -1.0)
    initial_up: tuple = (0.0, 1.0, 0.0)
    fov_deg: float = 45.0
    orthographic: bool = False
    ortho_width: float = 2.0
    jitter: bool = False
    jitter_seed: float = 0.0

    def struct(self, width: int, height: int) -> L.CameraStruct:
        c = L.CameraStruct()
        for i in range(3):
            c.position[i] = self.position[i]
            c.forward[i] = self.forward[i]
            c.up[i] = self.initial_up[i]
        c.fov_deg = self.fov_deg
        c.ortho_width = self.ortho_width
        c.projection = 1 if self.orthographic else 0
        c.width, c.height = width, height
        c.jitter = 1 if self.jitter else 0
        c.jitter_seed = self.jitter_seed
        return c


@dataclass
class Lights:
    """Directional lights, ambient and background (raytracer.cpp:183-192).
    Defaults are the reference's two hard-coded lights."""

    directions: list = field(default_factory=lambda: [(-1.0, -1.0, -0.2), (1.0, -1.0, -0.2)])
    colors: list = field(default_factory=lambda: [(1.0, 0.0, 0.0, 0.0), (0.0, 0.0, 2.0, 0.0)])
    ambient: tuple = (0.2, 0.2, 0.2, 1.0)
    background: tuple = (0.0, 0.0, 0.0, 1.0)
    shadow_mask: int = 0

    def struct(self) -> L.LightsStruct:
        s = L.LightsStruct()
        s.count = len(self.directions)
        for i, (d, c) in enumerate(zip(self.directions, self.colors)):
            for k in range(3):
                s.direction[i][k] = d[k]
            for k in range(4):
                s.color[i][k] = c[k]
        for k in range(4):
            s.ambient[k] = self.ambient[k]
            s.background[k] = self.background[k]
        s.shadow_mask = self.shadow_mask
        return s


class Raytracer:
    """Renders a voxelized tree (Raytracer, raytracer.h:15-121) into device
    buffers (torch tensors): an rgba8 image and optionally hit records."""

    def __init__(self, ctx: Context, voxels: VoxelStorage):
        self.ctx = ctx
        self.voxels = voxels
        self.lights = Lights()

    def set_background_color(self, rgb) -> None:
        self.lights.background = (float(rgb[0]), float(rgb[1]), float(rgb[2]), 1.0)

    def trace(self, camera: Camera, tape_time: float = 0.0, width: int = 256, height: int = 256,
              hits: bool = False, out=None, stream=None):
        import torch
        dev = torch.device("cuda", self.ctx.device)
        if out is None:
            rgba = torch.empty((height, width, 4), dtype=torch.uint8, device=dev)
            hit_buf = torch.empty((height, width, 8), dtype=torch.int32, device=dev) if hits else None
        else:
            rgba, hit_buf = out
        img = L.Image(rgba.data_ptr() if rgba is not None else None,
                      hit_buf.data_ptr() if hit_buf is not None else None)
        cam = camera.struct(width, height)
        lights = self.lights.struct()
        L.check(L.lib().frep_render(self.ctx._h, self.voxels.tree, C.byref(cam), C.byref(lights),
                                    float(tape_time), C.byref(img), _stream_ptr(stream)))
        return rgba, hit_buf

    def trace_temporal(self, camera: Camera, tape_time: float = 0.0, width: int = 256, height: int = 256,
                       n_samples: int = 4, stream=None):
        """n_samples jittered frames (seeds camera.jitter_seed + i) averaged
        into one rgba8 image (the reference's temporal accumulation over an
        image array, renderer/triangle.frag). Returns (image, layers)."""
        import torch
        dev = torch.device("cuda", self.ctx.device)
        layers = torch.empty((n_samples, height, width, 4), dtype=torch.uint8, device=dev)
        rgba = torch.empty((height, width, 4), dtype=torch.uint8, device=dev)
        cam = camera.struct(width, height)
        lights = self.lights.struct()
        L.check(L.lib().frep_render_temporal(self.ctx._h, self.voxels.tree, C.byref(cam), C.byref(lights),
                                             float(tape_time), n_samples, layers.data_ptr(), rgba.data_ptr(),
                                             _stream_ptr(stream)))
        return rgba, layers


class CompactTree:
    """A compact tree (frep_compact): the voxelized tree with every level in
    depth-first preorder and no per-node child lists, optionally pruned as
    SceneBuilder::BuildNode does (scene_builder.cpp:91-156); renders like
    Raytracer.trace and round-trips through a host blob (frep.compact)."""

    def __init__(self, ctx: Context, handle: C.c_void_p):
        self.ctx = ctx
        self._h = handle
        self.lights = Lights()

    @classmethod
    def from_storage(cls, ctx: Context, voxels: VoxelStorage, prune: bool = False, stream=None) -> "CompactTree":
        h = C.c_void_p()
        L.check(L.lib().frep_tree_compact(ctx._h, voxels.tree, 1 if prune else 0, _stream_ptr(stream), C.byref(h)))
        return cls(ctx, h)

    @classmethod
    def from_blob(cls, ctx: Context, blob) -> "CompactTree":
        from .compact import as_bytes
        arr = as_bytes(blob)
        h = C.c_void_p()
        L.check(L.lib().frep_compact_import(ctx._h, _ptr(arr), arr.nbytes, C.byref(h)))
        return cls(ctx, h)

    def info(self) -> "L.CompactInfo":
        i = L.CompactInfo()
        L.check(L.lib().frep_compact_get_info(self._h, C.byref(i)))
        return i

    def export(self) -> np.ndarray:
        """The blob (uint8 array)."""
        size = C.c_uint64()
        L.check(L.lib().frep_compact_export(self._h, None, 0, C.byref(size)))
        out = np.zeros(size.value, np.uint8)
        L.check(L.lib().frep_compact_export(self._h, _ptr(out), out.nbytes, C.byref(size)))
        return out

    def trace(self, camera: Camera, tape_time: float = 0.0, width: int = 256, height: int = 256,
              hits: bool = False, out=None, stream=None):
        import torch
        dev = torch.device("cuda", self.ctx.device)
        if out is None:
            rgba = torch.empty((height, width, 4), dtype=torch.uint8, device=dev)
            hit_buf = torch.empty((height, width, 8), dtype=torch.int32, device=dev) if hits else None
        else:
            rgba, hit_buf = out
        img = L.Image(rgba.data_ptr() if rgba is not None else None,
                      hit_buf.data_ptr() if hit_buf is not None else None)
        cam = camera.struct(width, height)
        lights = self.lights.struct()
        L.check(L.lib().frep_render_compact(self.ctx._h, self._h, C.byref(cam), C.byref(lights), float(tape_time),
                                            C.byref(img), _stream_ptr(stream)))
        return rgba, hit_buf

    def close(self):
        if self._h is not None and self._h.value and L is not None and L._lib is not None:
            L.lib().frep_compact_destroy(self._h)
        self._h = C.c_void_p()

    def __del__(self):
        if L is not None and C is not None:
            self.close()


def resolve_layers(layers, stream=None):
    """Mean of rgba8 layers (device tensor (n, H, W, 4)) -> (H, W, 4)."""
    import torch
    n, h, w, _ = layers.shape
    out = torch.empty((h, w, 4), dtype=torch.uint8, device=layers.device)
    L.check(L.lib().frep_resolve_layers(layers.data_ptr(), n, w, h, out.data_ptr(), _stream_ptr(stream)))
    return out


class Batch:
    """Many scenes voxelized and rendered together (frep_batch): one launch per
    level pass over all trees, one launch for all frames, optionally replayed
    as a CUDA graph. Scenes keep their own VoxelStorage (tree and tape)."""

    def __init__(self, ctx: Context, storages: list):
        self.ctx = ctx
        self.storages = list(storages)
        arr = (C.c_void_p * len(self.storages))(*[s.tree.value for s in self.storages])
        self._h = C.c_void_p()
        L.check(L.lib().frep_batch_create(ctx._h, arr, len(self.storages), C.byref(self._h)))
        self._tapes = (C.c_void_p * len(self.storages))(*[s.tape.handle.value for s in self.storages])

    def close(self):
        if self._h is not None and self._h.value and L._lib is not None:
            L.lib().frep_batch_destroy(self._h)
        self._h = C.c_void_p()

    def __del__(self):
        if L is not None and C is not None:
            self.close()

    def set_tapes(self):
        self._tapes = (C.c_void_p * len(self.storages))(*[s.tape.handle.value for s in self.storages])

    @staticmethod
    def _times(tape_times):
        if tape_times is None:
            return None
        return (C.c_float * len(tape_times))(*[float(t) for t in tape_times])

    def info(self) -> "L.BatchInfo":
        out = L.BatchInfo()
        L.check(L.lib().frep_batch_get_info(self._h, C.byref(out)))
        return out

    def set_trees(self, storages: list) -> None:
        """Replaces the tree set (a serving loop's next step)."""
        self.storages = list(storages)
        arr = (C.c_void_p * len(self.storages))(*[s.tree.value for s in self.storages])
        L.check(L.lib().frep_batch_set_trees(self._h, arr, len(self.storages)))
        self.set_tapes()

    def render_frames(self, storages, cameras, sizes, rgba, hits=None, lights=None, tape_times=None, stream=None):
        """One launch rendering frame i of storages[i] (repeats allowed)."""
        trees = (C.c_void_p * len(storages))(*[s.tree.value for s in storages])
        cams, imgs = self._frames(cameras, sizes, rgba, hits)
        lt = (lights or Lights()).struct()
        L.check(L.lib().frep_batch_render_frames(self._h, trees, len(storages), cams, C.byref(lt),
                                                 self._times(tape_times), imgs, _stream_ptr(stream)))

    def set_tuning(self, interval_warps_per_block: int = 0, point_warps_per_block: int = 0) -> None:
        L.check(L.lib().frep_batch_set_tuning(self._h, interval_warps_per_block, point_warps_per_block))

    def set_profiling(self, enable: bool = True) -> None:
        L.check(L.lib().frep_batch_set_profiling(self._h, 1 if enable else 0))

    def timings(self) -> dict:
        """Device ms of the last profiled plain calls: {"level": [[interval,
        point K=4, point K=2] per level], "init": ms, "render": ms}."""
        arr = (C.c_float * (3 * L.MAX_LEVELS + 2))()
        L.check(L.lib().frep_batch_timings(self._h, arr))
        lv = [[arr[3 * l + k] for k in range(3)] for l in range(L.MAX_LEVELS)]
        return {"level": lv, "init": arr[3 * L.MAX_LEVELS], "render": arr[3 * L.MAX_LEVELS + 1]}

    def voxelize(self, tape_times=None, stream=None):
        L.check(L.lib().frep_batch_voxelize(self._h, self._tapes, self._times(tape_times), _stream_ptr(stream)))

    @staticmethod
    def _frames(cameras, sizes, rgba, hits):
        n = len(cameras)
        cams = (L.CameraStruct * n)(*[c.struct(w, h) for c, (w, h) in zip(cameras, sizes)])
        imgs = (L.Image * n)()
        for i in range(n):
            imgs[i].rgba8 = rgba[i].data_ptr()
            imgs[i].hits = hits[i].data_ptr() if hits is not None else None
        return cams, imgs

    def render(self, cameras, sizes, rgba, hits=None, lights=None, tape_times=None, stream=None):
        """rgba[i] / hits[i]: device tensors (H, W, 4) uint8 / (H, W, 8) int32."""
        cams, imgs = self._frames(cameras, sizes, rgba, hits)
        lt = (lights or Lights()).struct()
        L.check(L.lib().frep_batch_render(self._h, cams, C.byref(lt), self._times(tape_times), imgs,
                                          _stream_ptr(stream)))

    def run(self, cameras, sizes, rgba, hits=None, lights=None, tape_times=None, graph=True, stream=None):
        cams, imgs = self._frames(cameras, sizes, rgba, hits)
        lt = (lights or Lights()).struct()
        L.check(L.lib().frep_batch_run(self._h, self._tapes, self._times(tape_times), cams, C.byref(lt), imgs,
                                       1 if graph else 0, _stream_ptr(stream)))


REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED = range(4)


class Server:
    """Request loop with continuous batching (frep_server): scenes are
    registered once; each request (scene, camera, tape time, host image) joins
    the next step the scheduler forms; trees stay resident in a device arena
    of `hbm_budget_bytes` and are evicted least recently used."""

    def __init__(self, ctx: Context, hbm_budget_bytes: int = 0, max_batch: int = 0, max_inflight: int = 0,
                 lights: Lights | None = None, warps=(0, 0)):
        self.ctx = ctx
        cfg = L.ServerConfig(hbm_budget_bytes, max_batch, max_inflight, warps[0], warps[1])
        lt = (lights or Lights()).struct()
        self._h = C.c_void_p()
        L.check(L.lib().frep_server_create(ctx._h, C.byref(cfg), C.byref(lt), C.byref(self._h)))
        self._keep = {}  # request id -> host buffer (kept alive until done)

    def close(self):
        if self._h is not None and self._h.value and L._lib is not None:
            L.lib().frep_server_destroy(self._h)
        self._h = C.c_void_p()
        self._keep.clear()

    def __del__(self):
        if L is not None and C is not None:
            self.close()

    def add_scene(self, tape: Tape, grid_dims, low_vertex, world_size, node_words: int = 0, tape_words: int = 0,
                  point_cells_per_lane: int = 0, rounding: int = ROUND_OUTWARD) -> int:
        vs = VoxelStorage(grid_dims, low_vertex, world_size)
        g = vs.grid_struct()
        opts = L.VoxelizeOpts(rounding, 1, node_words, tape_words, point_cells_per_lane, 0)
        sid = C.c_uint64()
        L.check(L.lib().frep_server_add_scene(self._h, tape.handle, C.byref(g), C.byref(opts), C.byref(sid)))
        return sid.value

    def submit(self, scene: int, camera: Camera, tape_time: float, width: int, height: int, out) -> int:
        """out: a host uint8 tensor/array of height*width*4 bytes (pinned for
        an asynchronous copy); written when the request completes."""
        ptr = out.data_ptr() if hasattr(out, "data_ptr") else out.ctypes.data
        req = L.RequestStruct(scene, camera.struct(width, height), float(tape_time), ptr)
        rid = C.c_uint64()
        L.check(L.lib().frep_server_submit(self._h, C.byref(req), C.byref(rid)))
        self._keep[rid.value] = out
        return rid.value

    def poll(self, rid: int) -> L.RequestStatus:
        st = L.RequestStatus()
        L.check(L.lib().frep_server_poll(self._h, rid, C.byref(st)))
        if st.state in (REQ_DONE, REQ_FAILED):
            self._keep.pop(rid, None)
        return st

    def wait(self, rid: int, timeout_ms: int = 60000) -> L.RequestStatus:
        st = L.RequestStatus()
        L.check(L.lib().frep_server_wait(self._h, rid, timeout_ms, C.byref(st)))
        self._keep.pop(rid, None)
        return st

    def release(self, rid: int) -> None:
        """Forgets a finished request."""
        L.check(L.lib().frep_server_release(self._h, rid))
        self._keep.pop(rid, None)

    def drain(self, timeout_ms: int = 600000) -> None:
        L.check(L.lib().frep_server_drain(self._h, timeout_ms))
        self._keep.clear()

    def stats(self, reset: bool = False) -> dict:
        s = L.ServerStats()
        L.check(L.lib().frep_server_get_stats(self._h, 1 if reset else 0, C.byref(s)))
        return {k: getattr(s, k) for k, _ in L.ServerStats._fields_}
