"""Pool sizing and the batch autotuner: a thin wrapper of the C-ABI's
frep_fit_pools and frep_batch_autotune (csrc/autotune.cpp, host C++).

The reference fixes one scene's branching by hand (``gridDims`` in
vulkan/src/main.cpp:16) and sizes its buffers for the worst case
(voxel_storage.h:45-47, 512 MiB of tapes). A batch of hundreds of scenes needs
both chosen per scene:

* ``fit_pools`` voxelizes each scene once into a scratch tree and returns the
  node and tape words it used, so that resident trees hold what they need and
  no more;
* ``Autotuner`` picks, per (effective resolution, tape-size class), the grid
  branching and the cells per lane of the last-level pass by timing batched
  voxelize + render of a few scenes of that class on the device (the median of
  several runs; a candidate must beat the incumbent by a margin), and picks the
  tapes (warps) per block of the level passes for the whole batch. Choices are
  kept in a JSON file keyed by device name, so a later run reuses them.
"""
from __future__ import annotations

import ctypes as C
import json
import math
import os
from dataclasses import dataclass, field

from . import Context, Lights
from . import _lib as L

# Candidate branchings per effective resolution (csrc/autotune.cpp holds the
# table the tuner times; this copy documents it for Python callers).
BRANCHINGS = {
    64: [(16, 4), (8, 8), (4, 16), (4, 4, 4)],
    128: [(16, 8), (8, 16), (32, 4), (8, 4, 4)],
    256: [(16, 16), (16, 4, 4), (8, 8, 4), (32, 8)],
    512: [(16, 8, 4), (8, 8, 8), (16, 32), (32, 16)],
    1024: [(16, 16, 4), (16, 8, 8), (8, 8, 16), (32, 8, 4)],
}

SIZE_CLASSES = (256, 1024, 4096)  # tape-length class bounds (instructions)

# The tuning the benchmark uses by default: frep_batch_autotune's choices on a
# B200 for the 512-scene batch workload (regenerate with bench.py --retune).
DEFAULT_TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning_b200.json")


def size_class(n_instr: int) -> int:
    for i, b in enumerate(SIZE_CLASSES):
        if n_instr < b:
            return i
    return len(SIZE_CLASSES)


def _fine(dims) -> int:
    return math.prod(int(d) for d in dims)


@dataclass
class Pool:
    node_words: int
    tape_words: int

    @property
    def bytes(self) -> int:
        return 4 * self.node_words + 8 * self.tape_words


def fit_pools(ctx: Context, tapes, grids, low_vertex, world_size, tape_times=None, margin: float = 0.02,
              start_bytes: int = 1 << 30) -> list[Pool]:
    """Node and tape words each (tape, grid) needs (frep_fit_pools): one
    voxelization into a scratch tree per distinct grid (grown by doubling on
    overflow), plus `margin` and 4096 words of slack. Voxelization is
    deterministic up to the order of child ids, so a tree sized this way
    never overflows on the same tape and time."""
    n = len(tapes)
    if n == 0:
        return []
    handles = (C.c_void_p * n)(*[t.handle.value for t in tapes])
    gr = (L.Grid * n)()
    for i, dims in enumerate(grids):
        gr[i].levels = len(dims)
        for j, d in enumerate(dims):
            gr[i].dims[j] = int(d)
        gr[i].low_vertex[:] = [float(v) for v in low_vertex]
        gr[i].world_size = float(world_size)
    times = None if tape_times is None else (C.c_float * n)(*[float(t) for t in tape_times])
    nw = (C.c_uint64 * n)()
    tw = (C.c_uint64 * n)()
    L.check(L.lib().frep_fit_pools(ctx._h, handles, gr, times, n, float(margin), nw, tw))
    return [Pool(int(a), int(b)) for a, b in zip(nw, tw)]


@dataclass
class Choice:
    dims: tuple
    point_cells_per_lane: int = 0
    ms_per_scene: float = float("nan")


def load_table(path, device: str | None = None) -> dict:
    """The tuned choices of a cache file ("res:class" -> Choice) without
    touching a device: the entry of `device`, else of "NVIDIA B200", else the
    file's first entry. {} when the file is absent or unreadable."""
    if not path or not os.path.exists(path):
        return {}
    try:
        data = json.loads(open(path).read())
        entry = data.get(device) or data.get("NVIDIA B200") or next(iter(data.values()), {})
        return {k: Choice(tuple(v["dims"]), v["point_cells_per_lane"], v["ms_per_scene"])
                for k, v in entry.get("choices", {}).items()}
    except (ValueError, KeyError, TypeError, StopIteration, AttributeError):
        return {}


class Autotuner:
    """Measured choice of branching and last-level tile per scene class
    (frep_batch_autotune), with the tapes per block for the batch."""

    def __init__(self, ctx: Context, cache_path: str | None = None, per_class: int = 4, reps: int = 5,
                 margin: float = 0.03, save_path: str | None = "same"):
        """cache_path: tuning file to start from; save_path: where tune()
        writes the result ("same": cache_path; None: nowhere)."""
        self.ctx = ctx
        self.cache_path = cache_path
        self.save_path = save_path
        self.per_class = per_class
        self.reps = reps
        self.margin = margin
        self.log: list = []
        self._h = C.c_void_p()
        L.check(L.lib().frep_tuning_create(C.byref(self._h)))
        self.device = self._device_name()
        if cache_path and os.path.exists(cache_path):
            L.check(L.lib().frep_tuning_load(self._h, cache_path.encode(), self.device.encode()))

    def __del__(self):
        if L is not None and L._lib is not None and getattr(self, "_h", None) and self._h.value:
            L.lib().frep_tuning_destroy(self._h)
            self._h = C.c_void_p()

    @staticmethod
    def _device_name() -> str:
        try:
            import torch
            return torch.cuda.get_device_name()
        except Exception:
            return "unknown"

    def save(self, path: str | None = None) -> None:
        path = path or (self.cache_path if self.save_path == "same" else self.save_path)
        if path:
            os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
            L.check(L.lib().frep_tuning_save(self._h, path.encode(), self.device.encode()))

    @staticmethod
    def key(res: int, n_instr: int) -> str:
        return f"{int(res)}:{size_class(n_instr)}"

    @property
    def warps(self) -> tuple:
        a, b = C.c_uint32(), C.c_uint32()
        L.check(L.lib().frep_tuning_warps(self._h, C.byref(a), C.byref(b)))
        return int(a.value), int(b.value)

    def choice_for(self, res: int, n_instr: int) -> Choice | None:
        levels, k = C.c_uint32(), C.c_uint32()
        dims = (C.c_uint32 * L.MAX_LEVELS)()
        L.check(L.lib().frep_tuning_lookup(self._h, int(res), int(n_instr), C.byref(levels), dims, C.byref(k)))
        if levels.value == 0:
            return None
        return Choice(tuple(int(d) for d in dims[: levels.value]), int(k.value))

    def tune(self, scenes, force: bool = False, refine: bool = False) -> None:
        """Tunes every (resolution, size class) present in `scenes` that the
        cache lacks (all of them with force; cached ones re-timed against
        their cached choice with refine), then saves the cache."""
        import time
        t0 = time.perf_counter()
        n = len(scenes)
        tapes = (C.c_void_p * n)(*[s.shape.handle.value for s in scenes])
        res = (C.c_uint32 * n)(*[int(s.meta["res"]) for s in scenes])
        cams = (L.CameraStruct * n)(*[s.camera.struct(s.width, s.height) for s in scenes])
        lights = Lights(shadow_mask=scenes[0].shadow_mask).struct()
        low = (C.c_float * 3)(*[float(v) for v in scenes[0].low_vertex])
        opts = L.AutotuneOpts(self.per_class, self.reps, scenes[0].width, scenes[0].height, float(self.margin),
                              1 if force else 0, 1 if refine else 0)
        L.check(L.lib().frep_batch_autotune(self.ctx._h, tapes, res, cams, n, C.byref(lights), low,
                                            float(scenes[0].world_size), C.byref(opts), self._h))
        self.log.append({"tune_seconds": time.perf_counter() - t0})
        self.save()

    def apply(self, scene) -> tuple:
        """(grid dims, point cells per lane) for a scene: the tuned choice of
        its class, else its own grid dims with the automatic tile."""
        c = self.choice_for(scene.meta["res"], scene.shape.n_instr)
        if c is None:
            return tuple(scene.grid_dims), 0
        return tuple(c.dims), c.point_cells_per_lane
