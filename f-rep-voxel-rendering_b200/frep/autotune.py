"""Pool sizing and the batch autotuner.

The reference fixes one scene's branching by hand (``gridDims`` in
vulkan/src/main.cpp:16) and sizes its buffers for the worst case
(voxel_storage.h:45-47, 512 MiB of tapes). A batch of hundreds of scenes needs
both chosen per scene:

* ``fit_pools`` voxelizes each scene once into a scratch tree and returns the
  node and tape words it used, so that resident trees hold what they need and
  no more;
* ``Autotuner`` picks, per (effective resolution, tape-size class), the grid
  branching and the cells per lane of the last-level pass by timing batched
  voxelize + render of a few scenes of that class on the device, and picks the
  tapes (warps) per block of the level passes for the whole batch. Choices are
  cached in a JSON file keyed by device name, so a later run reuses them.
"""
from __future__ import annotations

import json
import math
import os
import time
from dataclasses import dataclass, field

from . import Batch, Context, Lights, ROUND_OUTWARD, Tape, VoxelStorage, Voxelizer
from . import _lib as L

# Candidate branchings per effective resolution: every level a multiple of 4
# from 4 to 32, two to four levels.
BRANCHINGS = {
    64: [(16, 4), (8, 8), (4, 16), (4, 4, 4)],
    128: [(16, 8), (8, 16), (32, 4), (8, 4, 4)],
    256: [(16, 16), (16, 4, 4), (8, 8, 4), (32, 8)],
    512: [(16, 8, 4), (8, 8, 8), (16, 32), (32, 16)],
    1024: [(16, 16, 4), (16, 8, 8), (8, 8, 16), (32, 8, 4)],
}

SIZE_CLASSES = (256, 1024, 4096)  # tape-length class bounds (instructions)


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
    """Node and tape words each (tape, grid) needs: one voxelization into a
    scratch tree per distinct grid (grown by doubling on overflow), plus
    `margin` and 4096 words of slack. Voxelization is deterministic up to the
    order of child ids, so a tree sized this way never overflows on the same
    tape and time."""
    scratch: dict[tuple, VoxelStorage] = {}
    sizes: dict[tuple, int] = {}
    out = []
    for i, (tape, dims) in enumerate(zip(tapes, grids)):
        key = tuple(int(d) for d in dims)
        t = 0.0 if tape_times is None else float(tape_times[i])
        while True:
            vs = scratch.get(key)
            if vs is None:
                b = sizes.setdefault(key, start_bytes)
                vs = VoxelStorage(key, low_vertex, world_size, rounding=ROUND_OUTWARD,
                                  node_words=b // 4 // 4, tape_words=b * 3 // 4 // 8)
                vs.init(ctx, tape)
                scratch[key] = vs
            vs.tape = tape
            Voxelizer(ctx, vs).voxelize(t)
            info = vs.sync(raise_on_overflow=False)
            if not info.overflow:
                break
            vs.cleanup()
            del scratch[key]
            sizes[key] *= 2
        out.append(Pool(int(info.node_words_used * (1 + margin)) + 4096,
                        int(info.tape_words_used * (1 + margin)) + 4096))
    for vs in scratch.values():
        vs.cleanup()
    return out


@dataclass
class Choice:
    dims: tuple
    point_cells_per_lane: int = 0
    ms_per_scene: float = float("nan")


@dataclass
class Autotuner:
    """Measured choice of branching and last-level tile per scene class."""

    ctx: Context
    cache_path: str | None = None
    per_class: int = 4        # scenes timed per class
    reps: int = 3             # timed batched runs per candidate
    choices: dict = field(default_factory=dict)   # "res:class" -> Choice
    warps: tuple = (0, 0)     # interval / point warps per block for the batch
    log: list = field(default_factory=list)

    def __post_init__(self):
        self.device = self._device_name()
        if self.cache_path and os.path.exists(self.cache_path):
            try:
                data = json.loads(open(self.cache_path).read()).get(self.device, {})
                for k, v in data.get("choices", {}).items():
                    self.choices[k] = Choice(tuple(v["dims"]), v["point_cells_per_lane"], v["ms_per_scene"])
                self.warps = tuple(data.get("warps", (0, 0)))
            except (ValueError, KeyError, TypeError):
                self.choices = {}

    @staticmethod
    def _device_name() -> str:
        try:
            import torch
            return torch.cuda.get_device_name()
        except Exception:
            return "unknown"

    def save(self) -> None:
        if not self.cache_path:
            return
        data = {}
        if os.path.exists(self.cache_path):
            try:
                data = json.loads(open(self.cache_path).read())
            except ValueError:
                data = {}
        data[self.device] = {
            "choices": {k: {"dims": list(c.dims), "point_cells_per_lane": c.point_cells_per_lane,
                            "ms_per_scene": c.ms_per_scene} for k, c in self.choices.items()},
            "warps": list(self.warps),
        }
        os.makedirs(os.path.dirname(os.path.abspath(self.cache_path)), exist_ok=True)
        with open(self.cache_path, "w") as f:
            json.dump(data, f, indent=1)

    @staticmethod
    def key(res: int, n_instr: int) -> str:
        return f"{int(res)}:{size_class(n_instr)}"

    def choice_for(self, res: int, n_instr: int) -> Choice | None:
        return self.choices.get(self.key(res, n_instr))

    # ---- measurement ----------------------------------------------------------------

    def _time_batch(self, scenes, dims_of, k_of, warps=(0, 0)) -> float:
        """Device ms per scene of batched voxelize + render (graph replay)."""
        import torch
        tapes = [s.shape for s in scenes]
        grids = [dims_of(s) for s in scenes]
        pools = fit_pools(self.ctx, tapes, grids, scenes[0].low_vertex, scenes[0].world_size)
        storages = []
        for s, g, p in zip(scenes, grids, pools):
            vs = VoxelStorage(g, s.low_vertex, s.world_size, rounding=ROUND_OUTWARD, node_words=p.node_words,
                              tape_words=p.tape_words, point_cells_per_lane=k_of(s, g))
            storages.append(vs.init(self.ctx, s.shape))
        batch = Batch(self.ctx, storages)
        batch.set_tuning(*warps)
        dev = torch.device("cuda", self.ctx.device)
        rgba = [torch.empty((s.height, s.width, 4), dtype=torch.uint8, device=dev) for s in scenes]
        cams = [s.camera for s in scenes]
        sizes = [(s.width, s.height) for s in scenes]
        lights = Lights(shadow_mask=scenes[0].shadow_mask)
        stream = torch.cuda.current_stream()
        batch.run(cams, sizes, rgba, lights=lights, graph=True, stream=stream)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record(stream)
        for _ in range(self.reps):
            batch.run(cams, sizes, rgba, lights=lights, graph=True, stream=stream)
        ev[1].record(stream)
        torch.cuda.synchronize()
        ms = ev[0].elapsed_time(ev[1]) / self.reps / len(scenes)
        batch.close()
        for vs in storages:
            vs.cleanup()
        return ms

    def tune(self, scenes, force: bool = False) -> None:
        """Fills `choices` for every (resolution, size class) present in
        `scenes` (those already cached are kept unless `force`), then the
        batch's warps per block on a mixed sample."""
        t0 = time.perf_counter()
        classes: dict[str, list] = {}
        for s in scenes:
            classes.setdefault(self.key(s.meta["res"], s.shape.n_instr), []).append(s)
        for key, members in sorted(classes.items()):
            if key in self.choices and not force:
                continue
            res = int(key.split(":")[0])
            sample = members[:: max(1, len(members) // self.per_class)][: self.per_class]
            best = None
            for dims in BRANCHINGS[res]:
                ks = [0] if dims[-1] < 8 else [4, 2]
                for k in ks:
                    ms = self._time_batch(sample, lambda s, d=dims: d, lambda s, g, k=k: k)
                    self.log.append({"class": key, "dims": list(dims), "point_cells_per_lane": k, "ms": ms})
                    if best is None or ms < best.ms_per_scene:
                        best = Choice(tuple(dims), k, ms)
            self.choices[key] = best
        # batch-wide tapes per block, on up to 32 scenes spread over the classes
        if force or self.warps == (0, 0):
            mixed = scenes[:: max(1, len(scenes) // 32)][:32]
            dims_of = lambda s: self.apply(s)[0]
            k_of = lambda s, g: self.apply(s)[1]
            best_w, best_ms = (0, 0), None
            for w in [(0, 0), (1, 1), (4, 4), (1, 4), (4, 1)]:
                ms = self._time_batch(mixed, dims_of, k_of, w)
                self.log.append({"warps": list(w), "ms": ms})
                if best_ms is None or ms < best_ms:
                    best_w, best_ms = w, ms
            self.warps = best_w
        self.log.append({"tune_seconds": time.perf_counter() - t0})
        self.save()

    def apply(self, scene) -> tuple:
        """(grid dims, point cells per lane) for a scene: the tuned choice of
        its class, else its own grid dims with the automatic tile."""
        c = self.choice_for(scene.meta["res"], scene.shape.n_instr)
        if c is None:
            return tuple(scene.grid_dims), 0
        return tuple(c.dims), c.point_cells_per_lane
