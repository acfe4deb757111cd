"""Benchmark: scenes/s of voxelize + render, batched vs plain, on one B200.

Default workload (`--workload batch`): 512 independent scenes, each a random
CSG of sphere / box / capsule primitives (sizes U[0.02, 0.2]) combined by a
random binary tree of min / max / max(a,-b) / polynomial smooth-min, with
primitive counts log-uniform in [4, 1024] and effective resolutions drawn from
{64, 128, 256, 512, 1024}^3; every scene rendered at 512x512 from its own
orbit camera (60 degrees) with one shadow ray per hit. Branching, last-level
tile and tapes per block are chosen by the autotuner before timing. One step =
the whole batch voxelized and rendered (one frep_batch_run, CUDA graph
replay). The same trees are also run as 512 sequential plain launches
(frep_voxelize + frep_render per scene) for the batched/plain ratio.

`--workload small`: the min-union of 16 spheres on a {16, 4} = 64^3 tree over
[-1.5, 1.5]^3, 256x256 orthographic, one ray per pixel; one step = one
voxelization + one frame.

`--workload large`: one scene of 256 primitives on a {16, 16, 8} = 2048^3
tree, 1920x1080 perspective + shadow rays; one step = one voxelization + one
frame.

Seeded synthetic scenes (the reference ships no dataset).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank renders its own scene replica (the path has no
cross-scene exchange: replicas only, weak scaling); rank 0 prints one JSON line.
`--impl reference` times the reference path's CPU implementation (the oracle's
C++ restatement of its shaders; the reference's GLSL cannot run without a
graphics stack) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "f-rep-voxel-rendering_b200"))

METRIC = "scenes/s (voxelize+render)"
SM_COUNT = 148
FP32_LANES_PER_SM = 128


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", choices=("batch", "small", "large", "stress", "animated"), default="batch")
    ap.add_argument("--frames", type=int, default=30, help="stress: animation frames (T = frame / frames)")
    ap.add_argument("--no-reuse", action="store_true",
                    help="animated: re-voxelize every frame in full (no reuse of the previous frame's tree)")
    ap.add_argument("--scenes", type=int, default=512, help="batch: number of scenes")
    ap.add_argument("--plain-steps", type=int, default=2, help="batch: timed passes of the plain launch loop")
    ap.add_argument("--no-tune", action="store_true", help="batch: default branching, no autotuning")
    ap.add_argument("--tune-cache", default=None,
                    help="batch: tuning file to start from and to write (default: read the committed "
                         "f-rep-voxel-rendering_b200/frep/tuning_b200.json, write nothing)")
    ap.add_argument("--retune", action="store_true",
                    help="batch: re-time every class against its tuned choice (the incumbent is kept "
                         "unless beaten by the tuner's margin)")
    ap.add_argument("--serve-inflight", type=int, default=0,
                    help="batch: steps the server keeps on the device (0 = library default)")
    ap.add_argument("--budget-gb", type=int, default=150, help="HBM budget of the context, GB")
    ap.add_argument("--serve-seconds", type=float, default=60.0,
                    help="batch: seconds of the serving run after the batch measurements (0 = none)")
    ap.add_argument("--serve-rate", type=float, default=1000.0, help="batch: Poisson request rate, requests/s")
    ap.add_argument("--serve-sweep", default="200,2000",
                    help="batch: extra request rates (comma separated, requests/s), each served for "
                         "--serve-seconds after the main serving phase; results under serving_sweep")
    ap.add_argument("--serve-budget-gb", type=int, default=120, help="batch: tree arena of the server, GB")
    ap.add_argument("--grid", default=None,
                    help="large / stress: tree branching per level (default 16,16,8 / 16,16,4,4)")
    ap.add_argument("--res", default=None, help="render resolution WxH (batch 512x512, large 1920x1080)")
    ap.add_argument("--pool-mb", type=int, default=3072, help="large: node + tape pool size of the tree, MB")
    ap.add_argument("--point-k", type=int, default=0, choices=(0, 2, 4, 8),
                    help="large / stress / animated: cells per lane of the last-level pass (0 = library default)")
    ap.add_argument("--no-compact", action="store_true",
                    help="large: skip the compact-tree measurements (compaction time, bytes, render time)")
    args = ap.parse_args()
    if args.grid is None:
        args.grid = {"stress": "16,16,4,4", "small": "16,4"}.get(args.workload, "16,16,8")
    args.grid_dims = tuple(int(v) for v in args.grid.split(","))
    if args.res is None:
        args.res = {"batch": "512x512", "small": "256x256"}.get(args.workload, "1920x1080")
    args.width, args.height = (int(v) for v in args.res.lower().split("x"))
    fine = 1
    for d in args.grid_dims:
        fine *= d
    if args.workload == "batch":
        args.workload_name = (f"batch_{args.scenes}scenes_4-1024prim_64-1024cube_{args.width}x{args.height}_shadow")
    elif args.workload == "stress":
        args.workload_name = (f"stress_twisted_gyroid_64spheres_{fine}cube_{args.width}x{args.height}_shadow_"
                              f"{args.frames}frames")
    elif args.workload == "small":
        args.workload_name = f"spheres16_union_{fine}cube_{args.width}x{args.height}_ortho"
    elif args.workload == "animated":
        args.workload_name = (f"animated_csg_256prim_4orbiting_{fine}cube_{args.width}x{args.height}_shadow_"
                              f"60fps_{'full' if args.no_reuse else 'reuse'}")
    else:
        args.workload_name = f"random_csg_256prim_{fine}cube_{args.width}x{args.height}_shadow"
    return args


def dist_setup(args):
    """One process per GPU (torchrun sets RANK / LOCAL_RANK / WORLD_SIZE):
    NCCL on GPUs; gloo on a host without CUDA (the reference arm's ranks and
    the CPU tests of this plumbing)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, value: float) -> float:
    """The largest of the ranks' values (timings are reported as the slowest
    rank's)."""
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text())
    return {"hbm_gbs": 6650.0, "sm_max_mhz": 1965.0, "fallback": True}


def make_scene(args, grid_dims=None):
    from frep import scenes
    dims = grid_dims or args.grid_dims
    if args.workload == "stress":
        return scenes.stress_gyroid(grid_dims=dims, width=args.width, height=args.height)
    if args.workload == "animated":
        return scenes.animated_csg(256, 4, seed=2, grid_dims=dims, width=args.width, height=args.height)
    if args.workload == "small":
        # min-union of 16 spheres over [-1.5, 1.5]^3, orthographic view down +z
        sc = scenes.spheres_union(16, width=args.width, height=args.height)
        sc.grid_dims = list(dims)
        return sc
    return scenes.random_csg(256, seed=2, grid_dims=dims, width=args.width, height=args.height, shadows=True)


def frame_times(args):
    """Tape time of each step: the stress animation sweeps T over [0, 1); the
    animated scene advances T by 1/60 per frame (4 s per revolution of its
    spheres; the list is long enough never to wrap within a run)."""
    if args.workload == "stress":
        return [f / args.frames for f in range(args.frames)]
    if args.workload == "animated":
        return [0.3 + f / 60.0 for f in range(100000)]
    return [0.0]


def cpu_baseline(scene, threads: int, tape_time: float = 0.0):
    """The oracle (C++ restatement of the reference's shaders) on the host:
    one full voxelization + one full render, all host threads."""
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle
    import frep
    tape = scene.shape if isinstance(scene.shape, frep.Tape) else frep.Tape(scene.shape)
    t0 = time.perf_counter()
    tree = oracle.OracleTree(tape.wide(), tape.n_slots, scene.grid_dims, scene.low_vertex, scene.world_size,
                             tape_time=tape_time, rounding=1, threads=threads)
    t1 = time.perf_counter()
    lights = frep.Lights(shadow_mask=scene.shadow_mask)
    tree.render(oracle.camera_vector(scene.camera, scene.width, scene.height), lights, tape_time=tape_time,
                threads=threads)
    t2 = time.perf_counter()
    return t2 - t0, t1 - t0, t2 - t1


def run_reference(args, world, rank):
    """--impl reference: the CPU path on the host cores, same metric/config."""
    if rank != 0:
        return
    # the stress scene at 4096^3 would take hours on the host: its sample is the
    # same scene and frames on the first three levels of the grid (1024^3)
    sample_dims = args.grid_dims[:3] if args.workload == "stress" else args.grid_dims
    scene = make_scene(args, sample_dims)
    threads = os.cpu_count() or 1
    tt = frame_times(args)
    if args.warmup > 0:
        cpu_baseline(scene, threads, tt[0])  # one warm-up scene (the oracle has no caches to warm)
    times = [cpu_baseline(scene, threads, tt[i % len(tt)])[0] for i in range(args.steps)]
    total = sum(times)
    value = args.steps / total
    line = {
        "metric": METRIC, "value": value, "unit": "scenes/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": args.workload_name, "grid": list(args.grid_dims), "resolution": [args.width, args.height],
                   "shadow_rays": 1 if scene.shadow_mask else 0, "rounding": "outward"},
        "cpu_baseline": {"value": value, "unit": "scenes/s", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} scenes on grid {list(sample_dims)} (voxelize + "
                                   f"{args.width}x{args.height} render), oracle C++ port, {threads} threads"},
        "e2e": {"value": value, "unit": "scenes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, world, rank, local):
    import torch
    import frep

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    scene = make_scene(args)
    tt = frame_times(args)
    if args.workload == "stress":
        from frep.autotune import fit_pools
        ctx = frep.Context(local, hbm_budget_bytes=args.budget_gb << 30)
        tape = frep.Tape(scene.shape)
        fits = fit_pools(ctx, [tape] * 4, [scene.grid_dims] * 4, scene.low_vertex, scene.world_size,
                         tape_times=[tt[i * len(tt) // 4] for i in range(4)], start_bytes=8 << 30)
        node_words = int(max(p.node_words for p in fits) * 1.15)
        tape_words = int(max(p.tape_words for p in fits) * 1.15)
        scene.shape = tape
    else:
        ctx = frep.Context(local, hbm_budget_bytes=48 << 30)
        pool = args.pool_mb << 20
        node_words, tape_words = pool // 4 // 4, pool * 3 // 4 // 8
    vs = frep.VoxelStorage(scene.grid_dims, scene.low_vertex, scene.world_size, rounding=frep.ROUND_OUTWARD,
                           node_words=node_words, tape_words=tape_words, point_cells_per_lane=args.point_k)
    vs.init(ctx, scene.shape)
    vox = frep.Voxelizer(ctx, vs)
    # the animated scene alternates two trees, each frame reusing the other
    anim = args.workload == "animated"
    reuse = anim and not args.no_reuse
    storages = [vs]
    if anim:
        storages.append(frep.VoxelStorage(scene.grid_dims, scene.low_vertex, scene.world_size,
                                          rounding=frep.ROUND_OUTWARD, node_words=node_words,
                                          tape_words=tape_words, point_cells_per_lane=args.point_k).init(ctx, vs.tape))
    rt = frep.Raytracer(ctx, vs)
    rt.lights = frep.Lights(shadow_mask=scene.shadow_mask)
    W, H = scene.width, scene.height
    rgba = torch.empty((H, W, 4), dtype=torch.uint8, device=dev)
    host_img = torch.empty((H, W, 4), dtype=torch.uint8, pin_memory=True)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2
    stream = torch.cuda.current_stream()

    frame = [0]

    def voxelize_frame():
        """Voxelizes the next frame; returns its tape time and storage."""
        f = frame[0]
        frame[0] += 1
        t = tt[f % len(tt)]
        cur = storages[f % len(storages)]
        prev = storages[(f - 1) % 2] if reuse and f > 0 else None
        frep.Voxelizer(ctx, cur).voxelize(t, stream, reuse=prev)
        rt.voxels = cur
        return t, cur

    def step():
        t, _ = voxelize_frame()
        rt.trace(scene.camera, t, W, H, out=(rgba, None), stream=stream)

    for _ in range(args.warmup):
        step()
    for st in storages:
        info = st.sync()
    if not anim:  # (the animation runs on instead: every timed frame follows another frame)
        frame[0] = 0
    L = vs.grid_levels
    launches_per_step = 1 + 2 * L + 1  # init + (work scan + level pass) per level + render
    if reuse:
        launches_per_step += 1 + (L - 1) + L  # match passes (root, each child level) + copy passes

    # ---- device-resident timing (value) -------------------------------------
    torch.cuda.synchronize()
    barrier(world)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local) as clocks:
        for s, e in evs:
            flush.fill_(1)
            s.record(stream)
            step()
            e.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    t_ms = sum(s.elapsed_time(e) for s, e in evs)
    t_ms = max_over_ranks(world, t_ms)
    value = world * args.steps / (t_ms / 1e3)

    # ---- per-kernel timing of the dominant kernel (level passes) -----------
    for st in storages:
        st.set_profiling(True)
    level_ms = [0.0] * vs.grid_levels
    render_ms = 0.0
    reps = max(3, min(args.steps, 10))
    for _ in range(reps):
        flush.fill_(1)
        if not anim:
            frame[0] = 0  # (the profiled voxelization is at tape time tt[0])
        t, cur = voxelize_frame()
        rs, re_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        rs.record(stream)
        rt.trace(scene.camera, t, W, H, out=(rgba, None), stream=stream)
        re_.record(stream)
        lt = cur.level_timings()
        torch.cuda.synchronize()
        level_ms = [a + b / reps for a, b in zip(level_ms, lt)]
        render_ms += rs.elapsed_time(re_) / reps
    for st in storages:
        st.set_profiling(False)
    fp32_ops = cur.fp32_ops()   # of the last profiled voxelization (evaluated nodes only)
    cell_instr = cur.work()
    if not anim:
        frame[0] = 0

    # ---- end to end through the public API with host buffers ---------------
    torch.cuda.synchronize()
    barrier(world)
    e2e_evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for i, (s, e) in enumerate(e2e_evs):
        flush.fill_(1)
        s.record(stream)
        t, _ = voxelize_frame()   # host tape -> device (pinned staging + H2D)
        rt.trace(scene.camera, t, W, H, out=(rgba, None), stream=stream)
        host_img.copy_(rgba, non_blocking=True)  # result -> host
        e.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    e2e_ms = max_over_ranks(world, sum(s.elapsed_time(e) for s, e in e2e_evs))
    e2e_value = world * args.steps / (e2e_ms / 1e3)
    h2d = 8 * info.root_tape_words
    d2h = W * H * 4

    # ---- compact trees (large scene): compaction time, bytes, render time ---
    compact_stats = None
    if args.workload == "large" and not args.no_compact:
        compact_stats = measure_compact(args, ctx, vs, scene, rt.lights, tt[0], rgba, flush, stream, render_ms)

    # ---- roofline of the dominant kernel -------------------------------------
    peaks = measured_peaks()
    dom = max(range(vs.grid_levels), key=lambda l: level_ms[l])
    sm_mhz = float(peaks.get("sm_max_mhz", 1965.0))
    fp32_peak_tops = SM_COUNT * FP32_LANES_PER_SM * sm_mhz * 1e6 / 1e12
    achieved = fp32_ops[dom] / (level_ms[dom] / 1e3) / 1e12
    roofline = {
        "bound": "fp32", "kernel": "point_level_kernel" if dom == vs.grid_levels - 1 else "interval_level_kernel",
        "level": dom, "achieved": achieved, "peak": fp32_peak_tops, "unit": "TFLOP/s",
        "frac": achieved / fp32_peak_tops, "traffic": None,
        "peak_source": "nominal FP32 issue: 148 SMs x 128 lanes x MEASURED_PEAKS.json sm_max_mhz "
                       "(the file holds no FP32 figure)",
        "algorithmic_ops_per_launch": fp32_ops[dom], "cell_instr_per_launch": cell_instr[dom],
        "ms_per_launch": level_ms[dom],
    }

    line = {
        "metric": METRIC, "value": value, "unit": "scenes/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload_name, "grid": scene.grid_dims, "resolution": [W, H],
                   "shadow_rays": 1 if scene.shadow_mask else 0,
                   "tape_instructions": vs.tape.n_instr, "rounding": "outward", "point_cells_per_lane": args.point_k or "default",
                   "nodes_per_level": list(info.node_count[:vs.grid_levels]),
                   "l2": "flushed between timed steps (256 MB write, outside the step events)",
                   "parallelism": f"replicas x{world}"},
        "roofline": roofline,
        "level_ms": level_ms, "render_ms": render_ms,
        **({"reuse": {"previous_frame_tree": reuse,
                      "cell_instr_per_level": cell_instr}} if anim else {}),
        **({"compact": compact_stats} if compact_stats else {}),
        "e2e": {"value": e2e_value, "unit": "scenes/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "clocks": clocks.summary(),
        "gpu_launches": launches_per_step * args.steps,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        sample_dims = args.grid_dims[:3] if args.workload == "stress" else args.grid_dims
        total, t_vox, t_ren = cpu_baseline(make_scene(args, sample_dims), threads, tt[0])
        line["cpu_baseline"] = {"value": 1.0 / total, "unit": "scenes/s", "cores": threads, "kind": "port",
                                "sample": f"1 scene on grid {list(sample_dims)} (voxelize {t_vox:.2f} s + "
                                          f"{W}x{H} render {t_ren:.2f} s), oracle C++ port, {threads} threads"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    for st in storages:
        st.cleanup()
    ctx.close()

def measure_compact(args, ctx, vs, scene, lights, t, rgba, flush, stream, render_ms_full):
    """Compacts the last voxelized tree both ways (frep_tree_compact) and
    renders each: device time of the compaction (CUDA events around the
    blocking call), bytes held, render time of one frame, blob size."""
    import torch
    import frep

    frep.Voxelizer(ctx, vs).voxelize(t, stream)
    info = vs.sync()
    out = {"source_bytes": info.node_words_used * 4 + info.tape_words_used * 8,
           "source_node_bytes": info.node_words_used * 4, "source_tape_bytes": info.tape_words_used * 8,
           "render_ms_source": render_ms_full}
    W, H = scene.width, scene.height
    for name, prune in (("layout", False), ("prune", True)):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ms = []
        for _ in range(3):
            flush.fill_(1)
            a.record(stream)
            ct = frep.CompactTree.from_storage(ctx, vs, prune=prune, stream=stream)
            b.record(stream)
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
            if len(ms) < 3:
                ct.close()
        ct.lights = lights
        rms = []
        for _ in range(max(3, min(args.steps, 10))):
            flush.fill_(1)
            a.record(stream)
            ct.trace(scene.camera, t, W, H, out=(rgba, None), stream=stream)
            b.record(stream)
            torch.cuda.synchronize()
            rms.append(a.elapsed_time(b))
        ci = ct.info()
        size = len(ct.export())
        out[name] = {"compact_ms": sorted(ms)[1], "device_bytes": ci.device_bytes,
                     "node_bytes": ci.node_words * 4, "tape_bytes": ci.tape_words * 8,
                     "nodes_per_level": list(ci.node_count[:ci.levels]), "blob_bytes": size,
                     "render_ms": sum(rms) / len(rms)}
        ct.close()
    return out


# ---- many-scene batch ----------------------------------------------------------------

def make_batch_scenes(args, world: int = 1, indices=None):
    """The batch workload with one orbit camera per scene (seeded); with
    `indices`, only those scenes (same shapes and cameras as in the full set)."""
    import numpy as np
    from frep import scenes
    rng = np.random.default_rng(11)
    cams = [scenes.orbit_camera(rng) for _ in range(args.scenes)]
    if indices is not None:
        jobs = scenes.batch_jobs(args.scenes, seed=3, width=args.width, height=args.height)
        scs = [scenes.batch_scene(jobs[i]) for i in indices]
        for sc, i in zip(scs, indices):
            sc.camera = cams[i]
        return scs
    procs = max(1, min(32, (os.cpu_count() or 1) // max(1, world)))
    scs = scenes.batch_workload(args.scenes, seed=3, width=args.width, height=args.height, processes=procs)
    for sc, cam in zip(scs, cams):
        sc.camera = cam
    return scs


def oracle_scene_seconds(scene, dims, threads: int) -> float:
    """Oracle (C++ restatement of the reference's shaders): one voxelization +
    one frame of `scene` on `threads` host threads, in seconds."""
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle
    import frep
    tape = scene.shape
    t0 = time.perf_counter()
    tree = oracle.OracleTree(tape.wide(), tape.n_slots, list(dims), scene.low_vertex, scene.world_size,
                             rounding=1, threads=threads)
    tree.render(oracle.camera_vector(scene.camera, scene.width, scene.height),
                frep.Lights(shadow_mask=scene.shadow_mask), threads=threads)
    return time.perf_counter() - t0


def cpu_sample_order(n: int):
    import numpy as np
    return [int(i) for i in np.random.default_rng(17).permutation(n)]


# DRAM bytes (read + write) per launch of each (level, kind) level pass of the
# default workload (512 scenes at 512x512, the committed tuning table), kinds
# 0 interval, 1 point 4 cells/lane, 2 point 2 cells/lane: one ncu capture of
# dram__bytes_read.sum + dram__bytes_write.sum (one pass per launch) of
#   python bench.py --steps 2 --warmup 3 --no-cpu-baseline --serve-seconds 0 --serve-sweep '' --plain-steps 1
# summarised in profiles/batch_512scenes_dram_per_launch.txt.
NCU_DRAM_BYTES_512 = {(0, 0): 9.666e9, (1, 0): 18.210e9, (1, 1): 1.195e9, (1, 2): 0.513e9,
                      (2, 1): 0.337e9, (2, 2): 11.455e9}


def tuning_table():
    """The committed tuning of the batch workload (frep.autotune.DEFAULT_TABLE),
    None when absent."""
    from frep.autotune import DEFAULT_TABLE
    return DEFAULT_TABLE if os.path.exists(DEFAULT_TABLE) else None


# The CPU figures of the batch workload (the reference arm and the GPU arm's
# cpu_baseline leg) time the same scenes: the first CPU_SAMPLE of a seeded
# permutation of the batch, each at the grid the GPU arm runs it with.
CPU_SAMPLE = 20


def tuned_grid(table: dict, sc):
    """(grid dims, point cells per lane) of a batch scene under a tuning table
    (frep.autotune.load_table); the default branching where it has no entry."""
    from frep import scenes as S
    from frep.autotune import Autotuner
    c = table.get(Autotuner.key(sc.meta["res"], sc.shape.n_instr))
    if c is None:
        return tuple(S.DEFAULT_BRANCHING[sc.meta["res"]]), 0
    return tuple(c.dims), c.point_cells_per_lane


def run_reference_batch(args, world, rank):
    """--impl reference on the batch workload: step i is scene i of the CPU
    sample (the GPU arm's cpu_baseline scenes, at the grids the GPU arm's
    tuning table gives them), voxelized + rendered by the oracle on all host
    threads; warm-up steps run the first scenes of the sample once more.
    value = scenes / total seconds."""
    if rank != 0:
        return
    from frep.autotune import load_table
    table = load_table(args.tune_cache or tuning_table())
    order = cpu_sample_order(args.scenes)
    idx = [order[i % CPU_SAMPLE] for i in range(max(args.steps, args.warmup))]
    built = {i: sc for i, sc in zip(sorted(set(idx)), make_batch_scenes(args, indices=sorted(set(idx))))}
    threads = os.cpu_count() or 1
    for i in range(args.warmup):
        sc = built[idx[i]]
        oracle_scene_seconds(sc, tuned_grid(table, sc)[0], threads)
    times = []
    for i in range(args.steps):
        sc = built[idx[i]]
        times.append(oracle_scene_seconds(sc, tuned_grid(table, sc)[0], threads))
    total = sum(times)
    value = args.steps / total
    sample = (f"{args.steps} scenes of the batch (the first {min(args.steps, CPU_SAMPLE)} of a seeded permutation, "
              f"the GPU arm's cpu_baseline sample), each voxelized at the grid the GPU arm's tuning table "
              f"({'given' if args.tune_cache else ('committed' if tuning_table() else 'none: default')} branchings) gives it + rendered "
              f"{args.width}x{args.height}; oracle C++ port, {threads} threads")
    line = {
        "metric": METRIC, "value": value, "unit": "scenes/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
        "config": {"workload": args.workload_name, "scenes": args.scenes, "resolution": [args.width, args.height],
                   "shadow_rays": 1, "rounding": "outward"},
        "cpu_baseline": {"value": value, "unit": "scenes/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "scenes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def serve_phase(args, ctx, scs, chosen, pools, warps):
    """Serving: a Poisson request stream at args.serve_rate for
    args.serve_seconds. Each request is a scene plus an orbit camera pose at
    the batch resolution: with probability 0.3 a repeat of one of the 64 most
    recently requested scenes (a re-render when it is still resident), else a
    new scene of the batching distribution (a batch scene's tape with its
    constants scaled by U[0.9, 1.1], at that scene's tuned branching). Trees
    stay resident in an arena of args.serve_budget_gb GB, evicted least
    recently used. Latency = submit -> image in (pinned) host memory."""
    import collections
    import numpy as np
    import torch
    import frep
    from frep import scenes as S

    W, H = args.width, args.height
    rng = np.random.default_rng(23)
    n_req = max(1, int(args.serve_rate * args.serve_seconds))
    arrivals = np.cumsum(rng.exponential(1.0 / args.serve_rate, n_req))
    srv = frep.Server(ctx, hbm_budget_bytes=args.serve_budget_gb << 30, lights=frep.Lights(shadow_mask=1),
                      warps=warps, max_inflight=args.serve_inflight)
    wides = [sc.shape.wide() for sc in scs]
    recent = collections.deque(maxlen=64)
    plan = []
    n_new = 0

    def new_scene():
        b = int(rng.integers(len(scs)))
        tape = S.jitter_tape(wides[b], rng)
        dims, k = chosen[b]
        # jittered sizes change the surface by up to ~20 %: start with more pool
        return srv.add_scene(tape, dims, scs[b].low_vertex, scs[b].world_size,
                             node_words=int(pools[b].node_words * 1.5) + 4096,
                             tape_words=int(pools[b].tape_words * 1.5) + 4096, point_cells_per_lane=k)

    for i in range(n_req):
        if recent and rng.random() < 0.3:
            sid = recent[int(rng.integers(len(recent)))]
        else:
            sid = new_scene()
            n_new += 1
        recent.append(sid)
        plan.append((sid, S.orbit_camera(rng)))
    ring = min(n_req, 4096)  # pinned host images in rotation (4 GB at 512x512)
    bufs = [torch.empty((H, W, 4), dtype=torch.uint8, pin_memory=True) for _ in range(ring)]
    # warm-up (plans, upload areas, first trees): not measured
    warm = [srv.submit(new_scene(), S.orbit_camera(rng), 0.0, W, H, bufs[i % ring]) for i in range(min(64, ring))]
    srv.drain(600000)
    before = srv.stats(reset=True)
    ids = [0] * n_req
    lag = np.zeros(n_req)  # submit - scheduled arrival
    t0 = time.perf_counter()
    for i, (sid, cam) in enumerate(plan):
        target = t0 + arrivals[i]
        while True:
            now = time.perf_counter()
            if now >= target:
                break
            time.sleep(min(target - now, 0.0005))
        if i >= ring:
            srv.wait(ids[i - ring], 600000)  # the host buffer is reused
        lag[i] = time.perf_counter() - target
        ids[i] = srv.submit(sid, cam, 0.0, W, H, bufs[i % ring])
    srv.drain(600000)
    st = srv.stats()
    # open-loop latency: from the scheduled arrival, so that a late submit counts
    server_ms = np.array([srv.poll(r).latency_ms for r in ids])
    open_ms = server_ms + 1e3 * lag
    for r in ids:
        srv.release(r)
    failed = st["failed"]
    srv.close()
    return {
        "rate_req_s": args.serve_rate, "seconds": args.serve_seconds, "requests": n_req,
        "new_scenes": n_new, "resolution": [W, H], "arena_gb": args.serve_budget_gb,
        "p50_ms": float(np.percentile(open_ms, 50)), "p99_ms": float(np.percentile(open_ms, 99)),
        "mean_ms": float(open_ms.mean()), "max_ms": float(open_ms.max()),
        "server_p50_ms": st["p50_ms"], "server_p99_ms": st["p99_ms"],
        "scenes_per_s": st["scenes_per_s"], "completed": st["completed"] - before["completed"],
        "failed": failed - before["failed"], "voxelized": st["voxelized"] - before["voxelized"],
        "rerendered": st["rerendered"] - before["rerendered"], "evictions": st["evictions"] - before["evictions"],
        "steps": st["steps"] - before["steps"], "max_submit_lag_ms": float(1e3 * lag.max()),
        "max_plan_ms": st["max_plan_ms"], "max_enqueue_ms": st["max_enqueue_ms"],
        "max_step_evictions": st["max_step_evictions"],
        "latency": "scheduled arrival -> image in pinned host memory (p50/p99_ms); server_*: submit -> image",
    }


def batch_cpu_baseline(args, scs, chosen) -> dict:
    """The oracle on the CPU sample (CPU_SAMPLE scenes, at the grids the GPU
    arm ran them with) on all host threads; beside it the same path on one
    thread for the sample's first scene, and the reference's own csg::Tape::Eval
    point-sampling every finest voxel (SceneBuilder::BuildNode semantics,
    scene_builder.cpp:91-156) of the 16-sphere scene."""
    threads = os.cpu_count() or 1
    order = cpu_sample_order(len(scs))[:CPU_SAMPLE]
    spent = sum(oracle_scene_seconds(scs[i], chosen[i][0], threads) for i in order)
    one = oracle_scene_seconds(scs[order[0]], chosen[order[0]][0], 1)
    all_first = oracle_scene_seconds(scs[order[0]], chosen[order[0]][0], threads)
    out = {"value": len(order) / spent, "unit": "scenes/s", "cores": threads, "kind": "port",
           "sample": f"{len(order)} scenes of the batch (the first of a seeded permutation; the reference "
                     f"arm's steps), each at the grid this run used, voxelize + {args.width}x{args.height} "
                     f"render, oracle C++ port, {threads} threads",
           "single_core": {"value": 1.0 / one, "unit": "scenes/s", "cores": 1,
                           "sample": f"scene {order[0]} of the batch ({scs[order[0]].shape.n_instr} "
                                     f"instructions) on one thread; {1.0 / all_first:.3f} scenes/s on "
                                     f"{threads} threads"}}
    ref = reference_point_sampling()
    if ref:
        out["reference_tape_eval"] = ref
    return out


def reference_point_sampling():
    """The reference's own csg::Tape::Eval (compiled from the reference's
    sources into oracle/_ref) on every finest voxel of the 16-sphere scene
    (64^3 = 262,144 points, one thread): SceneBuilder's point-only
    voxelization (scene_builder.cpp:91-156). None when oracle/_ref is absent."""
    sys.path.insert(0, str(REPO / "oracle"))
    import numpy as np
    import oracle
    if not oracle.ref_available():
        return None
    from frep import scenes
    sc = scenes.spheres_union(16, seed=1)
    ops, in0, in1, consts, root = sc.shape.flatten()
    rt = oracle.RefTape(ops, in0, in1, consts, root)
    fine = 64
    g = (np.arange(fine, dtype=np.float32) + np.float32(0.0))
    cs = np.float32(sc.world_size) / np.float32(fine)
    ax = np.float32(sc.low_vertex[0]) + g * cs
    X, Y, Z = np.meshgrid(ax, ax, ax, indexing="ij")
    pts = np.stack([X.ravel(), Y.ravel(), Z.ravel(), np.zeros(fine ** 3, np.float32)], 1)
    rt.eval(pts[:1024])
    t0 = time.perf_counter()
    v = rt.eval(pts)
    dt = time.perf_counter() - t0
    return {"value": len(pts) / dt, "unit": "point evals/s", "cores": 1, "kind": "reference",
            "sample": f"csg::Tape::Eval of the 16-sphere scene ({rt.n_instr} instructions) at all {fine}^3 "
                      f"finest voxels ({int((v < 0).sum())} inside), {dt:.3f} s"}


def run_ours_batch(args, world, rank, local):
    import numpy as np
    import torch
    import frep
    from frep.autotune import Autotuner, fit_pools

    scs = make_batch_scenes(args, world)  # spawned workers, before any CUDA work
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    ctx = frep.Context(local, hbm_budget_bytes=args.budget_gb << 30)
    stream = torch.cuda.current_stream()

    # ---- untimed setup: autotune, size the pools, build resident trees -------
    t0 = time.perf_counter()
    tuner = Autotuner(ctx, cache_path=args.tune_cache or tuning_table(), save_path=args.tune_cache)
    if not args.no_tune:
        tuner.tune(scs, refine=args.retune)
    t_tune = time.perf_counter() - t0
    chosen = [tuner.apply(sc) for sc in scs]
    pools = fit_pools(ctx, [sc.shape for sc in scs], [d for d, _ in chosen], scs[0].low_vertex, scs[0].world_size)
    storages = []
    for sc, (dims, k), p in zip(scs, chosen, pools):
        vs = frep.VoxelStorage(dims, sc.low_vertex, sc.world_size, rounding=frep.ROUND_OUTWARD,
                               node_words=p.node_words, tape_words=p.tape_words, point_cells_per_lane=k)
        storages.append(vs.init(ctx, sc.shape))
    batch = frep.Batch(ctx, storages)
    batch.set_tuning(*tuner.warps)
    W, H = args.width, args.height
    n = len(scs)
    rgba = torch.empty((n, H, W, 4), dtype=torch.uint8, device=dev)
    frames = [rgba[i] for i in range(n)]
    host_img = torch.empty((n, H, W, 4), dtype=torch.uint8, pin_memory=True)
    cams = [sc.camera for sc in scs]
    sizes = [(W, H)] * n
    lights = frep.Lights(shadow_mask=scs[0].shadow_mask)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2

    def step():
        batch.run(cams, sizes, frames, lights=lights, graph=True, stream=stream)

    for _ in range(max(1, args.warmup)):
        step()
    torch.cuda.synchronize()
    binfo = batch.info()

    # ---- batched, device-resident (value) ------------------------------------
    barrier(world)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    torch.cuda.nvtx.range_push("batched_steps")  # lets a profiler select the timed launches
    with ClockSampler(local) as clocks:
        for s, e in evs:
            flush.fill_(1)
            s.record(stream)
            step()
            e.record(stream)
        torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    barrier(world)
    t_ms = max_over_ranks(world, sum(s.elapsed_time(e) for s, e in evs))
    value = world * n * args.steps / (t_ms / 1e3)

    # ---- plain: one frep_voxelize + frep_render per scene, in sequence --------
    voxs = [frep.Voxelizer(ctx, vs) for vs in storages]
    rts = []
    for vs in storages:
        rt = frep.Raytracer(ctx, vs)
        rt.lights = lights
        rts.append(rt)

    def plain_pass():
        for i in range(n):
            voxs[i].voxelize(0.0, stream)
            rts[i].trace(cams[i], 0.0, W, H, out=(frames[i], None), stream=stream)

    plain_pass()
    torch.cuda.synchronize()
    barrier(world)
    pevs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
            for _ in range(args.plain_steps)]
    torch.cuda.nvtx.range_push("plain_passes")
    for s, e in pevs:
        flush.fill_(1)
        s.record(stream)
        plain_pass()
        e.record(stream)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    barrier(world)
    p_ms = max_over_ranks(world, sum(s.elapsed_time(e) for s, e in pevs))
    plain_value = world * n * args.plain_steps / (p_ms / 1e3)

    # ---- per-launch timing of the batched passes (plain batch calls + events) -
    batch.set_profiling(True)
    reps = 3
    acc = None
    for _ in range(reps):
        flush.fill_(1)
        batch.voxelize(stream=stream)
        batch.render(cams, sizes, frames, lights=lights, stream=stream)
        tm = batch.timings()
        grid_ms = np.array(tm["level"]) / reps
        acc = grid_ms if acc is None else acc + grid_ms
        render_ms = tm["render"]
    batch.set_profiling(False)
    # op-weighted FP32 work of each (level, kind) launch, summed over the trees
    ops = np.zeros_like(acc)
    cinstr = np.zeros_like(acc)
    for vs, (dims, k) in zip(storages, chosen):
        f = vs.fp32_ops()
        c = vs.work()
        kk = vs.point_cells_per_lane or (4 if (dims[-1] ** 3 // 32) % 4 == 0 else 2)
        for l in range(len(dims)):
            kind = 0 if l < len(dims) - 1 else (1 if kk == 4 else 2)
            ops[l, kind] += f[l]
            cinstr[l, kind] += c[l]
    max_levels = max(len(d) for d, _ in chosen)
    dom = np.unravel_index(int(np.argmax(acc)), acc.shape)
    dom_ms = float(acc[dom])
    peaks = measured_peaks()
    sm_mhz = float(peaks.get("sm_max_mhz", 1965.0))
    fp32_peak = SM_COUNT * FP32_LANES_PER_SM * sm_mhz * 1e6 / 1e12
    achieved = float(ops[dom]) / (dom_ms / 1e3) / 1e12
    kind_name = ["interval_level_kernel", "point_level_kernel (4 cells/lane)", "point_level_kernel (2 cells/lane)"]
    total_ops = float(ops.sum())
    default_workload = (n == 512 and (W, H) == (512, 512) and not args.tune_cache and not args.retune
                        and tuning_table() is not None)
    traffic = NCU_DRAM_BYTES_512.get((int(dom[0]), int(dom[1]))) if default_workload else None
    roofline = {
        "bound": "fp32", "kernel": kind_name[dom[1]], "level": int(dom[0]), "achieved": achieved,
        "peak": fp32_peak, "unit": "TFLOP/s", "frac": achieved / fp32_peak, "traffic": traffic,
        "traffic_unit": "bytes per launch",
        "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum of this launch kind on this workload "
                           "(profiles/batch_512scenes_dram_per_launch.txt)") if traffic else None,
        "peak_source": "nominal FP32 issue: 148 SMs x 128 lanes x MEASURED_PEAKS.json sm_max_mhz "
                       "(the file holds no FP32 figure)",
        "algorithmic_ops_per_launch": float(ops[dom]), "cell_instr_per_launch": float(cinstr[dom]),
        "ms_per_launch": dom_ms,
        "all_level_passes": {"ops": total_ops, "ms": float(acc.sum()),
                             "frac": total_ops / (float(acc.sum()) / 1e3) / 1e12 / fp32_peak},
    }
    # the interval kernel's longest launch (the FP32-issue target names the interval kernel)
    iv_l = int(np.argmax(acc[:, 0]))
    iv_ms = float(acc[iv_l, 0])
    if iv_ms > 0.0:
        iv_achieved = float(ops[iv_l, 0]) / (iv_ms / 1e3) / 1e12
        roofline["interval_kernel"] = {
            "level": iv_l, "ms_per_launch": iv_ms, "achieved": iv_achieved, "frac": iv_achieved / fp32_peak,
            "algorithmic_ops_per_launch": float(ops[iv_l, 0]), "cell_instr_per_launch": float(cinstr[iv_l, 0]),
            "traffic": NCU_DRAM_BYTES_512.get((iv_l, 0)) if default_workload else None}

    # ---- end to end: public API with host buffers ----------------------------
    torch.cuda.synchronize()
    barrier(world)
    e2e_evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
    for s, e in e2e_evs:
        flush.fill_(1)
        s.record(stream)
        step()                                     # host tapes + frame args -> device inside
        host_img.copy_(rgba, non_blocking=True)    # all frames -> host
        e.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    e2e_ms = max_over_ranks(world, sum(s.elapsed_time(e) for s, e in e2e_evs))
    e2e_value = world * n * args.steps / (e2e_ms / 1e3)

    branching = {}
    for sc, (dims, k) in zip(scs, chosen):
        branching.setdefault(str(sc.meta["res"]), set()).add((tuple(dims), k))
    instr = np.array([sc.shape.n_instr for sc in scs])
    used = ctx.memory()[0]
    line = {
        "metric": METRIC, "value": value, "unit": "scenes/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload_name, "scenes": n, "resolution": [W, H], "shadow_rays": 1,
                   "rounding": "outward", "tape_instructions": {"min": int(instr.min()),
                                                                "median": float(np.median(instr)),
                                                                "max": int(instr.max())},
                   "branching": {r: sorted([list(d), k] for d, k in v) for r, v in sorted(branching.items())},
                   "warps_per_block": [binfo.interval_warps_per_block, binfo.point_warps_per_block],
                   "autotune_seconds": round(t_tune, 1), "resident_bytes": int(used),
                   "l2": "flushed between timed steps (256 MB write, outside the step events)",
                   "graph": "one CUDA graph per step (upload, level passes, frames)",
                   "parallelism": f"replicas x{world}"},
        "plain": {"value": plain_value, "unit": "scenes/s", "ms_per_pass": p_ms / args.plain_steps,
                  "passes": args.plain_steps,
                  "what": "same trees, frep_voxelize + frep_render per scene in sequence on one stream"},
        "batched_over_plain": value / plain_value,
        "roofline": roofline,
        "level_ms": acc[:max_levels].round(3).tolist(),
        "level_cell_instr": cinstr[:max_levels].tolist(),
        "level_kinds": ["interval", "point 4 cells/lane", "point 2 cells/lane"],
        "render_ms": render_ms,
        "e2e": {"value": e2e_value, "unit": "scenes/s", "h2d_bytes_per_step": int(binfo.upload_bytes),
                "d2h_bytes_per_step": int(n * W * H * 4)},
        "clocks": clocks.summary(),
        "gpu_launches": int((binfo.voxelize_launches + 1) * args.steps),
    }
    batch.close()
    for vs in storages:
        vs.cleanup()
    if args.serve_seconds > 0:
        torch.cuda.synchronize()
        line["serving"] = serve_phase(args, ctx, scs, chosen, pools, tuner.warps)
        sweep = []
        for rate in (float(v) for v in args.serve_sweep.split(",") if v.strip()):
            a = argparse.Namespace(**vars(args))
            a.serve_rate = rate
            r = serve_phase(a, ctx, scs, chosen, pools, tuner.warps)
            sweep.append({k: r[k] for k in ("rate_req_s", "p50_ms", "p99_ms", "max_ms", "scenes_per_s",
                                            "voxelized", "rerendered", "evictions", "failed",
                                            "max_submit_lag_ms", "max_plan_ms", "max_enqueue_ms")})
        if sweep:
            line["serving_sweep"] = sweep
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = batch_cpu_baseline(args, scs, chosen)
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            (run_reference_batch if args.workload == "batch" else run_reference)(args, world, rank)
        else:
            (run_ours_batch if args.workload == "batch" else run_ours)(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
