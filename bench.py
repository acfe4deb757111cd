"""Benchmark: scenes/s of voxelize + render on the large single-scene workload.

Workload (BASELINE's large scene): 256 primitives (sphere / box / capsule,
sizes U[0.02, 0.2]) combined by a random binary tree of min / max / max(a,-b)
/ polynomial smooth-min; 3-level tree {16, 16, 8} = 2048^3 effective; 1920x1080
perspective render at 60 degrees with one shadow ray per hit. Seeded synthetic
scene (the reference ships no dataset).

One step = one full voxelization (every level pass) + one rendered frame.

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
    ap.add_argument("--grid", default="16,16,8",
                    help="tree branching per level (profiling uses a smaller grid of the same scene)")
    ap.add_argument("--res", default="1920x1080", help="render resolution WxH")
    ap.add_argument("--pool-mb", type=int, default=3072, help="node + tape pool size of the tree, MB")
    args = ap.parse_args()
    args.grid_dims = tuple(int(v) for v in args.grid.split(","))
    args.width, args.height = (int(v) for v in args.res.lower().split("x"))
    fine = 1
    for d in args.grid_dims:
        fine *= d
    args.workload = f"random_csg_256prim_{fine}cube_{args.width}x{args.height}_shadow"
    return args


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, value: float) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device="cuda")
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


def make_scene(args):
    from frep import scenes
    return scenes.random_csg(256, seed=2, grid_dims=args.grid_dims, width=args.width, height=args.height,
                             shadows=True)


def cpu_baseline(scene, threads: int):
    """The oracle (C++ restatement of the reference's shaders) on the host:
    one full voxelization + one full render, all host threads."""
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle
    import frep
    tape = frep.Tape(scene.shape)
    t0 = time.perf_counter()
    tree = oracle.OracleTree(tape.wide(), tape.n_slots, scene.grid_dims, scene.low_vertex, scene.world_size,
                             rounding=1, threads=threads)
    t1 = time.perf_counter()
    lights = frep.Lights(shadow_mask=scene.shadow_mask)
    tree.render(oracle.camera_vector(scene.camera, scene.width, scene.height), lights, threads=threads)
    t2 = time.perf_counter()
    return t2 - t0, t1 - t0, t2 - t1


def run_reference(args, world, rank):
    """--impl reference: the CPU path on the host cores, same metric/config."""
    if rank != 0:
        return
    scene = make_scene(args)
    threads = os.cpu_count() or 1
    if args.warmup > 0:
        cpu_baseline(scene, threads)  # one warm-up scene (the oracle has no caches to warm)
    times = [cpu_baseline(scene, threads)[0] for _ in range(args.steps)]
    total = sum(times)
    value = args.steps / total
    line = {
        "metric": METRIC, "value": value, "unit": "scenes/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": args.workload, "grid": list(args.grid_dims), "resolution": [args.width, args.height],
                   "shadow_rays": 1, "rounding": "outward"},
        "cpu_baseline": {"value": value, "unit": "scenes/s", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} full scenes (voxelize + 1080p render), oracle C++ port, "
                                   f"{threads} threads"},
        "e2e": {"value": value, "unit": "scenes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, world, rank, local):
    import torch
    import frep

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    scene = make_scene(args)
    ctx = frep.Context(local, hbm_budget_bytes=48 << 30)
    pool = args.pool_mb << 20
    vs = frep.VoxelStorage(scene.grid_dims, scene.low_vertex, scene.world_size, rounding=frep.ROUND_OUTWARD,
                           node_words=pool // 4 // 4, tape_words=pool * 3 // 4 // 8)
    vs.init(ctx, scene.shape)
    vox = frep.Voxelizer(ctx, vs)
    rt = frep.Raytracer(ctx, vs)
    rt.lights = frep.Lights(shadow_mask=scene.shadow_mask)
    W, H = scene.width, scene.height
    rgba = torch.empty((H, W, 4), dtype=torch.uint8, device=dev)
    host_img = torch.empty((H, W, 4), dtype=torch.uint8, pin_memory=True)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2
    stream = torch.cuda.current_stream()

    def step():
        vox.voxelize(0.0, stream)
        rt.trace(scene.camera, 0.0, W, H, out=(rgba, None), stream=stream)

    for _ in range(args.warmup):
        step()
    info = vs.sync()
    fp32_ops = vs.fp32_ops()
    cell_instr = vs.work()
    launches_per_step = 1 + 2 * vs.grid_levels + 1  # init + (work scan + level pass) per level + render

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
    vs.set_profiling(True)
    level_ms = [0.0] * vs.grid_levels
    render_ms = 0.0
    reps = max(3, min(args.steps, 10))
    for _ in range(reps):
        flush.fill_(1)
        vox.voxelize(0.0, stream)
        rs, re_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        rs.record(stream)
        rt.trace(scene.camera, 0.0, W, H, out=(rgba, None), stream=stream)
        re_.record(stream)
        lt = vs.level_timings()
        torch.cuda.synchronize()
        level_ms = [a + b / reps for a, b in zip(level_ms, lt)]
        render_ms += rs.elapsed_time(re_) / reps
    vs.set_profiling(False)

    # ---- end to end through the public API with host buffers ---------------
    torch.cuda.synchronize()
    barrier(world)
    e2e_evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for s, e in e2e_evs:
        flush.fill_(1)
        s.record(stream)
        vox.voxelize(0.0, stream)   # host tape -> device (pinned staging + H2D)
        rt.trace(scene.camera, 0.0, W, H, out=(rgba, None), stream=stream)
        host_img.copy_(rgba, non_blocking=True)  # result -> host
        e.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    e2e_ms = max_over_ranks(world, sum(s.elapsed_time(e) for s, e in e2e_evs))
    e2e_value = world * args.steps / (e2e_ms / 1e3)
    h2d = 8 * info.root_tape_words
    d2h = W * H * 4

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
        "config": {"workload": args.workload, "grid": scene.grid_dims, "resolution": [W, H], "shadow_rays": 1,
                   "tape_instructions": vs.tape.n_instr, "rounding": "outward",
                   "nodes_per_level": list(info.node_count[:vs.grid_levels]),
                   "l2": "flushed between timed steps (256 MB write, outside the step events)",
                   "parallelism": f"replicas x{world}"},
        "roofline": roofline,
        "level_ms": level_ms, "render_ms": render_ms,
        "e2e": {"value": e2e_value, "unit": "scenes/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "clocks": clocks.summary(),
        "gpu_launches": launches_per_step * args.steps,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        total, t_vox, t_ren = cpu_baseline(scene, threads)
        line["cpu_baseline"] = {"value": 1.0 / total, "unit": "scenes/s", "cores": threads, "kind": "port",
                                "sample": f"1 full scene (voxelize {t_vox:.2f} s + 1080p render {t_ren:.2f} s), "
                                          f"oracle C++ port, {threads} threads"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    vs.cleanup()
    ctx.close()


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
