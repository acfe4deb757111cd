"""bench.py's multi-process plumbing on the CPU (gloo, world size 2): process
group set-up, the barrier and the max-over-ranks timing every multi-GPU
number goes through, and the reference arm under torchrun (rank 0 alone
measures and prints, the other ranks exit 0). The path shards as independent
replicas, so there is no data-path collective to test beyond these."""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import torch.multiprocessing as mp

REPO = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "CUDA_VISIBLE_DEVICES": ""})
    sys.path.insert(0, str(REPO))
    import torch.distributed as dist

    import bench
    w, r, _ = bench.dist_setup(None)
    assert (w, r) == (world, rank) and dist.get_backend() == "gloo"
    bench.barrier(w)
    out[rank] = bench.max_over_ranks(w, 1.5 * (rank + 1))
    bench.barrier(w)
    dist.destroy_process_group()


def test_max_over_ranks_with_gloo():
    world = 2
    out = mp.get_context("spawn").Manager().dict()
    mp.start_processes(_rank_main, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    assert dict(out) == {0: 3.0, 1: 3.0}


def test_reference_arm_under_torchrun_prints_once():
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), str(REPO / "bench.py"),
           "--impl", "reference", "--gpus", "2", "--workload", "large", "--grid", "8,4", "--res", "32x32",
           "--steps", "1", "--warmup", "0"]
    p = subprocess.run(cmd, cwd=REPO, env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [json.loads(l) for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, p.stdout
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0
