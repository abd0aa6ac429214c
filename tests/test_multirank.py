"""CPU: the multi-rank plumbing of bench.py with gloo, world size 2.

The benchmark runs one independent replica per rank (no collective on the
data path); ranks meet only at barriers and in the max-over-ranks timing.
These tests cover that host logic without a GPU.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    ws, r, _ = bench.dist_setup(world)
    try:
        bench.barrier(ws)
        v = bench.max_over_ranks(1.5 + r, ws)
        with open(os.path.join(out_dir, f"r{r}.txt"), "w") as f:
            f.write(repr(v))
    finally:
        import torch.distributed as dist
        dist.destroy_process_group()


def test_max_over_ranks_gloo(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.spawn(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    vals = [float(open(tmp_path / f"r{r}.txt").read()) for r in range(2)]
    assert vals == [2.5, 2.5]


def test_reference_arm_prints_once_under_torchrun():
    """Under torchrun only rank 0 runs the CPU reference arm and prints."""
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl",
           "reference", "--gpus", "2", "--workload", "c1", "--cpu-budget", "0.2"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "GB/s" and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"

