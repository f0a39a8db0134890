"""The N > 1 path of bench.py on the CPU: one process per rank, world size 2, gloo.

The decoder shards by code block with no data-path exchange (replicas), so the only collectives
are the timing barrier and the max-over-ranks reduction of the elapsed time; both are checked
here, and the reference arm is run as torchrun launches it (rank 0 measures and prints, the
other rank exits 0 without work)."""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_RANK_SCRIPT = """
import argparse, json, sys
sys.path.insert(0, {root!r})
import torch.distributed as dist
import bench
world, rank, local = bench.dist_setup(argparse.Namespace(impl="reference"))
bench.barrier(world)
m = bench.max_over_ranks(1.5 + rank, world)
print(json.dumps({{"rank": rank, "world": world, "max": m, "backend": dist.get_backend()}}))
dist.destroy_process_group()
"""


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_barrier_and_max_over_ranks_with_two_gloo_ranks():
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2",
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", _RANK_SCRIPT.format(root=ROOT)],
                                      env=env, stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                                      text=True))
    outs = [p.communicate(timeout=180) for p in procs]
    for p, (out, err) in zip(procs, outs):
        assert p.returncode == 0, err[-2000:]
    recs = sorted((json.loads(o.strip().splitlines()[-1]) for o, _ in outs), key=lambda r: r["rank"])
    assert [r["rank"] for r in recs] == [0, 1]
    assert all(r["world"] == 2 and r["max"] == 2.5 and r["backend"] == "gloo" for r in recs)


def test_reference_arm_under_torchrun_two_ranks():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl",
           "reference", "--gpus", "2", "--steps", "1", "--warmup", "0", "--cpu-seconds", "3"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout  # rank 0 alone prints
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["cores"] >= 1
