"""bench.py's multi-rank plumbing on CPU: two ranks over gloo (127.0.0.1).

The per-rank work of the GPU arm needs a GPU; what runs here is the
rendezvous, the max-over-ranks reduction and the barrier that the GPU arm
uses, and the reference arm end to end (rank 0 times the CPU restatement,
rank 1 exits without work)."""
import json
import os
import re
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


WORKER = r"""
import os, sys
sys.path.insert(0, sys.argv[1])
import bench
rank, world, local, dist = bench.dist_setup(2)
assert world == 2 and dist is not None
v = bench.allmax(dist, float(10 + rank), local)
bench.barrier(dist, local)
print(f"rank {rank} max {v}", flush=True)
dist.destroy_process_group()
"""


def _torchrun(args, timeout=240):
    env = dict(os.environ, OMP_NUM_THREADS="2")
    for attempt in range(3):
        # a port found free can be taken before the rendezvous binds it
        port = _free_port()
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
               "--master-addr=127.0.0.1", f"--master-port={port}"] + args
        out = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout, cwd=ROOT, env=env)
        if out.returncode == 0 or "address already in use" not in (out.stderr + out.stdout).lower():
            return out
    return out


def test_two_rank_max_and_barrier(tmp_path):
    w = tmp_path / "worker.py"
    w.write_text(WORKER)
    out = _torchrun([str(w), ROOT])
    assert out.returncode == 0, out.stderr[-2000:]
    # the two ranks share one stdout pipe: their lines may interleave
    found = sorted(re.findall(r"rank (\d) max ([0-9.]+)", out.stdout))
    assert found == [("0", "11.0"), ("1", "11.0")]


def test_reference_arm_two_ranks_prints_one_line():
    out = _torchrun(["bench.py", "--impl", "reference", "--gpus", "2", "--steps", "3", "--warmup", "3"])
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference" and rec["n_gpus"] == 2 and rec["value"] > 0
    assert rec["cpu_baseline"]["kind"] == "port" and rec["e2e"]["h2d_bytes_per_step"] == 0
