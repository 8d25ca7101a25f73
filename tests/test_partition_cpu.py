"""Replica placement over several GPUs (fmd_partition_replicas), on CPU.

The path shards by replica: independent melts are placed on GPUs by a
greedy longest-processing-time bin-pack of their atom counts, with no
data-path exchange between GPUs.  Checked here: the placement against a
plain-Python restatement of the rule, its balance bound, determinism, and a
two-rank gloo run in which both ranks compute the batched case's (256 uneven
replicas) placement independently and agree on it."""
import os
import re
import socket
import subprocess
import sys

import numpy as np
import pytest

import fastmd_b200 as fm

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _lpt(costs, nparts):
    """The rule restated: decreasing cost (stable), each to the least-loaded
    part (lowest index on ties)."""
    order = sorted(range(len(costs)), key=lambda i: -costs[i])
    load = [0] * nparts
    part = [0] * len(costs)
    for i in order:
        p = min(range(nparts), key=lambda q: (load[q], q))
        part[i] = p
        load[p] += costs[i]
    return part, load


@pytest.mark.parametrize("seed,n,parts", [(0, 256, 8), (1, 17, 4), (2, 3, 8), (3, 100, 1), (4, 64, 2)])
def test_partition_matches_the_rule(seed, n, parts):
    costs = np.random.default_rng(seed).integers(500, 20000, size=n)
    part, load = fm.partition_replicas(costs, parts)
    want_part, want_load = _lpt(costs.tolist(), parts)
    assert part.tolist() == want_part and load.tolist() == want_load
    assert np.bincount(part, minlength=parts).sum() == n
    if n >= parts:
        # greedy bound: the most loaded part exceeds the least by at most one item
        assert load.max() - load.min() <= costs.max()


def test_partition_ties_and_empty_input():
    part, load = fm.partition_replicas([5, 5, 5, 5], 2)
    assert part.tolist() == [0, 1, 0, 1] and load.tolist() == [10, 10]
    part, load = fm.partition_replicas([], 4)
    assert len(part) == 0 and load.tolist() == [0, 0, 0, 0]
    with pytest.raises(fm.FastMDError):
        fm.partition_replicas([1, -2], 2)


def test_c3_placement_is_balanced():
    sys.path.insert(0, ROOT)
    import bench
    for world in (1, 2, 4, 8):
        reps, part, load = bench.c3_assignment(fm, world)
        assert len(part) == 256 and set(part.tolist()) <= set(range(world))
        assert load.sum() == sum(nc * cl for nc, cl, _, _ in reps)
        assert load.max() / load.mean() < 1.02   # 256 replicas of 500-20,000 atoms pack within 2 %


WORKER = r"""
import os, sys
sys.path.insert(0, sys.argv[1])
import bench
import fastmd_b200 as fm
rank, world, local, dist = bench.dist_setup(2)
reps, part, load = bench.c3_assignment(fm, world)
mine = sorted(k for k in range(len(reps)) if part[k] == rank)
everyone = [None, None]
dist.all_gather_object(everyone, (part.tolist(), mine))
if rank == 0:
    parts = [e[0] for e in everyone]
    assert parts[0] == parts[1], "ranks disagree on the placement"
    union = sorted(everyone[0][1] + everyone[1][1])
    assert union == list(range(len(reps))), "replicas lost or duplicated"
    print(f"placement ok {len(everyone[0][1])} {len(everyone[1][1])} {load.tolist()}", flush=True)
dist.destroy_process_group()
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_placement_agrees(tmp_path):
    w = tmp_path / "worker.py"
    w.write_text(WORKER)
    env = dict(os.environ, OMP_NUM_THREADS="2")
    for attempt in range(3):
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
               "--master-addr=127.0.0.1", f"--master-port={_free_port()}", str(w), ROOT]
        out = subprocess.run(cmd, capture_output=True, text=True, timeout=240, cwd=ROOT, env=env)
        if out.returncode == 0 or "address already in use" not in (out.stderr + out.stdout).lower():
            break
    assert out.returncode == 0, out.stderr[-2000:]
    m = re.search(r"placement ok (\d+) (\d+) \[(\d+), (\d+)\]", out.stdout)
    assert m and int(m.group(1)) + int(m.group(2)) == 256
    assert abs(int(m.group(3)) - int(m.group(4))) <= 20000
