"""Benchmark: aggregate atom-steps/s of the bead-spring MD step on B200.

Workload (one GPU): 64 independent Kremer-Grest melts of 300 chains x 100
beads (30,000 beads each, density 0.85, L = 32.80), LJ eps = sig = 1,
rc = 2.5, skin = 0.3, FENE k = 30, R0 = 1.5 with WCA, harmonic angle k = 5,
theta0 = 180 deg; nvt_langevin T = 1, Tdamp = 1, seed = replica index (+ 1000
* rank), dt = 0.001.  Each replica is a seeded random-walk melt pushed off for
2,000 capped-force (|F| <= 50) Langevin steps on the device.  One bench step
advances every replica by one MD step in the mixed form (FP32 forces on
cell-relative positions, FP64 reductions), batched in CUDA graphs.  The device
working set (~1.5 GB) is far larger than L2, so no flush is needed.

Timing: W untimed warm-up steps, then K timed steps on the library's own
stream with CUDA events, barrier + synchronize on both sides, max over ranks.
Multi-GPU: one process per GPU, each with its own 64 replicas (weak scaling,
no data-path collective; the barrier and the max reduction use
torch.distributed).

Also reported (rank 0, N = 1): the force kernel's roofline from a live
CUDA-event timing of the kernel alone, the end-to-end rate through the public
C API (fmd_batch_run in thermo-sized chunks + thermo readout), the FP64 plain
form on one 30K replica, and the CPU baseline (the FP64 oracle port on the
host cores, a bounded sample).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "atom-steps/s (aggregate over replicas), Kremer-Grest melt, 30K beads per replica"
NCHAINS, CHAIN_LEN, DENSITY = 300, 100, 0.85
PUSHOFF = 2000


def run_conf(seed, nsteps=10_000_000):
    # thermo every 100 steps, as the reference's runs of this melt print it:
    # energies and virial come from the step itself on those steps
    return (f"ntypes 1\nrc 2.5\nskin 0.3\ndt 0.001\nnsteps {nsteps}\nnvt_langevin 1.0 1.0 1.0 {seed}\n"
            "lj 0 0 1.0 1.0\nbond_type 0 30.0 1.5 1.0 1.0\nangle_type 0 5.0 180.0\nthermo 1 100 thermo.dat\n")


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiler_range(start):
    """cudaProfilerStart / Stop around the timed region, so that a profiler
    run with --profile-from-start off sees exactly the timed launches."""
    import ctypes as C
    try:
        rt = C.CDLL("libcudart.so.12")
    except OSError:
        return
    (rt.cudaProfilerStart if start else rt.cudaProfilerStop)()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                line = out.stdout.strip().splitlines()[0]
                self.samples.append([x.strip() for x in line.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for k, n in enumerate(names):
                if len(s) > 5 + k and "Active" in s[5 + k] and "Not" not in s[5 + k]:
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def dist_setup(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        import datetime
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        return rank, world, local, dist
    return 0, 1, 0, None


def allmax(dist, value, local):
    if dist is None:
        return value
    import torch
    dev = torch.device("cuda", local) if torch.cuda.is_available() else torch.device("cpu")
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist, local):
    if dist is None:
        return
    import torch
    if torch.cuda.is_available():
        dist.barrier(device_ids=[local])
    else:
        dist.barrier()


# --------------------------------------------------------------------- CPU
def cpu_oracle_rate(desc, seconds=12.0, threads=None):
    """FP64 oracle port (OpenMP over the host cores) stepping one 30K replica."""
    from oracle import pyoracle as po
    threads = threads or os.cpu_count() or 1
    s = po.System(xyz=desc["xyz"], L=desc["L"], type=desc["type"], mass=np.ones(1), lj=np.ones((1, 1, 2)),
                  bonds=desc["bonds"], bond_type=np.zeros(len(desc["bonds"]), np.int32),
                  fene=np.array([[30.0, 1.5, 1.0, 1.0]]), angles=desc["angles"],
                  angle_type=np.zeros(len(desc["angles"]), np.int32), angle_p=np.array([[5.0, np.pi]]),
                  mol=desc["mol"], vel=desc["vel"], image=desc["image"])
    sim = po.Sim(s, ensemble="langevin", T=(1.0, 1.0, 1.0), seed=1, nsteps=10**7, nthreads=threads)
    sim.step(2)
    t0 = time.perf_counter()
    sim.step(5)
    per = (time.perf_counter() - t0) / 5
    nsteps = max(5, int(seconds / max(per, 1e-6)))
    t0 = time.perf_counter()
    sim.step(nsteps)
    dt = time.perf_counter() - t0
    n = len(desc["type"])
    return n * nsteps / dt, threads, f"one {n}-bead replica of the workload, {nsteps} steps, FP64 oracle port, " \
                                    f"{threads} OpenMP threads, {dt:.1f} s"


def bench_replica_state():
    """Replica 0 of the workload after its push-off, from the committed
    fixture (tests/golden/make_bench_replica.py made it on a GPU), with the
    implied topology: linear chains of CHAIN_LEN beads in atom order."""
    p = os.path.join(ROOT, "tests", "golden", "kg30k_replica0.npz")
    z = np.load(p)
    n = len(z["xyz"])
    nch, cl = int(z["nchains"][0]), int(z["chain_length"][0])
    ids = np.arange(n, dtype=np.int32).reshape(nch, cl)
    bonds = np.stack([ids[:, :-1].ravel(), ids[:, 1:].ravel()], axis=1).astype(np.int32)
    angles = np.stack([ids[:, :-2].ravel(), ids[:, 1:-1].ravel(), ids[:, 2:].ravel()], axis=1).astype(np.int32)
    mol = np.repeat(np.arange(1, nch + 1, dtype=np.int32), cl)
    return dict(xyz=z["xyz"].astype(np.float64), L=float(z["box_L"][0]), type=np.zeros(n, np.int32), bonds=bonds,
                angles=angles, mol=mol, vel=z["vel"].astype(np.float64), image=z["image"].astype(np.int32),
                seed=int(z["seed"][0]))


def headline_config(world, graph_steps, replicas):
    return {"workload": "kg_melt_64x30k_langevin_batched", "replicas_per_gpu": replicas,
            "beads_per_replica": NCHAINS * CHAIN_LEN, "chains": NCHAINS, "chain_length": CHAIN_LEN,
            "density": DENSITY, "rc": 2.5, "skin": 0.3, "dt": 0.001, "ensemble": "nvt_langevin T=1 Tdamp=1",
            "l2": "working set > L2 (no flush needed)", "parallelism": f"replicas x{world} (no collective)"}


def run_reference(args, rank, world, local, dist):
    """--impl reference: the reference has no CPU stepping path, so its CPU
    arm is the FP64 oracle port (OpenMP over the host cores) stepping replica
    0 of the same workload (the pushed-off state from the committed fixture,
    the same Langevin settings and seed, no force cap): one replica per step
    is the bounded sample.  Loads no library of this repository."""
    if rank != 0:
        return
    from oracle import pyoracle as po
    desc = bench_replica_state()
    threads = os.cpu_count() or 1
    s = po.System(xyz=desc["xyz"], L=desc["L"], type=desc["type"], mass=np.ones(1), lj=np.ones((1, 1, 2)),
                  bonds=desc["bonds"], bond_type=np.zeros(len(desc["bonds"]), np.int32),
                  fene=np.array([[30.0, 1.5, 1.0, 1.0]]), angles=desc["angles"],
                  angle_type=np.zeros(len(desc["angles"]), np.int32), angle_p=np.array([[5.0, np.pi]]),
                  mol=desc["mol"], vel=desc["vel"], image=desc["image"])
    sim = po.Sim(s, ensemble="langevin", T=(1.0, 1.0, 1.0), seed=desc["seed"], nsteps=10**7, nthreads=threads)
    sim.step(args.warmup)
    t0 = time.perf_counter()
    sim.step(args.steps)
    dt = time.perf_counter() - t0
    n = len(desc["type"])
    v = n * args.steps / dt
    sample = (f"replica 0 of the workload ({n} beads, pushed off), {args.steps} steps (+{args.warmup} warm-up), "
              "FP64 oracle port (the reference has no CPU stepping path)")
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "atom-steps/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded random-walk melt, "
        "2,000-step capped push-off; replica 0 from tests/golden/kg30k_replica0.npz)",
        "config": headline_config(world, None, args.replicas),
        "cpu_baseline": {"value": v, "unit": "atom-steps/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": "atom-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    assert "fastmd_b200" not in sys.modules, "the reference arm must not load this repository's library"
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------- GPU
def reference_gpu_leg(fm, xyz, vel, image, steps):
    """The reference's own FP32 GPU engine (src/main.cu and its core library,
    built for sm_100a into oracle/_ref/fastMD_ref by `make -C oracle refbin`)
    stepping one 30K replica of the same melt: one system per process, its
    own wall clock (the "Steps/s" it prints, main.cu:750-756).  A datapoint
    beside the batched number, not a bench arm."""
    exe = os.path.join(ROOT, "oracle", "_ref", "fastMD_ref")
    if not os.path.exists(exe):
        return {"unavailable": "reference GPU engine not built (make -C oracle refbin)"}
    import tempfile
    d = fm.generate_melt(NCHAINS, CHAIN_LEN, density=DENSITY, seed=0)
    d.xyz, d.vel, d.image = xyz, vel, image
    with tempfile.TemporaryDirectory() as td:
        data = os.path.join(td, "melt.data")
        fm.write_lammps_data(data, d)
        conf = os.path.join(td, "run.conf")
        with open(conf, "w") as f:
            # the reference sizes its arrays from natoms (main.cu:62-99)
            f.write(run_conf(42, nsteps=steps) + f"natoms {len(d.type)}\nlammps_data_file {data}\n")
        out = subprocess.run([exe, conf], capture_output=True, text=True, timeout=600, cwd=td)
    m = re.search(r"Steps/s:\s*([0-9.]+)", out.stdout)
    if out.returncode != 0 or not m:
        tail = (out.stdout + out.stderr).strip().splitlines()[-3:]
        return {"unavailable": f"reference run failed (rc {out.returncode}): {' | '.join(tail)}"}
    sps = float(m.group(1))
    n = len(d.type)
    return {"value": n * sps, "unit": "atom-steps/s", "steps": steps, "natoms": n,
            "how": "oracle/_ref/fastMD_ref <run.conf> on a LAMMPS data file of replica 0, its printed Steps/s"}


def force_profile_traffic():
    """Per-launch DRAM bytes of the force kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "k_force_kg30k_langevin.md")
    if not os.path.exists(p):
        return None
    m = re.search(r"dram_bytes_per_launch_full_workload:\s*([0-9.eE+]+)", open(p).read())
    return float(m.group(1)) if m else None


# --------------------------------------------------------------- workloads
# The scope table's reported cases beside the headline (one JSON line each):
#   c0  3,000 beads (30 x 100), Langevin, 5,000 steps: mixed vs plain FP64 vs CPU oracle
#   c1  30,000 beads: force RMS error vs the FP64 oracle on 10 snapshots; <T>, <P>, Rg
#       of the mixed form against the plain FP64 form; NVT conserved-quantity drift
#   c2  1,000,000 beads, two types, NPT: throughput and conserved-quantity drift
#   c3  256 replicas of uneven size: batched vs the plain form one at a time
#   c4  served request stream (Poisson arrivals): p50 / p99 latency, throughput


def _conf(ens, nsteps, ntypes=1, lj=((0, 0, 1.0, 1.0),), thermo=0):
    text = (f"ntypes {ntypes}\nrc 2.5\nskin 0.3\ndt 0.001\nnsteps {nsteps}\n{ens}\n"
            "bond_type 0 30.0 1.5 1.0 1.0\nangle_type 0 5.0 180.0\n")
    text += "".join(f"lj {a} {b} {e} {g}\n" for a, b, e, g in lj)
    if thermo:
        text += f"thermo 1 {thermo} thermo.dat\n"
    return text


GRAPH_CAPTURE_STEPS = 50  # one replay of a batch's default step graph
# force-kernel variants, in the library's order (fastmd_b200/csrc/mixed_kernels.cu, force_kernels)
FORCE_VARIANTS = ["m8 k1 t3", "m8 k2 t3", "m8 k1 a5", "m8 k2 a5", "m8 k1 a5 x2", "m8 k2 a5 x2", "m7 k1 a5 x2",
                  "m9 k1 a5 x2", "m6 k1 a5", "m8 k1 a5 x2 l2", "m8 k1 a5 x2 l4",
                  "m8 k1 a5 x2 r3", "m8 k1 a5 x2 r4", "m8 k1 a5 x2 r2", "m9 k1 a5 x2 r2"]


def _dev_run(fm, b, nsteps):
    """Advance a batch nsteps; device milliseconds between events on its stream."""
    import ctypes as C
    lib = fm.lib()
    lib.fmd_batch_mark(b._h, 0)
    b.run(nsteps)
    lib.fmd_batch_mark(b._h, 1)
    ms = C.c_double()
    lib.fmd_batch_elapsed_ms(b._h, C.byref(ms))
    return ms.value


def _oracle_sim(desc, ens_kw, nthreads=None):
    from oracle import pyoracle as po
    s = po.System(xyz=desc.xyz, L=desc.box_L, type=desc.type, mass=np.ones(max(1, int(desc.type.max()) + 1)),
                  lj=np.ones((1, 1, 2)), bonds=desc.bonds, bond_type=np.zeros(len(desc.bonds), np.int32),
                  fene=np.array([[30.0, 1.5, 1.0, 1.0]]), angles=desc.angles,
                  angle_type=np.zeros(len(desc.angles), np.int32), angle_p=np.array([[5.0, np.pi]]),
                  mol=desc.mol, vel=desc.vel, image=desc.image)
    return po, s


def wl_c0(args, fm):
    conf = _conf("nvt_langevin 1.0 1.0 1.0 42", 5000, thermo=100)
    b = fm.Batch(max_replicas=1, max_atoms=4096, device=0)
    s = b.add(conf, gen=dict(nchains=30, chain_length=100, density=DENSITY, seed=42, pushoff_steps=PUSHOFF))
    b.run(1)  # push-off and setup
    x0, v0, i0 = b.state(s)
    b.run(GRAPH_CAPTURE_STEPS)  # captures the step graph outside the timed steps
    timed_steps = 4999 - GRAPH_CAPTURE_STEPS
    ms = _dev_run(fm, b, timed_steps)
    n = 3000
    mixed = n * timed_steps / (ms * 1e-3)
    t_mixed = b.thermo(s)
    d = fm.generate_melt(30, 100, density=DENSITY, seed=42)
    d.xyz, d.vel, d.image = x0, v0, i0
    ps = fm.Simulation(conf, desc=d, form=fm.FMD_FORM_PLAIN_FP64)
    t0 = time.perf_counter()
    ps.step(4999)
    plain = n * 4999 / (time.perf_counter() - t0)
    t_plain = ps.thermo()
    ps.close()
    po, sysm = _oracle_sim(d, None)
    threads = os.cpu_count() or 1
    sim = po.Sim(sysm, ensemble="langevin", T=(1.0, 1.0, 1.0), seed=42, nsteps=5000, nthreads=threads)
    t0 = time.perf_counter()
    sim.step(4999)
    cpu = n * 4999 / (time.perf_counter() - t0)
    return {"workload": "c0_3k_langevin_5000", "metric": "atom-steps/s", "unit": "atom-steps/s",
            "mixed_device": mixed, "plain_fp64_wall": plain, "cpu_oracle": cpu, "cpu_threads": threads,
            "T_final": {"mixed": t_mixed.temp, "plain_fp64": t_plain.temp},
            "steps": 4999, "mixed_timed_steps": timed_steps,
            "note": "one replica; mixed timed on the device after its step graph is captured, plain and CPU by wall clock"}


def wl_c1(args, fm):
    from oracle import pyoracle as po
    conf = _conf("nvt_langevin 1.0 1.0 1.0 7", 10 ** 7)
    b = fm.Batch(max_replicas=2, max_atoms=65536, device=0)
    s = b.add(conf, gen=dict(nchains=NCHAINS, chain_length=CHAIN_LEN, density=DENSITY, seed=7, pushoff_steps=PUSHOFF))
    b.run(200)
    d = fm.generate_melt(NCHAINS, CHAIN_LEN, density=DENSITY, seed=7)
    errs = []
    for k in range(10):
        b.run(100)
        x, v, img = b.state(s)
        f, _, _ = b.forces(s)
        osys = po.System(xyz=x, L=d.box_L, type=d.type, mass=np.ones(1), lj=np.ones((1, 1, 2)), bonds=d.bonds,
                         bond_type=np.zeros(len(d.bonds), np.int32), fene=np.array([[30.0, 1.5, 1.0, 1.0]]),
                         angles=d.angles, angle_type=np.zeros(len(d.angles), np.int32),
                         angle_p=np.array([[5.0, np.pi]]), mol=d.mol)
        fo, _, _ = po.forces(osys)
        errs.append(float(np.sqrt(np.mean((f - fo) ** 2)) / np.sqrt(np.mean(fo ** 2))))
    # <T>, <P>, Rg: mixed, plain FP64 and the FP64 oracle from the same state,
    # c1_stat_steps steps sampled every 100
    x, v, img = b.state(s)
    d.xyz, d.vel, d.image = x, v, img
    nsamp = max(10, args.c1_stat_steps // 100)

    def p_of(st):
        return (st[0] + st[3] + st[5]) / 3.0

    def sample_batch():
        out = []
        for _ in range(nsamp):
            b.run(100)
            t = b.thermo(s)
            out.append((t.temp, p_of(t.stress), b.rg(s)))
        return np.array(out)

    def sample_plain():
        ps = fm.Simulation(conf, desc=d, form=fm.FMD_FORM_PLAIN_FP64)
        out = []
        for _ in range(nsamp):
            ps.step(100)
            t = ps.thermo()
            out.append((t.temp, p_of(t.stress), ps.rg()))
        ps.close()
        return np.array(out)

    def sample_oracle():
        osys = po.System(xyz=x, L=d.box_L, type=d.type, mass=np.ones(1), lj=np.ones((1, 1, 2)), bonds=d.bonds,
                         bond_type=np.zeros(len(d.bonds), np.int32), fene=np.array([[30.0, 1.5, 1.0, 1.0]]),
                         angles=d.angles, angle_type=np.zeros(len(d.angles), np.int32),
                         angle_p=np.array([[5.0, np.pi]]), mol=d.mol, vel=v, image=img)
        osim = po.Sim(osys, ensemble="langevin", T=(1.0, 1.0, 1.0), seed=7, nsteps=10 ** 7)
        out = []
        for _ in range(nsamp):
            osim.step(100)
            o = osim.thermo()
            out.append((o[2], (o[3] + o[6] + o[8]) / 3.0, osim.rg()))
        return np.array(out)

    mb, pl, orc = sample_batch(), sample_plain(), sample_oracle()

    def ms(a):
        # mean and standard error with 10 blocks (correlated series)
        blocks = np.array([blk.mean(axis=0) for blk in np.array_split(a, 10)])
        return a.mean(axis=0).tolist(), (blocks.std(axis=0, ddof=1) / np.sqrt(len(blocks))).tolist()

    (m_mean, m_err), (p_mean, p_err), (o_mean, o_err) = ms(mb), ms(pl), ms(orc)
    sigma = [abs(a - c) / max(np.hypot(ea, ec), 1e-300) for a, ea, c, ec in zip(m_mean, m_err, o_mean, o_err)]
    # NVT conserved-quantity drift (nose_hoover test definition), mixed form
    cn = _conf("nvt_nh 1.0 1.0 0.5 3", 10 ** 7, thermo=0)
    b2 = fm.Batch(max_replicas=1, max_atoms=65536, device=0)
    s2 = b2.add(cn, desc=d)
    b2.run(10)
    # 100 samples over c1_drift_steps: the conserved quantity's step-to-step
    # fluctuation (FP32 forces, dt = 0.001) swamps a slope fitted over a
    # short run
    e = []
    chunk = max(1, args.c1_drift_steps // 100)
    for _ in range(100):
        b2.run(chunk)
        e.append(b2.thermo(s2).conserved)
    e = np.array(e)
    steps = np.arange(1, len(e) + 1) * float(chunk)
    slope = float(np.polyfit(steps, e, 1)[0]) if len(e) > 1 else 0.0
    rel_per_1e6 = slope * 1e6 / abs(e[0]) if len(e) else 0.0
    return {"workload": "c1_30k", "force_rel_rms_vs_fp64_oracle": {"max": max(errs), "mean": float(np.mean(errs)),
                                                                   "snapshots": len(errs), "target": 1e-5},
            "langevin_T_P_Rg": {"mixed": {"mean": m_mean, "stderr": m_err},
                                "plain_fp64": {"mean": p_mean, "stderr": p_err},
                                "fp64_oracle": {"mean": o_mean, "stderr": o_err},
                                "mixed_vs_oracle_sigmas": sigma,
                                "samples": f"{nsamp} per form, every 100 steps, {nsamp * 100} steps from the same "
                                           "state; standard errors from 10 block averages"},
            "nvt_conserved_drift": {"steps": int(steps[-1]) if len(e) else 0, "E0": float(e[0]) if len(e) else 0.0,
                                    "slope_per_step": slope, "relative_per_1e6_steps": rel_per_1e6,
                                    "target_relative_per_1e6": 1e-4}}


def wl_c2(args, fm):
    conf = _conf("npt_nh 1.0 1.0 0.1 0.0 0.0 1.0 3", 10 ** 7, ntypes=2,
                 lj=((0, 0, 1.0, 1.0), (1, 1, 1.0, 1.0), (0, 1, 0.9, 1.0)))
    b = fm.Batch(max_replicas=1, max_atoms=1_000_200, device=0)
    t0 = time.perf_counter()
    s = b.add(conf, gen=dict(nchains=10_000, chain_length=100, density=DENSITY, seed=2, pushoff_steps=PUSHOFF,
                             type_block=50))
    b.run(GRAPH_CAPTURE_STEPS)  # settles the push-off
    b.autotune(10)              # kernel variants and list buffer, as for the headline
    b.run(GRAPH_CAPTURE_STEPS)  # captures the step graph
    setup = time.perf_counter() - t0
    # the configured 20,000 steps, sampled every 1,000 (--drift-chunks of them)
    e, L, ms_total = [], [], 0.0
    for _ in range(args.drift_chunks):
        ms_total += _dev_run(fm, b, 1000)
        row = b.thermo(s)
        e.append(row.conserved)
        L.append(row.box_L)
    if args.timeline:
        kernel_timeline(b, args.timeline_steps, args.timeline)
    e = np.array(e)
    steps = np.arange(1, len(e) + 1) * 1000.0
    slope = float(np.polyfit(steps, e, 1)[0]) if len(e) > 1 else 0.0
    h = len(e) // 2
    slope2 = float(np.polyfit(steps[h:], e[h:], 1)[0]) if len(e) - h > 1 else 0.0
    n = 1_000_000
    return {"workload": "c2_1m_npt_two_types", "value": n * steps[-1] / (ms_total * 1e-3), "unit": "atom-steps/s",
            "steps": int(steps[-1]), "setup_s": setup, "box_L": [round(x, 4) for x in L],
            "conserved_drift": {"E0": float(e[0]), "slope_per_step": slope,
                                "relative_per_1e6_steps": slope * 1e6 / abs(e[0]),
                                "second_half_relative_per_1e6_steps": slope2 * 1e6 / abs(e[h]),
                                "samples": [round(float(x), 7) for x in e]}}


def wl_tiles(args, fm):
    """The warp-per-tile LJ (fmd_launch_lj_tiles over fmd_launch_tile_list's
    32-atom tile pairs at rc) against the per-atom Verlet-list LJ
    (fmd_launch_lj over fmd_launch_verlet_build's list at rc + skin), both in
    the reference's layout, on the same pushed-off one-type melt of
    --tiles-chains x 100 beads with atoms in 30-bit Morton order (compact
    tiles) and the 1-2 bonds excluded; each LJ pass timed alone with CUDA
    events over 20 launches after 3.  Pair work per atom: tile pairs x 32
    evaluated, against the list entries and the pairs inside rc."""
    import ctypes as C
    import torch
    lib = fm.lib()
    nch = args.tiles_chains
    b = fm.Batch(max_replicas=1, max_atoms=nch * 100 + 4096, device=0)
    s = b.add(_conf("nvt_langevin 1.0 1.0 1.0 7", 10 ** 7), gen=dict(nchains=nch, chain_length=100, density=DENSITY,
                                                                     seed=5, pushoff_steps=PUSHOFF))
    b.run(100)
    x, _, _ = b.state(s)
    L = b.info(s).box_L
    b.close()
    n = len(x)
    q = np.clip((x / L * 1024).astype(np.int64), 0, 1023)
    key = np.zeros(n, np.int64)
    for bit in range(10):
        for d in range(3):
            key |= ((q[:, d] >> bit) & 1) << (3 * bit + d)
    order = np.argsort(key, kind="stable")
    rank = np.empty_like(order)
    rank[order] = np.arange(n)
    x = x[order]
    k = np.arange(n) % 100
    first = np.nonzero(k < 99)[0]
    bonds = np.sort(rank[np.stack([first, first + 1], axis=1)], axis=1)
    per = [[] for _ in range(n)]
    for a_, c_ in bonds:
        per[a_].append(c_)
        per[c_].append(a_)
    xo = np.zeros(n + 1, np.int32)
    xo[1:] = np.cumsum([len(p_) for p_ in per])
    xl = np.array([j for p_ in per for j in sorted(p_)], np.int32)
    p4 = np.zeros((n, 4), np.float32)
    p4[:, :3] = x
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    pos, eo, el = dev(p4), dev(xo), dev(xl)
    rc, rcs = 2.5, 2.8
    Lf, invL = C.c_float(L), C.c_float(1.0 / L)
    ptr = lambda t: C.c_void_p(t.data_ptr())
    # tile list at rc
    T = (n + 31) // 32
    sb = C.c_size_t()
    lib.fmd_tile_list_scratch_bytes(C.c_int32(n), C.byref(sb))
    tscr = torch.empty(sb.value, dtype=torch.uint8, device="cuda")
    toff = torch.zeros(T + 1, dtype=torch.int32, device="cuda")
    npairs = C.c_int32()
    # count first (capacity 0: FMD_ERR_OVERFLOW with the count), then build
    st = lib.fmd_launch_tile_list(ptr(pos), C.c_int32(n), Lf, C.c_float(rc), ptr(toff), None, C.c_int32(0),
                                  C.byref(npairs), ptr(tscr), C.c_size_t(sb.value), None)
    assert st in (0, 5), st
    cap = max(1, npairs.value)
    tnbr = torch.zeros(cap, dtype=torch.int32, device="cuda")
    assert lib.fmd_launch_tile_list(ptr(pos), C.c_int32(n), Lf, C.c_float(rc), ptr(toff), ptr(tnbr), C.c_int32(cap),
                                    C.byref(npairs), ptr(tscr), C.c_size_t(sb.value), None) == 0
    # Verlet list at rc + skin
    vs = C.c_size_t()
    lib.fmd_verlet_scratch_bytes(C.c_int32(n), C.c_float(rcs), Lf, C.byref(vs))
    vscr = torch.empty(vs.value, dtype=torch.uint8, device="cuda")
    M = 128
    nbr = torch.zeros(M * n, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(n, dtype=torch.int32, device="cuda")
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert lib.fmd_launch_verlet_build(ptr(pos), C.c_int32(n), Lf, ptr(eo), ptr(el), C.c_float(rcs), C.c_int32(M),
                                       ptr(nbr), ptr(cnt), ptr(vscr), C.c_size_t(vs.value), ptr(flag), None) == 0
    torch.cuda.synchronize()
    assert int(flag.item()) == 0
    ljp = torch.tensor([1.0, 1.0], dtype=torch.float32, device="cuda")
    f_t = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    f_v = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    vir = torch.zeros(6, dtype=torch.float32, device="cuda")
    rc2 = C.c_float(rc * rc)

    def tiles():
        return lib.fmd_launch_lj_tiles(ptr(pos), ptr(f_t), ptr(vir), ptr(ljp), ptr(toff), ptr(tnbr), ptr(eo), ptr(el),
                                       C.c_int32(n), C.c_int32(1), rc2, Lf, invL, None)

    def verlet():
        return lib.fmd_launch_lj(ptr(pos), ptr(f_v), ptr(vir), ptr(ljp), ptr(nbr), ptr(cnt), C.c_int32(n),
                                 C.c_int32(1), rc2, Lf, invL, None)

    def timed(fn):
        for _ in range(3):
            assert fn() == 0
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(20):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 20

    ms_t, ms_v = timed(tiles), timed(verlet)
    ft, fv = f_t.cpu().numpy()[:, :3], f_v.cpu().numpy()[:, :3]
    diff = float(np.sqrt(np.mean(np.sum((ft - fv) ** 2, 1)) / np.mean(np.sum(fv ** 2, 1))))
    entries = float(cnt.float().mean().item())
    from oracle import pyoracle as po
    inside = 2.0 * len(po.pairs_brute(x, L, rc, bonds=bonds)[0]) / n if n <= 100_000 else None
    return {"workload": "lj_tiles_vs_verlet", "natoms": n, "box_L": L,
            "tile_pairs": int(npairs.value), "tile_pairs_per_tile": npairs.value / T,
            "pairs_evaluated_per_atom": {"tiles": 32.0 * npairs.value / T, "verlet_list_entries": entries,
                                         "inside_rc": inside},
            "ms_per_launch": {"lj_tiles": ms_t, "lj_verlet": ms_v}, "ns_per_atom": {"lj_tiles": ms_t * 1e6 / n,
                                                                                   "lj_verlet": ms_v * 1e6 / n},
            "force_rel_rms_tiles_vs_verlet": diff,
            "note": "reference layout (absolute FP32 positions, one thread per atom for the list form); the product "
                    "force kernel k_force works on the cell-offset layout and also evaluates the bonded terms"}


def c3_replicas():
    """The 256 uneven replicas of the batched case: (chains, chain length, T, seed)."""
    rng = np.random.default_rng(3)
    reps = []
    for i in range(256):
        cl = int(rng.choice([10, 20, 50, 100, 200]))
        beads = float(np.exp(rng.uniform(np.log(500), np.log(20000))))
        nc = max(1, int(round(beads / cl)))
        T = float(rng.uniform(0.5, 1.5))
        reps.append((nc, cl, T, i))
    return reps


def c3_assignment(fm, world):
    """Replicas of the batched case placed on `world` GPUs by atom count
    (greedy longest-processing-time bin-pack, the same on every rank)."""
    reps = c3_replicas()
    part, load = fm.partition_replicas([nc * cl for nc, cl, _, _ in reps], world)
    return reps, part, load


def wl_c3(args, fm, rank=0, world=1, local=0, dist=None):
    reps_all, part, load = c3_assignment(fm, world)
    mine = [k for k in range(len(reps_all)) if part[k] == rank]
    reps = [reps_all[k] for k in mine]
    b = fm.Batch(max_replicas=max(1, len(reps)), max_atoms=sum(nc * cl + 128 for nc, cl, _, _ in reps) + 4096,
                 device=local)
    slots = [b.add(_conf(f"nvt_langevin {T} {T} 1.0 {i}", 10 ** 7),
                   gen=dict(nchains=nc, chain_length=cl, density=DENSITY, seed=i, pushoff_steps=PUSHOFF))
             for nc, cl, T, i in reps]
    b.run(20)
    b.autotune(10)
    b.run(GRAPH_CAPTURE_STEPS)  # the autotuner's choices invalidate the step graph: capture it untimed
    k = 1000
    barrier(dist, local)
    ms = allmax(dist, _dev_run(fm, b, k), local)
    natoms_all = [nc * cl for nc, cl, _, _ in reps_all]
    batched = sum(natoms_all) * k / (ms * 1e-3)
    out = {"workload": "c3_256_uneven_replicas", "value": batched, "unit": "atom-steps/s", "steps": k,
           "total_atoms": int(sum(natoms_all)), "n_gpus": world,
           "placement": {"rule": "greedy longest-processing-time by atom count", "atoms_per_gpu": load.tolist(),
                         "replicas_per_gpu": np.bincount(part, minlength=world).tolist()}}
    if rank != 0:
        b.close()
        return out
    # plain FP64, one replica at a time: timed on 8 replicas spread over the
    # sizes, per-step cost interpolated in size for all 256
    natoms = [nc * cl for nc, cl, _, _ in reps]
    order = np.argsort(natoms)
    pick = [int(order[j]) for j in np.linspace(0, len(order) - 1, 8).astype(int)]
    sizes, per_step = [], []
    for j in pick:
        x, v, img = b.state(slots[j])
        nc, cl, T, i = reps[j]
        d = fm.generate_melt(nc, cl, density=DENSITY, seed=i)
        d.xyz, d.vel, d.image = x, v, img
        ps = fm.Simulation(_conf(f"nvt_langevin {T} {T} 1.0 {i}", 10 ** 7), desc=d, form=fm.FMD_FORM_PLAIN_FP64)
        ps.step(10)
        t0 = time.perf_counter()
        ps.step(200)
        per_step.append((time.perf_counter() - t0) / 200)
        sizes.append(natoms[j])
        ps.close()
    b.close()
    est = float(np.sum(np.interp(natoms_all, sizes, per_step))) * k
    plain = sum(natoms_all) * k / est
    out.update({"plain_fp64_one_at_a_time": plain, "speedup": batched / plain,
                "plain_sample": {"sizes": sizes, "s_per_step": per_step}})
    return out


def wl_c4(args, fm):
    rng = np.random.default_rng(4)
    srv = fm.Server(max_replicas=256, hbm_budget_gb=150.0, steps_per_round=200, device=0)
    rate, dur = 20.0, args.serve_seconds
    t_start = time.perf_counter()
    t_next, ids, work = 0.0, {}, {}
    while t_next < dur:
        now = time.perf_counter() - t_start
        if now < t_next:
            time.sleep(min(0.01, t_next - now))
            continue
        cl = int(rng.choice([20, 50, 100]))
        beads = float(np.exp(rng.uniform(np.log(1e3), np.log(1e5))))
        nc = max(1, int(round(beads / cl)))
        T = float(rng.uniform(0.8, 1.2))
        nsteps = int(np.exp(rng.uniform(np.log(1e3), np.log(5e4))) * args.serve_step_scale)
        rid = srv.submit(_conf(f"nvt_langevin {T} {T} 1.0 {len(ids) + 1}", max(nsteps, 100)),
                         dict(nchains=nc, chain_length=cl, density=DENSITY, seed=len(ids) + 1, pushoff_steps=1000))
        ids[rid] = time.perf_counter() - t_start
        work[rid] = nc * cl * max(nsteps, 100)
        t_next += float(rng.exponential(1.0 / rate))
    srv.drain(3600.0)
    res = srv.poll(len(ids) + 8)
    stats = srv.stats()
    timing = srv.timing()
    srv.close()
    lat = np.array([r.finish_time - r.submit_time for r in res if r.status == 0])
    failed = {}
    for r in res:
        if r.status != 0:
            failed[str(r.status)] = failed.get(str(r.status), 0) + 1
    span = max(r.finish_time for r in res) - min(r.submit_time for r in res)
    return {"workload": "c4_served_stream", "requests": len(ids), "completed": int(len(lat)),
            "failed_by_status": failed,
            "arrival_rate_per_s": rate, "duration_s": dur, "nsteps_scale": args.serve_step_scale,
            "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                          "mean": float(lat.mean())},
            "value": stats["atom_steps"] / span, "unit": "atom-steps/s",
            "offered_atom_steps_per_s": sum(work.values()) / dur, "server_thread": timing}


def wl_npt_drift(args, fm):
    """Nose-Hoover NPT conserved-quantity drift on a box already at P = 0:
    the C0 melt (3,000 beads, two types as in C2, npt_nh T = 1 Tdamp = 0.1,
    P = 0 Pdamp = 1.0, chain 3) relaxed for --npt-equil steps in the mixed
    form, then the same simulated time (--npt-time tau) at dt and dt / 2 in
    the mixed form, the plain FP64 form and the FP64 oracle, each from the
    relaxed state with a fresh chain and barostat.  Extended energy: KE + PE
    + chain terms + v_eps^2 / (2 W) + P V (P = 0).  A slope fitted to 100
    samples; reported per unit time and relative per 10^6 steps."""
    from oracle import pyoracle as po
    lj = ((0, 0, 1.0, 1.0), (1, 1, 1.0, 1.0), (0, 1, 0.9, 1.0))
    ens = "npt_nh 1.0 1.0 0.1 0.0 0.0 1.0 3"
    pre = fm.Batch(max_replicas=1, max_atoms=8192, device=0)
    s0 = pre.add(_conf(ens, 10 ** 8, ntypes=2, lj=lj),
                 gen=dict(nchains=30, chain_length=100, density=DENSITY, seed=42, pushoff_steps=PUSHOFF,
                          type_block=50))
    pre.run(args.npt_equil)
    x0, v0, i0 = pre.state(s0)
    L0 = pre.info(s0).box_L
    pre.close()
    d = fm.generate_melt(30, 100, density=DENSITY, seed=42, type_block=50)
    d.xyz, d.vel, d.image, d.box_L = x0, v0, i0, L0
    tab = np.ones((2, 2, 2))
    tab[0, 1, 0] = tab[1, 0, 0] = 0.9
    out = {"workload": "npt_drift_c0_two_types", "relaxed_box_L": L0, "equil_steps": args.npt_equil,
           "sim_time_tau": args.npt_time, "runs": []}
    n = len(d.type)
    for dt in (0.001, 0.0005):
        nsteps = int(round(args.npt_time / dt))
        every = max(1, nsteps // 100)
        conf = (f"ntypes 2\nrc 2.5\nskin 0.3\ndt {dt}\nnsteps {10 ** 8}\n{ens}\n"
                "bond_type 0 30.0 1.5 1.0 1.0\nangle_type 0 5.0 180.0\n"
                + "".join(f"lj {a} {b} {e} {g}\n" for a, b, e, g in lj))
        series = {}
        for form, name in ((fm.FMD_FORM_MIXED, "mixed"), (fm.FMD_FORM_PLAIN_FP64, "plain_fp64")):
            sim = fm.Simulation(conf, desc=d, form=form)
            e = []
            for _ in range(nsteps // every):
                sim.step(every)
                e.append(sim.thermo().conserved)
            sim.close()
            series[name] = np.array(e)
        osys = po.System(xyz=x0, L=L0, type=d.type, mass=np.ones(2), lj=tab, bonds=d.bonds,
                         bond_type=np.zeros(len(d.bonds), np.int32), fene=np.array([[30.0, 1.5, 1.0, 1.0]]),
                         angles=d.angles, angle_type=np.zeros(len(d.angles), np.int32),
                         angle_p=np.array([[5.0, np.pi]]), mol=d.mol, vel=v0, image=i0)
        osim = po.Sim(osys, ensemble="npt_nh", dt=dt, T=(1.0, 1.0, 0.1), P=(0.0, 0.0, 1.0), chain=3, nsteps=10 ** 8)
        e, em = [], []
        for _ in range(nsteps // every):
            osim.step(every)
            e.append(osim.conserved() / n)
            em.append(osim.conserved_mtk() / n)
        series["fp64_oracle"] = np.array(e)
        # the same run's extended energy with the work of the barostat force's
        # kinetic term (3 / N_f) 2 KE, which the reference's barostat omits
        series["fp64_oracle_with_mtk_term"] = np.array(em)
        t = np.arange(1, nsteps // every + 1) * every * dt
        row = {"dt": dt, "steps": nsteps}
        for name, e in series.items():
            slope = float(np.polyfit(t, e, 1)[0])  # per atom per tau
            row[name] = {"E0": float(e[0]), "slope_per_tau": slope,
                         "relative_per_1e6_steps": slope * dt * 1e6 / abs(e[0]),
                         "rms_fluctuation": float(np.std(e - np.polyval(np.polyfit(t, e, 1), t)))}
        out["runs"].append(row)
    return out


def cutoff_jump_energy(x, L, lj, tb, rc=2.5):
    """-sum over non-bonded pairs within rc of U(rc) (the LJ energy at the
    cutoff, per pair type) at positions x in a box of edge L (chains of
    CHAIN_LEN beads, types in blocks of tb along each chain): what shifting
    the truncated LJ to zero at rc would add to the potential energy."""
    from oracle import pyoracle as po
    n = len(x)
    k = np.arange(n) % CHAIN_LEN
    first = np.nonzero(k < CHAIN_LEN - 1)[0]
    bonds = np.stack([first, first + 1], axis=1)
    nbr, cnt, _ = po.verlet_lists(x, L, rc, bonds=bonds, max_nbr=256)
    typ = (k // tb) % 2 if tb > 0 else np.zeros(n, np.int64)
    eps = np.ones((2, 2))
    for a, c, e, _ in lj:
        eps[a, c] = eps[c, a] = e
    src = np.repeat(np.arange(n), cnt)
    dst = np.concatenate([nbr[i, :cnt[i]] for i in range(n)]) if n else np.zeros(0, np.int64)
    sr6 = (1.0 / rc) ** 6
    u_rc = 4.0 * eps[typ[src], typ[dst]] * (sr6 * sr6 - sr6)
    return -0.5 * float(np.sum(u_rc))   # each pair listed from both ends


def wl_drift(args, fm):
    """Conserved-quantity drift of the Nose-Hoover ensembles, batched for
    statistics: --drift-reps replicas of 30,000 beads each (seeded melts,
    pushed off, relaxed --drift-relax steps in the same ensemble), then
    --drift-run steps sampled 100 times; a line per replica, relative slope
    per 10^6 steps, mean and standard error over the replicas.  NVT (nvt_nh
    T = 1, Tdamp = 0.5) at dt and dt / 2 (the same simulated time), NPT
    (two types as C2, npt_nh T = 1 Tdamp = 0.1, P = 0 Pdamp = 1, chain 3) at
    dt, and the plain FP64 form on two NVT replicas for comparison."""
    lj2 = ((0, 0, 1.0, 1.0), (1, 1, 1.0, 1.0), (0, 1, 0.9, 1.0))
    npt = "npt_nh 1.0 1.0 0.1 0.0 0.0 1.0 3"
    cases = [("nvt", "nvt_nh 1.0 1.0 0.5 3", 1, ((0, 0, 1.0, 1.0),), 0, 0.001),
             ("nvt", "nvt_nh 1.0 1.0 0.5 3", 1, ((0, 0, 1.0, 1.0),), 0, 0.0005),
             ("npt", npt, 2, lj2, 50, 0.001),
             ("npt", npt, 2, lj2, 50, 0.0005),
             # the same with the chain's upper accelerations carried between half steps
             ("nptc", npt + "\nnh_chain_carry 1", 2, lj2, 50, 0.001),
             ("nptc", npt + "\nnh_chain_carry 1", 2, lj2, 50, 0.0005)]
    wanted = set(args.drift_cases.split(","))
    cases = [c for c in cases if f"{c[0]}{c[5]}" in wanted or c[0] in wanted]
    out = {"workload": "nh_drift_batched", "replicas": args.drift_reps, "beads_per_replica": NCHAINS * CHAIN_LEN,
           "cases": []}

    def conf_for(ens, nt, lj, dt):
        return (f"ntypes {nt}\nrc 2.5\nskin 0.3\ndt {dt}\nnsteps {10 ** 9}\n{ens}\n"
                "bond_type 0 30.0 1.5 1.0 1.0\nangle_type 0 5.0 180.0\n"
                + "".join(f"lj {a} {b_} {e} {g}\n" for a, b_, e, g in lj))

    def slopes(series, t):
        rel = [np.polyfit(t, e, 1)[0] / abs(e[0]) for e in series.T]
        return np.array(rel)

    for name, ens, nt, lj, tb, dt in cases:
        b = fm.Batch(max_replicas=args.drift_reps, max_atoms=args.drift_reps * 30080 + 4096, device=0)
        slots = [b.add(conf_for(ens, nt, lj, dt), gen=dict(nchains=NCHAINS, chain_length=CHAIN_LEN, density=DENSITY,
                                                           seed=500 + r, pushoff_steps=PUSHOFF, type_block=tb))
                 for r in range(args.drift_reps)]
        b.run(int(args.drift_relax * 0.001 / dt))
        nrun = int(args.drift_run * 0.001 / dt)
        every = max(1, nrun // 100)
        e = np.zeros((nrun // every, len(slots)))
        nshift = min(args.drift_shift_check, len(slots)) if name.startswith("npt") else 0
        es = np.zeros((nrun // every, nshift))
        vol = np.zeros((nrun // every, len(slots)))
        for k in range(nrun // every):
            b.run(every)
            for j, s in enumerate(slots):
                e[k, j] = b.thermo(s).conserved
                vol[k, j] = b.info(s).box_L ** 3
            for j in range(nshift):
                es[k, j] = e[k, j] + cutoff_jump_energy(*b.force_frame(slots[j]), lj, tb) / (NCHAINS * CHAIN_LEN)
        t = np.arange(1, nrun // every + 1) * float(every)
        rel = slopes(e, t) * 1e6
        row = {"ensemble": ens.replace("\n", "; "), "dt": dt, "steps": nrun, "relative_per_1e6_steps": float(rel.mean()),
               "stderr": float(rel.std(ddof=1) / np.sqrt(len(rel))), "per_replica": rel.tolist(),
               "relative_per_tau": float(rel.mean() / (1e6 * dt))}
        if name.startswith("npt"):
            vrel = slopes(vol, t) * 1e6
            row["volume_relative_per_1e6_steps"] = {"mean": float(vrel.mean()),
                                                    "stderr": float(vrel.std(ddof=1) / np.sqrt(len(vrel)))}
        if nshift:
            rs = slopes(es, t) * 1e6
            row["with_shifted_lj_energy"] = {
                "relative_per_1e6_steps": rs.tolist(), "same_replicas_unshifted": rel[:nshift].tolist(),
                "how": "extended energy with the LJ energy of every pair within rc shifted by -U(rc) (the "
                       "forces are unchanged): the jump U(rc) a pair carries across the cutoff, which the "
                       "instantaneous virial (hence the barostat) does not see, is taken out"}
        if dt == 0.001 and args.drift_plain > 0:
            # the plain FP64 form from the relaxed states of the first replicas
            pl, pls, plv = [], [], []
            for s in slots[:args.drift_plain]:
                x, v, img = b.state(s)
                d = fm.generate_melt(NCHAINS, CHAIN_LEN, density=DENSITY, seed=0, type_block=tb)
                d.xyz, d.vel, d.image, d.box_L = x, v, img, b.info(s).box_L
                ps = fm.Simulation(conf_for(ens, nt, lj, dt), desc=d, form=fm.FMD_FORM_PLAIN_FP64)
                ee, es_, vv = [], [], []
                for _ in range(nrun // every):
                    ps.step(every)
                    th = ps.thermo()
                    ee.append(th.conserved)
                    vv.append(th.box_L ** 3)
                    if name.startswith("npt"):
                        es_.append(th.conserved + cutoff_jump_energy(ps.state()[0], th.box_L, lj, tb)
                                   / (NCHAINS * CHAIN_LEN))
                ps.close()
                pl.append(ee)
                pls.append(es_)
                plv.append(vv)
            prel = slopes(np.array(pl).T, t) * 1e6
            row["plain_fp64"] = {"relative_per_1e6_steps": prel.tolist(), "replicas": len(pl),
                                 "volume_relative_per_1e6_steps": (slopes(np.array(plv).T, t) * 1e6).tolist(),
                                 "note": "from the mixed replicas' relaxed states"}
            if name.startswith("npt"):
                row["plain_fp64"]["with_shifted_lj_energy"] = (slopes(np.array(pls).T, t) * 1e6).tolist()
        b.close()
        out["cases"].append(row)
    return out


WORKLOADS = {"c0": wl_c0, "c1": wl_c1, "c2": wl_c2, "c3": wl_c3, "c4": wl_c4, "npt_drift": wl_npt_drift,
             "drift": wl_drift, "tiles": wl_tiles}


def kernel_timeline(b, steps, path):
    """Kernel timeline of `steps` graph steps, from the CUDA activity records
    the torch profiler collects over CUPTI (kernels inside the step graph's
    conditional nodes included): per-kernel totals, step durations (k_pre to
    k_pre) and the kernels of the first step with a rebuild.  Written to path
    as text; the run's timing is not taken from it."""
    import collections
    import tempfile

    import numpy as np
    import torch
    from torch.profiler import ProfilerActivity, profile

    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        b.run(steps)
        torch.cuda.synchronize()
    with tempfile.TemporaryDirectory() as td:
        tp = os.path.join(td, "trace.json")
        prof.export_chrome_trace(tp)
        with open(tp) as f:
            ev = [e for e in json.load(f)["traceEvents"] if e.get("cat") == "kernel"]
    ev.sort(key=lambda e: e["ts"])

    def short(n):
        return n.replace("void fmd::mixed::", "").replace("fmd::mixed::", "").split("(")[0]

    tot, cnt = collections.defaultdict(float), collections.Counter()
    for e in ev:
        tot[short(e["name"])] += e["dur"]
        cnt[short(e["name"])] += 1
    pre = [e for e in ev if short(e["name"]).startswith("k_pre")]
    dur = np.array([pre[i + 1]["ts"] - pre[i]["ts"] for i in range(len(pre) - 1)])
    out = [f"kernels {len(ev)}, steps {len(dur)}: step us mean {dur.mean():.1f}, median {np.median(dur):.1f}, "
           f"p90 {np.percentile(dur, 90):.1f}, max {dur.max():.1f}", "",
           "| kernel | launches | total us | mean us |", "|---|---|---|---|"]
    for k, v in sorted(tot.items(), key=lambda x: -x[1]):
        out.append(f"| `{k}` | {cnt[k]} | {v:.1f} | {v / cnt[k]:.2f} |")
    # steps by what ran beside the force kernel: a rebuild, a list filter only, nothing
    cls = collections.defaultdict(list)
    for i in range(len(pre) - 1):
        a, z = pre[i]["ts"], pre[i + 1]["ts"]
        names = [short(e["name"]) for e in ev if a <= e["ts"] < z]
        force = sum(e["dur"] for e in ev if a <= e["ts"] < z and short(e["name"]).startswith("k_force<"))
        kind = ("rebuild" if any(n.startswith("k_neighbors") for n in names)
                else "filter only" if any(n.startswith(("k_prune", "k_force_rb")) for n in names) else "neither")
        cls[kind].append((z - a, force))
    # rebuild steps by the list kernel's duration (grows with the atoms rebuilt)
    rb = []
    for i in range(len(pre) - 1):
        a, z = pre[i]["ts"], pre[i + 1]["ts"]
        nb = sum(e["dur"] for e in ev if a <= e["ts"] < z and short(e["name"]).startswith("k_neighbors"))
        if nb > 0:
            rb.append((nb, z - a))
    rb_lines = []
    if len(rb) >= 8:
        rb = np.array(sorted(rb))
        rb_lines = ["", "| rebuild steps by list-kernel time | steps | list kernel us mean | step us mean |",
                    "|---|---|---|---|"]
        for q, part in enumerate(np.array_split(rb, 4)):
            rb_lines.append(f"| quartile {q + 1} | {len(part)} | {part[:, 0].mean():.1f} | {part[:, 1].mean():.1f} |")
    out += ["", "| step kind | steps | step us mean | step us median | k_force us mean |", "|---|---|---|---|---|"]
    for kind in ("neither", "filter only", "rebuild"):
        if cls[kind]:
            v = np.array(cls[kind])
            out.append(f"| {kind} | {len(v)} | {v[:, 0].mean():.1f} | {np.median(v[:, 0]):.1f} | {v[:, 1].mean():.1f} |")
    out += rb_lines
    for i in range(len(pre) - 1):
        a, z = pre[i]["ts"], pre[i + 1]["ts"]
        win = [e for e in ev if a <= e["ts"] < z]
        if any("k_neighbors" in e["name"] for e in win):
            out += ["", f"first step with a rebuild ({z - a:.1f} us; start offset, duration, stream, kernel):", ""]
            out += [f"    {e['ts'] - a:8.1f} +{e['dur']:7.1f}  s{e['args'].get('stream')}  {short(e['name'])}"
                    for e in win]
            break
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


def graph_steps_for(steps, requested):
    """Steps per CUDA-graph launch: the largest divisor of the timed steps not
    above the requested length, so every timed step is a graph replay
    (requested < 0: direct launches, for kernel profilers)."""
    if requested < 0:
        return requested
    cap = max(1, min(requested or 50, steps))
    return max(d for d in range(1, cap + 1) if steps % d == 0)


def _kg_oracle_system(po, x, L, natoms):
    nch = natoms // CHAIN_LEN
    ids = np.arange(natoms, dtype=np.int32).reshape(nch, CHAIN_LEN)
    bonds = np.stack([ids[:, :-1].ravel(), ids[:, 1:].ravel()], axis=1).astype(np.int32)
    angles = np.stack([ids[:, :-2].ravel(), ids[:, 1:-1].ravel(), ids[:, 2:].ravel()], axis=1).astype(np.int32)
    return po.System(xyz=x, L=L, type=np.zeros(natoms, np.int32), mass=np.ones(1), lj=np.ones((1, 1, 2)),
                     bonds=bonds, bond_type=np.zeros(len(bonds), np.int32), fene=np.array([[30.0, 1.5, 1.0, 1.0]]),
                     angles=angles, angle_type=np.zeros(len(angles), np.int32), angle_p=np.array([[5.0, np.pi]]),
                     mol=np.repeat(np.arange(1, nch + 1, dtype=np.int32), CHAIN_LEN))


def force_rms_vs_oracle(fm, b, slots):
    """Force RMS error relative to the FP64 oracle of the benchmarked
    replicas at the end of the timed run (the forces the kernels produce
    for the current positions, read in FP64)."""
    from oracle import pyoracle as po
    errs = []
    for s in slots:
        x, _, _ = b.state(s)
        f, _, _ = b.forces(s)
        fo, _, _ = po.forces(_kg_oracle_system(po, x, b.info(s).box_L, len(x)))
        errs.append(float(np.sqrt(np.mean((f - fo) ** 2)) / np.sqrt(np.mean(fo ** 2))))
    return {"max": max(errs), "per_replica": errs, "replicas": len(errs), "tolerance": 1e-5,
            "how": "mixed-form forces of the timed replicas' final states vs the FP64 oracle on the same positions"}


def nvt_drift(fm, b, slots, steps, device):
    """Nose-Hoover NVT conserved-quantity drift (extended energy per atom,
    thermostat terms included) of the benchmarked replicas' final states run
    under nvt_nh T = 1, Tdamp = 0.5, chain 3 for `steps` steps: a line fitted
    per replica, relative slope per 10^6 steps, mean and standard error over
    the replicas."""
    conf = ("ntypes 1\nrc 2.5\nskin 0.3\ndt 0.001\nnsteps 100000000\nnvt_nh 1.0 1.0 0.5 3\n"
            "lj 0 0 1.0 1.0\nbond_type 0 30.0 1.5 1.0 1.0\nangle_type 0 5.0 180.0\n")
    nb = fm.Batch(max_replicas=len(slots), max_atoms=len(slots) * 30080 + 4096, device=device)
    ns = []
    for s in slots:
        x, v, img = b.state(s)
        d = fm.generate_melt(NCHAINS, CHAIN_LEN, density=DENSITY, seed=0)
        d.xyz, d.vel, d.image = x, v, img
        ns.append(nb.add(conf, desc=d))
    nb.run(50)
    samples = 50
    chunk = max(50, steps // samples // 50 * 50)
    e = np.zeros((samples, len(ns)))
    for k in range(samples):
        nb.run(chunk)
        for j, s in enumerate(ns):
            e[k, j] = nb.thermo(s).conserved
    nb.close()
    t = np.arange(1, samples + 1) * float(chunk)
    rel = np.array([np.polyfit(t, e[:, j], 1)[0] * 1e6 / abs(e[0, j]) for j in range(len(ns))])
    return {"relative_per_1e6_steps": float(rel.mean()),
            "stderr": float(rel.std(ddof=1) / np.sqrt(len(rel))) if len(rel) > 1 else None,
            "per_replica": rel.tolist(), "steps": int(t[-1]), "replicas": len(ns), "target": 1e-4,
            "ensemble": "nvt_nh T=1 Tdamp=0.5 chain 3, from the timed replicas' final states"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=100)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--replicas", type=int, default=64)
    ap.add_argument("--no-extras", action="store_true", help="skip e2e / plain / CPU / reference-GPU legs")
    ap.add_argument("--ref-gpu-steps", type=int, default=5000, help="steps of the reference GPU datapoint")
    ap.add_argument("--graph-steps", type=int, default=50,
                    help="longest CUDA graph (steps per launch; the largest divisor of --steps not above it is "
                         "used); < 0 launches every step directly (for kernel profilers)")
    ap.add_argument("--drift-steps", type=int, default=100_000,
                    help="NVT conserved-quantity drift leg: steps (0 skips it)")
    ap.add_argument("--workload", default="headline", choices=["headline"] + sorted(WORKLOADS),
                    help="headline = the 64 x 30K benchmark; c0..c4 = the reported cases (one GPU)")
    ap.add_argument("--timeline", default="", help="after the timed run, write a kernel timeline of "
                    "--timeline-steps graph steps (torch profiler / CUPTI) to this file")
    ap.add_argument("--timeline-steps", type=int, default=200)
    ap.add_argument("--drift-chunks", type=int, default=20, help="c2: conserved-quantity samples")
    ap.add_argument("--c1-drift-steps", type=int, default=200_000, help="c1: NVT steps of the drift fit")
    ap.add_argument("--c1-stat-steps", type=int, default=20_000, help="c1: steps of the <T>, <P>, Rg comparison")
    ap.add_argument("--npt-equil", type=int, default=20_000, help="npt_drift: relaxation steps at P = 0")
    ap.add_argument("--drift-reps", type=int, default=16, help="drift: replicas per case")
    ap.add_argument("--drift-cases", default="nvt,npt,nptc",
                    help="drift: nvt, npt, nptc (NPT, chain accelerations carried), or nvt0.001 / npt0.0005 ...")
    ap.add_argument("--drift-plain", type=int, default=2, help="drift: plain FP64 replicas at dt = 0.001")
    ap.add_argument("--drift-shift-check", type=int, default=4,
                    help="drift: NPT replicas whose extended energy is also reported with the LJ shifted at rc")
    ap.add_argument("--drift-relax", type=int, default=20_000, help="drift: relaxation steps (at dt = 0.001)")
    ap.add_argument("--tiles-chains", type=int, default=300, help="tiles: chains of 100 beads in the melt")
    ap.add_argument("--force-variant", type=int, default=-1,
                    help="after the autotuner, pin this force-kernel variant (default: its pick)")
    ap.add_argument("--drift-run", type=int, default=200_000, help="drift: measured steps (at dt = 0.001)")
    ap.add_argument("--npt-time", type=float, default=20.0, help="npt_drift: simulated time per run (tau)")
    ap.add_argument("--serve-seconds", type=float, default=30.0, help="c4: arrival window")
    ap.add_argument("--serve-step-scale", type=float, default=0.25, help="c4: scale of the requests' nsteps")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    rank, world, local, dist = dist_setup(args.gpus)
    if args.workload != "headline" and args.impl == "ours":
        import fastmd_b200 as fm
        if args.workload == "c3":
            res = wl_c3(args, fm, rank, world, local, dist)
        elif rank == 0:
            res = WORKLOADS[args.workload](args, fm)
        else:
            res = None
        if rank == 0:
            print(json.dumps(res), flush=True)
        if dist is not None:
            barrier(dist, local)
            dist.destroy_process_group()
        return
    if args.impl == "reference":
        run_reference(args, rank, world, local, dist)
        if dist is not None:
            dist.destroy_process_group()
        return

    import fastmd_b200 as fm

    R = args.replicas
    gsteps = graph_steps_for(args.steps, args.graph_steps)
    b = fm.Batch(max_replicas=R, max_atoms=R * 30080 + 4096, hbm_budget_gb=150.0, graph_steps=gsteps,
                 device=local)
    t_setup = time.perf_counter()
    slots = []
    for r in range(R):
        seed = r + 1000 * rank
        slots.append(b.add(run_conf(seed), gen=dict(nchains=NCHAINS, chain_length=CHAIN_LEN, density=DENSITY,
                                                    seed=seed, pushoff_steps=PUSHOFF)))
    t_setup = time.perf_counter() - t_setup
    natoms = sum(b.info(s).natoms for s in slots)
    lib = fm.lib()

    # warm-up, then the force-kernel autotuner on the live state
    b.run(args.warmup)
    variant, variant_ms = b.autotune(20)
    if args.force_variant >= 0:  # a pinned variant (profiling one variant)
        b.set_variants(args.force_variant, -1)
        variant = args.force_variant
    # The autotuner's choices invalidate the step graph: replay one graph's
    # worth of steps untimed so that its capture (host work while the device
    # idles) is not inside the timed region.  The graph length divides the
    # timed steps, so every timed step is a graph replay.
    b.run(max(3, gsteps))
    barrier(dist, local)
    counts0 = b.launch_counts()
    rebuilds0 = sum(b.info(s).rebuilds for s in slots)
    with ClockSampler(local) as clk:
        profiler_range(True)
        lib.fmd_batch_mark(b._h, 0)
        b.run(args.steps)
        lib.fmd_batch_mark(b._h, 1)
        profiler_range(False)
        import ctypes as C
        ms = C.c_double()
        lib.fmd_batch_elapsed_ms(b._h, C.byref(ms))
    counts1 = b.launch_counts()
    rebuilds1 = sum(b.info(s).rebuilds for s in slots)
    barrier(dist, local)
    dev_ms = allmax(dist, ms.value, local)
    total_atoms = allmax(dist, float(natoms), local) * world  # equal per rank
    value = total_atoms * args.steps / (dev_ms * 1e-3)
    for s in slots:
        st = b.info(s).status_word
        if st != 0:
            raise SystemExit(f"replica {s} faulted with status {st}")

    line = {
        "metric": METRIC, "value": value, "unit": "atom-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 forces / f64 reductions",
        "data": "synthetic (seeded random-walk melts, 2,000-step capped push-off)",
        "config": headline_config(world, gsteps, R),
        "form": "mixed (FP32 cell-offset forces, FP64 reductions)",
        "path": "graph" if gsteps > 0 else "direct launches",
        "graph_steps": gsteps,
    }

    if rank == 0:
        line["clocks"] = clk.summary()
        launched = {k: counts1[k] - counts0[k] for k in counts0}
        line["gpu_launches"] = int(sum(launched.values()))
        nf = b.variants()[2]
        line["autotune"] = {"force_variant": variant, "neighbor_variant": int(variant_ms[nf + 3]),
                            "ms_per_full_rebuild": {"ballot m8": round(float(variant_ms[nf]), 4),
                                                    "rows m6": round(float(variant_ms[nf + 1]), 4),
                                                    "ballot m6": round(float(variant_ms[nf + 2]), 4)},
                            "ms_per_variant": [round(float(x), 4) for x in variant_ms[:nf]],
                            "variants": FORCE_VARIANTS[:nf],
                            "legend": "m = min blocks per SM, k = batches of 4 list entries per compensated add, "
                                      "t3 = shift from the 125-entry 3D table, a5 = per-axis 5-value table, "
                                      "x2 = pairs two at a time in packed FP32x2 arithmetic, l2 / l4 = two / "
                                      "four lanes per atom (one otherwise), r2 / r3 / r4 = list rows staged through "
                                      "a shared-memory ring 1 / 2 / 3 batches ahead by asynchronous copies (otherwise "
                                      "the next batch's list words are loaded ahead into registers)"}
        line["launches_by_kernel"] = launched
        line["replica_rebuilds"] = {"total": int(rebuilds1 - rebuilds0),
                                    "mean_interval_steps": args.steps * len(slots) / max(1, rebuilds1 - rebuilds0),
                                    "policy": "displacement trigger only (forced cadence lifted by the "
                                              "autotuner; the reference forces one every 20 steps)",
                                    "list_buffer": round(b.list_buffer(slots[0]), 4),
                                    "list_buffer_policy": "run.conf skin 0.3 widened by the autotuner to the "
                                                          "cell edge minus rc (replicas with a pruned list; the "
                                                          "forces walk the pairs within rc + 0.12 either way)"}
        # ---- roofline of the force kernel
        entries = C.c_int64()
        mx = C.c_int32()
        lib.fmd_batch_list_stats(b._h, C.byref(entries), C.byref(mx))
        fms = C.c_double()
        lib.fmd_batch_time_force(b._h, 50, C.byref(fms))
        per_atom_fixed = 88  # pos_i, pos_j set, force write, list count, bonded count, bond and angle tables
        alg_bytes = natoms * per_atom_fixed + 4 * entries.value
        achieved = alg_bytes / (fms.value * 1e-3) / 1e9
        peak, kind = measured_peaks()
        traffic = force_profile_traffic()
        line["roofline"] = {"kernel": "k_force (LJ + FENE + angle, gathered)", "bound": "hbm", "achieved": achieved,
                            "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_kind": kind,
                            "traffic": traffic, "alg_bytes_per_launch": alg_bytes,
                            "ms_per_launch": fms.value, "mean_neighbors": entries.value / natoms,
                            "max_neighbors": mx.value}
        if args.timeline:
            kernel_timeline(b, args.timeline_steps, args.timeline)
        if not args.no_extras:
            # ---- end to end through the public C API: run in thermo-sized
            # chunks (100 steps) and read every replica's thermo row.
            chunk = 100 if gsteps <= 0 or 100 % gsteps == 0 else gsteps * -(-100 // gsteps)
            nchunks = max(1, args.steps // chunk)
            # start on a thermo step, as a run printing every 100 steps does
            lead = (-b.info(slots[0]).step) % chunk
            if lead:
                b.run(lead)
            t0 = time.perf_counter()
            lib.fmd_batch_mark(b._h, 0)
            rows = 0
            for _ in range(nchunks):
                b.run(chunk)
                for s in slots:
                    b.thermo(s)
                    rows += 1
            lib.fmd_batch_mark(b._h, 1)
            wall = time.perf_counter() - t0
            e2e_ms = C.c_double()
            lib.fmd_batch_elapsed_ms(b._h, C.byref(e2e_ms))
            e2e_s = max(wall, e2e_ms.value * 1e-3)
            rep_bytes = 3072 * R  # replica table up + down per run() call
            line["e2e"] = {"value": natoms * chunk * nchunks / e2e_s, "unit": "atom-steps/s",
                           "h2d_bytes_per_step": rep_bytes / chunk, "d2h_bytes_per_step": rep_bytes / chunk,
                           "how": "fmd_batch_run(100) + fmd_batch_thermo for every replica per chunk, wall clock"}
            # ---- plain FP64 form, one 30K replica at a time (host-driven like the reference)
            try:
                x, v, img = b.state(slots[0])
                d = fm.generate_melt(NCHAINS, CHAIN_LEN, density=DENSITY, seed=0)
                d.xyz, d.vel, d.image = x, v, img
                ps = fm.Simulation(run_conf(0), desc=d, form=fm.FMD_FORM_PLAIN_FP64)
                ps.step(20)
                k = 200
                t0 = time.perf_counter()
                ps.step(k)
                pt = time.perf_counter() - t0
                line["plain_fp64_one_replica"] = {"value": len(d.type) * k / pt, "unit": "atom-steps/s",
                                                  "steps": k, "note": "one 30K replica, host wall clock"}
                line["speedup_vs_plain_fp64"] = value / line["plain_fp64_one_replica"]["value"]
                ps.close()
            except Exception as e:  # reported, not fatal
                line["plain_fp64_one_replica"] = {"error": str(e)}
            # ---- the reference's own FP32 GPU engine on one replica
            try:
                x, v, img = b.state(slots[0])
                line["reference_gpu_fp32_one_replica"] = reference_gpu_leg(fm, x, v, img, args.ref_gpu_steps)
            except Exception as e:
                line["reference_gpu_fp32_one_replica"] = {"unavailable": str(e)}
            # ---- CPU baseline (FP64 oracle port on the host cores)
            try:
                x, v, img = b.state(slots[0])
                d = fm.generate_melt(NCHAINS, CHAIN_LEN, density=DENSITY, seed=0)
                desc = dict(xyz=x, L=d.box_L, type=d.type, bonds=d.bonds, angles=d.angles, mol=d.mol, vel=v,
                            image=img)
                cv, cores, sample = cpu_oracle_rate(desc, seconds=12.0)
                line["cpu_baseline"] = {"value": cv, "unit": "atom-steps/s", "cores": cores, "kind": "port",
                                        "sample": sample}
            except Exception as e:
                line["cpu_baseline"] = {"error": str(e)}
            # ---- force RMS error of the timed state against the FP64 oracle
            try:
                line["force_rms_vs_oracle"] = force_rms_vs_oracle(fm, b, slots[:2])
            except Exception as e:
                line["force_rms_vs_oracle"] = {"error": str(e)}
            # ---- Nose-Hoover conserved-quantity drift from the timed states
            if args.drift_steps > 0:
                try:
                    line["nvt_drift"] = nvt_drift(fm, b, slots[:8], args.drift_steps, local)
                except Exception as e:
                    line["nvt_drift"] = {"error": str(e)}
        line["setup_s"] = t_setup
        print(json.dumps(line), flush=True)
    b.close()
    if dist is not None:
        barrier(dist, local)
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
