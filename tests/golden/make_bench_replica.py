"""Generate kg30k_replica0.npz: replica 0 of the benchmark workload (300
chains x 100 beads, density 0.85, seed 0) after its 2,000-step capped-force
push-off, as `bench.py` creates it on the GPU.

`bench.py --impl reference` times the FP64 CPU oracle stepping this state, so
that its input is the benchmark's own replica without loading the library
(the push-off runs on the device).  Positions and velocities are stored in
FP32 (the push-off is a preparation step; the timed stepping starts from these
values), image flags as int16.  Topology is implied: linear chains of 100
beads in atom order (bonds i, i+1 and angles i, i+1, i+2 inside a chain).

Run on a machine with a GPU, from the repository root:

    python tests/golden/make_bench_replica.py [out.npz]
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

NCHAINS, CHAIN_LEN, DENSITY, PUSHOFF, SEED = 300, 100, 0.85, 2000, 0


def main():
    import fastmd_b200 as fm

    out = sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.path.dirname(__file__), "kg30k_replica0.npz")
    conf = (f"ntypes 1\nrc 2.5\nskin 0.3\ndt 0.001\nnsteps 10000000\nnvt_langevin 1.0 1.0 1.0 {SEED}\n"
            "lj 0 0 1.0 1.0\nbond_type 0 30.0 1.5 1.0 1.0\nangle_type 0 5.0 180.0\nthermo 1 100 thermo.dat\n")
    b = fm.Batch(max_replicas=1, max_atoms=30080 + 4096, device=0)
    s = b.add(conf, gen=dict(nchains=NCHAINS, chain_length=CHAIN_LEN, density=DENSITY, seed=SEED,
                             pushoff_steps=PUSHOFF))
    b.run(0)  # completes the push-off
    x, v, img = b.state(s)
    L = b.info(s).box_L
    b.close()
    np.savez_compressed(out, xyz=x.astype(np.float32), vel=v.astype(np.float32), image=img.astype(np.int16),
                        box_L=np.array([L]), nchains=np.array([NCHAINS]), chain_length=np.array([CHAIN_LEN]),
                        seed=np.array([SEED]), pushoff_steps=np.array([PUSHOFF]))
    print(f"wrote {out}: {len(x)} beads, L = {L:.6f}")


if __name__ == "__main__":
    main()
