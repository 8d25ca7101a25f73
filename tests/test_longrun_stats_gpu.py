"""Long-run statistics of the mixed form against the FP64 oracle (C0).

The third oracle check: the C0 melt (30 chains x 100 beads, density 0.85,
pushed off) run for 5,000 steps of Langevin T = 1 (Tdamp = 1, seed 42,
dt = 0.001) in the mixed form on the GPU and in the FP64 CPU oracle from the
same state; <T>, <P> (the pressure tensor's trace / 3) and <Rg> sampled every
25 steps after a 500-step settling window must agree within four combined
standard errors, each from 10 block averages (the series are correlated).
The two runs share the noise stream (same Philox keys), so they stay close
for a while and then decorrelate: the comparison is statistical, not
pointwise."""
import numpy as np
import pytest

import fastmd_b200 as fm
from oracle import pyoracle as po
from tests.util import oracle_system, run_conf

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

STEPS, EVERY, SETTLE = 5000, 25, 500


def _mean_se(a):
    blocks = np.array_split(np.asarray(a), 10)
    m = np.array([b.mean() for b in blocks])
    return float(np.mean(a)), float(m.std(ddof=1) / np.sqrt(len(m)))


def test_c0_langevin_averages_match_the_oracle():
    pre = fm.Simulation(run_conf(), gen=dict(nchains=30, chain_length=100, density=0.85, seed=42, pushoff_steps=2000),
                        form=fm.FMD_FORM_MIXED)
    x0, v0, i0 = pre.state()
    pre.close()
    d = fm.generate_melt(30, 100, density=0.85, seed=42)
    d.xyz, d.vel, d.image = x0, v0, i0
    conf = run_conf(ensemble="nvt_langevin 1.0 1.0 1.0 42", nsteps=STEPS)
    sim = fm.Simulation(conf, desc=d, form=fm.FMD_FORM_MIXED)
    osim = po.Sim(oracle_system(d, xyz=x0, vel=v0, image=i0), ensemble="langevin", T=(1.0, 1.0, 1.0), seed=42,
                  dt=0.001, nsteps=STEPS)
    gpu, cpu = [], []
    for k in range(STEPS // EVERY):
        sim.step(EVERY)
        osim.step(EVERY)
        if (k + 1) * EVERY <= SETTLE:
            continue
        t = sim.thermo()
        ot = osim.thermo()  # ke, pe, T, then the six pressure components
        gpu.append((t.temp, (t.stress[0] + t.stress[3] + t.stress[5]) / 3.0, sim.rg()))
        cpu.append((ot[2], (ot[3] + ot[6] + ot[8]) / 3.0, osim.rg()))
    sim.close()
    gpu, cpu = np.array(gpu), np.array(cpu)
    for c, name in enumerate(["T", "P", "Rg"]):
        mg, sg = _mean_se(gpu[:, c])
        mc, sc = _mean_se(cpu[:, c])
        assert abs(mg - mc) < 4.0 * np.hypot(sg, sc) + 1e-12, (name, mg, sg, mc, sc)
    assert abs(np.mean(gpu[:, 0]) - 1.0) < 0.05   # the thermostat holds T = 1
