"""The Langevin thermostat of the mixed form holds the target temperature.

Free particles (no bonds, LJ eps = 0) under BAOAB Langevin dynamics have the
stationary velocity variance kT/m exactly, whatever the time step, so any
bias of the FP32 noise transform (Box-Muller on the Philox words) or of the
velocity update shows directly in <T>.  200,000 particles at T = 1.3
(Tdamp = 0.5) for 20,000 steps, sampled every 250 steps after 5,000: the
mean must be within 4 standard errors (block averages) and 0.1 % of T."""
import numpy as np
import pytest

import fastmd_b200 as fm
from tests.util import run_conf

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


def test_free_particles_reach_the_target_temperature():
    n, L = 200_000, 60.0
    rng = np.random.default_rng(5)
    d = fm.SystemDesc(xyz=rng.uniform(0, L, (n, 3)), box_L=L, type=np.zeros(n, np.int32),
                      mol=np.arange(1, n + 1, dtype=np.int32))
    conf = run_conf(ensemble="nvt_langevin 1.3 1.3 0.5 17", nsteps=10 ** 7, lj=[(0, 0, 0.0, 1.0)], bond=None,
                    angle=None)
    b = fm.Batch(max_replicas=1, max_atoms=n + 4096)
    s = b.add(conf, desc=d)
    b.run(5000)
    temps = []
    for _ in range(60):
        b.run(250)
        temps.append(b.thermo(s).temp)
    b.close()
    t = np.array(temps)
    blocks = np.array([x.mean() for x in np.array_split(t, 10)])
    se = blocks.std(ddof=1) / np.sqrt(len(blocks))
    assert abs(t.mean() - 1.3) < max(4 * se, 1e-12), (t.mean(), se)
    assert abs(t.mean() - 1.3) < 1.3e-3, (t.mean(), se)
