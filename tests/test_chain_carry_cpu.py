"""The opt-in Nose-Hoover chain scheme (run.conf nh_chain_carry 1), on CPU.

The reference's chain half step (integrate/nose_hoover.cu:86-178, :356-447)
starts the upper chain elements' accelerations from zero in every half step,
so its downward sweep drives them with nothing; LAMMPS's fix nh, whose
splitting it follows, carries them over from the previous half step's upward
sweep.  The reset makes the chain update irreversible to first order in dt,
and the extended energy then rises steadily under stiff coupling.  Checked
here with the FP64 oracle, which implements both schemes: a 300-bead melt at
Tdamp = 100 dt gains energy at a steady rate under the reference's scheme
and holds it with the carried accelerations; and the run.conf key is
parsed."""
import numpy as np
import pytest

import fastmd_b200 as fm
from oracle import pyoracle as po


def _melt_state():
    d = fm.generate_melt(3, 100, density=0.85, seed=4)
    bonds = np.asarray(d.bonds).reshape(-1, 2)
    angles = np.asarray(d.angles).reshape(-1, 3)
    n = len(d.type)

    def system(x, L, v, img):
        return po.System(xyz=x, L=L, type=np.zeros(n, np.int32), mass=np.ones(1), lj=np.ones((1, 1, 2)),
                         bonds=bonds, bond_type=np.zeros(len(bonds), np.int32),
                         fene=np.array([[30.0, 1.5, 1.0, 1.0]]), angles=angles,
                         angle_type=np.zeros(len(angles), np.int32), angle_p=np.array([[5.0, np.pi]]), mol=d.mol,
                         vel=v, image=img)

    pre = po.Sim(system(d.xyz, d.box_L, d.vel, d.image), ensemble="langevin", dt=0.001, T=(1.0, 1.0, 1.0),
                 nsteps=10 ** 8, force_cap=50.0, nthreads=4)
    pre.step(2000)
    st = pre.state()
    return system, st, pre.scalars()["L"]


def _slope(system, st, L, carry, steps=20_000, samples=40):
    sim = po.Sim(system(st["x"], L, st["v"], st["image"]), ensemble="nvt_nh", dt=0.001, T=(1.0, 1.0, 0.1),
                 chain=3, nsteps=10 ** 8, nthreads=4, chain_carry=carry)
    sim.step(2000)
    e = []
    for _ in range(samples):
        sim.step(steps // samples)
        e.append(sim.conserved())
    t = np.arange(1, samples + 1) * (steps // samples) * 0.001
    return float(np.polyfit(t, e, 1)[0])  # kT per tau, whole system


def test_carried_chain_accelerations_hold_the_extended_energy():
    system, st, L = _melt_state()
    ref = _slope(system, st, L, carry=0)
    kept = _slope(system, st, L, carry=1)
    assert ref > 0.2                 # the reference's scheme: a steady gain (0.3-1.2 kT per tau here)
    assert abs(kept) < 0.1 * ref     # carried: flat to within the fit's noise (|slope| ~ 0.01)


def test_run_conf_key():
    base = "ntypes 1\nrc 2.5\nskin 0.3\ndt 0.001\nnvt_nh 1.0 1.0 0.1 3\n"
    for v in (0, 1):
        assert fm.parse_run_conf(base + f"nh_chain_carry {v}\n")["chain_length"] == 3
    with pytest.raises(fm.FastMDError):
        fm.parse_run_conf(base + "nh_chain_carry 2\n")


def test_barostat_kinetic_term_diagnostic():
    """orc_sim_conserved_mtk adds the summed work of the (3 / N_f) 2 KE term
    the reference's barostat force leaves out: zero under NVT, nonzero and
    small (next to the extended energy) under NPT."""
    system, st, L = _melt_state()
    for ens, kw in (("nvt_nh", {}), ("npt_nh", dict(P=(0.0, 0.0, 1.0)))):
        sim = po.Sim(system(st["x"], L, st["v"], st["image"]), ensemble=ens, dt=0.001, T=(1.0, 1.0, 0.5),
                     chain=3, nsteps=10 ** 8, nthreads=4, **kw)
        sim.step(500)
        gap = sim.conserved_mtk() - sim.conserved()
        if ens == "nvt_nh":
            assert gap == 0.0
        else:
            assert gap != 0.0 and abs(gap) < 1e-3 * abs(sim.conserved())
