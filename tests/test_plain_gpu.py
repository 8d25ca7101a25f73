"""FP64 plain form on the GPU against the FP64 CPU oracle (same inputs).

Tolerances: the pair set is compared exactly; LJ forces are summed in the same
neighbor order with no fused multiply-add on either side, FENE / angle forces
are scattered with atomics (order-dependent rounding), so forces are checked
to 1e-12 relative RMS; one integration step to 1e-12."""
import numpy as np
import pytest

import fastmd_b200 as fm
from oracle import pyoracle as po
from tests.util import oracle_system, pair_set, rel_rms, run_conf

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-12
STEP_TOL = 1e-12


def _melt(nchains, length, seed=7, density=0.85, type_block=0):
    return fm.generate_melt(nchains, length, density=density, seed=seed, type_block=type_block)


@pytest.mark.parametrize("nchains,length", [(10, 30), (30, 100)])
def test_plain_forces_and_pairs_match_oracle(nchains, length):
    d = _melt(nchains, length)
    sim = fm.Simulation(run_conf(), desc=d, form=fm.FMD_FORM_PLAIN_FP64)
    x, v, img = sim.state()
    f, pe, vir = sim.forces()
    osys = oracle_system(d, xyz=x)
    fo, peo, viro = po.forces(osys)
    assert rel_rms(f, fo) < FORCE_TOL
    assert rel_rms(pe, peo) < FORCE_TOL
    assert np.max(np.abs(vir - viro)) / np.max(np.abs(viro)) < FORCE_TOL
    pi, pj = sim.pairs()
    oi, oj = po.pairs_brute(x, d.box_L, 2.8, bonds=d.bonds)
    assert pair_set(pi, pj) == pair_set(oi, oj)


@pytest.mark.parametrize("ens", ["nvt_langevin 1.0 1.2 1.0 42", "nvt_nh 1.0 1.0 0.5 3",
                                 "npt_nh 1.0 1.0 0.5 0.5 0.5 1.0 3"])
def test_plain_steps_match_oracle(ens):
    d = _melt(20, 30, seed=11)
    conf = run_conf(ensemble=ens, nsteps=100)
    sim = fm.Simulation(conf, desc=d, form=fm.FMD_FORM_PLAIN_FP64)
    x0, v0, i0 = sim.state()
    name = ens.split()[0]
    args = [float(t) for t in ens.split()[1:]]
    kw = {}
    if name == "nvt_langevin":
        kw = dict(ensemble="langevin", T=tuple(args[:3]), seed=int(args[3]))
    elif name == "nvt_nh":
        kw = dict(ensemble="nvt_nh", T=tuple(args[:3]), chain=int(args[3]))
    else:
        kw = dict(ensemble="npt_nh", T=tuple(args[:3]), P=tuple(args[3:6]), chain=int(args[6]))
    osim = po.Sim(oracle_system(d, xyz=x0, vel=v0, image=i0), dt=0.001, nsteps=100, **kw)
    for nstep in (1, 4):
        sim.step(nstep)
        osim.step(nstep)
        x, v, img = sim.state()
        o = osim.state()
        L = sim.box_L
        dx = x - o["x"]
        dx -= L * np.round(dx / L)
        assert np.max(np.abs(dx)) < STEP_TOL * 10, name
        assert rel_rms(v, o["v"]) < STEP_TOL * 10, name
        assert abs(L - osim.scalars()["L"]) < 1e-12 * L
        t = sim.thermo()
        ot = osim.thermo()
        assert np.allclose(t.as_array(), ot, rtol=1e-10, atol=1e-12), name


def test_plain_thermo_rg_known_answers():
    # tests/test_thermo.cu: N=96, v=(1,0,0) -> KE/atom 0.5, T = 1/3.
    n = 96
    L = 10.0
    xyz = np.random.default_rng(0).uniform(0, L, (n, 3))
    d = fm.SystemDesc(xyz=xyz, box_L=L, type=np.zeros(n, np.int32), vel=np.tile([1.0, 0, 0], (n, 1)),
                      mol=np.repeat(np.arange(1, 9), 12).astype(np.int32))
    sim = fm.Simulation(run_conf(bond=None, angle=None), desc=d, form=fm.FMD_FORM_PLAIN_FP64)
    t = sim.thermo()
    assert abs(t.ke - 0.5) < 1e-12
    assert abs(t.temp - 1.0 / 3.0) < 1e-12
    # tests/test_rg.cu:45-77: chain at x = 9, 1+10, 3+10 (images) -> Rg 1.63299
    xyz = np.array([[9.0, 0, 0], [1.0, 0, 0], [3.0, 0, 0]])
    img = np.array([[0, 0, 0], [1, 0, 0], [1, 0, 0]], np.int32)
    d = fm.SystemDesc(xyz=xyz, box_L=10.0, type=np.zeros(3, np.int32), image=img, mol=np.ones(3, np.int32))
    sim = fm.Simulation(run_conf(bond=None, angle=None, rc=2.5), desc=d, form=fm.FMD_FORM_PLAIN_FP64)
    assert abs(sim.rg() - np.sqrt(8.0 / 3.0)) < 1e-12


def _nh_kw(ens):
    name = ens.split()[0]
    a = [float(t) for t in ens.split()[1:]]
    if name == "nvt_nh":
        return dict(ensemble="nvt_nh", T=tuple(a[:3]), chain=int(a[3]))
    return dict(ensemble="npt_nh", T=tuple(a[:3]), P=tuple(a[3:6]), chain=int(a[6]))


@pytest.mark.parametrize("form", ["plain", "mixed"])
@pytest.mark.parametrize("ens", ["nvt_nh 1.0 1.0 0.1 3", "npt_nh 1.0 1.0 0.1 0.5 0.5 1.0 3"])
def test_chain_carry_follows_the_oracle(ens, form):
    """run.conf nh_chain_carry 1 (chain accelerations carried between half
    steps): after 100 steps at Tdamp = 100 dt the extended energy per atom is
    the oracle's with the same option (plain form: to FP64 round-off; mixed:
    much closer than the two schemes are to each other), and the two schemes
    have parted."""
    pre = fm.Simulation(run_conf(), gen=dict(nchains=20, chain_length=30, density=0.85, seed=11, pushoff_steps=2000),
                        form=fm.FMD_FORM_MIXED)
    d = _melt(20, 30, seed=11)
    d.xyz, d.vel, d.image = pre.state()
    pre.close()
    n = len(d.type)
    conf = run_conf(ensemble=ens, nsteps=1000, extra="nh_chain_carry 1")
    sim = fm.Simulation(conf, desc=d, form=fm.FMD_FORM_PLAIN_FP64 if form == "plain" else fm.FMD_FORM_MIXED)
    x0, v0, i0 = sim.state()
    kw = _nh_kw(ens)
    o1 = po.Sim(oracle_system(d, xyz=x0, vel=v0, image=i0), dt=0.001, nsteps=1000, chain_carry=1, **kw)
    o0 = po.Sim(oracle_system(d, xyz=x0, vel=v0, image=i0), dt=0.001, nsteps=1000, chain_carry=0, **kw)
    for _ in range(5):
        sim.step(20)
        o1.step(20)
        o0.step(20)
    e = sim.thermo().conserved
    e1, e0 = o1.conserved() / n, o0.conserved() / n
    assert abs(e1 - e0) > 1e-7 * abs(e1)
    if form == "plain":
        assert abs(e - e1) < 1e-10 * abs(e1)
    else:
        assert abs(e - e1) < 0.2 * abs(e1 - e0)
