"""Mixed form (FP32 forces on cell-relative positions, FP64 reductions and
thermostat scalars) on the GPU against the FP64 oracle on the same inputs.

Tolerances (stated targets): force RMS error <= 1e-5 relative to the FP64
oracle; positions after one step within 2e-6 sigma (FP32 offsets); thermo
values within 1e-5 relative; the neighbor list holds every pair within rc and
every pair within rc + skin except pairs within 1e-4 of the rc + skin boundary."""
import numpy as np
import pytest

import fastmd_b200 as fm
from oracle import pyoracle as po
from tests.util import oracle_system, pair_set, rel_rms, run_conf

pytestmark = pytest.mark.gpu

FORCE_RMS_TOL = 1e-5


def _melt(nchains, length, seed=7, type_block=0):
    return fm.generate_melt(nchains, length, density=0.85, seed=seed, type_block=type_block)


@pytest.mark.parametrize("nchains,length", [(6, 20), (10, 30), (30, 100), (50, 100)])
def test_mixed_forces_match_oracle(nchains, length):
    d = _melt(nchains, length)
    sim = fm.Simulation(run_conf(), desc=d, form=fm.FMD_FORM_MIXED)
    x, v, img = sim.state()
    f, pe, vir = sim.forces()
    fo, peo, viro = po.forces(oracle_system(d, xyz=x))
    assert rel_rms(f, fo) < FORCE_RMS_TOL
    assert abs(pe.sum() - peo.sum()) / abs(peo.sum()) < 1e-5
    assert np.max(np.abs(vir - viro)) / np.max(np.abs(viro)) < 1e-5


def test_mixed_two_types_forces():
    d = _melt(20, 100, seed=3, type_block=50)
    lj = [(0, 0, 1.0, 1.0), (1, 1, 1.0, 1.0), (0, 1, 0.9, 1.0)]
    sim = fm.Simulation(run_conf(ntypes=2, lj=lj), desc=d, form=fm.FMD_FORM_MIXED)
    x, _, _ = sim.state()
    f, _, _ = sim.forces()
    tab = np.ones((2, 2, 2))
    tab[0, 1, 0] = tab[1, 0, 0] = 0.9
    fo, _, _ = po.forces(oracle_system(d, xyz=x, lj_table=tab))
    assert rel_rms(f, fo) < FORCE_RMS_TOL


def test_mixed_pair_list_covers_oracle():
    d = _melt(30, 100, seed=5)
    sim = fm.Simulation(run_conf(), desc=d, form=fm.FMD_FORM_MIXED)
    x, _, _ = sim.state()
    pi, pj = sim.pairs()
    got = pair_set(pi, pj)
    oi, oj = po.pairs_brute(x, d.box_L, 2.8, bonds=d.bonds)
    want = pair_set(oi, oj)
    # every oracle pair within rc + skin - 1e-4 must be present
    ii, jj = po.pairs_brute(x, d.box_L, 2.8 - 1e-4, bonds=d.bonds)
    core = pair_set(ii, jj)
    assert core <= got
    # nothing beyond rc + skin + 1e-4
    oi2, oj2 = po.pairs_brute(x, d.box_L, 2.8 + 1e-4, bonds=d.bonds)
    assert got <= pair_set(oi2, oj2)
    assert len(got ^ want) <= 2


@pytest.mark.parametrize("ens", ["nvt_langevin 1.0 1.2 1.0 42", "nvt_nh 1.0 1.0 0.5 3",
                                 "npt_nh 1.0 1.0 0.5 0.5 0.5 1.0 3"])
def test_mixed_steps_track_oracle(ens):
    # Start from a pushed-off melt: a raw random walk keeps overlaps whose
    # clamped LJ forces make trajectories chaotic from the first step.
    pre = fm.Simulation(run_conf(), gen=dict(nchains=20, chain_length=50, density=0.85, seed=11, pushoff_steps=2000),
                        form=fm.FMD_FORM_MIXED)
    x0, v0, i0 = pre.state()
    d = _melt(20, 50, seed=11)
    d.xyz, d.vel, d.image = x0, v0, i0
    conf = run_conf(ensemble=ens, nsteps=100)
    sim = fm.Simulation(conf, desc=d, form=fm.FMD_FORM_MIXED)
    x0, v0, i0 = sim.state()
    name = ens.split()[0]
    a = [float(t) for t in ens.split()[1:]]
    if name == "nvt_langevin":
        kw = dict(ensemble="langevin", T=tuple(a[:3]), seed=int(a[3]))
    elif name == "nvt_nh":
        kw = dict(ensemble="nvt_nh", T=tuple(a[:3]), chain=int(a[3]))
    else:
        kw = dict(ensemble="npt_nh", T=tuple(a[:3]), P=tuple(a[3:6]), chain=int(a[6]))
    osim = po.Sim(oracle_system(d, xyz=x0, vel=v0, image=i0), dt=0.001, nsteps=100, **kw)
    for n in (1, 4, 5):
        sim.step(n)
        osim.step(n)
        x, v, img = sim.state()
        o = osim.state()
        L = sim.box_L
        ux = x - o["x"]
        ux -= L * np.round(ux / L)
        assert np.max(np.abs(ux)) < 2e-5, (name, n, float(np.max(np.abs(ux))), int(np.argmax(np.abs(ux)) // 3))
        assert rel_rms(v, o["v"]) < 1e-4, name
        t = sim.thermo().as_array()
        ot = osim.thermo()
        assert np.allclose(t, ot, rtol=2e-4, atol=2e-4), (name, t, ot)
        assert abs(sim.rg() - osim.rg()) < 1e-5 * osim.rg(), (name, sim.rg(), osim.rg())


def test_batch_alone_equals_in_mix():
    """Each replica's trajectory is bit-identical alone and in a mixed batch."""
    confs = [run_conf(ensemble=f"nvt_langevin {T} {T} 1.0 {s}", nsteps=200) for T, s in
             [(1.0, 1), (0.7, 2), (1.3, 3)]]
    confs.append(run_conf(ensemble="nvt_nh 1.0 1.0 0.5 3", nsteps=200))
    melts = [_melt(10, 20, seed=1), _melt(25, 40, seed=2), _melt(7, 100, seed=3), _melt(12, 30, seed=4)]
    mix = fm.Batch(max_replicas=8, max_atoms=1 << 16)
    slots = [mix.add(c, desc=m) for c, m in zip(confs, melts)]
    mix.run(60)
    for c, m, s in zip(confs, melts, slots):
        alone = fm.Batch(max_replicas=1, max_atoms=1 << 14)
        a = alone.add(c, desc=m)
        alone.run(60)
        xa, va, ia = alone.state(a)
        xm, vm, im = mix.state(s)
        assert np.array_equal(xa, xm) and np.array_equal(va, vm) and np.array_equal(ia, im)
        ta = alone.thermo(a).as_array()
        tm = mix.thermo(s).as_array()
        assert np.array_equal(ta, tm)
        alone.close()


@pytest.mark.parametrize("ens", ["nvt_langevin 1.0 1.0 1.0 7", "npt_nh 1.0 1.0 0.5 12.0 12.0 0.3 3"])
def test_trigger_only_rebuilds_keep_list_complete(ens):
    """With the forced cadence lifted, rebuilds follow the displacement and
    box-shrink trigger alone, and the forces computed from the list in use
    stay the oracle's (a missing pair would show as a large error).  The NPT
    case drives the box down with a high target pressure."""
    pre = fm.Simulation(run_conf(), gen=dict(nchains=20, chain_length=50, density=0.85, seed=11, pushoff_steps=2000),
                        form=fm.FMD_FORM_MIXED)
    x0, v0, i0 = pre.state()
    d = _melt(20, 50, seed=11)
    d.xyz, d.vel, d.image = x0, v0, i0
    b = fm.Batch(max_replicas=2, max_atoms=1 << 14)
    s = b.add(run_conf(ensemble=ens, nsteps=600), desc=d)
    b.set_rebuild_cadence(s, 0)
    L0 = b.info(s).box_L
    for _ in range(12):
        b.run(50)
        f, _, _ = b.forces(s)
        x, Lf = b.force_frame(s)
        info = b.info(s)
        fo, _, _ = po.forces(oracle_system(d, xyz=x, L=Lf))
        assert rel_rms(f, fo) < FORCE_RMS_TOL, (ens, info.step, rel_rms(f, fo))
        assert info.status_word == 0
    if ens.startswith("npt"):
        assert b.info(s).box_L < 0.995 * L0
    b.close()


@pytest.mark.parametrize("nchains,length", [(6, 20), (10, 30)])
def test_small_box_lists_over_rebuilds(nchains, length):
    """Boxes under three cells per axis (G = 1 at 120 beads, G = 2 at 300)
    get their lists from the small-box list kernel: rebuilt on every step
    (direct launches and graph steps) beside a larger replica that takes the
    ballot kernel, their forces stay the oracle's."""
    pre = fm.Simulation(run_conf(), gen=dict(nchains=nchains, chain_length=length, density=0.85, seed=11,
                                             pushoff_steps=2000), form=fm.FMD_FORM_MIXED)
    x0, v0, i0 = pre.state()
    d = _melt(nchains, length, seed=11)
    d.xyz, d.vel, d.image = x0, v0, i0
    b = fm.Batch(max_replicas=2, max_atoms=1 << 14)
    s = b.add(run_conf(ensemble="nvt_langevin 1.0 1.0 1.0 9", nsteps=400), desc=d)
    b.add(run_conf(ensemble="nvt_langevin 1.0 1.0 1.0 10", nsteps=400),
          gen=dict(nchains=20, chain_length=50, density=0.85, seed=6, pushoff_steps=300))
    b.set_rebuild_cadence(s, 1)
    assert d.box_L < 3 * 2.8
    r0 = b.info(s).rebuilds
    for n in (25, 25, 50, 50):  # direct launches, then the step graph
        b.run(n)
        f, _, _ = b.forces(s)
        x, Lf = b.force_frame(s)
        fo, _, _ = po.forces(oracle_system(d, xyz=x, L=Lf))
        assert rel_rms(f, fo) < FORCE_RMS_TOL, (nchains, rel_rms(f, fo))
        assert b.info(s).status_word == 0
    assert b.info(s).rebuilds - r0 >= 150
    b.close()


def test_pushoff_then_langevin_is_stable():
    conf = run_conf(ensemble="nvt_langevin 1.0 1.0 1.0 42", nsteps=2000)
    sim = fm.Simulation(conf, gen=dict(nchains=30, chain_length=100, density=0.85, seed=42, pushoff_steps=2000),
                        form=fm.FMD_FORM_MIXED)
    f, _, _ = sim.forces()
    assert np.max(np.linalg.norm(f, axis=1)) < 2000
    sim.step(1000)
    t = sim.thermo()
    assert 0.8 < t.temp < 1.2
    assert np.isfinite(t.pe)
    assert sim.counters()["status_word"] == 0


@pytest.mark.parametrize("ens", ["nvt_langevin 1.0 1.0 1.0 7", "nvt_nh 1.0 1.0 0.5 3",
                                 "npt_nh 1.0 1.0 0.5 0.5 0.5 1.0 3"])
def test_graph_steps_equal_direct_steps(ens):
    """A CUDA-graph run (conditional rebuild / force / post nodes, Langevin
    post-force kicks folded into the next pre-force) gives bit-identical
    states to launching every kernel of every step directly."""
    conf = run_conf(ensemble=ens, nsteps=10_000)
    melts = [_melt(10, 30, seed=21), _melt(12, 50, seed=22)]
    out = []
    for gs in (-1, 10):
        b = fm.Batch(max_replicas=4, max_atoms=1 << 14, graph_steps=gs)
        slots = [b.add(conf, desc=m) for m in melts]
        b.run(37)
        b.run(25)
        out.append([(b.state(s), b.thermo(s).as_array()) for s in slots])
        b.close()
    for (sa, ta), (sb, tb) in zip(out[0], out[1]):
        for a, c in zip(sa, sb):
            assert np.array_equal(a, c)
        assert np.array_equal(ta, tb)


@pytest.mark.parametrize("ens", ["nvt_langevin 1.0 1.0 1.0 9", "nvt_nh 1.0 1.0 0.5 3"])
def test_observing_does_not_perturb(ens):
    """Reading thermo / Rg / forces between runs re-evaluates energies with
    the energy flavour of the force kernel; the trajectory stays bit-identical
    to an unobserved run."""
    conf = run_conf(ensemble=ens, nsteps=10_000)
    m = _melt(15, 40, seed=31)
    a = fm.Batch(max_replicas=2, max_atoms=1 << 13)
    sa = a.add(conf, desc=m)
    a.run(120)
    b = fm.Batch(max_replicas=2, max_atoms=1 << 13)
    sb = b.add(conf, desc=m)
    for _ in range(4):
        b.run(30)
        b.thermo(sb)
        b.rg(sb)
        b.forces(sb)
    for x, y in zip(a.state(sa), b.state(sb)):
        assert np.array_equal(x, y)
    assert np.array_equal(a.thermo(sa).as_array(), b.thermo(sb).as_array())
    a.close()
    b.close()


@pytest.mark.parametrize("fv", [-1, 9, 10, 11])
def test_observing_every_step_does_not_perturb(fv):
    """Forces read after every step, so also right after the steps whose
    work-list force launch rebuilt or re-filtered the pruned list while
    evaluating the forces: the re-evaluation over the pruned list it wrote
    reproduces those forces bit for bit, and the trajectory stays identical
    to an unobserved one.  fv: the default force variant, the two
    lanes-per-atom variants (which filter first, then walk the new list) and
    a shared-memory ring variant (whose work-list kernel loads ahead into
    registers instead)."""
    conf = run_conf(ensemble="nvt_langevin 1.0 1.0 1.0 9", nsteps=10_000)
    m = _melt(15, 40, seed=33)
    a = fm.Batch(max_replicas=2, max_atoms=1 << 13)
    a.set_variants(fv, -1)
    sa = a.add(conf, desc=m)
    b = fm.Batch(max_replicas=2, max_atoms=1 << 13)
    b.set_variants(fv, -1)
    sb = b.add(conf, desc=m)
    for _ in range(150):
        a.run(1)
    r0 = b.info(sb).rebuilds
    for _ in range(150):
        b.run(1)
        f, _, _ = b.forces(sb)
        assert np.all(np.isfinite(f))
    assert b.info(sb).rebuilds - r0 >= 2
    for x, y in zip(a.state(sa), b.state(sb)):
        assert np.array_equal(x, y)
    assert np.array_equal(a.thermo(sa).as_array(), b.thermo(sb).as_array())
    a.close()
    b.close()


def test_server_results_equal_alone_and_in_mix():
    """Continuous batching: requests admitted while others run, retired and
    back-filled, give the same final thermo row and Rg as the same request
    run alone."""
    reqs = []
    for k, (nc, cl, steps) in enumerate([(10, 20, 300), (8, 50, 500), (20, 30, 200), (5, 100, 400), (12, 40, 350)]):
        T = 0.8 + 0.1 * k
        conf = run_conf(ensemble=f"nvt_langevin {T} {T} 1.0 {k + 1}", nsteps=steps)
        gen = dict(nchains=nc, chain_length=cl, density=0.85, seed=100 + k, pushoff_steps=300)
        reqs.append((conf, gen))
    srv = fm.Server(max_replicas=3, hbm_budget_gb=8.0, steps_per_round=50)
    ids = []
    for conf, gen in reqs:
        ids.append(srv.submit(conf, gen))
    srv.drain(600.0)
    got = {r.request_id: r for r in srv.poll(64)}
    srv.close()
    assert sorted(got) == sorted(ids)
    for rid, (conf, gen) in zip(ids, reqs):
        r = got[rid]
        assert r.status == 0
        alone = fm.Batch(max_replicas=1, max_atoms=1 << 14)
        s = alone.add(conf, gen=gen)
        alone.run(10_000)  # stops at the request's nsteps
        assert alone.info(s).step == r.steps
        assert np.array_equal(alone.thermo(s).as_array(), np.asarray(r.thermo.as_array()))
        assert alone.rg(s) == r.rg
        alone.close()


@pytest.mark.parametrize("ens", ["nvt_langevin 1.0 1.0 1.0 5", "npt_nh 1.0 1.0 0.5 1.0 1.0 1.0 3"])
def test_stress_acf_matches_oracle_correlator(ens, tmp_path):
    """The device correlator equals the oracle correlator fed with the thermo
    pressure tensor of every stress step (the same doubles), in the rows of
    the reference's stress file."""
    freq, nsamp = 3, 300
    conf = run_conf(ensemble=ens, nsteps=freq * nsamp, extra=f"stress 1 {freq} acf.dat")
    d = _melt(10, 30, seed=9)
    b = fm.Batch(max_replicas=2, max_atoms=1 << 13)
    s = b.add(conf, desc=d)
    acf = po.StressACF(freq)
    for _ in range(nsamp):
        b.run(freq)
        acf.push(b.thermo(s).stress)
    lag, val, cnt = b.stress_acf(s)
    olag, oval, ocnt = acf.rows()
    assert np.array_equal(lag, olag) and np.array_equal(cnt, ocnt)
    assert np.allclose(val, oval, rtol=1e-12, atol=1e-14 * np.max(np.abs(oval)))
    p = tmp_path / "acf.dat"
    b.write_stress_acf(s, p)
    rows = np.loadtxt(p)
    assert rows.shape == (len(lag), 8)
    assert np.array_equal(rows[:, 0].astype(np.int64), lag) and np.array_equal(rows[:, 7].astype(np.int64), cnt)
    b.close()


def test_trajectory_frames_are_the_force_frame(tmp_path):
    """Dumped frames (reference dump format) hold the positions the forces
    belong to, in single precision and atom-id order, with step and box."""
    conf = run_conf(ensemble="npt_nh 1.0 1.0 0.5 2.0 2.0 1.0 3", nsteps=400)
    d = _melt(8, 25, seed=4)
    b = fm.Batch(max_replicas=2, max_atoms=1 << 12)
    s = b.add(conf, desc=d)
    p = tmp_path / "traj.bin"
    want = []
    with fm.Trajectory(p, d.natoms if hasattr(d, "natoms") else len(d.type), ntypes=1) as t:
        for _ in range(5):
            b.run(37)
            x, Lf = b.force_frame(s)
            want.append((b.info(s).step, np.float32(b.info(s).box_L), x.astype(np.float32)))
            t.write(b, s)
    tr = fm.read_trajectory(p)
    assert tr["natoms"] == len(d.type) and tr["ntypes"] == 1 and len(tr["steps"]) == 5
    for k, (st, L, x) in enumerate(want):
        assert tr["steps"][k] == st and tr["box_L"][k] == L
        assert np.array_equal(tr["xyz"][k], x)
    b.close()


def test_trajectory_of_a_simulation(tmp_path):
    d = _melt(6, 20, seed=2)
    for form in (fm.FMD_FORM_MIXED, fm.FMD_FORM_PLAIN_FP64):
        sim = fm.Simulation(run_conf(nsteps=100), desc=d, form=form)
        p = tmp_path / f"traj{form}.bin"
        with fm.Trajectory(p, sim.natoms) as t:
            sim.step(10)
            t.write(sim)
            sim.step(10)
            t.write(sim)
        tr = fm.read_trajectory(p)
        assert list(tr["steps"]) == [10, 20]
        x, _, _ = sim.state()
        assert np.max(np.abs(tr["xyz"][1] - x.astype(np.float32))) < 1e-4 * sim.box_L


def _soft_table(path, keyword, n=2001, rlo=0.05, rhi=2.5):
    """A smooth tabulated pair: E = A cos^2(pi r / (2 rhi)), force column
    F/r = -dE/dr / r."""
    r = np.linspace(rlo, rhi, n)
    A = 5.0
    e = A * np.cos(np.pi * r / (2 * rhi)) ** 2
    f = A * np.pi / rhi * np.cos(np.pi * r / (2 * rhi)) * np.sin(np.pi * r / (2 * rhi)) / r
    lines = [keyword, f"N {n} R {rlo} {rhi}", ""]
    lines += [f"{k + 1} {a:.9g} {b:.9g} {c:.9g}" for k, (a, b, c) in enumerate(zip(r, e, f))]
    path.write_text("\n".join(lines) + "\n")


def test_table_forces_match_oracle(tmp_path):
    p = tmp_path / "soft.table"
    _soft_table(p, "SOFT")
    d = _melt(20, 50, seed=6)
    conf = run_conf(lj=[(0, 0, 0.0, 0.0)], extra=f"table 0 0 {p} SOFT")
    sim = fm.Simulation(conf, desc=d, form=fm.FMD_FORM_MIXED)
    x, _, _ = sim.state()
    f, pe, vir = sim.forces()
    tb = fm.read_pair_table(p, "SOFT")
    ft, pet, virt = po.table_forces(x, d.box_L, 2.5, d.type, [[0]], [tb], bonds=d.bonds)
    fb, peb, virb = po.forces(oracle_system(d, xyz=x, lj_table=np.zeros((1, 1, 2))))
    fo = fb + ft
    assert rel_rms(f, fo) < FORCE_RMS_TOL
    assert abs(pe.sum() - (peb.sum() + pet.sum())) < 1e-5 * abs(peb.sum() + pet.sum())
    assert np.max(np.abs(vir - (virb + virt))) < 1e-5 * np.max(np.abs(virb + virt))


def test_lj_shaped_table_reproduces_lj(tmp_path):
    # force/table.cu's own check (tests/test_table.cu:7-104): a 10,000-point
    # table of the clamped LJ force and energy matches the LJ kernel.
    n, rlo, rc = 10000, 0.01, 2.5
    r = np.linspace(rlo, rc, n)
    sr6 = (1.0 / r ** 2) ** 3
    fcol = np.clip(24.0 / r ** 2 * (2 * sr6 * sr6 - sr6), -1000, 1000)
    ecol = 4.0 * (sr6 * sr6 - sr6)
    p = tmp_path / "lj.table"
    p.write_text("LJT\n" + f"N {n} R {rlo} {rc}\n\n" +
                 "\n".join(f"{k + 1} {a:.9g} {b:.9g} {c:.9g}" for k, (a, b, c) in enumerate(zip(r, ecol, fcol))) + "\n")
    d = _melt(20, 50, seed=8)
    pre = fm.Simulation(run_conf(), gen=dict(nchains=20, chain_length=50, density=0.85, seed=8, pushoff_steps=2000),
                        form=fm.FMD_FORM_MIXED)
    x0, v0, i0 = pre.state()
    d.xyz, d.vel, d.image = x0, v0, i0
    lj_sim = fm.Simulation(run_conf(), desc=d, form=fm.FMD_FORM_MIXED)
    tb_sim = fm.Simulation(run_conf(lj=[(0, 0, 0.0, 0.0)], extra=f"table 0 0 {p} LJT"), desc=d,
                           form=fm.FMD_FORM_MIXED)
    f1, pe1, _ = lj_sim.forces()
    f2, pe2, _ = tb_sim.forces()
    assert np.max(np.abs(f1 - f2)) < 1e-2 * max(1.0, np.max(np.abs(f1)))
    assert abs(pe1.sum() - pe2.sum()) < 1e-3 * abs(pe1.sum())


def test_table_replica_alone_equals_in_mix(tmp_path):
    p = tmp_path / "soft.table"
    _soft_table(p, "SOFT")
    tconf = run_conf(ensemble="nvt_langevin 1.0 1.0 1.0 3", nsteps=200, lj=[(0, 0, 0.0, 0.0)],
                     extra=f"table 0 0 {p} SOFT\nthermo 1 7 th.dat")
    lconf = run_conf(ensemble="nvt_nh 1.0 1.0 0.5 3", nsteps=200)
    mt, ml = _melt(12, 30, seed=1), _melt(9, 40, seed=2)
    mix = fm.Batch(max_replicas=4, max_atoms=1 << 13)
    st = mix.add(tconf, desc=mt)
    mix.add(lconf, desc=ml)
    mix.run(80)
    alone = fm.Batch(max_replicas=1, max_atoms=1 << 12)
    a = alone.add(tconf, desc=mt)
    alone.run(80)
    xa, va, _ = alone.state(a)
    xm, vm, _ = mix.state(st)
    assert np.array_equal(xa, xm) and np.array_equal(va, vm)
    assert np.array_equal(alone.thermo(a).as_array(), mix.thermo(st).as_array())
    assert np.all(np.isfinite(xa)) and alone.info(a).status_word == 0
    alone.close()
    mix.close()


def test_thermo_rows_of_a_batch_in_any_order():
    """Reading one replica's thermo row re-evaluates every stale replica in
    one pass; the rows and the trajectories that follow do not depend on the
    order or number of rows read."""
    confs = [run_conf(ensemble=f"nvt_langevin 1.0 1.0 1.0 {s}", nsteps=500) for s in (5, 6)]
    confs.append(run_conf(ensemble="nvt_nh 1.0 1.0 0.5 3", nsteps=500))
    melts = [_melt(8, 25, seed=11), _melt(6, 30, seed=12), _melt(10, 20, seed=13)]

    def make():
        b = fm.Batch(max_replicas=4, max_atoms=1 << 13)
        return b, [b.add(c, desc=m) for c, m in zip(confs, melts)]

    a, sa = make()
    b, sb = make()
    a.run(37)
    b.run(37)
    ra = [a.thermo(s).as_array() for s in sa]
    rb = {s: b.thermo(s).as_array() for s in reversed(sb)}
    for s1, s2, row in zip(sa, sb, ra):
        assert np.array_equal(row, rb[s2])
    a.run(20)
    b.run(20)
    b.thermo(sb[1])  # read one row only
    for s1, s2 in zip(sa, sb):
        xa, va, _ = a.state(s1)
        xb, vb, _ = b.state(s2)
        assert np.array_equal(xa, xb) and np.array_equal(va, vb)
        assert np.array_equal(a.thermo(s1).as_array(), b.thermo(s2).as_array())
    a.close()
    b.close()


def test_pruned_list_forces_equal_full_list():
    """The pruned list (pairs within rc + 0.12, the default outside NPT) gives
    the full list's forces up to summation order, at the start and after
    many filters; switching it off and on keeps the forces."""
    pre = fm.Simulation(run_conf(), gen=dict(nchains=20, chain_length=50, density=0.85, seed=21, pushoff_steps=2000),
                        form=fm.FMD_FORM_MIXED)
    x0, v0, i0 = pre.state()
    d = _melt(20, 50, seed=21)
    d.xyz, d.vel, d.image = x0, v0, i0
    conf = run_conf(ensemble="nvt_langevin 1.0 1.0 1.0 9", nsteps=2000)
    b = fm.Batch(max_replicas=2, max_atoms=1 << 13)
    sp = b.add(conf, desc=d)   # pruned (default)
    sf = b.add(conf, desc=d)
    b.set_list_prune(sf, 0.0)  # full list
    fp, pep, _ = b.forces(sp)
    ff, pef, _ = b.forces(sf)
    assert rel_rms(fp, ff) < 1e-6 and abs(pep.sum() - pef.sum()) < 1e-6 * abs(pef.sum())
    for _ in range(6):
        b.run(100)
        x, _, _ = b.state(sp)
        f, _, _ = b.forces(sp)
        fo, _, _ = po.forces(oracle_system(d, xyz=x))
        assert rel_rms(f, fo) < FORCE_RMS_TOL
        assert b.info(sp).status_word == 0
    # off mid-interval (the rebuild bound keeps the filters' displacements),
    # then on again (filtered at once)
    for delta in (0.0, 0.12):
        b.set_list_prune(sp, delta)
        for _ in range(2):
            b.run(100)
            x, _, _ = b.state(sp)
            f, _, _ = b.forces(sp)
            assert rel_rms(f, po.forces(oracle_system(d, xyz=x))[0]) < FORCE_RMS_TOL
    b.close()


def test_list_buffer_widened_by_autotune_keeps_forces():
    """The autotuner widens the Verlet-list margin of a replica with a pruned
    list to the cell edge; rebuilds come further apart and the forces stay
    the oracle's.  The run.conf skin can be restored, and a margin the list
    capacity cannot hold is refused."""
    pre = fm.Simulation(run_conf(), gen=dict(nchains=30, chain_length=100, density=0.85, seed=41, pushoff_steps=2000),
                        form=fm.FMD_FORM_MIXED)
    x0, v0, i0 = pre.state()
    d = _melt(30, 100, seed=41)
    d.xyz, d.vel, d.image = x0, v0, i0
    b = fm.Batch(max_replicas=2, max_atoms=1 << 13)
    s = b.add(run_conf(ensemble="nvt_langevin 1.0 1.0 1.0 5", nsteps=10_000), desc=d)
    assert b.list_buffer(s) == pytest.approx(0.3)
    b.autotune(3)
    wide = b.list_buffer(s)
    assert wide > 0.45, wide
    r0 = b.info(s).rebuilds
    for _ in range(8):
        b.run(50)
        f, _, _ = b.forces(s)
        x, Lf = b.force_frame(s)
        assert rel_rms(f, po.forces(oracle_system(d, xyz=x, L=Lf))[0]) < FORCE_RMS_TOL
        assert b.info(s).status_word == 0
    assert b.info(s).rebuilds - r0 >= 2
    b.set_list_buffer(s, 0.3)
    assert b.list_buffer(s) == pytest.approx(0.3)
    b.run(50)
    f, _, _ = b.forces(s)
    x, Lf = b.force_frame(s)
    assert rel_rms(f, po.forces(oracle_system(d, xyz=x, L=Lf))[0]) < FORCE_RMS_TOL
    with pytest.raises(fm.FastMDError):
        b.set_list_buffer(s, 3.0)
    b.close()


def test_table_replica_over_rebuilds_and_filters(tmp_path):
    """A tabulated-pair replica stepped through rebuilds and pruned-list
    filters (the table pass then walks the pruned list the work-list force
    launch wrote), with the list buffer widened by the autotuner: the forces
    stay the oracle's."""
    p = tmp_path / "soft.table"
    _soft_table(p, "SOFT")
    d = _melt(30, 100, seed=12)
    b = fm.Batch(max_replicas=2, max_atoms=1 << 13)
    s = b.add(run_conf(ensemble="nvt_langevin 1.0 1.0 1.0 4", nsteps=10_000, lj=[(0, 0, 0.0, 0.0)],
                       extra=f"table 0 0 {p} SOFT"), desc=d)
    b.autotune(3)
    assert b.list_buffer(s) > 0.45
    tb = fm.read_pair_table(p, "SOFT")
    r0 = b.info(s).rebuilds
    for _ in range(6):
        b.run(50)
        f, _, _ = b.forces(s)
        x, Lf = b.force_frame(s)
        ft, _, _ = po.table_forces(x, Lf, 2.5, d.type, [[0]], [tb], bonds=d.bonds)
        fb, _, _ = po.forces(oracle_system(d, xyz=x, L=Lf, lj_table=np.zeros((1, 1, 2))))
        assert rel_rms(f, fb + ft) < FORCE_RMS_TOL
        assert b.info(s).status_word == 0
    assert b.info(s).rebuilds - r0 >= 1
    b.close()


def test_chain_carry_survives_the_pushoff():
    """A replica added with a push-off starts its run with a fresh chain;
    run.conf nh_chain_carry 1 still applies to it.  At Tdamp = 100 dt, after
    2,000 steps of settling, the extended energy of the 600-bead melt rises
    steadily under the reference's scheme (about 0.6 kT per tau for the
    system in the FP64 oracle) and holds with the accelerations carried:
    slopes fitted to 16 samples over 16,000 steps."""
    slope = {}
    for carry in (0, 1):
        b = fm.Batch(max_replicas=1, max_atoms=1 << 13)
        s = b.add(run_conf(ensemble="nvt_nh 1.0 1.0 0.1 3", nsteps=100_000, extra=f"nh_chain_carry {carry}"),
                  gen=dict(nchains=20, chain_length=30, density=0.85, seed=11, pushoff_steps=2000))
        n = b.info(s).natoms
        b.run(2000)
        e = []
        for _ in range(16):
            b.run(1000)
            e.append(b.thermo(s).conserved * n)
        slope[carry] = float(np.polyfit(np.arange(1, 17) * 1.0, e, 1)[0])  # kT per tau, whole melt
        b.close()
    assert slope[0] > 0.15 and abs(slope[1]) < 0.3 * slope[0], slope


@pytest.mark.parametrize("fv", [9, 10, 11, 13])
@pytest.mark.parametrize("ens", ["nvt_langevin 1.0 1.0 1.0 5", "npt_nh 1.0 1.0 0.5 0.5 0.5 1.0 3"])
def test_two_type_forces_lanes_and_ring_variants(ens, fv):
    """The lanes-per-atom and shared-memory ring force variants on a two-type
    melt (per-pair parameter lookup), through 60 steps of their own (pruned
    list with filters under Langevin, the full list under NPT): forces at the
    force frame against the FP64 oracle."""
    lj = [(0, 0, 1.0, 1.0), (1, 1, 1.0, 1.0), (0, 1, 0.9, 1.0)]
    b = fm.Batch(max_replicas=1, max_atoms=1 << 13)
    b.set_variants(fv, -1)
    s = b.add(run_conf(ensemble=ens, ntypes=2, lj=lj, nsteps=1000),
              gen=dict(nchains=20, chain_length=100, density=0.85, seed=3, pushoff_steps=1000, type_block=50))
    b.run(60)
    assert b.variants()[0] == fv
    f, _, _ = b.forces(s)
    x, L = b.force_frame(s)
    d = _melt(20, 100, seed=3, type_block=50)
    tab = np.ones((2, 2, 2))
    tab[0, 1, 0] = tab[1, 0, 0] = 0.9
    fo, _, _ = po.forces(oracle_system(d, xyz=x, L=L, lj_table=tab))
    assert rel_rms(f, fo) < FORCE_RMS_TOL
    assert b.info(s).status_word == 0
    b.close()
