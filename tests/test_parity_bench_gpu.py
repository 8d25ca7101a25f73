"""Parity at the benchmarked configurations: the mixed form against the FP64
oracle on the benchmark's own replica shapes.

* The 64 x 30K workload's replica (300 chains x 100 beads, density 0.85,
  2,000-step capped push-off, Langevin T = 1) with the benchmark's settings
  (autotuned list buffer widened to the cell edge, pruned pair list, rebuild
  cadence lifted): forces, per-atom energies and the virial against the
  oracle for EVERY force-kernel variant (the stored forces of the step's own
  kernel flavour and the energy flavour's re-evaluation) and the pair list of
  EVERY neighbor-list variant against the oracle's pair sets.
* A two-type NPT replica of 30,000 beads tracked against the oracle's NPT
  step loop for 200 steps through several rebuilds (the scaled-down C2 melt).
* One snapshot of the 1,000,000-bead two-type melt (C2): forces against the
  oracle.
* Integer image flags after runs that wrap atoms many periods: exact for the
  plain FP64 form; exact for the mixed form wherever the oracle's wrapped
  coordinate is not within the FP32 tolerance of a box face (there FP32 and
  FP64 may legitimately land on different sides), with unwrapped positions
  in tolerance.

Tolerances: force RMS error <= 1e-5 relative (the stated target); per-atom
energy sum 1e-5 relative; the virial as a pressure-tensor error, |d W| / V
<= 1e-5 eps / sigma^3 (the total virial of a melt near zero pressure is a
small residual of large cancelling per-atom sums, each accumulated in FP32,
so its error grows with sqrt(N) while the total does not: relative to the
largest component it is about 1.5e-5 at 30,000 beads, in pressure units
1e-6); tracked NPT positions 5e-4 sigma after
200 steps (FP32 forces against FP64: the difference grows with the melt's
Lyapunov exponent, about 1e-6 after one step), box edge 1e-6 relative,
thermo values 2e-3 relative."""
import numpy as np
import pytest

import fastmd_b200 as fm
from oracle import pyoracle as po
from tests.util import oracle_system, pair_set, rel_rms, run_conf

pytestmark = pytest.mark.gpu

FORCE_RMS_TOL = 1e-5
LJ2 = [(0, 0, 1.0, 1.0), (1, 1, 1.0, 1.0), (0, 1, 0.9, 1.0)]


def _lj2_table():
    tab = np.ones((2, 2, 2))
    tab[0, 1, 0] = tab[1, 0, 0] = 0.9
    return tab


@pytest.fixture(scope="module")
def headline():
    """The benchmark's replica 0 (seed 0) after push-off and 50 steps, in a
    batch autotuned as the benchmark does it."""
    conf = run_conf(ensemble="nvt_langevin 1.0 1.0 1.0 0", nsteps=10_000_000, extra="thermo 1 100 thermo.dat")
    b = fm.Batch(max_replicas=2, max_atoms=2 * 30080 + 4096)
    s = b.add(conf, gen=dict(nchains=300, chain_length=100, density=0.85, seed=0, pushoff_steps=2000))
    b.run(20)
    b.autotune(2)
    b.run(30)
    d = fm.generate_melt(300, 100, density=0.85, seed=0)
    yield b, s, d
    b.close()


def _virial_ok(vir, viro, L):
    """Pressure-tensor error |d W| / V within 1e-5 eps / sigma^3."""
    return np.max(np.abs(vir - viro)) / L ** 3 < 1e-5


def _check_forces(b, s, d, f_stored=None):
    x, _, _ = b.state(s)
    f, pe, vir = b.forces(s)
    fo, peo, viro = po.forces(oracle_system(d, xyz=x))
    assert rel_rms(f, fo) < FORCE_RMS_TOL
    assert abs(pe.sum() - peo.sum()) < 1e-5 * abs(peo.sum())
    assert _virial_ok(vir, viro, b.info(s).box_L), (vir, viro)
    if f_stored is not None:
        xf, Lf = b.force_frame(s)
        fo2, _, _ = po.forces(oracle_system(d, xyz=xf, L=Lf))
        assert rel_rms(f_stored, fo2) < FORCE_RMS_TOL


def test_headline_replica_settings(headline):
    b, s, d = headline
    L = b.info(s).box_L
    # the benchmark's list buffer: the cell edge minus rc
    G = int(L / (2.5 + 0.3) / 1.0001)
    assert abs(b.list_buffer(s) - (L / (1.0002 * G) - 2.5)) < 1e-9
    assert b.list_buffer(s) > 0.4


@pytest.mark.parametrize("fv", range(15))
def test_headline_replica_forces_every_force_variant(headline, fv):
    b, s, d = headline
    assert b.variants()[2] == 15
    b.set_variants(fv, -1)
    b.run(23)   # direct steps with this variant's plain flavour (and its filter walk)
    assert b.variants()[0] == fv
    f_stored = b.last_forces(s)
    _check_forces(b, s, d, f_stored)
    assert b.info(s).status_word == 0


def test_ring_variants_equal_register_lookahead_bitwise(headline):
    """The shared-memory ring variants change only how the list words reach
    the lanes: forces, per-atom energies and the virial are bitwise those of
    the variant with the same batches and arithmetic that loads the next
    batch's words into registers (m8 k1 a5 x2)."""
    b, s, d = headline
    out = {}
    for fv in (4, 11, 12, 13):
        b.set_variants(fv, -1)
        out[fv] = b.forces(s)
    for fv in (11, 12, 13):
        for x, y in zip(out[4], out[fv]):
            assert np.array_equal(x, y)


@pytest.mark.parametrize("nv", range(3))
def test_headline_replica_pairs_every_neighbor_variant(headline, nv):
    b, s, d = headline
    b.set_variants(-1, nv)
    buf = b.list_buffer(s)
    b.set_list_buffer(s, buf)   # rebuilds the list now, with this variant
    x, _, _ = b.state(s)
    pi, pj = b.pairs(s)
    got = pair_set(pi, pj)
    L = b.info(s).box_L
    rcs = 2.5 + buf
    core = pair_set(*po.pairs_brute(x, L, rcs - 1e-4, bonds=d.bonds))
    outer = pair_set(*po.pairs_brute(x, L, rcs + 1e-4, bonds=d.bonds))
    assert core <= got <= outer
    b.run(20)
    _check_forces(b, s, d, b.last_forces(s))


def test_npt_two_type_30k_tracks_oracle():
    conf = run_conf(ensemble="npt_nh 1.0 1.0 0.1 0.0 0.0 1.0 3", ntypes=2, lj=LJ2, nsteps=10_000)
    pre = fm.Batch(max_replicas=1, max_atoms=30080 + 4096)
    s0 = pre.add(run_conf(ntypes=2, lj=LJ2), gen=dict(nchains=300, chain_length=100, density=0.85, seed=2,
                                                      pushoff_steps=2000, type_block=50))
    pre.run(0)
    x0, v0, i0 = pre.state(s0)
    pre.close()
    d = fm.generate_melt(300, 100, density=0.85, seed=2, type_block=50)
    d.xyz, d.vel, d.image = x0, v0, i0
    b = fm.Batch(max_replicas=1, max_atoms=30080 + 4096)
    s = b.add(conf, desc=d)
    x0, v0, i0 = b.state(s)
    osim = po.Sim(oracle_system(d, xyz=x0, vel=v0, image=i0, lj_table=_lj2_table()), ensemble="npt_nh",
                  T=(1.0, 1.0, 0.1), P=(0.0, 0.0, 1.0), chain=3, dt=0.001, nsteps=10_000)
    done = 0
    for upto, tol in ((1, 2e-5), (50, 1e-4), (200, 5e-4)):
        b.run(upto - done)
        osim.step(upto - done)
        done = upto
        x, v, img = b.state(s)
        o = osim.state()
        L = b.info(s).box_L
        assert abs(L - osim.scalars()["L"]) < 1e-6 * L
        ux = (x + img * L) - (o["x"] + o["image"] * L)
        assert np.max(np.abs(ux)) < tol, (upto, float(np.max(np.abs(ux))))
        assert rel_rms(v, o["v"]) < 50 * tol
        t = b.thermo(s).as_array()
        assert np.allclose(t, osim.thermo(), rtol=2e-3, atol=2e-3), (upto, t, osim.thermo())
    assert b.info(s).rebuilds >= 3
    xf, Lf = b.force_frame(s)
    f, pe, vir = b.forces(s)
    fo, peo, viro = po.forces(oracle_system(d, xyz=xf, L=Lf, lj_table=_lj2_table()))
    assert rel_rms(f, fo) < FORCE_RMS_TOL
    assert _virial_ok(vir, viro, Lf), (vir, viro)
    b.close()


def test_c2_million_bead_snapshot_forces():
    conf = run_conf(ensemble="npt_nh 1.0 1.0 0.1 0.0 0.0 1.0 3", ntypes=2, lj=LJ2, nsteps=10_000)
    b = fm.Batch(max_replicas=1, max_atoms=1_000_200 + 4096)
    s = b.add(conf, gen=dict(nchains=10_000, chain_length=100, density=0.85, seed=2, pushoff_steps=2000,
                             type_block=50))
    b.run(30)
    xf, Lf = b.force_frame(s)
    f, pe, vir = b.forces(s)
    d = fm.generate_melt(10_000, 100, density=0.85, seed=2, type_block=50)
    fo, peo, viro = po.forces(oracle_system(d, xyz=xf, L=Lf, lj_table=_lj2_table()))
    assert rel_rms(f, fo) < FORCE_RMS_TOL
    assert abs(pe.sum() - peo.sum()) < 1e-5 * abs(peo.sum())
    assert _virial_ok(vir, viro, Lf), (vir, viro)
    b.close()


def _wrapped_start(seed=11):
    """A pushed-off 1,000-bead melt whose positions are given unwrapped,
    each coordinate shifted by a random whole number of periods in [-3, 3]
    (image flags zero): loading must wrap them into the box and count the
    periods in the image flags."""
    pre = fm.Simulation(run_conf(), gen=dict(nchains=20, chain_length=50, density=0.85, seed=seed,
                                             pushoff_steps=2000), form=fm.FMD_FORM_MIXED)
    x, v, img = pre.state()
    pre.close()
    d = fm.generate_melt(20, 50, density=0.85, seed=seed)
    k = np.random.default_rng(seed).integers(-3, 4, size=x.shape)
    d.xyz = x + (img + k) * d.box_L
    d.vel = 1.5 * v   # a warm start: more atoms cross faces during the run
    d.image = np.zeros_like(img)
    return d, img + k


@pytest.mark.parametrize("form", [fm.FMD_FORM_PLAIN_FP64, fm.FMD_FORM_MIXED])
def test_image_flags_match_oracle_after_multi_period_runs(form):
    d, img_expect = _wrapped_start()
    conf = run_conf(ensemble="nvt_langevin 2.0 2.0 1.0 5", nsteps=1000)
    sim = fm.Simulation(conf, desc=d, form=form)
    x0, v0, i0 = sim.state()
    L = d.box_L
    assert np.array_equal(i0, img_expect)        # the periods given are counted exactly
    assert np.all((x0 >= 0) & (x0 < L))
    osim = po.Sim(oracle_system(d, xyz=x0, vel=v0, image=i0), ensemble="langevin", T=(2.0, 2.0, 1.0), seed=5,
                  dt=0.001, nsteps=1000)
    crossed = 0
    for n in (10, 40, 100):
        sim.step(n)
        osim.step(n)
        x, v, img = sim.state()
        o = osim.state()
        crossed = int(np.sum(img != i0))
        if form == fm.FMD_FORM_PLAIN_FP64:
            assert np.array_equal(img, o["image"])
            assert np.max(np.abs(x - o["x"])) < 1e-9
        else:
            # FP32 offsets: exact flags away from the faces, unwrapped positions in tolerance
            near = np.minimum(o["x"], L - o["x"]) < 1e-4
            assert np.array_equal(img[~near], o["image"][~near])
            ux = (x + img * L) - (o["x"] + o["image"] * L)
            assert np.max(np.abs(ux)) < 2e-4
    assert crossed > 20   # the run did move atoms across faces
