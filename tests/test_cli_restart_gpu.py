"""The `fastmd <run.conf>` program and exact restarts, on the GPU.

* Restart exactness: run N steps, write a restart (data file + state
  sidecar), run M more; a second simulation created from that data file runs
  M steps: positions, velocities, image flags and the thermo row must be
  bit-identical in the mixed form, for every ensemble (the Langevin noise is
  keyed on the step counter the sidecar carries; the Nose-Hoover chain and
  barostat state come from the sidecar).  The plain FP64 form scatters its
  bonded forces with atomics, as the reference does, so two of its runs agree
  to FP64 round-off (1e-10 here), not bit for bit; its image flags and step
  counter must still match exactly.
* The program over the C ABI: on a pushed-off 3,000-bead melt it writes the
  thermo and rg files with the reference's headers and row formats
  (analysis/thermo.cu:80, 190-192; analysis/rg.cu:95, 127-129), the restart
  files <base>_<step><ext> and <base>_final<ext> (io/lammps_data.cpp:255-267),
  traj.bin frames and the stress autocorrelation file, and its thermo rows
  equal those of the same run driven through the Python bindings."""
import os
import re
import struct
import subprocess

import numpy as np
import pytest

import fastmd_b200 as fm
from tests.util import run_conf

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "fastmd_b200", "bin", "fastmd")
ENSEMBLES = ["nvt_langevin 1.0 1.2 1.0 9", "nvt_nh 1.0 1.0 0.5 3", "npt_nh 1.0 1.0 0.5 0.5 0.5 1.0 3",
             # the carried chain accelerations come back from the sidecar too
             "npt_nh 1.0 1.0 0.1 0.5 0.5 1.0 3\nnh_chain_carry 1"]


def _pushed(nchains=20, length=50, seed=11):
    pre = fm.Simulation(run_conf(), gen=dict(nchains=nchains, chain_length=length, density=0.85, seed=seed,
                                             pushoff_steps=2000), form=fm.FMD_FORM_MIXED)
    x, v, img = pre.state()
    pre.close()
    d = fm.generate_melt(nchains, length, density=0.85, seed=seed)
    d.xyz, d.vel, d.image = x, v, img
    return d


@pytest.mark.parametrize("form", [fm.FMD_FORM_PLAIN_FP64, fm.FMD_FORM_MIXED])
@pytest.mark.parametrize("ens", ENSEMBLES)
def test_restart_resumes_bit_identically(tmp_path, form, ens):
    d = _pushed()
    conf = run_conf(ensemble=ens, nsteps=1000)
    a = fm.Simulation(conf, desc=d, form=form)
    a.step(37)
    path = str(tmp_path / "restart.data")
    a.write_restart(path)
    assert os.path.exists(path + ".state")
    a.step(45)
    xa, va, ia = a.state()
    ta = a.thermo().as_array()
    b = fm.Simulation(conf, data_path=path, form=form)
    assert b.step_count == 37
    b.step(45)
    xb, vb, ib = b.state()
    assert b.step_count == a.step_count == 82
    assert np.array_equal(ia, ib)
    if form == fm.FMD_FORM_MIXED:
        assert np.array_equal(xa, xb) and np.array_equal(va, vb)
        assert np.array_equal(ta, b.thermo().as_array())
    else:
        assert np.max(np.abs(xa - xb)) < 1e-10 and np.max(np.abs(va - vb)) < 1e-10
        assert np.allclose(ta, b.thermo().as_array(), rtol=1e-10, atol=1e-12)
    a.close()
    b.close()


def test_batch_restart_resumes_bit_identically(tmp_path):
    d = _pushed(seed=5)
    conf = run_conf(ensemble="nvt_nh 1.0 1.0 0.5 3", nsteps=1000)
    a = fm.Batch(max_replicas=2, max_atoms=1 << 14)
    sa = a.add(conf, desc=d)
    a.run(30)
    path = str(tmp_path / "rep.data")
    a.write_restart(sa, path)
    a.run(40)
    b = fm.Batch(max_replicas=2, max_atoms=1 << 14)
    sb = b.add(conf, data_path=path)
    assert b.info(sb).step == 30
    b.run(40)
    for x, y in zip(a.state(sa), b.state(sb)):
        assert np.array_equal(x, y)
    a.close()
    b.close()


THERMO_ROW = re.compile(r"^\d+(  -?\d+\.\d{4}){9}$")
RG_ROW = re.compile(r"^\d+  -?\d+\.\d{4}$")


def test_cli_writes_the_reference_outputs(tmp_path):
    assert os.path.exists(CLI), "fastmd_b200/bin/fastmd is not built (make -C fastmd_b200/csrc)"
    d = _pushed(nchains=30, length=100, seed=42)
    fm.write_lammps_data(str(tmp_path / "melt.data"), d)
    conf = run_conf(ensemble="nvt_langevin 1.0 1.0 1.0 42", nsteps=200,
                    extra="thermo 1 50 thermo.dat\nrg 1 50 rg.dat\nrestart 100 restart.data\ndump_freq 100\n"
                          "stress 1 10 stress.dat\nlammps_data_file melt.data")
    (tmp_path / "run.conf").write_text(conf)
    out = subprocess.run([CLI, "run.conf"], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    assert "Wall time:" in out.stdout and "Steps/s:" in out.stdout
    th = (tmp_path / "thermo.dat").read_text().splitlines()
    assert th[0] == "# step  KE  PE  T  Pxx  Pyy  Pzz  Pxy  Pxz  Pyz"
    assert [int(r.split()[0]) for r in th[1:]] == [50, 100, 150, 200]
    assert all(THERMO_ROW.match(r) for r in th[1:]), th[1:]
    rg = (tmp_path / "rg.dat").read_text().splitlines()
    assert rg[0] == "# step  Rg"
    assert [int(r.split()[0]) for r in rg[1:]] == [50, 100, 150, 200]
    assert all(RG_ROW.match(r) for r in rg[1:])
    for name in ("restart_100.data", "restart_final.data"):
        assert (tmp_path / name).exists() and (tmp_path / (name + ".state")).exists()
    assert not (tmp_path / "restart_200.data").exists()   # the last step writes only the final file
    raw = (tmp_path / "traj.bin").read_bytes()
    magic, n, nt = struct.unpack("<iii", raw[:12])
    assert magic == 0x4D444247 and n == 3000
    assert len(raw) == 12 + 2 * (8 + 4 + 4 + 12 * n)
    st = (tmp_path / "stress.dat").read_text().splitlines()
    assert st[0] == "# lag_steps  C_xx  C_xy  C_xz  C_yy  C_yz  C_zz  count" and len(st) > 1
    # the same run through the Python bindings gives the same rows
    sim = fm.Simulation(conf, data_path=str(tmp_path / "melt.data"))
    rows = []
    for k in range(4):
        sim.step(50)
        rows.append(fm.format_thermo_row(sim.thermo()))
        if sim.step_count == 100:
            sim.write_restart(str(tmp_path / "py_restart.data"))
    assert rows == th[1:]
    sim.close()
