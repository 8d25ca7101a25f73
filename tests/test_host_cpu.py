"""Host-side pieces of the library that need no GPU: the run.conf parser and
the LAMMPS data reader against the reference's own parsers (golden fixtures),
the melt generator, reference text rows, error codes, and the exported C ABI.
"""
import ctypes as C
import os
import re

import numpy as np
import pytest

import fastmd_b200 as fm
from fastmd_b200 import FastMDError
from oracle import pyoracle as po
from tests.util import pair_set, run_conf

HERE = os.path.dirname(os.path.abspath(__file__))
GD = os.path.join(HERE, "golden")
G = np.load(os.path.join(GD, "golden.npz"))
ROOT = os.path.dirname(HERE)

GOOD = ["kg_langevin", "two_type_npt", "nvt_default_chain", "langevin_default_seed"]
BAD = ["deprecated_temperature", "deprecated_seed", "zero_tdamp", "npt_zero_pdamp"]


@pytest.mark.parametrize("name", GOOD)
def test_run_conf_matches_reference_parser(name):
    text = open(os.path.join(GD, f"conf_{name}.conf")).read()
    assert G[f"conf_{name}_rc"][0] == 0
    c = fm.parse_run_conf(text)
    fo, io = G[f"conf_{name}_f"], G[f"conf_{name}_i"]
    got_f = [c["rc"], c["skin"], c["dt"], c["T_start"], c["T_stop"], c["Tdamp"], c["P_start"], c["P_stop"],
             c["Pdamp"]]
    assert np.allclose(got_f, fo, rtol=1e-6)
    assert c["natoms"] == io[0] and c["ntypes"] == io[1] and c["nsteps"] == io[2]
    assert c["ensemble"] == io[3] and c["chain_length"] == io[4]
    assert (c["thermo_on"], c["thermo_freq"], c["rg_on"], c["rg_freq"]) == tuple(io[5:9])
    assert np.allclose(c["lj"].reshape(-1), G[f"conf_{name}_lj"], rtol=1e-6)
    assert np.allclose(c["bond"].reshape(-1), G[f"conf_{name}_bond"], rtol=1e-6)
    assert np.allclose(c["angle"].reshape(-1), G[f"conf_{name}_angle"], rtol=1e-6)
    assert c["seed"] == int(G[f"conf_{name}_seed"][0])


@pytest.mark.parametrize("name", BAD)
def test_run_conf_rejects_like_reference(name):
    text = open(os.path.join(GD, f"conf_{name}.conf")).read()
    assert G[f"conf_{name}_rc"][0] == 1   # the reference throws
    with pytest.raises(FastMDError) as e:
        fm.parse_run_conf(text)
    assert e.value.code == 2


def test_run_conf_table_file_must_exist(tmp_path):
    # config.cpp:152 reads the table file while parsing; a missing file is an
    # I/O error, not a silently ignored key
    missing = tmp_path / "absent.table"
    with pytest.raises(FastMDError) as e:
        fm.parse_run_conf(f"ntypes 1\nrc 2.5\nskin 0.3\ndt 0.001\nnvt_langevin 1 1 1\ntable 0 0 {missing} KW\n")
    assert e.value.code == 3 and "absent.table" in str(e.value)


@pytest.mark.parametrize("name", ["full_style", "molecular_images", "atomic_velocities"])
def test_lammps_data_matches_reference_reader(name):
    d = fm.read_lammps_data(os.path.join(GD, f"data_{name}.data"))
    cnt = G[f"data_{name}_counts"]
    n, nb, na = int(cnt[0]), int(cnt[1]), int(cnt[2])
    assert len(d.type) == n and len(d.bonds) == nb and len(d.angles) == na
    assert abs(d.box_L - G[f"data_{name}_L"][0]) < 1e-6
    assert np.allclose(d.xyz.reshape(-1), G[f"data_{name}_xyz"], atol=1e-6)
    assert np.array_equal(d.type, G[f"data_{name}_type"])
    assert np.array_equal(d.mol, G[f"data_{name}_mol"])
    assert np.array_equal(d.image.reshape(-1), G[f"data_{name}_image"])
    assert np.allclose(d.vel.reshape(-1), G[f"data_{name}_vel"], atol=1e-6)
    if nb:
        assert np.array_equal(d.bonds.reshape(-1), G[f"data_{name}_bonds"][: 2 * nb])
        assert np.array_equal(d.bond_type, G[f"data_{name}_btype"][:nb])
    if na:
        assert np.array_equal(d.angles.reshape(-1), G[f"data_{name}_angles"][: 3 * na])
    assert np.allclose(d.mass, G[f"data_{name}_masses"][: len(d.mass)], atol=1e-6)


def test_lammps_data_errors():
    with pytest.raises(FastMDError) as e:
        fm.read_lammps_data("/nonexistent/file.data")
    assert e.value.code == 3
    p = os.path.join(HERE, "_tmp_noncubic.data")
    with open(p, "w") as f:
        f.write("x\n\n1 atoms\n\n0 10 xlo xhi\n0 11 ylo yhi\n0 10 zlo zhi\n\nAtoms # atomic\n\n1 1 1 1 1\n")
    try:
        with pytest.raises(FastMDError):
            fm.read_lammps_data(p)
    finally:
        os.remove(p)


def test_generator_is_seeded_and_respects_spec():
    a = fm.generate_melt(30, 100, density=0.85, seed=42)
    b = fm.generate_melt(30, 100, density=0.85, seed=42)
    c = fm.generate_melt(30, 100, density=0.85, seed=43)
    assert np.array_equal(a.xyz, b.xyz) and not np.array_equal(a.xyz, c.xyz)
    n = 3000
    assert abs(a.box_L - (n / 0.85) ** (1 / 3)) < 1e-12
    assert a.xyz.min() >= 0 and a.xyz.max() < a.box_L
    un = a.xyz + a.image * a.box_L
    bl = np.linalg.norm(un[a.bonds[:, 1]] - un[a.bonds[:, 0]], axis=1)
    assert np.allclose(bl, 0.97, atol=1e-9)
    assert len(a.bonds) == 30 * 99 and len(a.angles) == 30 * 98
    assert np.array_equal(np.unique(a.mol), np.arange(1, 31))
    # non-bonded beads mostly at least 0.8 apart
    pi, pj = po.pairs_brute(a.xyz, a.box_L, 0.8, bonds=a.bonds)
    assert len(pi) < 0.03 * n
    t = fm.generate_melt(4, 100, seed=1, type_block=50)
    assert np.array_equal(t.type[:100], np.repeat([0, 1], 50))


def test_text_rows_match_reference_format():
    r = fm.ThermoRow()
    r.step = 100
    r.ke, r.pe, r.temp = 1.5, -4.25, 1.0
    for k in range(6):
        r.stress[k] = 0.1 * (k + 1)
    s = fm.format_thermo_row(r)
    assert s == "100  1.5000  -4.2500  1.0000  0.1000  0.2000  0.3000  0.4000  0.5000  0.6000"
    assert fm.format_rg_row(200, 3.14159) == "200  3.1416"


def _header_symbols():
    text = open(os.path.join(ROOT, "include", "fastmd.h")).read()
    return sorted(set(re.findall(r"FMD_API\s+[\w\s\*]+?\b(fmd_\w+)\s*\(", text)))


def test_library_exports_every_header_symbol():
    lib = fm.lib()
    syms = _header_symbols()
    assert len(syms) > 30
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_no_device_is_reported_not_crashed():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(FastMDError) as e:
        fm.Simulation(run_conf(), gen=dict(nchains=20, chain_length=10, density=0.5, seed=1))
    assert e.value.code == 9


def test_bad_arguments_are_status_codes():
    lib = fm.lib()
    lib.fmd_step.restype = C.c_int32
    assert lib.fmd_step(None, C.c_int64(1)) == 1
    lib.fmd_batch_run.restype = C.c_int32
    assert lib.fmd_batch_run(None, C.c_int64(1)) == 1
    buf = C.create_string_buffer(128)
    lib.fmd_last_error(buf, 128)
    assert b"null" in buf.value


def test_lammps_data_writer_round_trip(tmp_path):
    d = fm.generate_melt(5, 20, density=0.85, seed=3, type_block=10)
    rng = np.random.default_rng(0)
    d.vel = rng.normal(size=d.xyz.shape)
    d.mass = np.array([1.0, 2.5])
    d.ntypes = 2
    p = tmp_path / "rt.data"
    fm.write_lammps_data(p, d, step=1234)
    text = p.read_text()
    assert text.startswith("# Restart from step 1234")
    assert "zlo zhi" in text and "Atoms # full" in text
    e = fm.read_lammps_data(str(p))
    assert np.array_equal(e.xyz, d.xyz) and np.array_equal(e.vel, d.vel)
    assert np.array_equal(e.image, d.image) and np.array_equal(e.type, d.type)
    assert np.array_equal(e.mol, d.mol) and np.array_equal(e.bonds, d.bonds)
    assert np.array_equal(e.angles, d.angles) and np.allclose(e.mass, d.mass)
    assert e.box_L == d.box_L


def test_lammps_data_writer_is_read_by_reference_reader(tmp_path):
    """The reference's own parser (io/lammps_data.cpp) reads the written file."""
    R = po.ref_lib()
    if R is None:
        pytest.skip("reference CPU code not built")
    d = fm.generate_melt(4, 10, density=0.85, seed=5)
    p = tmp_path / "ref.data"
    fm.write_lammps_data(p, d)
    counts = np.zeros(4, np.int32)
    Lc = C.c_float()
    err = C.create_string_buffer(256)
    assert R.ref_parse_lammps_data(str(p).encode(), counts, C.byref(Lc),
                                   *([None] * 10), err, 256) == 0, err.value
    n, nb, na = (int(x) for x in counts[:3])
    assert (n, nb, na) == (40, 36, 32)
    assert abs(Lc.value - d.box_L) < 1e-5
    xyz = np.zeros(3 * n, np.float32)
    i32 = lambda k: np.zeros(k, np.int32)
    # xyz, type, mol, image, vel, bonds, bond types, angles, angle types, masses
    arrs = [xyz, i32(n), i32(n), i32(3 * n), np.zeros(3 * n, np.float32), i32(2 * nb), i32(nb), i32(3 * na), i32(na),
            np.zeros(8, np.float32)]
    assert R.ref_parse_lammps_data(str(p).encode(), counts, C.byref(Lc),
                                   *[a.ctypes.data for a in arrs], err, 256) == 0
    assert np.allclose(xyz, d.xyz.reshape(-1), atol=1e-5)
    assert np.array_equal(arrs[3], d.image.reshape(-1))
    assert np.array_equal(arrs[5], d.bonds.reshape(-1)) and np.array_equal(arrs[7], d.angles.reshape(-1))
