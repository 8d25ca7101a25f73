"""Pair-table input: the library's table-file reader and run.conf 'table'
key against the reference's own parser (io/table_parser.cpp, compiled here
from the reference sources when present) and the rules of io/config.cpp:136-162.
Fixture files are generated here; no reference fixture is copied."""
import ctypes as C

import numpy as np
import pytest

import fastmd_b200 as fm
from oracle import pyoracle as po
from tests.util import run_conf


def _write_table(path, keyword, r, e, f, header="R", comment=True):
    lines = []
    if comment:
        lines.append("# generated pair table")
    lines.append("OTHER_SECTION")
    lines.append("N 2 R 0.1 0.2")
    lines.append("")
    lines.append("1 0.1 0 0")
    lines.append("2 0.2 0 0")
    lines.append(keyword)
    if header == "R":
        lines.append(f"N {len(r)} R {r[0]} {r[-1]}")
    else:
        lines.append(f"N {len(r)}")
    lines.append("")
    for k, (a, b, c) in enumerate(zip(r, e, f)):
        lines.append(f"{k + 1} {a:.6f} {b:.6f} {c:.6f}")
    path.write_text("\n".join(lines) + "\n")


def _ref_table(path, keyword):
    R = po.ref_lib()
    if R is None:
        pytest.skip("reference sources absent: oracle/_ref not built")
    grid = np.zeros(4, np.float32)
    n = C.c_int32()
    data = np.zeros(3 * 100000, np.float32)
    err = C.create_string_buffer(256)
    rc = R.ref_parse_table(str(path).encode(), keyword.encode(), grid, C.byref(n), data, 100000, err, 256)
    return rc, grid, n.value, data[:3 * n.value].reshape(-1, 3), err.value.decode()


@pytest.mark.parametrize("header", ["R", "N"])
def test_reader_matches_reference_parser(tmp_path, header):
    rng = np.random.default_rng(3)
    r = np.linspace(0.8, 2.5, 37)
    e = rng.normal(size=r.size)
    f = rng.normal(size=r.size) * 10
    p = tmp_path / "t.table"
    _write_table(p, "MY_PAIR", r, e, f, header=header)
    ours = fm.read_pair_table(p, "MY_PAIR")
    rc, grid, n, data, _ = _ref_table(p, "MY_PAIR")
    assert rc == 0 and n == len(ours["r"])
    assert np.array_equal(np.float32([ours["rmin"], ours["rmax"], ours["dr"], ours["inv_dr"]]), grid)
    assert np.array_equal(ours["r"], data[:, 0]) and np.array_equal(ours["f"], data[:, 1])
    assert np.array_equal(ours["e"], data[:, 2])


def test_reader_errors_as_reference(tmp_path):
    p = tmp_path / "bad.table"
    p.write_text("WRONG\nN 2 R 0 1\n\n1 0 0 0\n2 1 0 0\n")
    with pytest.raises(fm.FastMDError):
        fm.read_pair_table(p, "RIGHT")
    assert _ref_table(p, "RIGHT")[0] == 1
    p.write_text("K\nN 3\n\n1 0.5 0 0\n2 0.4 0 0\n3 0.6 0 0\n")  # r not increasing
    with pytest.raises(fm.FastMDError):
        fm.read_pair_table(p, "K")
    assert _ref_table(p, "K")[0] == 1
    p.write_text("K\nN 3\n\n1 0.5 0 0\n2 0.6 0 0\n")  # too few lines
    with pytest.raises(fm.FastMDError):
        fm.read_pair_table(p, "K")
    assert _ref_table(p, "K")[0] == 1


def test_run_conf_table_rules(tmp_path):
    p = tmp_path / "a.table"
    _write_table(p, "AA", np.linspace(0.5, 2.5, 11), np.zeros(11), np.zeros(11))
    _write_table(tmp_path / "b.table", "BB", np.linspace(0.5, 2.5, 11), np.zeros(11), np.zeros(11))
    lj = [(0, 0, 1.0, 1.0)]
    conf = run_conf(ntypes=3, lj=lj, extra=f"table 1 2 {p} AA\ntable 2 2 {p} AA\ntable 1 1 {tmp_path / 'b.table'} BB")
    tab, n = fm.run_conf_tables(conf)
    assert n == 2  # one table per distinct (file, keyword)
    assert tab[1, 2] == tab[2, 1] == tab[2, 2] == 0 and tab[1, 1] == 1
    assert tab[0, 0] == -1 and tab[0, 1] == -1
    # lj and table for the same pair is an error (config.cpp:143-146)
    with pytest.raises(fm.FastMDError):
        fm.run_conf_tables(run_conf(ntypes=1, lj=lj, extra=f"table 0 0 {p} AA"))
    with pytest.raises(fm.FastMDError):
        fm.run_conf_tables(run_conf(ntypes=2, lj=lj, extra=f"table 0 2 {p} AA"))
