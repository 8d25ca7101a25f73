"""Generate the golden fixtures in this directory from the reference's own CPU
code (oracle/_ref/libfmdref.so, compiled from the reference sources by
`make -C oracle ref REF=<reference checkout>`).

Run in a container that has the reference tree; the outputs are committed and
the tests read only the committed files.  Inputs follow the reference's unit
tests (paths within the fastMD project):
  tests/test_pbc.cu:29-41      five minimum-image pairs, L = 10
  tests/test_morton.cu:11-20   64 positions (i*3.7, i*5.3, i*7.1) mod 10
  tests/test_lj.cu:19-27       64 positions from srand(123), L = 8, rc = 2.5
  tests/test_fene.cu:11-20     3-bead chain, bonds 1.0 and 1.2
  tests/test_angle.cu:11-19    right angle, k = 100, theta0 = 120 degrees
  tests/test_tile_list.cu:16-25  128 positions from srand(42), L = 10, rc+skin 3
  tests/test_nose_hoover.cu:374-377  chain trials, KE = 0.5 N T (0.5 + 1.5 u)
glibc rand() streams are reproduced through ctypes and the generated arrays
are stored, so the fixtures do not depend on the C library at test time.
Additional inputs (a seeded melt snapshot, run.conf texts, LAMMPS data files)
are written by this script.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import pyoracle as po  # noqa: E402

libc = C.CDLL("libc.so.6")
RAND_MAX = np.float32(2147483647.0)


def crand_f32():
    return np.float32(libc.rand()) / RAND_MAX


def main():
    R = po.ref_lib()
    if R is None:
        raise SystemExit("oracle/_ref/libfmdref.so missing: run `make -C oracle ref REF=<reference checkout>`")
    out = {}

    # --- PBC minimum image (test_pbc.cu:29-41)
    r1 = np.array([[1, 2, 3], [9.5, 0.5, 5], [0.5, 0.5, 0.5], [5, 5, 5], [0.1, 9.9, 5]], np.float32)
    r2 = np.array([[2, 3, 4], [0.5, 9.5, 5], [9.5, 9.5, 9.5], [5, 5, 5], [9.9, 0.1, 5]], np.float32)
    dr = np.zeros_like(r1)
    for i in range(5):
        for a in range(3):
            dr[i, a] = R.ref_min_image(np.float32(r1[i, a] - r2[i, a]), 10.0, np.float32(0.1))
    out["pbc_r1"], out["pbc_r2"], out["pbc_dr"] = r1, r2, dr

    # --- Morton sort (test_morton.cu:11-20) and a larger seeded set
    i = np.arange(64, dtype=np.float32)
    mpos = np.stack([np.fmod(i * np.float32(3.7), np.float32(10.0)), np.fmod(i * np.float32(5.3), np.float32(10.0)),
                     np.fmod(i * np.float32(7.1), np.float32(10.0))], axis=1).astype(np.float32)
    perm = np.zeros(64, np.int32)
    R.ref_morton_sort(np.ascontiguousarray(mpos.reshape(-1)), 64, np.float32(0.1), perm)
    out["morton_pos"], out["morton_perm"] = mpos, perm
    rng = np.random.default_rng(2024)
    mpos2 = (rng.random((2000, 3)) * 15.0).astype(np.float32)
    perm2 = np.zeros(2000, np.int32)
    R.ref_morton_sort(np.ascontiguousarray(mpos2.reshape(-1)), 2000, np.float32(1.0 / 15.0), perm2)
    keys2 = np.array([R.ref_morton3d(*map(float, p), 1.0 / 15.0) for p in mpos2], np.uint32)
    out["morton2_pos"], out["morton2_perm"], out["morton2_keys"] = mpos2, perm2, keys2

    # --- LJ 64 atoms from srand(123), L = 8 (test_lj.cu)
    libc.srand(123)
    lpos = np.zeros((64, 3), np.float32)
    for k in range(64):
        for a in range(3):
            lpos[k, a] = np.float32(8.0) * crand_f32()
    f = np.zeros(192, np.float32)
    pe = np.zeros(64, np.float32)
    vir = np.zeros(6, np.float32)
    R.ref_brute_force_lj(np.ascontiguousarray(lpos.reshape(-1)), np.zeros(64, np.int32), 64,
                         np.array([1, 1], np.float32), 1, 2.5, 8.0, None, None, f, pe, vir)
    out["lj64_pos"], out["lj64_f"], out["lj64_pe"], out["lj64_vir"] = lpos, f.reshape(64, 3), pe, vir
    cap = 64 * 64
    pi = np.zeros(cap, np.int32)
    pj = np.zeros(cap, np.int32)
    m = R.ref_pairs_within(np.ascontiguousarray(lpos.reshape(-1)), 64, 8.0, 3.0, None, None, pi, pj, cap)
    out["lj64_pairs"] = np.stack([pi[:m], pj[:m]], axis=1)

    # --- FENE 3-bead chain (test_fene.cu) and angle triangle (test_angle.cu)
    fp = np.array([[2, 5, 5], [3, 5, 5], [4.2, 5, 5]], np.float32)
    f = np.zeros(9, np.float32)
    pe = np.zeros(3, np.float32)
    vir = np.zeros(6, np.float32)
    R.ref_brute_force_fene(np.ascontiguousarray(fp.reshape(-1)), 3, np.array([0, 1, 1, 2], np.int32),
                           np.zeros(2, np.int32), 2, np.array([30, 1.5, 1, 1], np.float32), 1, 10.0, f, pe, vir)
    out["fene3_pos"], out["fene3_f"], out["fene3_pe"], out["fene3_vir"] = fp, f.reshape(3, 3), pe.copy(), vir.copy()
    ap = np.array([[3, 5, 5], [5, 5, 5], [5, 7, 5]], np.float32)
    th0 = np.float32(np.pi * 120.0 / 180.0)
    f = np.zeros(9, np.float32)
    pe = np.zeros(3, np.float32)
    vir = np.zeros(6, np.float32)
    R.ref_brute_force_angle(np.ascontiguousarray(ap.reshape(-1)), 3, np.array([0, 1, 2], np.int32),
                            np.zeros(1, np.int32), 1, np.array([100.0, th0], np.float32), 1, 10.0, f, pe, vir)
    out["angle3_pos"], out["angle3_f"], out["angle3_pe"], out["angle3_vir"] = ap, f.reshape(3, 3), pe, vir
    out["angle3_theta0"] = np.array([th0], np.float32)

    # --- Tile pairs, 128 atoms from srand(42), L = 10, rc + skin = 3 (test_tile_list.cu)
    libc.srand(42)
    tpos = np.zeros((128, 3), np.float32)
    for k in range(128):
        for a in range(3):
            tpos[k, a] = np.float32(10.0) * crand_f32()
    tcap = 4 * 4 * 2
    tl = np.zeros(2 * tcap, np.int32)
    mt = R.ref_brute_force_tile_list(np.ascontiguousarray(tpos.reshape(-1)), 128, 4, 3.0, 10.0, tl, tcap)
    out["tile_pos"], out["tile_pairs"] = tpos, tl[: 2 * mt].reshape(-1, 2)
    pi = np.zeros(128 * 128, np.int32)
    pj = np.zeros(128 * 128, np.int32)
    m = R.ref_pairs_within(np.ascontiguousarray(tpos.reshape(-1)), 128, 10.0, 3.0, None, None, pi, pj, 128 * 128)
    out["tile_atom_pairs"] = np.stack([pi[:m], pj[:m]], axis=1)

    # --- Melt snapshot (library generator, 600 beads, bonds + angles): FP32
    # reference forces and pair set with 1-2 exclusions.
    import fastmd_b200 as fm  # host-only generator, no GPU needed
    d = fm.generate_melt(12, 50, density=0.85, seed=99)
    n = len(d.type)
    mx = d.xyz.astype(np.float32)
    bonds = d.bonds.astype(np.int32)
    angles = d.angles.astype(np.int32)
    eo = np.zeros(n + 1, np.int32)
    per = [[] for _ in range(n)]
    for a, b in bonds:
        per[a].append(b)
        per[b].append(a)
    el = []
    for k in range(n):
        lst = sorted(set(per[k]))
        eo[k] = len(el)
        el += lst
    eo[n] = len(el)
    el = np.array(el, np.int32)
    L32 = np.float32(d.box_L)
    f = np.zeros(3 * n, np.float32)
    pe = np.zeros(n, np.float32)
    vir = np.zeros(6, np.float32)
    R.ref_brute_force_lj(np.ascontiguousarray(mx.reshape(-1)), np.zeros(n, np.int32), n, np.array([1, 1], np.float32),
                         1, 2.5, L32, eo.ctypes.data, el.ctypes.data, f, pe, vir)
    out["melt_pos"], out["melt_L"] = mx, np.array([L32], np.float32)
    out["melt_bonds"], out["melt_angles"], out["melt_mol"] = bonds, angles, d.mol.astype(np.int32)
    out["melt_lj_f"], out["melt_lj_pe"], out["melt_lj_vir"] = f.reshape(n, 3), pe.copy(), vir.copy()
    f = np.zeros(3 * n, np.float32)
    pe = np.zeros(n, np.float32)
    vir = np.zeros(6, np.float32)
    R.ref_brute_force_fene(np.ascontiguousarray(mx.reshape(-1)), n, np.ascontiguousarray(bonds.reshape(-1)),
                           np.zeros(len(bonds), np.int32), len(bonds), np.array([30, 1.5, 1, 1], np.float32), 1, L32,
                           f, pe, vir)
    out["melt_fene_f"], out["melt_fene_pe"], out["melt_fene_vir"] = f.reshape(n, 3), pe.copy(), vir.copy()
    f = np.zeros(3 * n, np.float32)
    pe = np.zeros(n, np.float32)
    vir = np.zeros(6, np.float32)
    R.ref_brute_force_angle(np.ascontiguousarray(mx.reshape(-1)), n, np.ascontiguousarray(angles.reshape(-1)),
                            np.zeros(len(angles), np.int32), len(angles),
                            np.array([5.0, np.float32(np.pi)], np.float32), 1, L32, f, pe, vir)
    out["melt_angle_f"], out["melt_angle_pe"], out["melt_angle_vir"] = f.reshape(n, 3), pe.copy(), vir.copy()
    cap = n * 200
    pi = np.zeros(cap, np.int32)
    pj = np.zeros(cap, np.int32)
    m = R.ref_pairs_within(np.ascontiguousarray(mx.reshape(-1)), n, L32, np.float32(2.8), eo.ctypes.data,
                           el.ctypes.data, pi, pj, cap)
    out["melt_pairs"] = np.stack([pi[:m], pj[:m]], axis=1)

    # --- Nose-Hoover chain trials (test_nose_hoover.cu:343-444): the host
    # chain from a running state, KE = 0.5 N T (0.5 + 1.5 u), srand(12345).
    N, M, Tdamp, T, hdt = 100, 3, np.float32(0.5), np.float32(1.5), np.float32(0.001)
    xi = np.zeros(3, np.float32)
    vxi = np.zeros(3, np.float32)
    libc.srand(12345)
    rows = []
    Q = np.zeros(2, np.float32)
    for t in range(200):
        u = crand_f32()
        ke = np.float32(0.5) * np.float32(N) * T * (np.float32(0.5) + u * np.float32(1.5))
        x0, v0 = xi.copy(), vxi.copy()
        sc = C.c_float()
        R.ref_nh_chain(N, T, Tdamp, M, xi, vxi, ke, hdt, C.byref(sc), Q)
        rows.append(np.concatenate([[ke], x0, v0, [sc.value], xi, vxi]))
    out["nhc_trials"] = np.array(rows, np.float32)
    out["nhc_Q"] = Q.copy()

    # --- run.conf texts and LAMMPS data files through the reference parsers
    confs = {
        "kg_langevin": "# Kremer-Grest melt\nnatoms 3000\nntypes 1\nrc 2.5\nskin 0.3\ndt 0.001\nnsteps 5000\n"
                       "nvt_langevin 1.0 1.0 1.0 42\nthermo 1 100 thermo.dat\nrg 1 100 rg.dat\nlj 0 0 1.0 1.0\n"
                       "bond_type 0 30.0 1.5 1.0 1.0\nangle_type 0 5.0 180.0\nlammps_data_file melt.data\n",
        "two_type_npt": "natoms 1000000\nntypes 2\nrc 2.5\nskin 0.3\ndt 0.001\nnsteps 20000\n"
                        "npt_nh 1.0 1.0 0.1 0.0 0.0 1.0 3\nlj 0 0 1.0 1.0\nlj 1 1 1.0 1.0\nlj 0 1 0.9 1.0\n"
                        "bond_type 0 30.0 1.5 1.0 1.0\nangle_type 0 5.0 180.0\nthermo_freq 100\n",
        "nvt_default_chain": "ntypes 1\nrc 2.5\nskin 0.4\ndt 0.002\nnsteps 10\nnvt_nh 1.5 1.5 0.5\n"
                             "lj 0 0 1.0 1.0\n",
        "langevin_default_seed": "ntypes 1\nrc 2.5\nskin 0.3\ndt 0.001\nnsteps 100\nnvt_langevin 1.0 2.0 0.5\n"
                                 "lj 0 0 1.0 1.0\n",
    }
    bad_confs = {
        "deprecated_temperature": "ntypes 1\nrc 2.5\nskin 0.3\ndt 0.001\ntemperature 1.0\n",
        "deprecated_seed": "ntypes 1\nrc 2.5\nskin 0.3\ndt 0.001\nseed 5\n",
        "zero_tdamp": "ntypes 1\nrc 2.5\nskin 0.3\ndt 0.001\nnvt_langevin 1.0 1.0 0.0\nlj 0 0 1 1\n",
        "npt_zero_pdamp": "ntypes 1\nrc 2.5\nskin 0.3\ndt 0.001\nnpt_nh 1.0 1.0 0.5 0 0 0.0\nlj 0 0 1 1\n",
    }
    tmp = os.path.join(HERE, "_tmp_conf")
    parsed = {}
    for name, text in {**confs, **bad_confs}.items():
        with open(tmp, "w") as fh:
            fh.write(text)
        fo = np.zeros(9, np.float32)
        io = np.zeros(12, np.int32)
        lj = np.zeros(2 * 16 * 16, np.float32)
        bd = np.zeros(64, np.float32)
        an = np.zeros(64, np.float32)
        seed = C.c_uint64()
        err = C.create_string_buffer(256)
        rc = R.ref_parse_config(tmp.encode(), fo, io, lj, len(lj), bd, len(bd), an, len(an), C.byref(seed), err, 256)
        parsed[name] = dict(rc=rc, f=fo.copy(), i=io.copy(), lj=lj[: 2 * io[1] * io[1]].copy(),
                            bond=bd[: 4 * io[10]].copy(), angle=an[: 2 * io[11]].copy(), seed=seed.value)
        with open(os.path.join(HERE, f"conf_{name}.conf"), "w") as fh:
            fh.write(text)
    os.remove(tmp)
    for name, p in parsed.items():
        out[f"conf_{name}_rc"] = np.array([p["rc"]], np.int32)
        out[f"conf_{name}_f"] = p["f"]
        out[f"conf_{name}_i"] = p["i"]
        out[f"conf_{name}_lj"] = p["lj"]
        out[f"conf_{name}_bond"] = p["bond"]
        out[f"conf_{name}_angle"] = p["angle"]
        out[f"conf_{name}_seed"] = np.array([p["seed"]], np.uint64)

    data_files = {
        "full_style": _data_full(),
        "molecular_images": _data_molecular(),
        "atomic_velocities": _data_atomic(),
    }
    for name, text in data_files.items():
        path = os.path.join(HERE, f"data_{name}.data")
        with open(path, "w") as fh:
            fh.write(text)
        counts = np.zeros(4, np.int32)
        Lc = C.c_float()
        err = C.create_string_buffer(256)
        R.ref_parse_lammps_data(path.encode(), counts, C.byref(Lc), *([None] * 10), err, 256)
        n, nb, na, nm = (int(x) for x in counts)
        arrs = dict(xyz=np.zeros(3 * n, np.float32), type=np.zeros(n, np.int32), mol=np.zeros(n, np.int32),
                    image=np.zeros(3 * n, np.int32), vel=np.zeros(3 * n, np.float32),
                    bonds=np.zeros(2 * max(nb, 1), np.int32), btype=np.zeros(max(nb, 1), np.int32),
                    angles=np.zeros(3 * max(na, 1), np.int32), atype=np.zeros(max(na, 1), np.int32),
                    masses=np.zeros(max(nm, 1), np.float32))
        R.ref_parse_lammps_data(path.encode(), counts, C.byref(Lc), *[arrs[k].ctypes.data for k in
                                ("xyz", "type", "mol", "image", "vel", "bonds", "btype", "angles", "atype", "masses")],
                                err, 256)
        out[f"data_{name}_counts"] = counts.copy()
        out[f"data_{name}_L"] = np.array([Lc.value], np.float32)
        for k, v in arrs.items():
            out[f"data_{name}_{k}"] = v

    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)
    print("wrote", os.path.join(HERE, "golden.npz"), len(out), "arrays")


def _data_full():
    rng = np.random.default_rng(7)
    lines = ["LAMMPS data file: two 5-bead chains, atom style full", "", "10 atoms", "8 bonds", "6 angles", "",
             "2 atom types", "1 bond types", "1 angle types", "", "0.0 12.0 xlo xhi", "0.0 12.0 ylo yhi",
             "0.0 12.0 zlo zhi", "", "Masses", "", "1 1.0", "2 2.5", "", "Atoms # full", ""]
    ids = [3, 1, 2, 5, 4, 8, 6, 7, 10, 9]   # ids out of order on purpose
    for k, aid in enumerate(ids):
        mol = 1 if aid <= 5 else 2
        t = 1 if aid % 2 else 2
        x, y, z = rng.random(3) * 12.0
        lines.append(f"{aid} {mol} {t} 0.0 {x:.6f} {y:.6f} {z:.6f} {k % 2} 0 {-(k % 3)}")
    lines += ["", "Velocities", ""]
    for aid in range(1, 11):
        vx, vy, vz = rng.normal(size=3)
        lines.append(f"{aid} {vx:.6f} {vy:.6f} {vz:.6f}")
    lines += ["", "Bonds", ""]
    b = 1
    for c0 in (1, 6):
        for k in range(4):
            lines.append(f"{b} 1 {c0 + k} {c0 + k + 1}")
            b += 1
    lines += ["", "Angles", ""]
    a = 1
    for c0 in (1, 6):
        for k in range(3):
            lines.append(f"{a} 1 {c0 + k} {c0 + k + 1} {c0 + k + 2}")
            a += 1
    return "\n".join(lines) + "\n"


def _data_molecular():
    lines = ["molecular style with image flags", "", "4 atoms", "3 bonds", "2 angles", "", "1 atom types", "",
             "-2.0 8.0 xlo xhi", "-2.0 8.0 ylo yhi", "-2.0 8.0 zlo zhi", "", "Atoms # molecular", "",
             "1 7 1 1.0 2.0 3.0 0 0 0", "2 7 1 2.0 3.0 4.0 1 -1 0", "3 7 1 3.0 4.0 5.0 1 -1 2",
             "4 7 1 4.0 5.0 6.0", "", "Bonds", "", "1 1 1 2", "2 1 2 3", "3 1 3 4", "", "Angles", "",
             "1 1 1 2 3", "2 1 2 3 4"]
    return "\n".join(lines) + "\n"


def _data_atomic():
    lines = ["atomic style with velocities and comments", "", "3 atoms", "", "1 atom types", "",
             "0 5 xlo xhi", "0 5 ylo yhi", "0 5 zlo zhi", "", "Masses", "", "1 3.0", "",
             "Atoms # atomic", "", "1 1 0.5 0.5 0.5", "# a comment line", "2 1 1.5 1.5 1.5 0 0 1",
             "3 1 2.5 2.5 2.5", "", "Velocities", "", "2 0.1 0.2 0.3", "3 -1 -2 -3", "1 1 0 0"]
    return "\n".join(lines) + "\n"


if __name__ == "__main__":
    main()
