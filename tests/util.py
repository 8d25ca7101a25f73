"""Shared helpers for the tests: run.conf text, oracle systems built from the
same arrays the library gets, and tolerances."""
from __future__ import annotations

import numpy as np

from oracle import pyoracle as po

KG_BOND = (30.0, 1.5, 1.0, 1.0)      # FENE k, R0, WCA eps, sig
KG_ANGLE = (5.0, 180.0)              # k_theta, theta0 (degrees)


def run_conf(ensemble="nvt_langevin 1.0 1.0 1.0 42", ntypes=1, rc=2.5, skin=0.3, dt=0.001, nsteps=1000,
             lj=None, bond=KG_BOND, angle=KG_ANGLE, extra=""):
    lines = [f"ntypes {ntypes}", f"rc {rc}", f"skin {skin}", f"dt {dt}", f"nsteps {nsteps}", ensemble]
    if lj is None:
        lj = [(i, j, 1.0, 1.0) for i in range(ntypes) for j in range(i, ntypes)]
    for (i, j, e, s) in lj:
        lines.append(f"lj {i} {j} {e} {s}")
    if bond is not None:
        lines.append("bond_type 0 " + " ".join(str(x) for x in bond))
    if angle is not None:
        lines.append("angle_type 0 " + " ".join(str(x) for x in angle))
    if extra:
        lines.append(extra)
    return "\n".join(lines) + "\n"


def oracle_system(desc, xyz=None, rc=2.5, skin=0.3, lj_table=None, bond=KG_BOND, angle=KG_ANGLE, vel=None,
                  image=None, L=None):
    nt = desc.ntypes or int(np.max(desc.type)) + 1
    if lj_table is None:
        lj_table = np.ones((nt, nt, 2))
    return po.System(
        xyz=np.asarray(desc.xyz if xyz is None else xyz, dtype=np.float64).reshape(-1, 3),
        L=float(desc.box_L if L is None else L),
        type=np.asarray(desc.type, np.int32),
        mass=np.asarray(desc.mass if desc.mass is not None else np.ones(nt), np.float64),
        lj=np.asarray(lj_table, np.float64),
        bonds=np.asarray(desc.bonds if desc.bonds is not None else np.zeros((0, 2)), np.int32).reshape(-1, 2),
        bond_type=np.asarray(desc.bond_type if desc.bond_type is not None else np.zeros(0), np.int32),
        fene=np.array([bond], np.float64) if bond is not None else np.zeros((0, 4)),
        angles=np.asarray(desc.angles if desc.angles is not None else np.zeros((0, 3)), np.int32).reshape(-1, 3),
        angle_type=np.asarray(desc.angle_type if desc.angle_type is not None else np.zeros(0), np.int32),
        angle_p=np.array([[angle[0], angle[1] * np.pi / 180.0]]) if angle is not None else np.zeros((0, 2)),
        mol=np.asarray(desc.mol, np.int32) if desc.mol is not None else None,
        vel=None if vel is None else np.asarray(vel, np.float64).reshape(-1, 3),
        image=None if image is None else np.asarray(image, np.int32).reshape(-1, 3),
        rc=rc, skin=skin)


def rel_rms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(np.mean((a - b) ** 2)) / max(np.sqrt(np.mean(b ** 2)), 1e-300))


def pair_set(pi, pj):
    a = np.minimum(pi, pj).astype(np.int64)
    b = np.maximum(pi, pj).astype(np.int64)
    return set((a << 32 | b).tolist())
