"""ctypes bindings for the FP64 CPU oracle (liboracle.so) and for the
reference's own CPU code (_ref/libfmdref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py, as the checker.  The library never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")


class OrcSystem(C.Structure):
    _fields_ = [
        ("natoms", C.c_int32), ("ntypes", C.c_int32),
        ("type", C.c_void_p), ("mol", C.c_void_p), ("mass", C.c_void_p), ("lj", C.c_void_p),
        ("nbonds", C.c_int32), ("bonds", C.c_void_p), ("bond_type", C.c_void_p),
        ("nbond_types", C.c_int32), ("fene", C.c_void_p),
        ("nangles", C.c_int32), ("angles", C.c_void_p), ("angle_type", C.c_void_p),
        ("nangle_types", C.c_int32), ("angle_p", C.c_void_p),
        ("rc", C.c_double), ("skin", C.c_double),
        ("lj_clamp", C.c_int32), ("fene_clamp", C.c_int32),
    ]


class OrcRun(C.Structure):
    _fields_ = [
        ("ensemble", C.c_int32), ("dt", C.c_double),
        ("T_start", C.c_double), ("T_stop", C.c_double), ("Tdamp", C.c_double),
        ("P_start", C.c_double), ("P_stop", C.c_double), ("Pdamp", C.c_double),
        ("chain_length", C.c_int32), ("seed", C.c_uint64), ("nsteps", C.c_int64),
        ("max_steps_between_rebuilds", C.c_int32), ("force_cap", C.c_double),
        ("nthreads", C.c_int32), ("chain_carry", C.c_int32),
    ]


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle/liboracle.so is not built (run `make -C oracle`)")
        L = C.CDLL(path)
        L.orc_philox.argtypes = [u32p, C.c_uint32, C.c_uint32, u32p]
        L.orc_normal3.argtypes = [C.c_uint64, C.c_uint32, C.c_uint64, C.c_uint32, f64p]
        L.orc_min_image.restype = C.c_double
        L.orc_min_image.argtypes = [C.c_double] * 3
        L.orc_wrap.restype = C.c_double
        L.orc_wrap.argtypes = [C.c_double] * 3
        L.orc_min_image_f32.restype = C.c_float
        L.orc_min_image_f32.argtypes = [C.c_float] * 3
        L.orc_morton_key_f32.restype = C.c_uint32
        L.orc_morton_key_f32.argtypes = [C.c_float] * 4
        L.orc_morton_sort_f32.argtypes = [f32p, C.c_int32, C.c_float, i32p]
        L.orc_pairs_brute.restype = C.c_int64
        L.orc_pairs_brute.argtypes = [f64p, C.c_int32, C.c_double, C.c_double, C.c_void_p, C.c_int32,
                                      i32p, i32p, C.c_int64]
        L.orc_tile_list_aabb.restype = C.c_int64
        L.orc_tile_list_aabb.argtypes = [f32p, C.c_int32, C.c_float, C.c_float, i32p, i32p, C.c_int64]
        L.orc_pairs_brute_f32.restype = C.c_int64
        L.orc_pairs_brute_f32.argtypes = [f32p, C.c_int32, C.c_float, C.c_float, C.c_void_p, C.c_int32,
                                          i32p, i32p, C.c_int64]
        L.orc_verlet_lists.restype = C.c_int32
        L.orc_verlet_lists.argtypes = [f64p, C.c_int32, C.c_double, C.c_double, C.c_void_p, C.c_int32,
                                       C.c_int32, i32p, i32p]
        for name in ("orc_lj", "orc_fene", "orc_angle"):
            getattr(L, name).argtypes = [C.POINTER(OrcSystem), f64p, C.c_double, f64p, f64p, f64p]
        L.orc_forces.restype = C.c_int32
        L.orc_forces.argtypes = [C.POINTER(OrcSystem), f64p, C.c_double, f64p, f64p, f64p]
        L.orc_nhc_half.argtypes = [f64p, f64p, C.c_int32, C.c_double, C.c_double, C.c_double,
                                   C.c_int32, C.c_double, C.c_double, C.POINTER(C.c_double)]
        L.orc_thermo.argtypes = [f64p, i32p, f64p, f64p, f64p, C.c_int32, C.c_double, f64p]
        L.orc_rg.restype = C.c_double
        L.orc_rg.argtypes = [f64p, i32p, i32p, C.c_int32, C.c_double]
        L.orc_sim_create.restype = C.c_void_p
        L.orc_sim_create.argtypes = [C.POINTER(OrcSystem), C.POINTER(OrcRun), C.c_double, f64p, f64p,
                                     C.c_void_p]
        L.orc_sim_step.restype = C.c_int32
        L.orc_sim_step.argtypes = [C.c_void_p, C.c_int64]
        L.orc_sim_get.argtypes = [C.c_void_p] + [C.c_void_p] * 6
        L.orc_sim_scalars.argtypes = [C.c_void_p, f64p]
        L.orc_sim_thermo.argtypes = [C.c_void_p, f64p]
        L.orc_sim_rg.restype = C.c_double
        L.orc_sim_rg.argtypes = [C.c_void_p]
        L.orc_sim_conserved.restype = C.c_double
        L.orc_sim_conserved_mtk.restype = C.c_double
        L.orc_sim_conserved_mtk.argtypes = [C.c_void_p]
        L.orc_sim_conserved.argtypes = [C.c_void_p]
        L.orc_sim_destroy.argtypes = [C.c_void_p]
        _LIB = L
    return _LIB


def ref_lib():
    """The reference's own CPU code, or None when it was not built here."""
    global _REF
    if _REF is None:
        path = os.path.join(_HERE, "_ref", "libfmdref.so")
        if not os.path.exists(path):
            return None
        R = C.CDLL(path)
        R.ref_min_image.restype = C.c_float
        R.ref_min_image.argtypes = [C.c_float] * 3
        R.ref_morton3d.restype = C.c_uint32
        R.ref_morton3d.argtypes = [C.c_float] * 4
        R.ref_morton_sort.argtypes = [f32p, C.c_int32, C.c_float, i32p]
        R.ref_brute_force_lj.argtypes = [f32p, i32p, C.c_int32, f32p, C.c_int32, C.c_float, C.c_float,
                                         C.c_void_p, C.c_void_p, f32p, f32p, f32p]
        R.ref_brute_force_fene.argtypes = [f32p, C.c_int32, i32p, i32p, C.c_int32, f32p, C.c_int32,
                                           C.c_float, f32p, f32p, f32p]
        R.ref_brute_force_angle.argtypes = [f32p, C.c_int32, i32p, i32p, C.c_int32, f32p, C.c_int32,
                                            C.c_float, f32p, f32p, f32p]
        R.ref_brute_force_tile_list.restype = C.c_int64
        R.ref_brute_force_tile_list.argtypes = [f32p, C.c_int32, C.c_int32, C.c_float, C.c_float, i32p,
                                                C.c_int64]
        R.ref_pairs_within.restype = C.c_int64
        R.ref_pairs_within.argtypes = [f32p, C.c_int32, C.c_float, C.c_float, C.c_void_p, C.c_void_p, i32p, i32p,
                                       C.c_int64]
        R.ref_nh_chain.argtypes = [C.c_int32, C.c_float, C.c_float, C.c_int32, f32p, f32p, C.c_float,
                                   C.c_float, C.POINTER(C.c_float), f32p]
        R.ref_parse_config.restype = C.c_int32
        R.ref_parse_config.argtypes = [C.c_char_p, f32p, i32p, f32p, C.c_int32, f32p, C.c_int32, f32p,
                                       C.c_int32, C.POINTER(C.c_uint64), C.c_char_p, C.c_int32]
        R.ref_parse_lammps_data.restype = C.c_int32
        R.ref_parse_lammps_data.argtypes = [C.c_char_p, i32p, C.POINTER(C.c_float)] + [C.c_void_p] * 10 + [
            C.c_char_p, C.c_int32]
        R.ref_parse_table.restype = C.c_int32
        R.ref_parse_table.argtypes = [C.c_char_p, C.c_char_p, f32p, C.POINTER(C.c_int32), f32p, C.c_int32,
                                      C.c_char_p, C.c_int32]
        _REF = R
    return _REF


# ---------------------------------------------------------------------------
# Python-side model of a system, shared by tests and the CPU baseline.
# ---------------------------------------------------------------------------
@dataclass
class System:
    xyz: np.ndarray                    # (N, 3) float64, wrapped into [0, L)
    L: float
    type: np.ndarray                   # (N,) int32
    mass: np.ndarray                   # (ntypes,) float64
    lj: np.ndarray                     # (ntypes, ntypes, 2) float64
    bonds: np.ndarray = field(default_factory=lambda: np.zeros((0, 2), np.int32))
    bond_type: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    fene: np.ndarray = field(default_factory=lambda: np.zeros((0, 4)))
    angles: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.int32))
    angle_type: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    angle_p: np.ndarray = field(default_factory=lambda: np.zeros((0, 2)))
    mol: np.ndarray | None = None
    vel: np.ndarray | None = None
    image: np.ndarray | None = None
    rc: float = 2.5
    skin: float = 0.3
    lj_clamp: int = 1
    fene_clamp: int = 1

    def c_struct(self):
        """Build an OrcSystem; returns (struct, keepalive list)."""
        keep = []

        def arr(a, dt):
            a = np.ascontiguousarray(a, dtype=dt)
            keep.append(a)
            return a.ctypes.data if a.size else None

        n = len(self.type)
        s = OrcSystem()
        s.natoms = n
        s.ntypes = len(self.mass)
        s.type = arr(self.type, np.int32)
        s.mol = arr(self.mol if self.mol is not None else np.ones(n, np.int32), np.int32)
        s.mass = arr(self.mass, np.float64)
        s.lj = arr(self.lj, np.float64)
        s.nbonds = len(self.bonds)
        s.bonds = arr(self.bonds, np.int32)
        s.bond_type = arr(self.bond_type, np.int32)
        s.nbond_types = len(self.fene)
        s.fene = arr(self.fene, np.float64)
        s.nangles = len(self.angles)
        s.angles = arr(self.angles, np.int32)
        s.angle_type = arr(self.angle_type, np.int32)
        s.nangle_types = len(self.angle_p)
        s.angle_p = arr(self.angle_p, np.float64)
        s.rc = self.rc
        s.skin = self.skin
        s.lj_clamp = self.lj_clamp
        s.fene_clamp = self.fene_clamp
        return s, keep


def forces(sysm: System, which: str = "all"):
    L = lib()
    s, keep = sysm.c_struct()
    n = len(sysm.type)
    f = np.zeros(3 * n)
    pe = np.zeros(n)
    vir = np.zeros(6)
    x = np.ascontiguousarray(sysm.xyz, dtype=np.float64).reshape(-1)
    fn = {"all": L.orc_forces, "lj": L.orc_lj, "fene": L.orc_fene, "angle": L.orc_angle}[which]
    fn(C.byref(s), x, sysm.L, f, pe, vir)
    del keep
    return f.reshape(n, 3), pe, vir


def pairs_brute(xyz, L, rcs, bonds=None, f32=False):
    lb = lib()
    n = len(xyz)
    b = np.ascontiguousarray(bonds if bonds is not None else np.zeros((0, 2)), dtype=np.int32)
    cap = n * 400
    pi = np.zeros(cap, np.int32)
    pj = np.zeros(cap, np.int32)
    if f32:
        x = np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1)
        m = lb.orc_pairs_brute_f32(x, n, np.float32(L), np.float32(rcs), b.ctypes.data if b.size else None,
                                   len(b), pi, pj, cap)
    else:
        x = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1)
        m = lb.orc_pairs_brute(x, n, L, rcs, b.ctypes.data if b.size else None, len(b), pi, pj, cap)
    assert m <= cap
    return pi[:m].copy(), pj[:m].copy()


def tile_list_aabb(pos4, L, rc_skin):
    """Tile list of 32-atom tiles (neighbor/tile_list.cu semantics, FP32):
    CSR (offsets[ntiles + 1], neighbors) of tile pairs whose boxes lie within
    rc_skin.  pos4: (N, 4) float32."""
    lb = lib()
    p = np.ascontiguousarray(pos4, dtype=np.float32)
    n = len(p)
    T = (n + 31) // 32
    off = np.zeros(T + 1, np.int32)
    cap = T * T
    nb = np.zeros(max(cap, 1), np.int32)
    m = lb.orc_tile_list_aabb(p.reshape(-1), n, np.float32(L), np.float32(rc_skin), off, nb, cap)
    return off, nb[:m].copy()


def verlet_lists(xyz, L, rcs, bonds=None, max_nbr=256):
    lb = lib()
    n = len(xyz)
    b = np.ascontiguousarray(bonds if bonds is not None else np.zeros((0, 2)), dtype=np.int32)
    nbr = np.zeros(n * max_nbr, np.int32)
    cnt = np.zeros(n, np.int32)
    x = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1)
    nx = lb.orc_verlet_lists(x, n, L, rcs, b.ctypes.data if b.size else None, len(b), max_nbr, nbr, cnt)
    return nbr.reshape(n, max_nbr), cnt, nx


def normal3(seed, stream, step, ids):
    lb = lib()
    out = np.zeros((len(ids), 3))
    tmp = np.zeros(3)
    for k, i in enumerate(ids):
        lb.orc_normal3(seed, stream, step, int(i), tmp)
        out[k] = tmp
    return out


ENSEMBLES = {"langevin": 0, "nvt_nh": 1, "npt_nh": 2}


class Sim:
    """FP64 whole-step simulation mirroring the reference's step loop."""

    def __init__(self, sysm: System, ensemble="langevin", dt=0.001, T=(1.0, 1.0, 1.0), P=(0.0, 0.0, 1.0),
                 chain=3, seed=42, nsteps=1000, force_cap=0.0, nthreads=0, max_between=20, chain_carry=0):
        L = lib()
        self._s, self._keep = sysm.c_struct()
        r = OrcRun()
        r.ensemble = ENSEMBLES[ensemble]
        r.dt = dt
        r.T_start, r.T_stop, r.Tdamp = T
        r.P_start, r.P_stop, r.Pdamp = P
        r.chain_length = chain
        r.seed = seed
        r.nsteps = nsteps
        r.max_steps_between_rebuilds = max_between
        r.force_cap = force_cap
        r.nthreads = nthreads
        r.chain_carry = chain_carry
        self._r = r
        self.n = len(sysm.type)
        x = np.ascontiguousarray(sysm.xyz, dtype=np.float64).reshape(-1)
        v = np.ascontiguousarray(sysm.vel if sysm.vel is not None else np.zeros((self.n, 3)),
                                 dtype=np.float64).reshape(-1)
        img = None
        if sysm.image is not None:
            self._img = np.ascontiguousarray(sysm.image, dtype=np.int32).reshape(-1)
            img = self._img.ctypes.data
        self._h = L.orc_sim_create(C.byref(self._s), C.byref(r), sysm.L, x, v, img)

    def step(self, n):
        return lib().orc_sim_step(self._h, n)

    def state(self):
        n = self.n
        x = np.zeros(3 * n)
        v = np.zeros(3 * n)
        img = np.zeros(3 * n, np.int32)
        f = np.zeros(3 * n)
        pe = np.zeros(n)
        vir = np.zeros(6)
        lib().orc_sim_get(self._h, x.ctypes.data, v.ctypes.data, img.ctypes.data, f.ctypes.data,
                          pe.ctypes.data, vir.ctypes.data)
        return dict(x=x.reshape(n, 3), v=v.reshape(n, 3), image=img.reshape(n, 3), f=f.reshape(n, 3), pe=pe,
                    vir=vir)

    def scalars(self):
        o = np.zeros(27)
        lib().orc_sim_scalars(self._h, o)
        return dict(L=o[0], step=int(o[1]), rebuilds=int(o[2]), xi=o[3:13].copy(), v_xi=o[13:23].copy(),
                    eps=o[23], v_eps=o[24], carry=o[25], nh_scale=o[26])

    def thermo(self):
        o = np.zeros(9)
        lib().orc_sim_thermo(self._h, o)
        return o

    def rg(self):
        return lib().orc_sim_rg(self._h)

    def conserved(self):
        return lib().orc_sim_conserved(self._h)

    def conserved_mtk(self):
        """NPT extended energy plus the summed work of the kinetic barostat
        term the reference's equations omit (a diagnostic)."""
        return lib().orc_sim_conserved_mtk(self._h)

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                lib().orc_sim_destroy(self._h)
                self._h = None
        except Exception:
            pass


class StressACF:
    """Multiple-tau stress autocorrelator, restated from the reference
    (analysis/correlator.cu:33-92 for the update, main.cu:758-783 for the
    rows): 16 levels x 16 points x 6 components; each pushed sample is stored
    at its level's insert position and multiplied with the samples 0 ..
    insert position back (the reference bounds the lags by the insert
    position, not by the samples held); every 16 samples of a level pass
    their average to the next level.  FP64, products and sums rounded
    separately (plain Python floats)."""

    LEVELS = POINTS = 16

    def __init__(self, freq):
        L, P = self.LEVELS, self.POINTS
        self.freq = freq
        self.buf = [[[0.0] * 6 for _ in range(P)] for _ in range(L)]
        self.corr = [[[0.0] * 6 for _ in range(P)] for _ in range(L)]
        self.cnt = [[0] * P for _ in range(L)]
        self.idx = [0] * L
        self.acc = [[0.0] * 6 for _ in range(L)]
        self.accn = [0] * L

    def push(self, sample):
        P = self.POINTS
        smp = [float(x) for x in sample]
        for level in range(self.LEVELS):
            idx = self.idx[level]
            self.buf[level][idx] = list(smp)
            for lag in range(min(idx + 1, P)):
                older = self.buf[level][(idx - lag + P) % P]
                row = self.corr[level][lag]
                for c in range(6):
                    row[c] = row[c] + smp[c] * older[c]
                self.cnt[level][lag] += 1
            self.idx[level] = (idx + 1) % P
            acc = self.acc[level]
            for c in range(6):
                acc[c] = acc[c] + smp[c]
            self.accn[level] += 1
            if self.accn[level] >= P:
                smp = [acc[c] / P for c in range(6)]
                self.acc[level] = [0.0] * 6
                self.accn[level] = 0
            else:
                break

    def rows(self):
        lag, val, cnt = [], [], []
        step = self.freq
        for level in range(self.LEVELS):
            for k in range(self.POINTS):
                n = self.cnt[level][k]
                if n == 0:
                    continue
                lag.append(step * (k + 1))
                val.append([self.corr[level][k][c] / n for c in range(6)])
                cnt.append(n)
            step *= self.POINTS
        return np.array(lag, np.int64), np.array(val).reshape(-1, 6), np.array(cnt, np.int64)


def table_forces(xyz, L, rc, types, table_of, tables, bonds=None):
    """FP64 tabulated pair forces (force/table.cu:60-110 semantics): every
    pair within rc (minimum image; 1-2 bonded pairs excluded, as from the
    Verlet list the reference's table kernel walks) whose type pair has a
    table; r clamped to [rmin, rmax], grid index clamped to [0, n - 2],
    linear interpolation of the force column (applied as F/r) and of the
    energy.  tables: list of dict(rmin, rmax, dr, inv_dr, f, e).
    Returns (forces [N, 3], per-atom energy [N], virial [6])."""
    xyz = np.asarray(xyz, np.float64)
    n = len(xyz)
    f = np.zeros((n, 3))
    pe = np.zeros(n)
    vir = np.zeros(6)
    ii, jj = pairs_brute(xyz, L, rc, bonds=bonds)
    for i, j in zip(ii, jj):
        t = table_of[types[i]][types[j]]
        if t < 0:
            continue
        tb = tables[t]
        d = xyz[i] - xyz[j]
        d -= L * np.round(d / L)
        r2 = float(d @ d)
        if not (r2 < rc * rc and r2 > 1e-10):
            continue
        r = min(max(np.sqrt(r2), tb["rmin"]), tb["rmax"])
        k = int((r - tb["rmin"]) * tb["inv_dr"])
        k = max(0, min(k, len(tb["f"]) - 2))
        u = (r - (tb["rmin"] + k * tb["dr"])) * tb["inv_dr"]
        fs = tb["f"][k] + u * (tb["f"][k + 1] - tb["f"][k])
        e = tb["e"][k] + u * (tb["e"][k + 1] - tb["e"][k])
        f[i] += fs * d
        f[j] -= fs * d
        pe[i] += 0.5 * e
        pe[j] += 0.5 * e
        fd = fs * d
        vir += np.array([fd[0] * d[0], fd[0] * d[1], fd[0] * d[2], fd[1] * d[1], fd[1] * d[2], fd[2] * d[2]])
    return f, pe, vir
