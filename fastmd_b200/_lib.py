"""ctypes layer over libfastmd_b200.so (include/fastmd.h)."""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

FMD_FORM_PLAIN_FP64 = 0
FMD_FORM_MIXED = 1
FMD_LANGEVIN, FMD_NVT_NH, FMD_NPT_NH = 0, 1, 2

STATUS_NAMES = {
    0: "OK", 1: "ERR_ARG", 2: "ERR_CONFIG", 3: "ERR_IO", 4: "ERR_CUDA", 5: "ERR_OVERFLOW",
    6: "ERR_TIMEOUT", 7: "ERR_FAULT", 8: "ERR_CAPACITY", 9: "ERR_NO_DEVICE", 10: "ERR_STATE",
}


class FastMDError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


def lib_path():
    return os.path.join(_HERE, "lib", "libfastmd_b200.so")


class MeltSpec(C.Structure):
    _fields_ = [
        ("nchains", C.c_int32), ("chain_length", C.c_int32), ("density", C.c_double), ("seed", C.c_uint64),
        ("type_block", C.c_int32), ("bond_length", C.c_double), ("min_dist", C.c_double),
        ("pushoff_steps", C.c_int32), ("pushoff_fcap", C.c_double), ("pushoff_dt", C.c_double),
    ]


class SystemDescC(C.Structure):
    _fields_ = [
        ("natoms", C.c_int32), ("ntypes", C.c_int32), ("box_L", C.c_double),
        ("xyz", C.c_void_p), ("vel", C.c_void_p), ("image", C.c_void_p), ("type", C.c_void_p),
        ("mol", C.c_void_p), ("mass", C.c_void_p),
        ("nbonds", C.c_int32), ("bonds", C.c_void_p), ("bond_type", C.c_void_p),
        ("nangles", C.c_int32), ("angles", C.c_void_p), ("angle_type", C.c_void_p),
    ]


class ThermoRow(C.Structure):
    _fields_ = [
        ("step", C.c_int64), ("ke", C.c_double), ("pe", C.c_double), ("temp", C.c_double),
        ("stress", C.c_double * 6), ("box_L", C.c_double), ("conserved", C.c_double),
    ]

    def as_array(self):
        return np.array([self.ke, self.pe, self.temp] + list(self.stress))


class BatchOpts(C.Structure):
    _fields_ = [
        ("device", C.c_int32), ("max_replicas", C.c_int32), ("max_atoms", C.c_int64),
        ("hbm_budget_gb", C.c_double), ("graph_steps", C.c_int32),
    ]


class ReplicaInfo(C.Structure):
    _fields_ = [
        ("slot", C.c_int32), ("natoms", C.c_int32), ("step", C.c_int64), ("nsteps", C.c_int64),
        ("status_word", C.c_int32), ("active", C.c_int32), ("box_L", C.c_double), ("rebuilds", C.c_int64),
    ]


class ServerOpts(C.Structure):
    _fields_ = [("batch", BatchOpts), ("steps_per_round", C.c_int32)]


class RequestResult(C.Structure):
    _fields_ = [
        ("request_id", C.c_int64), ("status", C.c_int32), ("natoms", C.c_int32), ("steps", C.c_int64),
        ("submit_time", C.c_double), ("start_time", C.c_double), ("finish_time", C.c_double),
        ("thermo", ThermoRow), ("rg", C.c_double),
    ]


def _acf_rows(call):
    cap = 16 * 16
    lag = np.zeros(cap, np.int64)
    val = np.zeros((cap, 6))
    cnt = np.zeros(cap, np.int64)
    n = C.c_int32()
    call(_ptr(lag), _ptr(val), _ptr(cnt), C.c_int32(cap), C.byref(n))
    k = n.value
    return lag[:k].copy(), val[:k].copy(), cnt[:k].copy()


def lib():
    """Load the shared library; raises if it was not built."""
    global _LIB
    if _LIB is None:
        p = lib_path()
        if not os.path.exists(p):
            raise ImportError(f"{p} is missing: build it with `make -C fastmd_b200/csrc` "
                              "(there is no CPU fallback)")
        L = C.CDLL(p)
        L.fmd_version.restype = C.c_char_p
        L.fmd_last_error.restype = C.c_int32
        L.fmd_last_error.argtypes = [C.c_char_p, C.c_size_t]
        _LIB = L
    return _LIB


def _err():
    buf = C.create_string_buffer(1024)
    lib().fmd_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def _call(name, *args):
    fn = getattr(lib(), name)
    fn.restype = C.c_int32
    st = fn(*args)
    if st != 0:
        raise FastMDError(st, _err())


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _c(a, dt):
    return None if a is None else np.ascontiguousarray(a, dtype=dt)


@dataclass
class SystemDesc:
    """An in-memory system (what a LAMMPS data file carries)."""
    xyz: np.ndarray
    box_L: float
    type: np.ndarray
    mol: np.ndarray | None = None
    vel: np.ndarray | None = None
    image: np.ndarray | None = None
    mass: np.ndarray | None = None
    bonds: np.ndarray | None = None
    bond_type: np.ndarray | None = None
    angles: np.ndarray | None = None
    angle_type: np.ndarray | None = None
    ntypes: int = 0

    def to_c(self):
        keep = []

        def arr(a, dt):
            a = _c(a, dt)
            keep.append(a)
            return _ptr(a)

        n = len(self.type)
        d = SystemDescC()
        d.natoms = n
        d.ntypes = self.ntypes or (int(np.max(self.type)) + 1 if n else 1)
        d.box_L = float(self.box_L)
        d.xyz = arr(np.asarray(self.xyz).reshape(-1), np.float64)
        d.vel = arr(None if self.vel is None else np.asarray(self.vel).reshape(-1), np.float64)
        d.image = arr(None if self.image is None else np.asarray(self.image).reshape(-1), np.int32)
        d.type = arr(self.type, np.int32)
        d.mol = arr(self.mol, np.int32)
        d.mass = arr(self.mass, np.float64)
        nb = 0 if self.bonds is None else len(self.bonds)
        d.nbonds = nb
        d.bonds = arr(None if nb == 0 else np.asarray(self.bonds).reshape(-1), np.int32)
        d.bond_type = arr(None if nb == 0 else (self.bond_type if self.bond_type is not None else np.zeros(nb)),
                          np.int32)
        na = 0 if self.angles is None else len(self.angles)
        d.nangles = na
        d.angles = arr(None if na == 0 else np.asarray(self.angles).reshape(-1), np.int32)
        d.angle_type = arr(None if na == 0 else (self.angle_type if self.angle_type is not None else np.zeros(na)),
                           np.int32)
        return d, keep


def write_lammps_data(path, desc: SystemDesc, step=0):
    """Write a system as a LAMMPS data file (the reference's restart layout)."""
    d, keep = desc.to_c()
    _call("fmd_write_lammps_data", str(path).encode(), C.byref(d), C.c_int64(step))


def generate_melt(nchains, chain_length, density=0.85, seed=42, type_block=0, bond_length=0.0, min_dist=0.0):
    """Host-side seeded random-walk melt (no push-off).  Returns a SystemDesc."""
    spec = MeltSpec(nchains=nchains, chain_length=chain_length, density=density, seed=seed,
                    type_block=type_block, bond_length=bond_length, min_dist=min_dist)
    counts = np.zeros(3, np.int32)
    L = C.c_double()
    _call("fmd_generate_melt", C.byref(spec), _ptr(counts), C.byref(L), None, None, None, None, None, None)
    n, nb, na = (int(x) for x in counts)
    xyz = np.zeros((n, 3))
    img = np.zeros((n, 3), np.int32)
    typ = np.zeros(n, np.int32)
    mol = np.zeros(n, np.int32)
    bonds = np.zeros((nb, 2), np.int32)
    angles = np.zeros((na, 3), np.int32)
    _call("fmd_generate_melt", C.byref(spec), _ptr(counts), C.byref(L), _ptr(xyz), _ptr(img), _ptr(typ), _ptr(mol),
          _ptr(bonds), _ptr(angles))
    nt = 2 if type_block > 0 else 1
    return SystemDesc(xyz=xyz, box_L=L.value, type=typ, mol=mol, image=img, mass=np.ones(nt), bonds=bonds,
                      bond_type=np.zeros(nb, np.int32), angles=angles, angle_type=np.zeros(na, np.int32), ntypes=nt)


def parse_run_conf(text):
    """Parse run.conf text; returns a dict of the reference's keys."""
    iout = np.zeros(11, np.int32)
    fout = np.zeros(9)
    lj = np.zeros(16 * 16 * 2)
    bond = np.zeros(4 * 64)
    angle = np.zeros(2 * 64)
    seed = C.c_uint64()
    _call("fmd_parse_run_conf", text.encode(), _ptr(iout), _ptr(fout), _ptr(lj), C.c_int32(len(lj)), _ptr(bond),
          C.c_int32(len(bond)), _ptr(angle), C.c_int32(len(angle)), C.byref(seed))
    nt = int(iout[1])
    return dict(natoms=int(iout[0]), ntypes=nt, nsteps=int(iout[2]), ensemble=int(iout[3]),
                chain_length=int(iout[4]), thermo_on=int(iout[5]), thermo_freq=int(iout[6]), rg_on=int(iout[7]),
                rg_freq=int(iout[8]), rc=fout[0], skin=fout[1], dt=fout[2], T_start=fout[3], T_stop=fout[4],
                Tdamp=fout[5], P_start=fout[6], P_stop=fout[7], Pdamp=fout[8],
                lj=lj[: nt * nt * 2].reshape(nt, nt, 2).copy(), bond=bond[: 4 * iout[9]].reshape(-1, 4).copy(),
                angle=angle[: 2 * iout[10]].reshape(-1, 2).copy(), seed=int(seed.value))


def read_pair_table(path, keyword):
    """One section of a pair_style table file: dict(rmin, rmax, dr, inv_dr,
    r, f, e) with the grid in single precision (the force column f is
    applied as F/r)."""
    grid = np.zeros(4, np.float32)
    n = C.c_int32()
    _call("fmd_read_pair_table", str(path).encode(), keyword.encode(), _ptr(grid), C.byref(n), None, C.c_int32(0))
    data = np.zeros((n.value, 3), np.float32)
    _call("fmd_read_pair_table", str(path).encode(), keyword.encode(), _ptr(grid), C.byref(n), _ptr(data),
          C.c_int32(n.value))
    return dict(rmin=float(grid[0]), rmax=float(grid[1]), dr=float(grid[2]), inv_dr=float(grid[3]),
                r=data[:, 0].copy(), f=data[:, 1].copy(), e=data[:, 2].copy())


def run_conf_tables(text):
    """(table index per type pair [ntypes, ntypes] (-1: none), number of tables) of a run.conf."""
    cap = 16 * 16
    t = np.full(cap, -1, np.int32)
    n = C.c_int32()
    _call("fmd_run_conf_tables", text.encode(), _ptr(t), C.c_int32(cap), C.byref(n))
    nt = parse_run_conf(text)["ntypes"]
    return t[:nt * nt].reshape(nt, nt), n.value


def read_lammps_data(path):
    counts = np.zeros(4, np.int32)
    L = C.c_double()
    _call("fmd_read_lammps_data", str(path).encode(), _ptr(counts), C.byref(L), *([None] * 10))
    n, nb, na, nt = (int(x) for x in counts)
    xyz = np.zeros((n, 3))
    img = np.zeros((n, 3), np.int32)
    typ = np.zeros(n, np.int32)
    mol = np.zeros(n, np.int32)
    vel = np.zeros((n, 3))
    bonds = np.zeros((nb, 2), np.int32)
    btype = np.zeros(nb, np.int32)
    angles = np.zeros((na, 3), np.int32)
    atype = np.zeros(na, np.int32)
    mass = np.zeros(nt)
    _call("fmd_read_lammps_data", str(path).encode(), _ptr(counts), C.byref(L), _ptr(xyz), _ptr(img), _ptr(typ),
          _ptr(mol), _ptr(vel), _ptr(bonds), _ptr(btype), _ptr(angles), _ptr(atype), _ptr(mass))
    return SystemDesc(xyz=xyz, box_L=L.value, type=typ, mol=mol, vel=vel, image=img, mass=mass, bonds=bonds,
                      bond_type=btype, angles=angles, angle_type=atype, ntypes=nt)


def format_thermo_row(row: ThermoRow) -> str:
    buf = C.create_string_buffer(512)
    _call("fmd_format_thermo_row", C.byref(row), buf, C.c_size_t(512))
    return buf.value.decode()


def format_rg_row(step: int, rg: float) -> str:
    buf = C.create_string_buffer(128)
    _call("fmd_format_rg_row", C.c_int64(step), C.c_double(rg), buf, C.c_size_t(128))
    return buf.value.decode()


def _melt_spec(gen):
    if gen is None:
        return None
    if isinstance(gen, MeltSpec):
        return gen
    return MeltSpec(**gen)


class Simulation:
    """One system: ``Simulation(run_conf_text, data_path=... | desc=... | gen=..., form=...)``."""

    def __init__(self, run_conf, data_path=None, desc: SystemDesc | None = None, gen=None,
                 form=FMD_FORM_MIXED):
        self._h = C.c_void_p()
        spec = _melt_spec(gen)
        dc, self._keep = (desc.to_c() if desc is not None else (None, None))
        _call("fmd_sim_create", run_conf.encode(), None if data_path is None else str(data_path).encode(),
              None if dc is None else C.byref(dc), None if spec is None else C.byref(spec), C.c_int32(form),
              C.byref(self._h))
        self.form = form
        n = C.c_int32()
        nb = C.c_int32()
        na = C.c_int32()
        _call("fmd_sim_info", self._h, C.byref(n), C.byref(nb), C.byref(na), None, None)
        self.natoms, self.nbonds, self.nangles = n.value, nb.value, na.value

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().fmd_sim_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n=1):
        _call("fmd_step", self._h, C.c_int64(n))

    @property
    def step_count(self):
        s = C.c_int64()
        _call("fmd_sim_info", self._h, None, None, None, C.byref(s), None)
        return s.value

    @property
    def box_L(self):
        L = C.c_double()
        _call("fmd_sim_info", self._h, None, None, None, None, C.byref(L))
        return L.value

    def forces(self):
        f = np.zeros((self.natoms, 3))
        pe = np.zeros(self.natoms)
        vir = np.zeros(6)
        _call("fmd_compute_forces", self._h, _ptr(f), _ptr(pe), _ptr(vir))
        return f, pe, vir

    def state(self):
        x = np.zeros((self.natoms, 3))
        v = np.zeros((self.natoms, 3))
        img = np.zeros((self.natoms, 3), np.int32)
        _call("fmd_get_state", self._h, _ptr(x), _ptr(v), _ptr(img))
        return x, v, img

    def set_state(self, xyz=None, vel=None, image=None):
        x = _c(None if xyz is None else np.asarray(xyz).reshape(-1), np.float64)
        v = _c(None if vel is None else np.asarray(vel).reshape(-1), np.float64)
        i = _c(None if image is None else np.asarray(image).reshape(-1), np.int32)
        _call("fmd_set_state", self._h, _ptr(x), _ptr(v), _ptr(i))

    def thermo(self) -> ThermoRow:
        r = ThermoRow()
        _call("fmd_thermo", self._h, C.byref(r))
        return r

    def rg(self):
        r = C.c_double()
        _call("fmd_rg", self._h, C.byref(r))
        return r.value

    def pairs(self):
        n = C.c_int64()
        _call("fmd_pairs", self._h, None, None, C.c_int64(0), C.byref(n))
        i = np.zeros(n.value, np.int32)
        j = np.zeros(n.value, np.int32)
        _call("fmd_pairs", self._h, _ptr(i), _ptr(j), C.c_int64(n.value), C.byref(n))
        return i, j

    def counters(self):
        r = C.c_int64()
        s = C.c_int32()
        m = C.c_int32()
        _call("fmd_sim_counters", self._h, C.byref(r), C.byref(s), C.byref(m))
        return dict(rebuilds=r.value, status_word=s.value, max_neighbors=m.value)

    def write_restart(self, path):
        _call("fmd_write_restart", self._h, str(path).encode())

    def stress_acf(self):
        """Stress autocorrelation rows: (lag in steps, 6 averaged products
        per row in thermo column order, number of products)."""
        return _acf_rows(lambda *a: _call("fmd_stress_acf", self._h, *a))

    def write_stress_acf(self, path):
        _call("fmd_write_stress_acf", self._h, str(path).encode())


class Batch:
    """Many replicas advanced together (the mixed form)."""

    def __init__(self, max_replicas=256, max_atoms=0, hbm_budget_gb=150.0, graph_steps=0, device=0):
        self._h = C.c_void_p()
        o = BatchOpts(device=device, max_replicas=max_replicas, max_atoms=max_atoms, hbm_budget_gb=hbm_budget_gb,
                      graph_steps=graph_steps)
        _call("fmd_batch_create", C.byref(o), C.byref(self._h))
        self._natoms = {}

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().fmd_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, run_conf, data_path=None, desc: SystemDesc | None = None, gen=None):
        slot = C.c_int32()
        spec = _melt_spec(gen)
        dc, keep = (desc.to_c() if desc is not None else (None, None))
        _call("fmd_batch_add_replica", self._h, run_conf.encode(),
              None if data_path is None else str(data_path).encode(), None if dc is None else C.byref(dc),
              None if spec is None else C.byref(spec), C.byref(slot))
        info = self.info(slot.value)
        self._natoms[slot.value] = info.natoms
        return slot.value

    def run(self, nsteps):
        _call("fmd_batch_run", self._h, C.c_int64(nsteps))

    def retire(self, slot):
        _call("fmd_batch_retire", self._h, C.c_int32(slot))
        self._natoms.pop(slot, None)

    def info(self, slot) -> ReplicaInfo:
        r = ReplicaInfo()
        _call("fmd_batch_replica_info", self._h, C.c_int32(slot), C.byref(r))
        return r

    def state(self, slot):
        n = self._natoms[slot]
        x = np.zeros((n, 3))
        v = np.zeros((n, 3))
        img = np.zeros((n, 3), np.int32)
        _call("fmd_batch_get_state", self._h, C.c_int32(slot), _ptr(x), _ptr(v), _ptr(img))
        return x, v, img

    def thermo(self, slot) -> ThermoRow:
        r = ThermoRow()
        _call("fmd_batch_thermo", self._h, C.c_int32(slot), C.byref(r))
        return r

    def rg(self, slot):
        r = C.c_double()
        _call("fmd_batch_rg", self._h, C.c_int32(slot), C.byref(r))
        return r.value

    def forces(self, slot):
        n = self._natoms[slot]
        f = np.zeros((n, 3))
        pe = np.zeros(n)
        vir = np.zeros(6)
        _call("fmd_batch_compute_forces", self._h, C.c_int32(slot), _ptr(f), _ptr(pe), _ptr(vir))
        return f, pe, vir

    def force_frame(self, slot):
        """Positions and box edge of the geometry the forces belong to (the
        box of the last pre-force update; differs from info().box_L under NPT
        after the barostat's post-force half step)."""
        x = np.zeros((self._natoms[slot], 3))
        L = C.c_double()
        _call("fmd_batch_get_force_frame", self._h, C.c_int32(slot), _ptr(x), C.byref(L))
        return x, L.value

    def pairs(self, slot):
        """The replica's Verlet pair set (i < j, data-file indices)."""
        n = C.c_int64()
        _call("fmd_batch_pairs", self._h, C.c_int32(slot), None, None, C.c_int64(0), C.byref(n))
        i = np.zeros(n.value, np.int32)
        j = np.zeros(n.value, np.int32)
        _call("fmd_batch_pairs", self._h, C.c_int32(slot), _ptr(i), _ptr(j), C.c_int64(n.value), C.byref(n))
        return i[: n.value], j[: n.value]

    def totals(self):
        a = C.c_int32()
        n = C.c_int64()
        b = C.c_int64()
        _call("fmd_batch_totals", self._h, C.byref(a), C.byref(n), C.byref(b))
        return dict(active=a.value, atoms=n.value, bytes=b.value)

    def write_restart(self, slot, path):
        _call("fmd_batch_write_restart", self._h, C.c_int32(slot), str(path).encode())

    def stress_acf(self, slot):
        """Stress autocorrelation rows of a replica (see Simulation.stress_acf)."""
        return _acf_rows(lambda *a: _call("fmd_batch_stress_acf", self._h, C.c_int32(slot), *a))

    def write_stress_acf(self, slot, path):
        _call("fmd_batch_write_stress_acf", self._h, C.c_int32(slot), str(path).encode())

    LAUNCH_KINDS = ("pre", "bin", "scan", "scatter", "cellsort", "permute", "topo", "neighbors", "force",
                    "force_ev", "post", "plan", "commit", "table")

    def set_list_prune(self, slot, delta):
        """Pruned pair list at rc + delta walked by the force kernels (on by
        default with delta = 0.12 outside NPT); delta <= 0 turns it off."""
        _call("fmd_batch_set_list_prune", self._h, C.c_int32(slot), C.c_double(delta))

    def set_list_buffer(self, slot, skin):
        """Verlet-list margin beyond rc (the run.conf skin by default; the
        autotuner widens it for replicas with a pruned list); rebuilds the
        replica's list at once."""
        _call("fmd_batch_set_list_buffer", self._h, C.c_int32(slot), C.c_double(skin))

    def list_buffer(self, slot):
        v = C.c_double()
        _call("fmd_batch_get_list_buffer", self._h, C.c_int32(slot), C.byref(v))
        return v.value

    def set_rebuild_cadence(self, slot, max_steps):
        """Force a neighbor-list rebuild at least every max_steps steps
        (20 by default, as the reference); max_steps <= 0 leaves rebuilds to
        the displacement / box-shrink trigger alone."""
        _call("fmd_batch_set_rebuild_cadence", self._h, C.c_int32(slot), C.c_int32(max_steps))

    def autotune(self, iters=20):
        """Pick the fastest force-kernel and neighbor-list variants on the
        current state and lift the forced rebuild cadence of the active
        replicas."""
        nf, nn = self.variants()[2:4]
        ms = np.zeros(nf + nn + 1)   # force variants, list variants, the chosen list variant
        v = C.c_int32()
        _call("fmd_batch_autotune", self._h, C.c_int32(iters), C.byref(v), _ptr(ms), C.c_int32(len(ms)))
        return v.value, ms

    def set_variants(self, force_variant=-1, nbr_variant=-1):
        """Pin the force-kernel and neighbor-list variants (< 0 keeps one)."""
        _call("fmd_batch_set_variants", self._h, C.c_int32(force_variant), C.c_int32(nbr_variant))

    def variants(self):
        """(force variant, neighbor variant, number of force variants, number of neighbor variants)."""
        a, b, c, d = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        _call("fmd_batch_get_variants", self._h, C.byref(a), C.byref(b), C.byref(c), C.byref(d))
        return a.value, b.value, c.value, d.value

    def last_forces(self, slot):
        """Forces of the last evaluation as stored (FP32 values, id order), not re-evaluated."""
        f = np.zeros((self._natoms[slot], 3))
        _call("fmd_batch_last_forces", self._h, C.c_int32(slot), _ptr(f))
        return f

    def launch_counts(self):
        """Kernel launches executed so far, per kernel (counted on the device)."""
        c = np.zeros(len(self.LAUNCH_KINDS), np.int64)
        _call("fmd_batch_launch_counts", self._h, _ptr(c), C.c_int32(len(c)))
        return dict(zip(self.LAUNCH_KINDS, c.tolist()))


class Trajectory:
    """Binary trajectory in the reference's dump format (io/dump.cu:12-56):
    frames of a Simulation or of a Batch replica, written by a background
    thread from pinned buffers."""

    def __init__(self, path, natoms, ntypes=1):
        self._h = C.c_void_p()
        _call("fmd_traj_open", str(path).encode(), C.c_int32(natoms), C.c_int32(ntypes), C.byref(self._h))

    def write(self, source, slot=None):
        if slot is None:
            _call("fmd_traj_write_sim", self._h, source._h)
        else:
            _call("fmd_traj_write_batch", self._h, source._h, C.c_int32(slot))

    def close(self):
        if self._h:
            h, self._h = self._h, None
            _call("fmd_traj_close", h)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def read_trajectory(path):
    """Parse a trajectory file: dict(natoms, ntypes, steps, box_L, xyz[frames, natoms, 3])."""
    raw = open(path, "rb").read()
    magic, natoms, ntypes = np.frombuffer(raw[:12], np.int32)
    if magic != 0x4D444247:
        raise ValueError("not a trajectory file")
    fsz = 8 + 4 + 4 + 12 * int(natoms)
    nf = (len(raw) - 12) // fsz
    steps, box, xyz = [], [], []
    for k in range(nf):
        o = 12 + k * fsz
        steps.append(int(np.frombuffer(raw[o:o + 8], np.int64)[0]))
        assert int(np.frombuffer(raw[o + 8:o + 12], np.int32)[0]) == natoms
        box.append(float(np.frombuffer(raw[o + 12:o + 16], np.float32)[0]))
        xyz.append(np.frombuffer(raw[o + 16:o + fsz], np.float32).reshape(int(natoms), 3))
    return dict(natoms=int(natoms), ntypes=int(ntypes), steps=np.array(steps), box_L=np.array(box, np.float32),
                xyz=np.array(xyz).reshape(nf, int(natoms), 3))


class Server:
    """Continuous-batching request loop on its own host thread."""

    def __init__(self, max_replicas=256, hbm_budget_gb=150.0, steps_per_round=0, graph_steps=0, device=0):
        self._h = C.c_void_p()
        o = ServerOpts(batch=BatchOpts(device=device, max_replicas=max_replicas, max_atoms=0,
                                       hbm_budget_gb=hbm_budget_gb, graph_steps=graph_steps),
                       steps_per_round=steps_per_round)
        _call("fmd_server_create", C.byref(o), C.byref(self._h))

    def submit(self, run_conf, gen):
        rid = C.c_int64()
        spec = _melt_spec(gen)
        _call("fmd_server_submit", self._h, run_conf.encode(), C.byref(spec), C.byref(rid))
        return rid.value

    def poll(self, cap=256):
        out = (RequestResult * cap)()
        n = C.c_int32()
        _call("fmd_server_poll", self._h, out, C.c_int32(cap), C.byref(n))
        return [out[k] for k in range(n.value)]

    def stats(self):
        q, r, f, a = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64()
        s = C.c_double()
        _call("fmd_server_stats", self._h, C.byref(q), C.byref(r), C.byref(f), C.byref(a), C.byref(s))
        return dict(queued=q.value, running=r.value, finished=f.value, atoms_resident=a.value, atom_steps=s.value)

    def timing(self):
        """Host seconds of the batch thread per phase, rounds, graph captures."""
        a, r, t = C.c_double(), C.c_double(), C.c_double()
        n, g = C.c_int64(), C.c_int64()
        _call("fmd_server_timing", self._h, C.byref(a), C.byref(r), C.byref(t), C.byref(n), C.byref(g))
        return dict(admit_s=a.value, run_s=r.value, retire_s=t.value, rounds=n.value, graph_captures=g.value)

    def drain(self, timeout_s=600.0):
        _call("fmd_server_drain", self._h, C.c_double(timeout_s))

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().fmd_server_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def partition_replicas(costs, nparts):
    """Greedy longest-processing-time placement of replicas on nparts GPUs
    (fmd_partition_replicas): returns (part of each replica, total cost per
    part).  Costs are atom counts or atoms x steps."""
    c = np.ascontiguousarray(costs, dtype=np.int64)
    part = np.zeros(len(c), np.int32)
    load = np.zeros(nparts, np.int64)
    _call("fmd_partition_replicas", _ptr(c), C.c_int32(len(c)), C.c_int32(nparts), _ptr(part), _ptr(load))
    return part, load


class ServerPool:
    """One continuous-batching server per listed device (a device may be
    listed twice); each request goes to the server with the least outstanding
    work (atoms x steps)."""

    def __init__(self, devices, max_replicas=256, hbm_budget_gb=150.0, steps_per_round=0, graph_steps=0):
        self._h = C.c_void_p()
        dev = np.ascontiguousarray(devices, dtype=np.int32)
        o = ServerOpts(batch=BatchOpts(device=0, max_replicas=max_replicas, max_atoms=0,
                                       hbm_budget_gb=hbm_budget_gb, graph_steps=graph_steps),
                       steps_per_round=steps_per_round)
        _call("fmd_server_pool_create", C.byref(o), _ptr(dev), C.c_int32(len(dev)), C.byref(self._h))

    def submit(self, run_conf, gen):
        """Returns (request id, index of the server it was placed on)."""
        rid = C.c_int64()
        srv = C.c_int32()
        spec = _melt_spec(gen)
        _call("fmd_server_pool_submit", self._h, run_conf.encode(), C.byref(spec), C.byref(rid), C.byref(srv))
        return rid.value, srv.value

    def poll(self, cap=256):
        out = (RequestResult * cap)()
        n = C.c_int32()
        _call("fmd_server_pool_poll", self._h, out, C.c_int32(cap), C.byref(n))
        return [out[k] for k in range(n.value)]

    def stats(self):
        q, r, f, a = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64()
        s = C.c_double()
        _call("fmd_server_pool_stats", self._h, C.byref(q), C.byref(r), C.byref(f), C.byref(a), C.byref(s))
        return dict(queued=q.value, running=r.value, finished=f.value, atoms_resident=a.value, atom_steps=s.value)

    def drain(self, timeout_s=600.0):
        _call("fmd_server_pool_drain", self._h, C.c_double(timeout_s))

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().fmd_server_pool_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
