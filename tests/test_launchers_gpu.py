"""Reference-layout launchers (fmd_launch_*) on the GPU against the golden
fixtures made from the reference's own CPU code.

Device buffers are torch tensors (memory only); the work runs in
libfastmd_b200.so.  Tolerances: pair sets and the Morton permutation exact
(the reference's FP32 predicate, evaluated without fused multiply-add on both
sides); LJ forces within 1e-5 relative RMS of the reference's FP32 brute
force (summation order differs)."""
import ctypes as C
import os

import numpy as np
import pytest

import fastmd_b200 as fm
from tests.util import pair_set, rel_rms

pytestmark = pytest.mark.gpu
G = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden.npz"))


def _torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def _pos4(xyz, types=None):
    n = len(xyz)
    p = np.zeros((n, 4), np.float32)
    p[:, :3] = xyz
    p[:, 3] = (np.zeros(n, np.int32) if types is None else types.astype(np.int32)).view(np.float32)
    return p


def _excl(n, bonds):
    per = [[] for _ in range(n)]
    for a, b in bonds:
        per[a].append(b)
        per[b].append(a)
    off = [0]
    lst = []
    for k in range(n):
        lst += sorted(set(per[k]))
        off.append(len(lst))
    return np.array(off, np.int32), np.array(lst if lst else [0], np.int32)


def verlet(xyz, L, rcs, bonds=None, max_nbr=256):
    torch = _torch()
    lib = fm.lib()
    n = len(xyz)
    pos = torch.from_numpy(_pos4(xyz)).cuda()
    nbr = torch.full((max_nbr * n,), -1, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(n, dtype=torch.int32, device="cuda")
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")
    sb = C.c_size_t()
    lib.fmd_verlet_scratch_bytes.restype = C.c_int32
    assert lib.fmd_verlet_scratch_bytes(C.c_int32(n), C.c_float(rcs), C.c_float(L), C.byref(sb)) == 0
    scratch = torch.empty(sb.value, dtype=torch.uint8, device="cuda")
    eo = el = None
    if bonds is not None and len(bonds):
        o, l_ = _excl(n, bonds)
        eo = torch.from_numpy(o).cuda()
        el = torch.from_numpy(l_).cuda()
    lib.fmd_launch_verlet_build.restype = C.c_int32
    st = lib.fmd_launch_verlet_build(C.c_void_p(pos.data_ptr()), C.c_int32(n), C.c_float(L),
                                     C.c_void_p(eo.data_ptr() if eo is not None else 0),
                                     C.c_void_p(el.data_ptr() if el is not None else 0), C.c_float(rcs),
                                     C.c_int32(max_nbr), C.c_void_p(nbr.data_ptr()), C.c_void_p(cnt.data_ptr()),
                                     C.c_void_p(scratch.data_ptr()), C.c_size_t(sb.value),
                                     C.c_void_p(flag.data_ptr()), None)
    assert st == 0
    torch.cuda.synchronize()
    return pos, nbr, cnt, flag


def list_pairs(nbr, cnt, n, max_nbr=256):
    nb = nbr.cpu().numpy().reshape(max_nbr, n)
    c = cnt.cpu().numpy()
    pi, pj = [], []
    for i in range(n):
        for k in range(c[i]):
            pi.append(i)
            pj.append(nb[k, i])
    return np.array(pi), np.array(pj)


def test_verlet_launcher_pair_set_lj64_exact():
    xyz = G["lj64_pos"]
    _, nbr, cnt, flag = verlet(xyz, 8.0, 3.0)
    pi, pj = list_pairs(nbr, cnt, len(xyz))
    assert int(flag.item()) == 0
    assert pair_set(pi, pj) == pair_set(G["lj64_pairs"][:, 0], G["lj64_pairs"][:, 1])


def test_verlet_launcher_pair_set_melt_with_exclusions_exact():
    xyz = G["melt_pos"]
    L = float(G["melt_L"][0])
    _, nbr, cnt, flag = verlet(xyz, L, np.float32(2.8), bonds=G["melt_bonds"])
    pi, pj = list_pairs(nbr, cnt, len(xyz))
    assert pair_set(pi, pj) == pair_set(G["melt_pairs"][:, 0], G["melt_pairs"][:, 1])


def test_verlet_launcher_reports_overflow():
    xyz = G["lj64_pos"]
    _, nbr, cnt, flag = verlet(xyz, 8.0, 3.0, max_nbr=4)
    assert int(flag.item()) == 1
    assert int(cnt.max().item()) == 4


def test_lj_launcher_matches_reference_forces():
    torch = _torch()
    lib = fm.lib()
    xyz = G["lj64_pos"]
    n = len(xyz)
    pos, nbr, cnt, _ = verlet(xyz, 8.0, 3.0)
    force = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    vir = torch.zeros(6, dtype=torch.float32, device="cuda")
    lj = torch.tensor([1.0, 1.0], dtype=torch.float32, device="cuda")
    lib.fmd_launch_lj.restype = C.c_int32
    st = lib.fmd_launch_lj(C.c_void_p(pos.data_ptr()), C.c_void_p(force.data_ptr()), C.c_void_p(vir.data_ptr()),
                           C.c_void_p(lj.data_ptr()), C.c_void_p(nbr.data_ptr()), C.c_void_p(cnt.data_ptr()),
                           C.c_int32(n), C.c_int32(1), C.c_float(6.25), C.c_float(8.0), C.c_float(0.125), None)
    assert st == 0
    f = force.cpu().numpy()
    # the reference kernel clamps F/r at 1000 (lj.cu:48); its CPU oracle does not
    mask = np.all(np.abs(G["lj64_f"]) < 500, axis=1)
    assert rel_rms(f[mask, :3], G["lj64_f"][mask]) < 1e-5
    # The kernel clamps F/r at 1000 (lj.cu:48) and these random positions have
    # overlapping pairs, so the virial is checked against the FP64 oracle with
    # the same clamp (test_lj.cu:69 tolerance, 1e-2).
    from oracle import pyoracle as po
    osys = po.System(xyz=xyz.astype(np.float64), L=8.0, type=np.zeros(n, np.int32), mass=np.ones(1),
                     lj=np.ones((1, 1, 2)), skin=0.5, lj_clamp=1)
    fo, _, vo = po.forces(osys, "lj")
    assert rel_rms(f[:, :3], fo) < 1e-5
    assert np.max(np.abs(vir.cpu().numpy() - vo) / np.abs(vo)) < 1e-2


@pytest.mark.parametrize("pos_key,perm_key,inv", [("morton_pos", "morton_perm", 0.1),
                                                  ("morton2_pos", "morton2_perm", 1.0 / 15.0)])
def test_morton_launcher_bit_exact(pos_key, perm_key, inv):
    torch = _torch()
    lib = fm.lib()
    xyz = G[pos_key]
    n = len(xyz)
    pos = torch.from_numpy(_pos4(xyz)).cuda()
    vel = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    vel[:, 0] = torch.arange(n, dtype=torch.float32, device="cuda")
    perm = torch.zeros(n, dtype=torch.int32, device="cuda")
    sb = C.c_size_t()
    lib.fmd_morton_scratch_bytes(C.c_int32(n), C.byref(sb))
    scratch = torch.empty(sb.value, dtype=torch.uint8, device="cuda")
    lib.fmd_launch_morton_sort.restype = C.c_int32
    st = lib.fmd_launch_morton_sort(C.c_void_p(pos.data_ptr()), C.c_void_p(vel.data_ptr()), C.c_int32(n),
                                    C.c_float(inv), C.c_void_p(perm.data_ptr()), C.c_void_p(scratch.data_ptr()),
                                    C.c_size_t(sb.value), None)
    assert st == 0
    torch.cuda.synchronize()
    p = perm.cpu().numpy()
    assert np.array_equal(p, G[perm_key])
    assert np.array_equal(pos.cpu().numpy()[:, :3], xyz[p])
    assert np.array_equal(vel.cpu().numpy()[:, 0], p.astype(np.float32))  # test_morton.cu:48


def tile_list(pos4, L, rcs, cap=None):
    torch = _torch()
    lib = fm.lib()
    n = len(pos4)
    T = (n + 31) // 32
    cap = T * T if cap is None else cap
    pos = torch.from_numpy(np.ascontiguousarray(pos4, np.float32)).cuda()
    off = torch.full((T + 1,), -1, dtype=torch.int32, device="cuda")
    nbr = torch.full((max(cap, 1),), -1, dtype=torch.int32, device="cuda")
    sb = C.c_size_t()
    lib.fmd_tile_list_scratch_bytes.restype = C.c_int32
    assert lib.fmd_tile_list_scratch_bytes(C.c_int32(n), C.byref(sb)) == 0
    scratch = torch.empty(sb.value, dtype=torch.uint8, device="cuda")
    npairs = C.c_int32()
    lib.fmd_launch_tile_list.restype = C.c_int32
    st = lib.fmd_launch_tile_list(C.c_void_p(pos.data_ptr()), C.c_int32(n), C.c_float(L), C.c_float(rcs),
                                  C.c_void_p(off.data_ptr()), C.c_void_p(nbr.data_ptr()), C.c_int32(cap),
                                  C.byref(npairs), C.c_void_p(scratch.data_ptr()), C.c_size_t(sb.value), None)
    return st, off.cpu().numpy(), nbr.cpu().numpy()[: min(npairs.value, cap)], npairs.value


def _compact(xyz, L, bits=10):
    """Atoms ordered by a 30-bit Morton key of their positions, so that the
    32-atom tiles are spatially compact (as a cell-sorted system's are)."""
    q = np.clip((xyz / L * (1 << bits)).astype(np.int64), 0, (1 << bits) - 1)
    key = np.zeros(len(xyz), np.int64)
    for b in range(bits):
        for d in range(3):
            key |= ((q[:, d] >> b) & 1) << (3 * b + d)
    return xyz[np.argsort(key, kind="stable")]


@pytest.mark.parametrize("case", ["golden128", "melt3000", "uniform100k"])
def test_tile_list_launcher_exact_against_oracle(case):
    from oracle import pyoracle as po
    if case == "golden128":
        xyz, L, rcs = G["tile_pos"], 10.0, 3.0
    elif case == "melt3000":
        d = fm.generate_melt(30, 100, density=0.85, seed=3)
        xyz, L, rcs = _compact(d.xyz, d.box_L), d.box_L, 2.8
    else:
        L = 49.0
        xyz, rcs = _compact(np.random.default_rng(8).uniform(0, L, (100_000, 3)), L), 2.8
    p4 = _pos4(xyz)
    st, off, nbr, npairs = tile_list(p4, L, rcs)
    assert st == 0
    ooff, onbr = po.tile_list_aabb(p4, L, rcs)
    assert np.array_equal(off, ooff) and np.array_equal(nbr, onbr) and npairs == len(onbr)
    T = len(off) - 1
    got = {(a, int(b)) for a in range(T) for b in nbr[off[a]:off[a + 1]]}
    if case == "golden128":
        # tests/test_tile_list.cu: every tile pair of the reference's brute force is listed
        assert {tuple(x) for x in G["tile_pairs"]} <= got
    elif case == "melt3000":
        # every atom pair within rc_skin lies in a listed tile pair (both orders)
        pi, pj = po.pairs_brute(xyz, L, rcs, f32=True)
        assert {(int(a) // 32, int(b) // 32) for a, b in zip(pi, pj)} <= got
        assert {(int(b) // 32, int(a) // 32) for a, b in zip(pi, pj)} <= got


def test_tile_list_launcher_reports_overflow():
    d = fm.generate_melt(30, 100, density=0.85, seed=3)
    st, off, nbr, npairs = tile_list(_pos4(_compact(d.xyz, d.box_L)), d.box_L, 2.8, cap=10)
    assert st == 5 and npairs > 10 and len(nbr) == 10   # FMD_ERR_OVERFLOW, the first 10 written


def _compact_order(xyz, L, bits=10):
    """The permutation _compact applies."""
    q = np.clip((xyz / L * (1 << bits)).astype(np.int64), 0, (1 << bits) - 1)
    key = np.zeros(len(xyz), np.int64)
    for b in range(bits):
        for d in range(3):
            key |= ((q[:, d] >> b) & 1) << (3 * b + d)
    return np.argsort(key, kind="stable")


def lj_tiles(p4, L, rc, off, nbr, excl=None):
    torch = _torch()
    lib = fm.lib()
    n = len(p4)
    pos = torch.from_numpy(np.ascontiguousarray(p4, np.float32)).cuda()
    toff = torch.from_numpy(np.ascontiguousarray(off, np.int32)).cuda()
    tnbr = torch.from_numpy(np.ascontiguousarray(nbr, np.int32)).cuda()
    force = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    vir = torch.zeros(6, dtype=torch.float32, device="cuda")
    lj = torch.tensor([1.0, 1.0], dtype=torch.float32, device="cuda")
    eo = el = None
    if excl is not None:
        eo = torch.from_numpy(excl[0]).cuda()
        el = torch.from_numpy(excl[1]).cuda()
    lib.fmd_launch_lj_tiles.restype = C.c_int32
    st = lib.fmd_launch_lj_tiles(C.c_void_p(pos.data_ptr()), C.c_void_p(force.data_ptr()),
                                 C.c_void_p(vir.data_ptr()), C.c_void_p(lj.data_ptr()), C.c_void_p(toff.data_ptr()),
                                 C.c_void_p(tnbr.data_ptr()), C.c_void_p(eo.data_ptr() if eo is not None else None),
                                 C.c_void_p(el.data_ptr() if el is not None else None), C.c_int32(n), C.c_int32(1),
                                 C.c_float(rc * rc), C.c_float(L), C.c_float(1.0 / L), None)
    assert st == 0
    return force.cpu().numpy(), vir.cpu().numpy()


def lj_verlet(p4, L, rc, rcs, bonds=None):
    torch = _torch()
    lib = fm.lib()
    n = len(p4)
    pos, nbr, cnt, flag = verlet(p4[:, :3], L, rcs, bonds=bonds)
    assert int(flag.item()) == 0
    force = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    vir = torch.zeros(6, dtype=torch.float32, device="cuda")
    lj = torch.tensor([1.0, 1.0], dtype=torch.float32, device="cuda")
    lib.fmd_launch_lj.restype = C.c_int32
    st = lib.fmd_launch_lj(C.c_void_p(pos.data_ptr()), C.c_void_p(force.data_ptr()), C.c_void_p(vir.data_ptr()),
                           C.c_void_p(lj.data_ptr()), C.c_void_p(nbr.data_ptr()), C.c_void_p(cnt.data_ptr()),
                           C.c_int32(n), C.c_int32(1), C.c_float(rc * rc), C.c_float(L), C.c_float(1.0 / L), None)
    assert st == 0
    return force.cpu().numpy(), vir.cpu().numpy()


@pytest.mark.parametrize("case", ["lj64", "melt3000"])
def test_lj_tiles_launcher_matches_oracle_and_verlet_lj(case):
    """The warp-per-tile LJ over the tile list against the FP64 oracle and
    the Verlet-list LJ launcher on the same positions: the same pairs and
    pair arithmetic, only the summation order differs."""
    from oracle import pyoracle as po
    if case == "lj64":
        xyz, L, bonds = G["lj64_pos"].astype(np.float64), 8.0, None
    else:
        d = fm.generate_melt(30, 100, density=0.85, seed=3)
        order = _compact_order(d.xyz, d.box_L)
        rank = np.empty_like(order)
        rank[order] = np.arange(len(order))
        xyz, L = d.xyz[order], d.box_L
        bonds = rank[np.asarray(d.bonds).reshape(-1, 2)]
    n = len(xyz)
    p4 = _pos4(xyz)
    rc = 2.5
    st, off, nbr, _ = tile_list(p4, L, rc)
    assert st == 0
    excl = _excl(n, bonds) if bonds is not None else None
    ft, vt = lj_tiles(p4, L, rc, off, nbr, excl)
    fv, vv = lj_verlet(p4, L, rc, 2.8, bonds=bonds)
    assert rel_rms(ft[:, :3], fv[:, :3]) < 1e-6
    assert abs(ft[:, 3].sum() - fv[:, 3].sum()) < 1e-5 * abs(fv[:, 3]).sum()
    assert np.max(np.abs(vt - vv)) < 1e-4 * np.max(np.abs(vv))
    osys = po.System(xyz=xyz, L=L, type=np.zeros(n, np.int32), mass=np.ones(1), lj=np.ones((1, 1, 2)), skin=0.3,
                     lj_clamp=1, bonds=bonds if bonds is not None else np.zeros((0, 2), np.int32))
    fo, peo, vo = po.forces(osys, "lj")
    assert rel_rms(ft[:, :3], fo) < 1e-5
    assert abs(ft[:, 3].sum() - peo.sum()) < 1e-5 * abs(peo).sum()


def test_lj_tiles_launcher_rejects_half_exclusions():
    torch = _torch()
    lib = fm.lib()
    pos = torch.zeros((32, 4), dtype=torch.float32, device="cuda")
    off = torch.zeros(2, dtype=torch.int32, device="cuda")
    lib.fmd_launch_lj_tiles.restype = C.c_int32
    st = lib.fmd_launch_lj_tiles(C.c_void_p(pos.data_ptr()), C.c_void_p(pos.data_ptr()), C.c_void_p(pos.data_ptr()),
                                 C.c_void_p(pos.data_ptr()), C.c_void_p(off.data_ptr()), C.c_void_p(off.data_ptr()),
                                 C.c_void_p(off.data_ptr()), None, C.c_int32(32), C.c_int32(1), C.c_float(6.25),
                                 C.c_float(8.0), C.c_float(0.125), None)
    assert st == 1   # FMD_ERR_ARG, nothing launched
