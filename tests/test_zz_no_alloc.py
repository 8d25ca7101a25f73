"""The allocation-free Verlet build (fmd_launch_verlet_build_static) against
the caller-scratch entry point (fmd_launch_verlet_build).

It serves callers that cannot allocate device memory (code inside another
framework's memory pool or a stream-capture region, or a process with a fixed
device footprint); its cell-list scratch is a static device array inside the
library.  Both entry points are called through the C ABI on the same inputs,
two calls in a row on different systems, and must give identical neighbor
lists (the build is deterministic, so the tolerance is exact equality, as in
the other pair-set tests).  This file is collected last on purpose."""
import ctypes as C
import os

import numpy as np
import pytest

import fastmd_b200 as fm

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden.npz"))


def _inputs(xyz, bonds):
    import torch
    n = len(xyz)
    p = np.zeros((n, 4), np.float32)
    p[:, :3] = xyz
    p[:, 3] = np.zeros(n, np.int32).view(np.float32)
    per = [[] for _ in range(n)]
    for a, b in bonds:
        per[a].append(b)
        per[b].append(a)
    off, lst = [0], []
    for k in range(n):
        lst += sorted(set(per[k]))
        off.append(len(lst))
    return (torch.from_numpy(p).cuda(), torch.tensor(off, dtype=torch.int32, device="cuda"),
            torch.tensor(lst or [0], dtype=torch.int32, device="cuda"))


def _build(static, pos, eo, el, n, L, rcs, max_nbr=256):
    import torch
    lib = fm.lib()
    nbr = torch.full((max_nbr * n,), -7, dtype=torch.int32, device="cuda")
    cnt = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")
    P = lambda t: C.c_void_p(t.data_ptr())
    if static:
        fn = lib.fmd_launch_verlet_build_static
        fn.restype = C.c_int32
        st = fn(P(pos), C.c_int32(n), C.c_float(L), P(eo), P(el), C.c_float(rcs), C.c_int32(max_nbr), P(nbr), P(cnt),
                P(flag), None)
    else:
        sb = C.c_size_t()
        lib.fmd_verlet_scratch_bytes(C.c_int32(n), C.c_float(rcs), C.c_float(L), C.byref(sb))
        scratch = torch.empty(sb.value, dtype=torch.uint8, device="cuda")
        fn = lib.fmd_launch_verlet_build
        fn.restype = C.c_int32
        st = fn(P(pos), C.c_int32(n), C.c_float(L), P(eo), P(el), C.c_float(rcs), C.c_int32(max_nbr), P(nbr), P(cnt),
                P(scratch), C.c_size_t(sb.value), P(flag), None)
    assert st == 0
    torch.cuda.synchronize()
    c = cnt.cpu().numpy()
    nb = nbr.cpu().numpy().reshape(max_nbr, n)
    lists = [nb[: c[i], i].copy() for i in range(n)]
    return c, lists, int(flag.item())


@pytest.mark.gpu
def test_static_scratch_build_matches_caller_scratch_build_twice():
    cases = [
        (G["melt_pos"], G["melt_bonds"], float(G["melt_L"][0]), np.float32(2.8)),
        (G["lj64_pos"], np.zeros((0, 2), np.int32), 8.0, np.float32(3.0)),
    ]
    for xyz, bonds, L, rcs in cases:   # two calls in a row, different systems
        n = len(xyz)
        pos, eo, el = _inputs(xyz, bonds)
        c_ref, l_ref, f_ref = _build(False, pos, eo, el, n, L, rcs)
        c_st, l_st, f_st = _build(True, pos, eo, el, n, L, rcs)
        assert f_ref == 0 and f_st == 0
        assert np.array_equal(c_ref, c_st)
        assert all(np.array_equal(a, b) for a, b in zip(l_ref, l_st))


@pytest.mark.gpu
def test_static_scratch_rejects_oversized_input():
    import torch
    lib = fm.lib()
    n = (1 << 17) + 1
    pos = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    nbr = torch.zeros(4 * n, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(n, dtype=torch.int32, device="cuda")
    fn = lib.fmd_launch_verlet_build_static
    fn.restype = C.c_int32
    st = fn(C.c_void_p(pos.data_ptr()), C.c_int32(n), C.c_float(100.0), None, None, C.c_float(2.8), C.c_int32(4),
            C.c_void_p(nbr.data_ptr()), C.c_void_p(cnt.data_ptr()), None, None)
    assert st == 8   # FMD_ERR_CAPACITY, nothing launched


def _no_device():
    try:
        import torch
        return not torch.cuda.is_available()
    except Exception:
        return True


# Argument checks that return before anything is launched.  The pointers
# below are never dereferenced: each call must fail on the host, so these run
# on a machine without a GPU only.
@pytest.mark.skipif(not _no_device(), reason="host-side argument checks; run where no GPU is visible")
@pytest.mark.parametrize("L,rcs,code", [
    (200.0, 2.8, 8),        # 71 cells per axis: beyond the 40-per-axis (65,536-cell) limit
    (5735.0, 2.8, 8),       # 2048 per axis: 2048^3 wraps a 32-bit cell count to 0
    (1.0e30, 2.8, 8),       # per-axis count beyond int
    (float("inf"), 2.8, 1),
    (float("nan"), 2.8, 1),
    (30.0, 0.0, 1),
    (30.0, -2.8, 1),
    (-30.0, 2.8, 1),
])
def test_static_scratch_rejects_bad_geometry_before_launch(L, rcs, code):
    lib = fm.lib()
    fn = lib.fmd_launch_verlet_build_static
    fn.restype = C.c_int32
    dummy = C.c_void_p(256)
    st = fn(dummy, C.c_int32(64), C.c_float(L), None, None, C.c_float(rcs), C.c_int32(4), dummy, dummy, None, None)
    assert st == code


@pytest.mark.skipif(not _no_device(), reason="host-side argument checks; run where no GPU is visible")
@pytest.mark.parametrize("L,rcs,code", [(5735.0, 2.8, 8), (1.0e30, 2.8, 8), (float("nan"), 2.8, 1), (30.0, 0.0, 1)])
def test_caller_scratch_sizing_rejects_bad_geometry(L, rcs, code):
    lib = fm.lib()
    sb = C.c_size_t(123)
    fn = lib.fmd_verlet_scratch_bytes
    fn.restype = C.c_int32
    assert fn(C.c_int32(64), C.c_float(rcs), C.c_float(L), C.byref(sb)) == code
