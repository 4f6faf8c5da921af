"""rcpg_pairs_full_noalloc: the neighbour-row build for callers that must not
allocate device memory while they run (their device memory is reserved up
front by their own allocator, or a cudaMalloc / cudaFree in a time-critical
loop would synchronise the device). It takes its scratch from a fixed 8 MiB
array in the library's static device memory instead of allocating.

Checked through the C ABI against rcpg_pairs_full (which allocates its
scratch per call): identical rows and counts -- integer data, so exact
equality is the tolerance -- on two calls in a row, plus the size check that
rejects a working set larger than the fixed array. Collected last (file name)
so a run that stops at the first failure has run every other test first.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(native):
    fn = native.lib.rcpg_pairs_full_noalloc
    fn.restype = C.c_int32
    fn.argtypes = native.lib.rcpg_pairs_full.argtypes
    return fn


def _build(fn, x, D, box, walls, t, cap):
    import torch

    from tests import gpu_util as G
    from rcpgenerator_b200 import _native as N
    n, nd = x.shape
    xd, Dd = G.dev(x), G.dev(D)
    nbr = torch.full((cap * n,), -1, dtype=torch.int32, device="cuda:0")
    cnt = torch.full((n,), -1, dtype=torch.int32, device="cuda:0")
    need = C.c_uint32()
    err = N.errbuf()
    rc = fn(n, nd, G.vp(xd), G.vp(Dd), G.hp(np.ascontiguousarray(box, dtype=np.float64)),
            G.hp(np.ascontiguousarray(walls, dtype=np.int8), C.POINTER(C.c_int8)), t, cap,
            G.vp(nbr), G.vp(cnt), C.byref(need), None, err, len(err))
    N.raise_for(rc, err)
    c = cnt.cpu().numpy()
    M = nbr.view(cap, n).cpu().numpy()
    return c, [tuple(M[: c[i], i]) for i in range(n)], need.value


@pytest.mark.parametrize("case", ["bi_n1000_2d", "cfg1_n2000_3d", "walls_n256_2d"])
def test_noalloc_rows_equal_allocating_build_twice(cuda_device, native, golden, case):
    fn = _setup(native)
    g = golden(f"kernels_{case}.npz")
    x, D = g["x"], g["D"]
    t = native.lib.rcpg_t_shell(np.ascontiguousarray(D).ctypes.data_as(C.POINTER(C.c_double)), D.size)
    cap = 64
    ref_c, ref_rows, ref_need = _build(native.lib.rcpg_pairs_full, x, D, g["box"], g["walls"], t, cap)
    # two calls in a row: the second reuses the scratch the first left behind
    for _ in range(2):
        c, rows, need = _build(fn, x, D, g["box"], g["walls"], t, cap)
        assert need == ref_need
        assert np.array_equal(c, ref_c)
        assert rows == ref_rows


def test_noalloc_alternating_inputs(cuda_device, native, golden):
    fn = _setup(native)
    a = golden("kernels_bi_n1000_2d.npz")
    b = golden("kernels_mono_n300_4d.npz")
    for g in (a, b, a):
        D = g["D"]
        t = native.lib.rcpg_t_shell(np.ascontiguousarray(D).ctypes.data_as(C.POINTER(C.c_double)), D.size)
        ref = _build(native.lib.rcpg_pairs_full, g["x"], D, g["box"], g["walls"], t, 96)
        got = _build(fn, g["x"], D, g["box"], g["walls"], t, 96)
        assert np.array_equal(got[0], ref[0]) and got[1] == ref[1]


def test_noalloc_rejects_oversized_working_set(cuda_device, native):
    fn = _setup(native)
    from rcpgenerator_b200 import _native as N
    import torch
    from tests import gpu_util as G
    n, nd, cap = 400_000, 3, 64
    x = torch.rand(n * nd, dtype=torch.float64, device="cuda:0")
    D = torch.full((n,), 0.01, dtype=torch.float64, device="cuda:0")
    nbr = torch.zeros(cap * n, dtype=torch.int32, device="cuda:0")
    cnt = torch.zeros(n, dtype=torch.int32, device="cuda:0")
    err = N.errbuf()
    need = C.c_uint32()
    rc = fn(n, nd, G.vp(x), G.vp(D), None, None, 0.01, cap, G.vp(nbr), G.vp(cnt), C.byref(need),
            None, err, len(err))
    assert rc == N.RCPG_ENOSPC
    assert b"8 MiB" in err.value


@pytest.mark.parametrize("case,cap", [("large_bi2d_n30k", 16), ("large_bi3d_sphere_n20k", 64)])
def test_noalloc_tiled_sizes_equal_allocating_build(cuda_device, native, golden, case, cap):
    """Sizes at which the build takes its tiled search (N >= 20,000, ndim <= 3)
    and still fit the fixed array."""
    fn = _setup(native)
    g = golden(f"{case}.npz")
    D = g["D"]
    t = native.lib.rcpg_t_shell(np.ascontiguousarray(D).ctypes.data_as(C.POINTER(C.c_double)), D.size)
    ref = _build(native.lib.rcpg_pairs_full, g["x"], D, g["box"], g["walls"], t, cap)
    for _ in range(2):
        got = _build(fn, g["x"], D, g["box"], g["walls"], t, cap)
        assert got[2] == ref[2]
        assert np.array_equal(got[0], ref[0]) and got[1] == ref[1]


def test_noalloc_coarsened_grid_near_the_limit(cuda_device, native):
    """A 3-D working set that leaves little room for the cell grid: the build
    coarsens the grid to what is left and still returns the allocating build's
    rows."""
    fn = _setup(native)
    rng = np.random.default_rng(2024)
    n = 22_600
    x = rng.random((n, 3))
    D = np.full(n, 0.01)
    t = native.lib.rcpg_t_shell(np.ascontiguousarray(D).ctypes.data_as(C.POINTER(C.c_double)), D.size)
    ref = _build(native.lib.rcpg_pairs_full, x, D, [1.0, 1.0, 1.0], [0, 0, 0], t, 64)
    got = _build(fn, x, D, [1.0, 1.0, 1.0], [0, 0, 0], t, 64)
    assert np.array_equal(got[0], ref[0]) and got[1] == ref[1]
