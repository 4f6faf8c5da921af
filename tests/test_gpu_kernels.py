"""Per-step kernels on the GPU, through the C ABI, against the reference's
outputs on identical inputs (tests/golden/kernels_*.npz) and the C oracle."""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = ["cfg1_n2000_3d", "bi_n1000_2d", "walls_n256_2d", "sphere_n500_3d", "mono_n300_4d"]


def half_rows(counts, ids):
    out, k = [], 0
    for c in counts:
        out.append(tuple(int(v) for v in ids[k:k + c]))
        k += c
    return out


@pytest.mark.parametrize("case", CASES)
def test_pairs_full_matches_reference_half_list(cuda_device, golden, case):
    from tests import gpu_util as G
    g = golden(f"kernels_{case}.npz")
    from rcpgenerator_b200 import _native as N
    t = N.lib.rcpg_t_shell(np.ascontiguousarray(g["D"]).ctypes.data_as(C.POINTER(C.c_double)), g["D"].size)
    nbr, cnt, cap = G.pairs_full(g["x"], g["D"], g["box"], g["walls"], t)
    rows = G.rows_from(nbr, cnt, cap)
    # full rows are sorted, contain no self, and are symmetric
    for i, r in enumerate(rows):
        assert list(r) == sorted(set(r)) and i not in r
    half = [tuple(j for j in r if j > i) for i, r in enumerate(rows)]
    assert half == half_rows(g["counts"], g["ids"])
    for i, r in enumerate(rows):
        for j in r:
            assert i in rows[j]


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("exact", [1, 0])
def test_forces_match_reference(cuda_device, golden, case, exact):
    from tests import gpu_util as G
    g = golden(f"kernels_{case}.npz")
    from rcpgenerator_b200 import _native as N
    t = N.lib.rcpg_t_shell(np.ascontiguousarray(g["D"]).ctypes.data_as(C.POINTER(C.c_double)), g["D"].size)
    nbr, cnt, cap = G.pairs_full(g["x"], g["D"], g["box"], g["walls"], t)
    F, sc = G.forces(g["x"], g["D"], g["box"], g["walls"], nbr, cnt, cap, float(g["mu"]), exact)
    # per-particle forces sum in ascending partner order: bit-exact either way
    assert np.array_equal(F, g["F"])
    ref = g["scalars"]  # U, max_min_dist, Lc, Fmean, dkappa
    if exact:
        assert np.array_equal(sc[:5], ref)
        assert sc[5] == float(g["mean_force"])
    else:
        # tree-order sums: 1e-12 relative (max overlap is order-free)
        assert sc[1] == ref[1]
        for k in (0, 2, 3, 4):
            assert abs(sc[k] - ref[k]) <= 1e-12 * abs(ref[k]), k
        assert abs(sc[5] - float(g["mean_force"])) <= 1e-12 * abs(float(g["mean_force"]))


@pytest.mark.parametrize("case", CASES)
def test_adam_step_bit_exact(cuda_device, golden, case):
    from tests import gpu_util as G
    from rcpgenerator_b200 import _native as N
    g = golden(f"kernels_{case}.npz")
    n, nd = g["x"].shape
    F, m, v, x = G.dev(g["F"].reshape(-1)), G.dev(g["m0"]), G.dev(g["v0"]), G.dev(g["x"].reshape(-1))
    box = np.ascontiguousarray(g["box"])
    err = N.errbuf()
    rc = N.lib.rcpg_adam_step(n, nd, G.vp(F), G.vp(m), G.vp(v), G.vp(x), G.hp(box), float(g["alpha"]),
                              int(g["t"]), None, err, len(err))
    G.check(rc, err)
    assert np.array_equal(m.cpu().numpy(), g["m1"])
    assert np.array_equal(v.cpu().numpy(), g["v1"])
    assert np.array_equal(x.cpu().numpy().reshape(n, nd), g["x1"])


def test_mean_force_and_refresh_against_oracle(cuda_device, oracle, golden):
    from tests import gpu_util as G
    from rcpgenerator_b200 import _native as N
    g = golden("kernels_bi_n1000_2d.npz")
    F = g["F"]
    out = C.c_double()
    err = N.errbuf()
    Fd = G.dev(F.reshape(-1))
    G.check(N.lib.rcpg_mean_force(F.shape[0], F.shape[1], G.vp(Fd), C.byref(out), None, err, len(err)), err)
    assert abs(out.value - oracle.mean_force(F)) <= 1e-12 * abs(out.value)
    rng = np.random.default_rng(1)
    n = 5000
    x_last = rng.random((n, 2))
    x = x_last + rng.normal(scale=0.01, size=(n, 2))
    D_last = np.full(n, 0.05)
    D = D_last * rng.uniform(0.97, 1.03, size=n)
    theta = np.full(n, 0.012)
    r_o, xl_o, Dl_o, th_o, n_o = oracle.refresh_check(x, x_last, D, D_last, theta, 0.011)
    xd, xld, Dd, Dld, thd = G.dev(x), G.dev(x_last), G.dev(D), G.dev(D_last), G.dev(theta)
    import torch
    r = torch.zeros(n, dtype=torch.uint8, device="cuda:0")
    cnt = C.c_uint64()
    G.check(N.lib.rcpg_refresh_check(n, 2, G.vp(xd), G.vp(xld), G.vp(Dd), G.vp(Dld), G.vp(thd), 0.011,
                                     G.vp(r), C.byref(cnt), None, err, len(err)), err)
    assert np.array_equal(r.cpu().numpy(), r_o)
    assert cnt.value == n_o
    assert np.array_equal(xld.cpu().numpy(), xl_o)
    assert np.array_equal(Dld.cpu().numpy(), Dl_o)
    assert np.array_equal(thd.cpu().numpy(), th_o)


def test_pairs_row_capacity_overflow_reports_need(cuda_device, golden):
    from tests import gpu_util as G
    from rcpgenerator_b200 import _native as N
    import torch
    g = golden("kernels_cfg1_n2000_3d.npz")
    n, nd = g["x"].shape
    xd, Dd = G.dev(g["x"]), G.dev(g["D"])
    nbr = torch.zeros(4 * n, dtype=torch.int32, device="cuda:0")
    cnt = torch.zeros(n, dtype=torch.int32, device="cuda:0")
    need = C.c_uint32()
    err = N.errbuf()
    rc = N.lib.rcpg_pairs_full(n, nd, G.vp(xd), G.vp(Dd), G.hp(np.ascontiguousarray(g["box"])),
                               G.hp(np.ascontiguousarray(g["walls"]), C.POINTER(C.c_int8)), 0.5 * float(g["D"].max()),
                               4, G.vp(nbr), G.vp(cnt), C.byref(need), None, err, len(err))
    assert rc == N.RCPG_ENOSPC and need.value > 4
