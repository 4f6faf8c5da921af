"""Sizing of the allocation-free neighbour build's fixed scratch array
(rcpgenerator_b200/csrc/rcpg_noalloc_plan.h), checked on the CPU through the
host emulation library, which compiles the same header.

The plan must accept every working set up to the documented bound (about
20,000 particles in 3-D at row capacity 64), keep every array 256-byte aligned
and inside the 8 MiB array without overlaps, and refuse sizes whose products
would not fit (including ones large enough to wrap a 64-bit product).
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

NAMES = ["ctl", "pos", "spos", "x_last", "caps", "cell_of", "cell_rank", "cell_list", "work", "nbr_cnt",
         "nbr", "scan_tmp", "cell_count", "cell_start"]


def _plan(hostemu, N, ndim, cap):
    fn = hostemu.lib.hostemu_noalloc_plan
    fn.restype = C.c_int
    fn.argtypes = [C.c_uint64, C.c_int, C.c_uint32, C.POINTER(C.c_uint64)]
    out = np.zeros(17, dtype=np.uint64)
    ok = fn(N, ndim, cap, out.ctypes.data_as(C.POINTER(C.c_uint64)))
    return bool(ok), out


def _sizes(N, ndim, cap, cells, ctl_end):
    P = (ndim + 2) & ~1
    return {"pos": 8 * N * P, "spos": 8 * N * P, "x_last": 8 * N * ndim, "caps": 4 * N, "cell_of": 4 * N,
            "cell_rank": 4 * N, "cell_list": 4 * N, "work": 4 * N, "nbr_cnt": 4 * N, "nbr": 4 * N * cap,
            "scan_tmp": 4 * (2 * 4096 + 16), "cell_count": 4 * (cells + 1), "cell_start": 4 * (cells + 1),
            "ctl": ctl_end}


def _check_layout(N, ndim, cap, out):
    offs = {k: int(out[i]) for i, k in enumerate(NAMES)}
    cells, used, total = int(out[14]), int(out[15]), int(out[16])
    sz = _sizes(N, ndim, cap, cells, offs["pos"] - offs["ctl"])
    spans = sorted((offs[k], offs[k] + sz[k], k) for k in NAMES)
    for (a0, a1, ka), (b0, _, kb) in zip(spans, spans[1:]):
        assert a1 <= b0, (ka, kb)
    for k in NAMES:
        assert offs[k] % 256 == 0, k
    assert spans[-1][1] == used <= total
    assert cells >= 1


@pytest.mark.parametrize("ndim,cap,bound", [(3, 64, 20000), (2, 16, 30000), (2, 64, 20000), (4, 96, 8000)])
def test_plan_accepts_every_size_up_to_the_bound(hostemu, ndim, cap, bound):
    Ns = sorted(set(list(range(1, 400)) + list(range(400, bound + 1, 37)) + [bound]))
    for N in Ns:
        ok, out = _plan(hostemu, N, ndim, cap)
        assert ok, (N, ndim, cap)
        _check_layout(N, ndim, cap, out)


def test_plan_grid_uses_the_space_that_is_left(hostemu):
    # 3-D at row capacity 64 near the bound: the grid gets what remains
    # (coarsened below one cell per particle), without exceeding the array
    for N in range(19000, 22800, 13):
        ok, out = _plan(hostemu, N, 3, 64)
        if not ok:
            # refusal only once the fixed arrays themselves leave no room
            P = 4
            fixed = N * (16 * P + 8 * 3 + 24 + 4 * 64)
            assert fixed > (8 << 20) - 64 * 1024, N
            continue
        _check_layout(N, 3, 64, out)
        # the grid takes what remains, up to its own cap of 8 cells per particle
        assert int(out[14]) == 8 * N + 1024 or int(out[16]) - int(out[15]) < 1024


def test_plan_refuses_oversized_and_wrapping_sizes(hostemu):
    assert not _plan(hostemu, 400_000, 3, 64)[0]
    assert not _plan(hostemu, 30_000, 3, 64)[0]
    assert not _plan(hostemu, 2 ** 62, 3, 64)[0]
    assert not _plan(hostemu, 1000, 3, 2 ** 32 - 1)[0]
    assert not _plan(hostemu, 0, 3, 64)[0]
