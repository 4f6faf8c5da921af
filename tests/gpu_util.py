"""Device-buffer helpers of the GPU tests: torch holds the memory, the C ABI computes."""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from rcpgenerator_b200 import _native as N

_dp = C.POINTER(C.c_double)
_i8p = C.POINTER(C.c_int8)


def dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda:0", dtype=dtype).contiguous()


def vp(t: torch.Tensor):
    return C.c_void_p(t.data_ptr())


def hp(a: np.ndarray, t=_dp):
    return a.ctypes.data_as(t)


def check(rc, err):
    N.raise_for(rc, err)


def pairs_full(x: np.ndarray, D: np.ndarray, box, walls, t_shell: float, cap: int = 128):
    x = np.ascontiguousarray(x, dtype=np.float64)
    n, nd = x.shape
    xd, Dd = dev(x), dev(D)
    box = np.ascontiguousarray(box, dtype=np.float64)
    walls = np.ascontiguousarray(walls, dtype=np.int8)
    while True:
        nbr = torch.zeros(cap * n, dtype=torch.int32, device="cuda:0")
        cnt = torch.zeros(n, dtype=torch.int32, device="cuda:0")
        need = C.c_uint32()
        err = N.errbuf()
        rc = N.lib.rcpg_pairs_full(n, nd, vp(xd), vp(Dd), hp(box), hp(walls, _i8p), t_shell, cap,
                                   vp(nbr), vp(cnt), C.byref(need), None, err, len(err))
        if rc == N.RCPG_ENOSPC:
            cap = int(need.value) + 8
            continue
        check(rc, err)
        return nbr, cnt, cap


def rows_from(nbr: torch.Tensor, cnt: torch.Tensor, cap: int):
    n = cnt.numel()
    M = nbr.view(cap, n).cpu().numpy().astype(np.int64)
    c = cnt.cpu().numpy()
    return [tuple(M[:c[i], i]) for i in range(n)]


def forces(x, D, box, walls, nbr, cnt, cap, mu, exact):
    x = np.ascontiguousarray(x, dtype=np.float64)
    n, nd = x.shape
    xd, Dd = dev(x), dev(D)
    F = torch.zeros(n * nd, dtype=torch.float64, device="cuda:0")
    sc = np.zeros(7)
    box = np.ascontiguousarray(box, dtype=np.float64)
    walls = np.ascontiguousarray(walls, dtype=np.int8)
    err = N.errbuf()
    rc = N.lib.rcpg_forces(n, nd, vp(xd), vp(Dd), hp(box), hp(walls, _i8p), vp(nbr), vp(cnt), cap, mu,
                           int(exact), vp(F), hp(sc), None, err, len(err))
    check(rc, err)
    return F.cpu().numpy().reshape(n, nd), sc
