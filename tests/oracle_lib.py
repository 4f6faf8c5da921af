"""ctypes loader of the C restatement (oracle/librcpg_oracle.so) -- test infrastructure."""

from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB = Path(__file__).resolve().parents[1] / "oracle" / "librcpg_oracle.so"
_dp = C.POINTER(C.c_double)
_u32p = C.POINTER(C.c_uint32)


class Oracle:
    def __init__(self):
        lib = C.CDLL(str(LIB))
        lib.rcpo_t_shell.restype = C.c_double
        lib.rcpo_t_shell.argtypes = [C.c_size_t, _dp]
        lib.rcpo_pairs_full.restype = C.c_size_t
        lib.rcpo_pairs_full.argtypes = [C.c_size_t, C.c_size_t, _dp, _dp, _dp, C.c_double, _u32p, _u32p, C.c_size_t]
        lib.rcpo_forces.restype = None
        lib.rcpo_forces.argtypes = [C.c_size_t, C.c_size_t, _dp, _dp, _dp, C.POINTER(C.c_int8), _u32p, _u32p,
                                    C.c_double, _dp, _dp]
        lib.rcpo_mean_force.restype = C.c_double
        lib.rcpo_mean_force.argtypes = [_dp, C.c_size_t, C.c_size_t]
        lib.rcpo_adam_step.restype = None
        lib.rcpo_adam_step.argtypes = [C.c_size_t, C.c_size_t, _dp, C.c_double, C.c_double, C.c_double, _dp,
                                       _dp, _dp, _dp]
        lib.rcpo_kappa_step.restype = C.c_double
        lib.rcpo_kappa_step.argtypes = [_dp, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double]
        lib.rcpo_refresh_check.restype = C.c_size_t
        lib.rcpo_refresh_check.argtypes = [C.c_size_t, C.c_size_t, _dp, _dp, _dp, _dp, _dp, C.c_double,
                                           C.POINTER(C.c_uint8)]
        lib.rcpo_reorder_perm.restype = None
        lib.rcpo_reorder_perm.argtypes = [C.c_size_t, C.c_size_t, _dp, _dp, _u32p]
        lib.rcpo_pair_caps.restype = None
        lib.rcpo_pair_caps.argtypes = [C.c_size_t, C.c_size_t, _dp, C.c_uint32, _u32p]
        self.lib = lib

    @staticmethod
    def _d(a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        return a, a.ctypes.data_as(_dp)

    def t_shell(self, D):
        D, p = self._d(D)
        return self.lib.rcpo_t_shell(D.size, p)

    def pairs_full(self, x, D, box, t_shell):
        x, px = self._d(x)
        D, pD = self._d(D)
        box, pb = self._d(box)
        N, nd = x.shape
        counts = np.zeros(N, dtype=np.uint32)
        total = self.lib.rcpo_pairs_full(N, nd, px, pD, pb, t_shell, counts.ctypes.data_as(_u32p), None, 0)
        ids = np.zeros(max(total, 1), dtype=np.uint32)
        self.lib.rcpo_pairs_full(N, nd, px, pD, pb, t_shell, counts.ctypes.data_as(_u32p),
                                 ids.ctypes.data_as(_u32p), total)
        return counts, ids[:total]

    def forces(self, x, D, box, walls, counts, ids, mu):
        x, px = self._d(x)
        D, pD = self._d(D)
        box, pb = self._d(box)
        walls = np.ascontiguousarray(walls, dtype=np.int8)
        counts = np.ascontiguousarray(counts, dtype=np.uint32)
        ids = np.ascontiguousarray(ids, dtype=np.uint32)
        N, nd = x.shape
        F = np.zeros((N, nd))
        sc = np.zeros(6)
        self.lib.rcpo_forces(N, nd, px, pD, pb, walls.ctypes.data_as(C.POINTER(C.c_int8)),
                             counts.ctypes.data_as(_u32p), ids.ctypes.data_as(_u32p), mu,
                             F.ctypes.data_as(_dp), sc.ctypes.data_as(_dp))
        return F, sc

    def mean_force(self, F):
        F, p = self._d(F)
        return self.lib.rcpo_mean_force(p, F.shape[0], F.shape[1])

    def adam_step(self, F, m, v, x, box, alpha, t):
        F, pF = self._d(F)
        m = np.array(m, dtype=np.float64)
        v = np.array(v, dtype=np.float64)
        x = np.array(x, dtype=np.float64)
        box, pb = self._d(box)
        N, nd = x.reshape(-1, box.size).shape
        ib1 = 1.0 / (1.0 - 0.9 ** float(t))
        ib2 = 1.0 / (1.0 - 0.999 ** float(t))
        self.lib.rcpo_adam_step(N, nd, pF, alpha, ib1, ib2, pb, m.ctypes.data_as(_dp),
                                v.ctypes.data_as(_dp), x.ctypes.data_as(_dp))
        return m, v, x

    def refresh_check(self, x, x_last, D, D_last, theta, theta_new):
        x, px = self._d(x)
        x_last = np.array(x_last, dtype=np.float64)
        D, pD = self._d(D)
        D_last = np.array(D_last, dtype=np.float64)
        theta = np.array(theta, dtype=np.float64)
        N, nd = x.shape
        r = np.zeros(N, dtype=np.uint8)
        n = self.lib.rcpo_refresh_check(N, nd, px, x_last.ctypes.data_as(_dp), pD, D_last.ctypes.data_as(_dp),
                                        theta.ctypes.data_as(_dp), theta_new, r.ctypes.data_as(C.POINTER(C.c_uint8)))
        return r, x_last, D_last, theta, n

    def reorder_perm(self, x, box):
        x, px = self._d(x)
        box, pb = self._d(box)
        N, nd = x.shape
        perm = np.zeros(N, dtype=np.uint32)
        self.lib.rcpo_reorder_perm(N, nd, px, pb, perm.ctypes.data_as(_u32p))
        return perm

    def pair_caps(self, D, ndim, neighbor_max=0):
        D, p = self._d(D)
        caps = np.zeros(D.size, dtype=np.uint32)
        self.lib.rcpo_pair_caps(D.size, ndim, p, neighbor_max, caps.ctypes.data_as(_u32p))
        return caps


def load() -> Oracle:
    return Oracle()
