"""ctypes loader of the host emulation (tests/hostemu/libhostemu.so) -- test infrastructure."""

from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB = Path(__file__).resolve().parent / "hostemu" / "libhostemu.so"
_dp = C.POINTER(C.c_double)


class HostEmu:
    def __init__(self):
        self.lib = C.CDLL(str(LIB))
        self.lib.hostemu_run_packing.restype = C.c_int

    def run(self, positions, diameters, box, walls, max_steps=0, neighbor_max=0, reorder=2000,
            fix_height=False, mu=None, fix_diameter=False, growth_steps=0):
        pos = np.ascontiguousarray(positions, dtype=np.float64)
        N, nd = pos.shape
        D = np.ascontiguousarray(diameters, dtype=np.float64)
        box = np.ascontiguousarray(box, dtype=np.float64) if len(box) else None
        walls = np.ascontiguousarray(walls, dtype=np.int8) if len(walls) else None
        cap = 200000
        po = np.zeros(N * nd)
        do = np.zeros(N)
        ho = np.zeros(7 * cap)
        oo = np.zeros(N, dtype=np.uint64)
        so = np.zeros(16)
        rc = self.lib.hostemu_run_packing(
            C.c_uint64(N), C.c_int(nd), pos.ctypes.data_as(_dp), D.ctypes.data_as(_dp),
            box.ctypes.data_as(_dp) if box is not None else None,
            walls.ctypes.data_as(C.POINTER(C.c_int8)) if walls is not None else None,
            C.c_uint32(neighbor_max), int(bool(fix_height)), C.c_uint64(max_steps),
            C.c_double(0.0 if mu is None else mu), int(mu is not None), int(bool(fix_diameter)),
            C.c_uint64(reorder), po.ctypes.data_as(_dp), do.ctypes.data_as(_dp), ho.ctypes.data_as(_dp),
            C.c_uint64(cap), oo.ctypes.data_as(C.POINTER(C.c_uint64)), so.ctypes.data_as(_dp),
            C.c_uint64(growth_steps))
        assert rc == 0
        s = int(so[0])
        names = ("phi_history", "force_history", "energy_history", "max_overlap_history",
                 "mu_history", "alpha_history", "mu_flag_history")
        out = {n: ho[k * cap:k * cap + s].copy() for k, n in enumerate(names)}
        out["mu_flag_history"] = out["mu_flag_history"].astype(np.int8)
        out.update(steps=s, phi=so[1], max_min_dist=so[2], force_magnitude=so[3], builds=int(so[4]),
                   positions=po.reshape(N, nd), diameters=do, particle_origin=oo)
        return out


def load() -> HostEmu:
    return HostEmu()
