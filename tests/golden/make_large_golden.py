"""Golden vectors at N >= 20,000 -- the sizes at which the engine's neighbour
build switches to its tiled search (ndim <= 3) -- from the reference engine.

Runs in a container that holds the reference tree: builds it with
oracle/Makefile into oracle/_ref and records, per case,

* the initializer's output digest (the test regenerates the input with this
  project's bit-exact initializer and checks the digest first);
* run_packing_observed(max_steps=K) at one OpenMP thread: the final state
  (positions, diameters, box, walls), steps, phi, max_min_dist and SHA-256
  digests of particle_origin and of every history -- the exact engine must
  reproduce this run bit for bit;
* on that final state: the reference's full-refresh half list
  (get_pairs_kdtree for ndim <= 3, ENG:2758-3526), get_forces_nd_3 (F and the
  five scalars, ENG:3597-4269, mu = 2.5e-4) and compute_mean_force
  (ENG:769-803).

Writes tests/golden/large_<case>.npz.

Usage:  python tests/golden/make_large_golden.py /path/to/RCPGenerator
"""

from __future__ import annotations

import ctypes as C
import hashlib
import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[2]
OUT = Path(__file__).resolve().parent
REF_DIR = REPO / "oracle" / "_ref"
MU = 2.5e-4

# (name, initializer config, steps K)
CASES = [
    # 2-D bidisperse like the N = 1M benchmark packing, heavy-overlap early phase
    ("bi2d_n30k", dict(phi=0.30, N=30000, Ndim=2, box=[1.0, 1.0], walls=[0, 0],
                       dist={"type": "bidisperse", "d1": 1.0, "d2": 1.4, "p": 0.5}, seed=123), 150),
    # 3-D monodisperse like the N = 2,000 packing, at 12x the size
    ("mono3d_n24k", dict(phi=0.08, N=24000, Ndim=3, box=[1.0, 1.0, 1.0], walls=[0, 0, 0],
                         dist={"type": "mono", "d": 1.0}, seed=123), 300),
    # 3-D bidisperse in a spherical container (curved containment in the build's fused forces)
    ("bi3d_sphere_n20k", dict(phi=0.2, N=20480, Ndim=3, box=[1.0, 1.0, 1.0], walls=[-3, 0, 0],
                              dist={"type": "bidisperse", "d1": 1.0, "d2": 1.4, "p": 0.5}, seed=5), 200),
    # 2-D monodisperse between hard walls on both axes
    ("walls2d_n25k", dict(phi=0.3, N=25000, Ndim=2, box=[1.0, 1.0], walls=[1, 1],
                          dist={"type": "mono", "d": 1.0}, seed=11), 150),
    # power law d^-3 on [0.1, 1] in a sphere (size ratio 10: one cell grid per size class)
    ("powerlaw3d_sphere_n25k", dict(phi=0.2, N=25000, Ndim=3, box=[1.0, 1.0, 1.0], walls=[-3, 0, 0],
                                    dist={"type": "powerlaw", "d_min": 0.1, "d_max": 1.0, "exponent": -3.0},
                                    seed=123), 100),
]


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(np.asarray(a)).tobytes()).hexdigest()


def main(ref_root: str) -> None:
    env = dict(os.environ)
    env.pop("OMP_NUM_THREADS", None)
    subprocess.run(["make", "-C", str(REPO / "oracle"), "PY=" + sys.executable,
                    "REF_ROOT=" + str(Path(ref_root) / "python_code" / "python")], check=True, env=env)
    sys.path.insert(0, str(REF_DIR))
    for k in list(os.environ):
        if k.startswith("RCP_"):
            del os.environ[k]
    import _rcpgenerator as ref  # noqa: E402

    ref.set_num_threads(1)
    shim = C.CDLL(str(REF_DIR / "librcpg_ref.so"))
    shim.ref_set_num_threads(1)
    shim.ref_mean_force.restype = C.c_double
    dp = C.POINTER(C.c_double)
    u32p = C.POINTER(C.c_uint32)
    for name, icfg, K in CASES:
        init = ref.initialize_particles(icfg)
        pos0 = np.asarray(init["positions"], dtype=np.float64)
        dia0 = np.asarray(init["diameters"], dtype=np.float64)
        cfg = {"box": init["box"], "walls": init["walls"], "neighbor_max": 0, "seed": 0}
        r = ref.run_packing_observed({"positions": init["positions"], "diameters": init["diameters"]},
                                     cfg, 0, False, 0, None, {"max_steps": K})["result"]
        x = np.ascontiguousarray(r["positions"], dtype=np.float64)
        D = np.ascontiguousarray(r["diameters"], dtype=np.float64)
        box = np.ascontiguousarray(r["box"], dtype=np.float64)
        walls = np.ascontiguousarray(r["walls"], dtype=np.int8)
        N, nd = x.shape
        counts = np.zeros(N, dtype=np.uint32)
        cap = N * 400
        ids = np.zeros(cap, dtype=np.uint32)
        total = C.c_size_t()
        err = C.create_string_buffer(1024)
        rc = shim.ref_pairs_full(C.c_size_t(N), C.c_size_t(nd), x.ctypes.data_as(dp), D.ctypes.data_as(dp),
                                 box.ctypes.data_as(dp), walls.ctypes.data_as(C.POINTER(C.c_int8)),
                                 C.c_uint32(0), counts.ctypes.data_as(u32p), ids.ctypes.data_as(u32p),
                                 C.c_size_t(cap), C.byref(total), err, 1024)
        assert rc == 0, err.value
        ids = ids[: total.value].copy()
        F = np.zeros(N * nd)
        sc = np.zeros(5)
        shim.ref_forces(C.c_size_t(N), C.c_size_t(nd), x.ctypes.data_as(dp), D.ctypes.data_as(dp),
                        box.ctypes.data_as(dp), walls.ctypes.data_as(C.POINTER(C.c_int8)),
                        counts.ctypes.data_as(u32p), ids.ctypes.data_as(u32p), C.c_double(MU),
                        F.ctypes.data_as(dp), sc.ctypes.data_as(dp))
        mf = shim.ref_mean_force(F.ctypes.data_as(dp), C.c_size_t(N), C.c_size_t(nd))
        hist = {h + "_sha256": np.asarray(digest(np.asarray(r[h], dtype=np.float64)))
                for h in ("phi_history", "force_history", "energy_history", "max_overlap_history",
                          "mu_history", "alpha_history")}
        np.savez_compressed(
            OUT / f"large_{name}.npz", config=np.asarray(json.dumps(icfg)), steps_run=np.asarray(K),
            input_positions_sha256=np.asarray(digest(pos0)), input_diameters_sha256=np.asarray(digest(dia0)),
            x=x, D=D, box=box, walls=walls,
            scalars_run=np.asarray([r["steps"], r["phi"], r["max_min_dist"], r["force_magnitude"]]),
            particle_origin_sha256=np.asarray(digest(np.asarray(r["particle_origin"], dtype=np.uint64))),
            mu_flag_history_sha256=np.asarray(digest(np.asarray(r["mu_flag_history"], dtype=np.int8))),
            counts=counts.astype(np.uint16 if counts.max() < 65535 else np.uint32), ids=ids,
            mu=np.asarray(MU), F=F.reshape(N, nd), scalars=sc, mean_force=np.asarray(mf), **hist)
        print(name, "N", N, "pairs", total.value, "U", sc[0], "maxov", sc[1], "phi", r["phi"])


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_large_golden.py /path/to/RCPGenerator")
    main(sys.argv[1])
