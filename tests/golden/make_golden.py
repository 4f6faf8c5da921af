"""Generate the golden vectors of tests/golden from the reference engine.

Runs in a container where the reference sources are present: builds them
with oracle/Makefile (outputs in oracle/_ref) and records, for fixed seeded
inputs, what the reference's own code returns:

* initializer.npz   initialize_particles for every distribution family
* kernels_<case>.npz one mid-run state per case and, on it, the reference's
                     full-refresh half list (get_pairs_kdtree / get_pairs_nd_3),
                     get_forces_nd_3 (F + scalars), compute_mean_force and one
                     adam_update + position step
* packs.npz         complete run_packing results of small cases (one OpenMP
                     thread): steps, phi, positions, diameters, origins, and
                     SHA-256 digests of every history

Usage:  python tests/golden/make_golden.py /path/to/RCPGenerator
"""

from __future__ import annotations

import ctypes as C
import hashlib
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[2]
OUT = Path(__file__).resolve().parent
REF_DIR = REPO / "oracle" / "_ref"

INIT_CASES = [
    dict(name="mono2d", phi=0.08, N=64, Ndim=2, box=[1.0, 1.0], walls=[0, 0],
         dist={"type": "mono", "d": 1.0}, seed=20240719),
    dict(name="bi3d", phi=0.1, N=128, Ndim=3, box=[1.0, 1.0, 1.0], walls=[0, 0, 0],
         dist={"type": "bidisperse", "d1": 1.0, "d2": 1.4, "p": 0.5}, seed=7),
    dict(name="gauss2d_walls", phi=0.11, N=64, Ndim=2, box=[1.0, 1.0], walls=[1, 1],
         dist={"type": "gaussian", "mu": 1.0, "sigma": 0.2}, seed=11),
    dict(name="bigauss3d", phi=0.05, N=100, Ndim=3, box=[1.0, 1.0, 2.0], walls=[0, 0, 1],
         dist={"type": "bigaussian", "mu1": 1.0, "sigma1": 0.1, "mu2": 2.0, "sigma2": 0.2, "p": 0.3},
         seed=5),
    dict(name="lognormal2d", phi=0.2, N=200, Ndim=2, box=[1.0, 1.0], walls=[0, 0],
         dist={"type": "lognormal", "mu": 0.0, "sigma": 0.3}, seed=9),
    dict(name="flat3d_sphere", phi=0.1, N=128, Ndim=3, box=[1.0, 1.0, 1.0], walls=[-3, 0, 0],
         dist={"type": "flat", "d_min": 0.5, "d_max": 1.5}, seed=21),
    dict(name="powerlaw3d", phi=0.15, N=300, Ndim=3, box=[1.0, 1.0, 1.0], walls=[0, 0, 0],
         dist={"type": "powerlaw", "d_min": 0.1, "d_max": 1.0, "exponent": -3.0}, seed=123),
    dict(name="expo2d_disk", phi=0.1, N=100, Ndim=2, box=[1.0, 1.0], walls=[-1, 0],
         dist={"type": "exponential", "d_min": 0.5, "d_max": 2.0}, seed=33),
    dict(name="weibull4d", phi=0.05, N=80, Ndim=4, box=[1.0, 1.0, 1.0, 1.0], walls=[0, 0, 0, 0],
         dist={"type": "weibull", "shape": 2.0, "scale": 1.0}, seed=4),
    dict(name="custom2d_fixh", phi=0.1, N=50, Ndim=2, box=[1.0, 1.0], walls=[0, 0],
         fix_height=True, dist={"type": "custom", "custom": [1.0 + 0.01 * k for k in range(50)]},
         seed=2),
]

# mid-run states for the kernel vectors: (case name, initializer config, steps run before)
KERNEL_CASES = [
    ("cfg1_n2000_3d", dict(phi=0.08, N=2000, Ndim=3, box=[1.0, 1.0, 1.0], walls=[0, 0, 0],
                           dist={"type": "mono", "d": 1.0}, seed=123), 3000),
    ("bi_n1000_2d", dict(phi=0.3, N=1000, Ndim=2, box=[1.0, 1.0], walls=[0, 0],
                         dist={"type": "bidisperse", "d1": 1.0, "d2": 1.4, "p": 0.5}, seed=123), 400),
    ("walls_n256_2d", dict(phi=0.11, N=256, Ndim=2, box=[1.0, 1.0], walls=[1, 1],
                           dist={"type": "mono", "d": 1.0}, seed=0), 300),
    ("sphere_n500_3d", dict(phi=0.2, N=500, Ndim=3, box=[1.0, 1.0, 1.0], walls=[-3, 0, 0],
                            dist={"type": "powerlaw", "d_min": 0.3, "d_max": 1.0, "exponent": -3.0},
                            seed=1), 800),
    ("mono_n300_4d", dict(phi=0.1, N=300, Ndim=4, box=[1.0] * 4, walls=[0] * 4,
                          dist={"type": "mono", "d": 1.0}, seed=8), 500),
]

_FH_RNG = np.random.default_rng(60)
_FH_POS = np.column_stack([_FH_RNG.uniform(0.0, 20.0, 60), _FH_RNG.uniform(0.0, 4.0, 60)])
_FH_D = np.where(_FH_RNG.uniform(size=60) < 0.5, 1.0, 1.4)

PACK_CASES = [
    ("n4_2d", {"positions": [[0.10, 0.10], [0.35, 0.25], [0.70, 0.55], [0.82, 0.85]],
               "diameters": [0.12, 0.10, 0.09, 0.08]},
     {"box": [1.0, 1.0], "walls": [], "neighbor_max": 0, "seed": 123}, {}),
    ("n16_2d", dict(phi=0.08, N=16, Ndim=2, box=[1.0, 1.0], walls=[0, 0],
                    dist={"type": "mono", "d": 1.0}, seed=20240719), None, {}),
    ("n64_3d_bi", dict(phi=0.1, N=64, Ndim=3, box=[1.0, 1.0, 1.0], walls=[0, 0, 0],
                       dist={"type": "bidisperse", "d1": 1.0, "d2": 1.4, "p": 0.5}, seed=7), None, {}),
    ("n64_2d_walls_500", dict(phi=0.11, N=64, Ndim=2, box=[1.0, 1.0], walls=[1, 1],
                              dist={"type": "mono", "d": 1.0}, seed=0), None, {"max_steps": 500}),
    ("n128_3d_sphere_3000", dict(phi=0.1, N=128, Ndim=3, box=[1.0, 1.0, 1.0], walls=[-3, 0, 0],
                                 dist={"type": "powerlaw", "d_min": 0.3, "d_max": 1.0, "exponent": -3.0},
                                 seed=3), None, {"max_steps": 3000}),
    ("n200_2d_disk_2500", dict(phi=0.1, N=200, Ndim=2, box=[1.0, 1.0], walls=[-1, 0],
                               dist={"type": "bidisperse", "d1": 1.0, "d2": 1.4, "p": 0.5}, seed=4),
     None, {"max_steps": 2500}),
    ("n300_4d_1500", dict(phi=0.1, N=300, Ndim=4, box=[1.0] * 4, walls=[0] * 4,
                          dist={"type": "mono", "d": 1.0}, seed=8), None, {"max_steps": 1500}),
    ("cfg1_n2000_3d", dict(phi=0.08, N=2000, Ndim=3, box=[1.0, 1.0, 1.0], walls=[0, 0, 0],
                           dist={"type": "mono", "d": 1.0}, seed=123), None, {}),
    # relax() options (PackingRunOptions, rcp_generator.hpp:102-123)
    ("n64_2d_target_phi", dict(phi=0.1, N=64, Ndim=2, box=[1.0, 1.0], walls=[0, 0],
                               dist={"type": "bidisperse", "d1": 1.0, "d2": 1.4, "p": 0.5}, seed=5),
     None, {"max_steps": 2500, "target_phi": 0.7}),
    ("n64_3d_fix_diameter", dict(phi=0.3, N=64, Ndim=3, box=[1.0, 1.0, 1.0], walls=[0, 0, 0],
                                 dist={"type": "mono", "d": 1.0}, seed=6),
     None, {"max_steps": 1500, "fix_diameter": True}),
    ("n100_2d_mu", dict(phi=0.1, N=100, Ndim=2, box=[1.0, 1.0], walls=[0, 0],
                        dist={"type": "mono", "d": 1.0}, seed=7), None, {"max_steps": 1500, "mu": 1e-3}),
    # fix_height: diameters of order one, box height given in units of D[0] (rcp_generator.cpp:4460-4491)
    ("n60_2d_fix_height_wall", {"positions": _FH_POS.tolist(), "diameters": _FH_D.tolist()},
     {"box": [20.0, 4.0], "walls": [0, 1], "neighbor_max": 0, "seed": 0, "fix_height": True},
     {"max_steps": 1500}),
    # size ratio 10 (power law d^-3 on [0.1, 1], spherical container), several grid size classes
    ("n600_3d_powerlaw10_sphere_1500", dict(phi=0.2, N=600, Ndim=3, box=[1.0, 1.0, 1.0], walls=[-3, 0, 0],
                                            dist={"type": "powerlaw", "d_min": 0.1, "d_max": 1.0, "exponent": -3.0},
                                            seed=123), None, {"max_steps": 1500}),
    ("n80_2d_no_reorder", dict(phi=0.1, N=80, Ndim=2, box=[1.0, 1.0], walls=[0, 0],
                               dist={"type": "mono", "d": 1.0}, seed=9), None,
     {"max_steps": 2500, "reorder_interval": 0}),
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
    dp = C.POINTER(C.c_double)
    u32p = C.POINTER(C.c_uint32)

    # ---- initializer ----
    init_out = {}
    for case in INIT_CASES:
        cfg = {k: v for k, v in case.items() if k != "name"}
        r = ref.initialize_particles(cfg)
        nm = case["name"]
        init_out[nm + "/positions"] = np.asarray(r["positions"], dtype=np.float64)
        init_out[nm + "/diameters"] = np.asarray(r["diameters"], dtype=np.float64)
        init_out[nm + "/box"] = np.asarray(r["box"], dtype=np.float64)
        init_out[nm + "/walls"] = np.asarray(r["walls"], dtype=np.int8)
        init_out[nm + "/scalars"] = np.asarray([r["diameter_scale_factor"], r["phi_modifier"]])
    np.savez_compressed(OUT / "initializer.npz", **init_out)

    # ---- kernels on mid-run states ----
    for name, icfg, nsteps in KERNEL_CASES:
        init = ref.initialize_particles(icfg)
        cfg = {"box": init["box"], "walls": init["walls"], "neighbor_max": 0, "seed": 0}
        res = ref.run_packing_observed({"positions": init["positions"], "diameters": init["diameters"]},
                                       cfg, 0, False, 0, None, {"max_steps": nsteps})["result"]
        x = np.ascontiguousarray(res["positions"], dtype=np.float64)
        D = np.ascontiguousarray(res["diameters"], dtype=np.float64)
        box = np.ascontiguousarray(res["box"], dtype=np.float64)
        walls = np.ascontiguousarray(res["walls"], dtype=np.int8)
        N, nd = x.shape
        counts = np.zeros(N, dtype=np.uint32)
        cap = N * 200
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
        mu = 2.5e-4
        shim.ref_forces(C.c_size_t(N), C.c_size_t(nd), x.ctypes.data_as(dp), D.ctypes.data_as(dp),
                        box.ctypes.data_as(dp), walls.ctypes.data_as(C.POINTER(C.c_int8)),
                        counts.ctypes.data_as(u32p), ids.ctypes.data_as(u32p), C.c_double(mu),
                        F.ctypes.data_as(dp), sc.ctypes.data_as(dp))
        shim.ref_mean_force.restype = C.c_double
        mf = shim.ref_mean_force(F.ctypes.data_as(dp), C.c_size_t(N), C.c_size_t(nd))
        rng = np.random.default_rng(99)
        m0 = rng.normal(scale=1e-3, size=N * nd)
        v0 = rng.uniform(1e-8, 1e-6, size=N * nd)
        m1, v1, x1 = m0.copy(), v0.copy(), x.reshape(-1).copy()
        ks = np.zeros(4)
        t, alpha = 7, 0.0045
        shim.ref_adam_step(C.c_size_t(N), C.c_size_t(nd), F.ctypes.data_as(dp), C.c_double(0.0),
                           C.c_size_t(t), C.c_double(alpha), box.ctypes.data_as(dp),
                           m1.ctypes.data_as(dp), v1.ctypes.data_as(dp), x1.ctypes.data_as(dp),
                           ks.ctypes.data_as(dp))
        np.savez_compressed(
            OUT / f"kernels_{name}.npz", x=x, D=D, box=box, walls=walls, counts=counts, ids=ids,
            mu=np.asarray(mu), F=F.reshape(N, nd), scalars=sc, mean_force=np.asarray(mf),
            m0=m0, v0=v0, t=np.asarray(t), alpha=np.asarray(alpha), m1=m1, v1=v1, x1=x1.reshape(N, nd),
            steps_before=np.asarray(nsteps))
        print(name, "pairs", total.value, "U", sc[0], "mean_force", mf)

    # ---- complete packings ----
    packs = {}
    for name, spec, cfg, opts in PACK_CASES:
        if cfg is None:
            init = ref.initialize_particles(spec)
            inp = {"positions": init["positions"], "diameters": init["diameters"]}
            cfg = {"box": init["box"], "walls": init["walls"], "neighbor_max": 0, "seed": 0}
        else:
            inp = spec
        r = ref.run_packing_observed(inp, cfg, 0, False, 0, None, dict(opts))["result"]
        packs[name + "/input_positions"] = np.asarray(inp["positions"], dtype=np.float64)
        packs[name + "/input_diameters"] = np.asarray(inp["diameters"], dtype=np.float64)
        packs[name + "/box_in"] = np.asarray(cfg["box"], dtype=np.float64)
        packs[name + "/walls_in"] = np.asarray(cfg["walls"], dtype=np.int8)
        packs[name + "/max_steps"] = np.asarray(opts.get("max_steps", 0))
        packs[name + "/fix_height"] = np.asarray(bool(cfg.get("fix_height", False)))
        for k, v in opts.items():  # run options, one array per key (PackingRunOptions)
            packs[name + "/opt/" + k] = np.asarray(v)
        packs[name + "/positions"] = np.asarray(r["positions"], dtype=np.float64)
        packs[name + "/diameters"] = np.asarray(r["diameters"], dtype=np.float64)
        packs[name + "/particle_origin"] = np.asarray(r["particle_origin"], dtype=np.uint64)
        packs[name + "/box"] = np.asarray(r["box"], dtype=np.float64)
        packs[name + "/scalars"] = np.asarray([r["steps"], r["phi"], r["max_min_dist"], r["force_magnitude"]])
        for h in ("phi_history", "force_history", "energy_history", "max_overlap_history",
                  "mu_history", "alpha_history"):
            a = np.asarray(r[h], dtype=np.float64)
            packs[name + "/" + h + "_sha256"] = np.asarray(digest(a))
            packs[name + "/" + h + "_every100"] = a[::100].copy()
        packs[name + "/mu_flag_history_sha256"] = np.asarray(digest(np.asarray(r["mu_flag_history"], dtype=np.int8)))
        print(name, r["steps"], r["phi"])
    np.savez_compressed(OUT / "packs.npz", **packs)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py /path/to/RCPGenerator")
    main(sys.argv[1])
