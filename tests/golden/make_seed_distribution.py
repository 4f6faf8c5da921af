"""Reference phi_J / steps / final max overlap of the 3-D monodisperse N = 2000 packing over seeds
0..63 (3-D monodisperse, N = 2000, initial phi 0.08, periodic unit box), one
OpenMP thread per packing, eight packings at a time. Writes
tests/golden/cfg1_seeds.npz. Needs the reference build in oracle/_ref
(see make_golden.py).

Usage:  python tests/golden/make_seed_distribution.py
"""

from __future__ import annotations

import multiprocessing as mp
import os
import sys
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[2]
OUT = Path(__file__).resolve().parent / "cfg1_seeds.npz"


def one(seed: int):
    sys.path.insert(0, str(REPO / "oracle" / "_ref"))
    for k in list(os.environ):
        if k.startswith("RCP_"):
            del os.environ[k]
    import _rcpgenerator as ref
    ref.set_num_threads(1)
    init = ref.initialize_particles({"phi": 0.08, "N": 2000, "Ndim": 3, "box": [1.0, 1.0, 1.0],
                                     "walls": [0, 0, 0], "dist": {"type": "mono", "d": 1.0},
                                     "seed": seed})
    r = ref.run_packing({"positions": init["positions"], "diameters": init["diameters"]},
                        {"box": init["box"], "walls": init["walls"], "neighbor_max": 0, "seed": seed})
    return seed, r["phi"], r["steps"], r["max_min_dist"]


def main():
    ctx = mp.get_context("spawn")
    with ctx.Pool(8) as pool:
        rows = sorted(pool.map(one, range(64)))
    a = np.asarray(rows, dtype=np.float64)
    np.savez_compressed(OUT, seed=a[:, 0].astype(np.int64), phi=a[:, 1], steps=a[:, 2].astype(np.int64),
                        max_overlap=a[:, 3])
    print("phi_J mean", a[:, 1].mean(), "sd", a[:, 1].std(ddof=1), "steps mean", a[:, 2].mean())


if __name__ == "__main__":
    main()
