"""Golden outputs of the reference engine for the failure-path tests
(tests/test_gpu_failures.py), recorded from the compiled reference
(oracle/_ref, built from its sources by oracle/Makefile) at one OpenMP thread:

* the RuntimeError text of a neighbour-capacity overflow (200 particles in a
  0.01-wide cluster, diameter 0.05, neighbor_max = 1; ENG:647-658);
* a run whose input holds one NaN coordinate, which the reference completes
  without an error: its steps, phi, phi history and final positions.

Writes tests/golden/failure_nan.npz.

Usage:  python tests/golden/make_failure_golden.py /path/to/RCPGenerator
"""

from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[2]
OUT = Path(__file__).resolve().parent / "failure_nan.npz"
REF_DIR = REPO / "oracle" / "_ref"


def main(ref_root: str) -> None:
    subprocess.run(["make", "-C", str(REPO / "oracle"), "PY=" + sys.executable,
                    "REF_ROOT=" + str(Path(ref_root) / "python_code" / "python")], check=True)
    sys.path.insert(0, str(REF_DIR))
    for k in list(os.environ):
        if k.startswith("RCP_"):
            del os.environ[k]
    import _rcpgenerator as ref  # noqa: E402

    ref.set_num_threads(1)
    rng = np.random.default_rng(0)
    clustered = 0.5 + 0.01 * rng.random((200, 2))
    try:
        ref.run_packing({"positions": clustered.tolist(), "diameters": [0.05] * 200},
                        {"box": [1.0, 1.0], "walls": [0, 0], "neighbor_max": 1, "seed": 0})
        raise SystemExit("the reference raised no overflow error")
    except RuntimeError as e:
        overflow = str(e)
    rng = np.random.default_rng(7)
    pos = rng.random((100, 2))
    pos[5, 0] = np.nan
    dia = np.full(100, 0.05)
    K = 1500
    r = ref.run_packing_observed({"positions": pos.tolist(), "diameters": dia.tolist()},
                                 {"box": [1.0, 1.0], "walls": [0, 0], "neighbor_max": 0, "seed": 0},
                                 0, False, 0, None, {"max_steps": K})["result"]
    np.savez_compressed(OUT, overflow_text=np.asarray(overflow), input_positions=pos, input_diameters=dia,
                        max_steps=np.asarray(K), steps=np.asarray(r["steps"]), phi=np.asarray(r["phi"]),
                        phi_history=np.asarray(r["phi_history"]), positions=np.asarray(r["positions"]),
                        particle_origin=np.asarray(r["particle_origin"], dtype=np.uint64))
    print("overflow:", overflow[:60], "| nan run:", r["steps"], r["phi"],
          "origin of first rows", r["particle_origin"][:8], "nan row",
          [i for i, p in enumerate(r["positions"]) if p[0] != p[0] or p[1] != p[1]])


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_failure_golden.py /path/to/RCPGenerator")
    main(sys.argv[1])
