"""Golden outputs of the reference's overlap_report (rcptools/overlap.py:7-113)
on the final states of the golden packings (packs.npz, written by the
reference engine) -- run in a container that holds the reference tree:

    python tests/golden/make_overlap_golden.py /path/to/RCPGenerator

Writes tests/golden/overlap_report.npz: per case the overlapping pairs
(sorted by (i, j)), their fractions (sum and min conventions, same order),
n_overlapping, n_candidate_pairs, max_overlap, mean_overlap. The reference
module is loaded from its file (it needs only NumPy and SciPy)."""

from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


class _State:
    def __init__(self, positions, diameters, box):
        self.positions = positions
        self.diameters = diameters
        self.box = box


def main(ref_root: str) -> None:
    src = Path(ref_root) / "python_code" / "python" / "rcptools" / "overlap.py"
    spec = importlib.util.spec_from_file_location("ref_overlap", src)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    z = np.load(HERE / "packs.npz")
    cases = sorted({k.split("/")[0] for k in z.files})
    out = {}
    for c in cases:
        st = _State(z[f"{c}/positions"], z[f"{c}/diameters"], z[f"{c}/box"])
        r = mod.overlap_report(st)
        pairs = np.asarray(r["pairs"], dtype=np.int64).reshape(-1, 2)
        order = np.lexsort((pairs[:, 1], pairs[:, 0]))
        out[f"{c}/pairs"] = pairs[order]
        out[f"{c}/fractions_sum"] = np.asarray(r["fractions_sum"])[order]
        out[f"{c}/fractions_min"] = np.asarray(r["fractions_min"])[order]
        out[f"{c}/counts"] = np.asarray([r["n_overlapping"], r["n_candidate_pairs"]], dtype=np.int64)
        out[f"{c}/max_mean"] = np.asarray([r["max_overlap"], r["mean_overlap"]])
        print(c, r["n_overlapping"], r["n_candidate_pairs"], r["max_overlap"])
    np.savez_compressed(HERE / "overlap_report.npz", **out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_overlap_golden.py /path/to/RCPGenerator")
    main(sys.argv[1])
