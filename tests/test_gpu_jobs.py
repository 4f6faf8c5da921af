"""The rcptools job loop on the batch engine and the GPU overlap report
(rcpgenerator_b200.jobs): the kernel against the reference's overlap_report
output on the golden packings and against the CPU oracle on random states
(periodic and open boxes, 2-5 dimensions, grids of 1, 2 and 3+ cells per
axis); run_jobs rows against one-job-at-a-time rows."""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import overlap_oracle as oo  # noqa: E402

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"


class _State:
    def __init__(self, positions, diameters, box=None):
        self.positions = positions
        self.diameters = diameters
        if box is not None:
            self.box = box


def _cases():
    z = np.load(GOLD / "overlap_report.npz")
    return sorted({k.split("/")[0] for k in z.files})


@pytest.mark.parametrize("case", _cases())
def test_overlap_report_matches_reference(cuda_device, case):
    from rcpgenerator_b200 import jobs
    g = np.load(GOLD / "overlap_report.npz")
    p = np.load(GOLD / "packs.npz")
    r = jobs.overlap_report(_State(p[f"{case}/positions"], p[f"{case}/diameters"], p[f"{case}/box"]))
    assert (r["n_overlapping"], r["n_candidate_pairs"]) == tuple(g[f"{case}/counts"])
    np.testing.assert_array_equal(r["pairs"].reshape(-1, 2), g[f"{case}/pairs"])
    np.testing.assert_allclose(r["fractions_sum"], g[f"{case}/fractions_sum"], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(r["fractions_min"], g[f"{case}/fractions_min"], rtol=1e-12, atol=1e-15)
    assert r["max_overlap"] == pytest.approx(g[f"{case}/max_mean"][0], rel=1e-12, abs=1e-15)


@pytest.mark.parametrize("n,nd,dmax,periodic", [(500, 2, 0.08, True), (700, 3, 0.21, True), (400, 4, 0.45, True),
                                               (300, 5, 0.6, True), (600, 3, 0.15, False), (50, 2, 0.7, True),
                                               (1, 3, 0.1, True), (0, 2, 0.1, True)])
def test_overlap_report_matches_oracle(cuda_device, n, nd, dmax, periodic):
    from rcpgenerator_b200 import jobs
    rng = np.random.default_rng(n * 10 + nd)
    box = rng.uniform(0.8, 1.3, nd)
    pos = rng.uniform(0, 1, (n, nd)) * box
    if not periodic:
        pos = pos * 1.7 - 0.3  # outside [0, box): the open case bins on its bounding box
    D = rng.uniform(0.3, 1.0, n) * dmax
    r = jobs.overlap_report(_State(pos, D, box if periodic else None))
    P, S, M, nc = oo.overlap_pairs(pos, D, box if periodic else None)
    assert r["n_candidate_pairs"] == nc and r["n_overlapping"] == len(P)
    np.testing.assert_array_equal(r["pairs"].reshape(-1, 2), P)
    np.testing.assert_array_equal(r["fractions_sum"], S)
    np.testing.assert_array_equal(r["fractions_min"], M)


def _jobs():
    rng = np.random.default_rng(5)
    out = []
    for k in range(6):
        n = int(rng.integers(64, 400))
        nd = 2 + k % 2
        d = rng.choice([1.0, 1.4], size=n) if k % 3 else rng.lognormal(0.0, 0.2, n)
        out.append({"diameters": d, "seed": 100 + k, "Ndim": nd, "phi_init": 0.5 if nd == 2 else 0.3,
                    "initializer_phi": 0.11 if nd == 2 else 0.05, "candidate": k // 2, "generation": 0,
                    "stage": "test", "theta": [0.1 * k]})
    # a pre-screen rejection: one huge particle in a small packing
    d = np.ones(40)
    d[0] = 60.0
    out.append({"diameters": d, "seed": 7, "Ndim": 2, "phi_init": 0.5, "initializer_phi": 0.11,
                "candidate": 9, "generation": 0, "stage": "test", "theta": [0.0],
                "prescreen": {"enabled": True, "phi_target": 0.85, "threshold": 2.5}})
    return out


def test_run_jobs_rows_equal_single_jobs(cuda_device):
    """Engines on streams (gpu_concurrency > 0) run the same kernels as a
    single pack(): the rows are equal value for value."""
    from rcpgenerator_b200 import jobs
    js = _jobs()
    rows = jobs.run_jobs(js, {"gpu_concurrency": 4})
    single = [jobs.run_packing_job(j) for j in js]
    assert len(rows) == len(js)
    for a, b in zip(rows, single):
        assert a["success"] and b["success"], (a.get("error"), b.get("error"))
        for key in ("rejected", "candidate", "seed", "steps", "phi", "phi_rcp", "phi_corr", "max_overlap",
                    "max_min_dist", "Dmin", "Dmax"):
            assert a[key] == b[key], key
    assert rows[-1]["rejected"] and rows[-1]["phi"] == 0.0
    for r in rows[:-1]:
        assert 0.0 < r["max_overlap"] < 5e-4 and r["phi_corr"] < r["phi"]


def test_overlap_report_of_a_packed_job(cuda_device):
    """The engine's max_min_dist (its gate statistic) is the overlap report's
    max_overlap of the final state (jobs.py:346-360)."""
    from rcpgenerator_b200 import jobs
    p = jobs.run_one_custom_packing(np.full(200, 1.0), seed=3, Ndim=2, phi_init=0.5)
    r = jobs.overlap_report(p)
    # the gate statistic is taken before the last position update
    assert r["max_overlap"] == pytest.approx(jobs.engine_max_overlap(p), rel=0.1)
    assert r["n_overlapping"] > 0 and r["n_candidate_pairs"] >= r["n_overlapping"]


def test_run_jobs_default_split_meets_the_gate(cuda_device):
    """The default split (persistent kernel for the small packings) sums in
    another order, so its rows are statistically, not bitwise, equal."""
    from rcpgenerator_b200 import jobs
    js = _jobs()
    rows = jobs.run_jobs(js)
    assert all(r["success"] for r in rows)
    for r in rows[:-1]:
        assert 0.0 < r["max_overlap"] < 5e-4
        assert 0.5 < r["phi"] < 0.9
