"""The overlap-report oracle (oracle/overlap_oracle.py) against the reference's
overlap_report on the final states of the golden packings
(tests/golden/overlap_report.npz, made by tests/golden/make_overlap_golden.py),
and phi_corrected / engine_max_overlap of the jobs client on the CPU."""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import overlap_oracle as oo  # noqa: E402

GOLD = Path(__file__).resolve().parent / "golden"


def _cases():
    z = np.load(GOLD / "overlap_report.npz")
    return sorted({k.split("/")[0] for k in z.files})


@pytest.mark.parametrize("case", _cases())
def test_oracle_matches_reference_overlap_report(case):
    g = np.load(GOLD / "overlap_report.npz")
    p = np.load(GOLD / "packs.npz")
    P, S, M, ncand = oo.overlap_pairs(p[f"{case}/positions"], p[f"{case}/diameters"], p[f"{case}/box"])
    np.testing.assert_array_equal(P, g[f"{case}/pairs"])
    assert (len(P), ncand) == tuple(g[f"{case}/counts"])
    np.testing.assert_allclose(S, g[f"{case}/fractions_sum"], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(M, g[f"{case}/fractions_min"], rtol=1e-12, atol=1e-15)


def test_phi_corrected_and_engine_max_overlap():
    from rcpgenerator_b200 import jobs
    assert jobs.phi_corrected(0.64, 1e-3, 3) == pytest.approx(0.64 * 0.999 ** 3, rel=1e-15)

    class P:
        max_min_dist = 4.5e-4
    assert jobs.engine_max_overlap(P()) == 4.5e-4
    assert jobs.engine_max_overlap(object()) == 0.0


def test_job_preparation_leaves_the_job_unchanged():
    """The seeded shuffle of run_packing_job works on a copy: the caller's
    job dict (and a second run of it) sees the original diameter order."""
    from rcpgenerator_b200 import jobs
    d = np.linspace(0.8, 1.2, 64)
    job = {"diameters": d.copy(), "seed": 4, "Ndim": 2, "phi_init": 0.5, "initializer_phi": 0.11}
    s1, D1, p1, r1 = jobs._prepare_job(job)
    np.testing.assert_array_equal(job["diameters"], d)
    s2, D2, p2, r2 = jobs._prepare_job(job)
    np.testing.assert_array_equal(D1, D2)
    assert r1 is None and np.allclose(sorted(p1.diameters), sorted(p2.diameters))


def test_prescreen_and_safe_phi():
    """The job loop's geometric pre-screen (jobs.py:137-143) and the sanity
    checked phi of a state (rcptools/_helpers.py:30-77)."""
    from rcpgenerator_b200 import jobs
    d = np.ones(40)
    d[0] = 60.0
    rej, dmax, L = jobs._prescreen_reject(d, 2, 0.85, 2.5)
    V = np.pi / 4 * (39 + 3600)
    assert rej and dmax == 60.0 and L == pytest.approx(np.sqrt(V / 0.85))
    assert not jobs._prescreen_reject(np.ones(40), 2, 0.85, 2.5)[0]

    class S:
        positions = np.array([[0.1, 0.2], [0.5, 0.9]])
        diameters = np.array([0.2, 0.2])
        box = np.array([1.0, 1.0])
        walls = [0, 0]
    assert jobs._safe_phi(S()) == pytest.approx(2 * np.pi * 0.01)
    S.positions = np.array([[0.1, 0.2], [0.5, 1.1]])  # outside the box
    assert jobs._safe_phi(S()) == 0.0
    S.positions = np.array([[0.1, 0.2], [0.5, 0.5]])
    S.walls = [-2, -1]  # disk container: phi relative to its area
    assert jobs._safe_phi(S()) == pytest.approx(2 * np.pi * 0.01 / (np.pi / 4))


def test_custom_packing_preparation():
    """run_one_custom_packing's preparation (jobs.py:34-134): a dilute mono
    initialisation, then the caller's diameters (non-finite dropped, floored
    at 1e-12) scaled so that the realised phi is phi_init."""
    from rcpgenerator_b200 import jobs
    d = np.array([1.0, 2.0, np.nan, 1.5, np.inf] + [1.0] * 60)
    p = jobs.prepare_custom_packing(d, seed=5, Ndim=3, phi_init=0.3, initializer_phi=0.05)
    D = np.asarray(p.diameters)
    assert len(D) == 63 and p.N == 63
    vol = np.sum(np.pi / 6 * D ** 3) / np.prod(p.box)
    assert vol == pytest.approx(0.3, rel=1e-12)
    np.testing.assert_allclose(D / D[0], np.array([1.0, 2.0, 1.5] + [1.0] * 60), rtol=1e-14)
    assert p.needs_pack and not p.needs_initialize and np.asarray(p.positions).shape == (63, 3)
