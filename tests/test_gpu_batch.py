"""Batches of independent packings (rcpg_run_batch / run_packing_batch).

Each packing of a batch runs on one engine of its own, on the stream of the
worker thread that took it, so its result must not depend on the batch: in
the exact engine a batch of golden packings reproduces the reference bit for
bit, and in the graph engine every packing equals the same packing run alone.
"""

from __future__ import annotations

import hashlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = ["n16_2d", "n64_3d_bi", "n64_2d_walls_500", "n128_3d_sphere_3000", "n200_2d_disk_2500",
         "n300_4d_1500"]


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def item(g, case, engine):
    inp = {"positions": g[f"{case}/input_positions"], "diameters": g[f"{case}/input_diameters"]}
    cfg = {"box": g[f"{case}/box_in"].tolist(), "walls": g[f"{case}/walls_in"].tolist(),
           "neighbor_max": 0, "engine": engine}
    return inp, cfg


def test_exact_batch_reproduces_reference(cuda_device, golden):
    import rcpgenerator_b200 as rb
    g = golden("packs.npz")
    # the golden cases with a step cap share it through the batch options only
    # when equal, so run the uncapped ones and the capped ones separately
    groups: dict[int, list[str]] = {}
    for c in CASES:
        groups.setdefault(int(g[f"{c}/max_steps"]), []).append(c)
    for ms, cases in groups.items():
        opts = {"max_steps": ms} if ms else {}
        out = rb.run_packing_batch([item(g, c, "exact") for c in cases], opts, concurrency=3)
        for c, r in zip(cases, out):
            sc = g[f"{c}/scalars"]
            assert r["steps"] == int(sc[0]), c
            assert np.array_equal(r["positions"], g[f"{c}/positions"]), c
            assert digest(r["phi_history"]) == str(g[f"{c}/phi_history_sha256"]), c


def test_graph_batch_equals_single_runs(cuda_device, golden):
    import rcpgenerator_b200 as rb
    g = golden("packs.npz")
    cases = ["n16_2d", "n64_3d_bi", "n200_2d_disk_2500"]
    opts = {"max_steps": 1500}
    out = rb.run_packing_batch([item(g, c, "graph") for c in cases] * 2, opts, concurrency=4)
    for k, c in enumerate(cases):
        inp, cfg = item(g, c, "graph")
        alone = rb.run_packing_observed(inp, cfg, 0, False, 0, None, opts, as_arrays=True)["result"]
        for r in (out[k], out[k + len(cases)]):
            assert r["steps"] == alone["steps"]
            assert np.array_equal(r["positions"], alone["positions"])
            assert np.array_equal(r["phi_history"], alone["phi_history"])


def test_hybrid_batch_matches_its_parts(cuda_device, golden):
    """concurrency=0 sends each packing to the persistent kernel or to an engine
    on a stream by its size; either way a packing's result equals the one of
    that path run alone."""
    import rcpgenerator_b200 as rb
    g = golden("packs.npz")
    items = [item(g, c, "graph") for c in ("n16_2d", "n64_3d_bi", "cfg1_n2000_3d")]
    opts = {"max_steps": 1200}
    mixed = rb.run_packing_batch(items, opts, concurrency=0)
    small = rb.run_packing_batch(items[:2], opts, concurrency=-1)
    large = rb.run_packing_batch(items[2:], opts, concurrency=1)
    for r, ref in zip(mixed, small + large):
        assert np.array_equal(r["positions"], ref["positions"])


def test_batch_reports_the_failing_packing(cuda_device, golden):
    import rcpgenerator_b200 as rb
    g = golden("packs.npz")
    good = item(g, "n16_2d", "graph")
    bad_inp, bad_cfg = item(g, "n16_2d", "graph")
    bad_cfg = dict(bad_cfg, box=[1.0, 1.0, 1.0])  # box length != ndim: the reference's error
    with pytest.raises((ValueError, RuntimeError), match="packing 1"):
        rb.run_packing_batch([good, (bad_inp, bad_cfg), good], {"max_steps": 50}, concurrency=2)


# ---- persistent batch engine (concurrency=-1): one thread block per packing ----

def cfg1_item(seed, precision="f64"):
    import rcpgenerator_b200 as rb
    init = rb.initialize_particles({"phi": 0.08, "N": 2000, "Ndim": 3, "box": [1.0, 1.0, 1.0],
                                    "walls": [0, 0, 0], "dist": {"type": "mono", "d": 1.0},
                                    "seed": seed})
    return ({"positions": np.asarray(init["positions"]), "diameters": np.asarray(init["diameters"])},
            {"box": init["box"], "walls": init["walls"], "neighbor_max": 0, "seed": seed,
             "pair_precision": precision})


def test_persistent_batch_is_deterministic_and_independent_of_its_batch(cuda_device, golden):
    """A packing is run by one thread block from start to end, so its result
    does not depend on the other packings of the launch or on the run."""
    import rcpgenerator_b200 as rb
    g = golden("packs.npz")
    items = [item(g, c, "graph") for c in ("n16_2d", "n200_2d_disk_2500", "n64_2d_walls_500")]
    opts = {"max_steps": 2500}
    a = rb.run_packing_batch(items, opts, concurrency=-1)
    b = rb.run_packing_batch(items[::-1], opts, concurrency=-1)[::-1]
    alone = rb.run_packing_batch(items[1:2], opts, concurrency=-1)[0]
    for ra, rb_ in zip(a, b):
        assert ra["steps"] == rb_["steps"]
        assert np.array_equal(ra["positions"], rb_["positions"])
        assert np.array_equal(ra["phi_history"], rb_["phi_history"])
    assert np.array_equal(a[1]["positions"], alone["positions"])


def test_persistent_batch_mixed_ndim_converges(cuda_device, golden):
    import rcpgenerator_b200 as rb
    g = golden("packs.npz")
    cases = ["n16_2d", "n64_3d_bi", "n300_4d_1500", "n128_3d_sphere_3000"]
    out = rb.run_packing_batch([item(g, c, "graph") for c in cases], {}, concurrency=-1)
    for c, r in zip(cases, out):
        assert np.isfinite(r["positions"]).all(), c
        assert len(r["phi_history"]) == r["steps"]
        assert r["max_min_dist"] < 5e-4 or r["steps"] >= 60000, c


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_persistent_batch_config1_phiJ_distribution_64_seeds(cuda_device, golden, precision):
    """The 3-D monodisperse N = 2000 packing over 64 seeds in one persistent launch against the
    reference's distribution on the same seeds: |mean phi_J - reference| <= 1e-3,
    mean step count within 5 %, every packing under the reference's gate."""
    import rcpgenerator_b200 as rb
    g = golden("cfg1_seeds.npz")
    out = rb.run_packing_batch([cfg1_item(int(s), precision) for s in g["seed"].tolist()], {},
                               concurrency=-1)
    phis = np.asarray([r["phi"] for r in out])
    steps = np.asarray([r["steps"] for r in out])
    assert abs(phis.mean() - g["phi"].mean()) <= 1e-3
    assert abs(steps.mean() - g["steps"].mean()) <= 0.05 * g["steps"].mean()
    assert (np.asarray([r["max_min_dist"] for r in out]) < 5e-4).all()


def test_batch_autotuner_picks_the_faster_measured_shape(cuda_device):
    import rcpgenerator_b200 as rb
    t = rb.batch_tuning(3, pair_precision="mixed")
    assert t["blocks_per_sm"] in (1, 2)
    assert min(t["steps_per_s"]) > 0.0
    assert t["steps_per_s"][t["blocks_per_sm"] - 1] == max(t["steps_per_s"])
    assert rb.batch_tuning(3, pair_precision="mixed") == t  # kept for the process
