"""Failure paths through the engine, each made on the host (no GPU fault):

* a neighbour row over the reference's per-particle capacity (tiny
  neighbor_max on a clustered input) raises the reference's RuntimeError,
  naming the same particle and capacity (ENG:647-658), in both engines, and
  the device stays usable for the next packing;
* a NaN position runs to completion as in the reference (which raises no
  error for it): the exact engine reproduces the reference's run
  (tests/golden/failure_nan.npz), the graph engine completes it;
* max_steps caps the run at exactly that many steps.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _clustered():
    rng = np.random.default_rng(0)
    return {"positions": 0.5 + 0.01 * rng.random((200, 2)), "diameters": np.full(200, 0.05)}


# the reference engine's text for this input (one thread; make_failure_golden.py)
OVERFLOW_TEXT = ("rcpgenerator: particle 0 exceeded its neighbor capacity (34 slots) during pair-list "
                 "construction (kdtree own-write). This usually means the per-particle neighbor allocation "
                 "is too small for the size ratio in this packing. Recommendation: pass a larger "
                 "neighbor_max (the per-particle base; e.g. neighbor_max=1500 -- capacity scales as "
                 "50*(D_i/D_min)^omega + neighbor_max), or reduce the size ratio.")


@pytest.mark.parametrize("engine", ["exact", "graph"])
def test_neighbour_overflow_raises_reference_error(cuda_device, golden, engine):
    import rcpgenerator_b200 as rb
    assert str(golden("failure_nan.npz")["overflow_text"]) == OVERFLOW_TEXT
    with pytest.raises(RuntimeError) as ei:
        rb.run_packing(_clustered(), {"box": [1.0, 1.0], "walls": [0, 0], "neighbor_max": 1,
                                      "engine": engine})
    assert str(ei.value) == OVERFLOW_TEXT
    # the device is still usable
    r = rb.run_packing_observed({"positions": np.random.default_rng(1).random((64, 2)),
                                 "diameters": np.full(64, 0.05)}, {"box": [1.0, 1.0], "engine": engine},
                                0, False, 0, None, {"max_steps": 50}, as_arrays=True)["result"]
    assert r["steps"] == 50 and np.isfinite(r["positions"]).all()


def test_nan_position_runs_like_reference(cuda_device, golden):
    import rcpgenerator_b200 as rb
    g = golden("failure_nan.npz")
    inp = {"positions": g["input_positions"], "diameters": g["input_diameters"]}
    K = int(g["max_steps"])
    r = rb.run_packing_observed(inp, {"box": [1.0, 1.0], "walls": [0, 0], "engine": "exact"}, 0, False, 0,
                                None, {"max_steps": K}, as_arrays=True)["result"]
    assert r["steps"] == int(g["steps"])
    assert r["phi"] == float(g["phi"])
    assert np.array_equal(r["phi_history"], g["phi_history"])
    # the reference's comparison sort leaves the NaN particle at an arbitrary
    # row (the others in x order); every other particle, in the same order,
    # is identical
    nan_r, nan_g = np.isnan(r["positions"]).any(1), np.isnan(g["positions"]).any(1)
    assert nan_r.sum() == nan_g.sum() == 1
    assert np.array_equal(r["positions"][~nan_r], g["positions"][~nan_g])
    assert np.array_equal(np.asarray(r["particle_origin"])[~nan_r], g["particle_origin"][~nan_g])
    # the graph engine completes the same number of steps
    r2 = rb.run_packing_observed(inp, {"box": [1.0, 1.0], "walls": [0, 0]}, 0, False, 0, None,
                                 {"max_steps": K}, as_arrays=True)["result"]
    assert r2["steps"] == int(g["steps"])
    assert np.isnan(r2["positions"]).any(1).sum() == 1


@pytest.mark.parametrize("engine", ["exact", "graph"])
@pytest.mark.parametrize("cap", [1, 31, 33, 100])
def test_max_steps_caps_the_run(cuda_device, engine, cap):
    import rcpgenerator_b200 as rb
    init = rb.initialize_particles({"phi": 0.1, "N": 300, "Ndim": 3, "box": [1.0] * 3, "walls": [0] * 3,
                                    "dist": {"type": "mono", "d": 1.0}, "seed": 3})
    r = rb.run_packing_observed({"positions": init["positions"], "diameters": init["diameters"]},
                                {"box": init["box"], "walls": init["walls"], "engine": engine}, 0, False, 0,
                                None, {"max_steps": cap}, as_arrays=True)["result"]
    assert r["steps"] == cap == len(r["phi_history"])
