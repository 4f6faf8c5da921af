"""Mixed-precision pair arithmetic (graph mode, pair_precision="mixed").

The pair terms (distance, force magnitude, energy, dkappa) are computed in FP32
from the FP64 minimum-image displacement while the max overlap of the last step
is >= mixed_switch (relative overlap, default 1e-5), and in FP64 from the first
step below it. Positions, ADAM state, diameters, the neighbour shell test and
every global sum stay FP64. Checked here:

* the first steps track the FP64 graph engine (FP32 rounding of the forces);
* the run reports the final state's energy / force error of the FP32 terms
  against FP64 terms on the same rows, and the step of the switch;
* the 3-D monodisperse N = 2000 packing over 64 seeds matches the reference's phi_J distribution
  (|mean phi_J - reference mean| <= 1e-3) and every packing meets the gate.
"""

from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def cfg1(seed=123):
    import rcpgenerator_b200 as rb
    init = rb.initialize_particles({"phi": 0.08, "N": 2000, "Ndim": 3, "box": [1.0, 1.0, 1.0],
                                    "walls": [0, 0, 0], "dist": {"type": "mono", "d": 1.0},
                                    "seed": seed})
    inp = {"positions": np.asarray(init["positions"]), "diameters": np.asarray(init["diameters"])}
    cfg = {"box": init["box"], "walls": init["walls"], "neighbor_max": 0, "seed": seed}
    return inp, cfg


def run(inp, cfg, precision, opts=None, **extra):
    import rcpgenerator_b200 as rb
    c = dict(cfg, engine="graph", pair_precision=precision, **extra)
    return rb.run_packing_observed(inp, c, 0, False, 0, None, dict(opts or {}), as_arrays=True)["result"]


@pytest.mark.parametrize("steps,tol", [(3, 2e-5), (40, 5e-2)])
def test_mixed_first_steps_track_f64(cuda_device, steps, tol):
    """FP32 pair terms perturb each pair force by about 1e-7 relative. A force
    component whose pair terms nearly cancel keeps a larger relative error,
    and ADAM's normalised step (epsilon 1e-8) passes part of it on: after 3
    steps the positions differ by about 1.6e-6 Dmin, after 40 steps by about
    1e-2 Dmin (chaotic early dynamics, step size about 0.07 Dmin). Tolerances
    are absolute position differences relative to the smallest diameter."""
    inp, cfg = cfg1()
    a = run(inp, cfg, "f64", {"max_steps": steps})
    b = run(inp, cfg, "mixed", {"max_steps": steps})
    assert a["steps"] == b["steps"] == steps
    dmin = a["diameters"].min()
    dx = np.abs(a["positions"] - b["positions"]).max()
    assert dx <= tol * dmin, dx / dmin
    assert np.abs(a["phi_history"] - b["phi_history"]).max() <= (1e-9 if steps <= 3 else 1e-6) * a["phi_history"].max()
    st = b["engine_stats"]
    assert st["fp64_switch_step"] == 0  # large overlaps: still FP32
    assert 0.0 <= st["pair_energy_rel_error"] < 1e-4
    assert 0.0 <= st["pair_force_rel_error"] < 1e-4
    assert math.isnan(a["engine_stats"]["pair_force_rel_error"])


def test_mixed_switch_is_one_way(cuda_device):
    """A switch above every overlap turns FP64 on after step 1 for good."""
    inp, cfg = cfg1()
    b = run(inp, cfg, "mixed", {"max_steps": 30}, mixed_switch=10.0)
    assert b["engine_stats"]["fp64_switch_step"] == 1
    assert b["engine_stats"]["pair_force_rel_error"] < 1e-4


def test_mixed_config1_phiJ_distribution_64_seeds(cuda_device, golden):
    g = golden("cfg1_seeds.npz")
    phis, steps, ovs, ferr = [], [], [], []
    for seed in g["seed"].tolist():
        inp, cfg = cfg1(int(seed))
        r = run(inp, cfg, "mixed")
        phis.append(r["phi"])
        steps.append(r["steps"])
        ovs.append(r["max_min_dist"])
        ferr.append(r["engine_stats"]["pair_force_rel_error"])
    phis = np.asarray(phis)
    assert abs(phis.mean() - g["phi"].mean()) <= 1e-3
    assert abs(np.mean(steps) - g["steps"].mean()) <= 0.05 * g["steps"].mean()
    assert (np.asarray(ovs) < 5e-4).all()
    assert np.isfinite(ferr).all()
