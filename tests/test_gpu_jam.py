"""A packing of the N = 1M 2-D bidisperse workload's kind at N = 100,000, run
to the reference's convergence gate (ENG:5603-5655: max overlap < 5e-4 three
checks in a row; its mean-force term reads the history entry of the step not
yet run, which is zero) in mixed and in FP64 pair
precision. Mixed precision would switch to FP64 pair terms once the max
overlap fell below 1e-5, which a run that ends at the gate's 5e-4 does not
reach; its jamming fraction must stay within 1e-3 of the FP64 run's (the
tolerance the mixed path is held to); both runs end by the gate, not by the
step cap.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CFG = dict(phi=0.30, N=100_000, Ndim=2, box=[1.0, 1.0], walls=[0, 0],
           dist={"type": "bidisperse", "d1": 1.0, "d2": 1.4, "p": 0.5}, seed=123)


def test_mixed_precision_jams_within_1e3_of_fp64(cuda_device):
    import rcpgenerator_b200 as rb
    init = rb.initialize_particles(CFG)
    inp = {"positions": init["positions"], "diameters": init["diameters"]}
    out = {}
    for prec in ("mixed", "f64"):
        out[prec] = rb.run_packing_observed(inp, {"box": init["box"], "walls": init["walls"],
                                                  "pair_precision": prec}, 0, False, 0, None, {},
                                            as_arrays=True)["result"]
    m, f = out["mixed"], out["f64"]
    for prec, r in out.items():
        why = (prec, r["steps"], r["phi"], r["max_min_dist"], r["force_history"][-4:],
               r["max_overlap_history"][-4:], r["engine_stats"])
        # ended by the convergence gate: the final max overlap below its threshold
        assert r["max_min_dist"] < 5e-4, why
        # the mean force is the reference's (ENG:769-801): the mean |F_i| over
        # the particles with |F_i|^2 > 1e-16, NaN when there is none -- which
        # happens near jamming at this box scale (|F_i| ~ 1e-9); the gate
        # reads the entry of the step not yet run (zero), so it does not
        # depend on it
        fh = r["force_history"]
        assert np.isfinite(fh[: len(fh) // 2]).all(), why
        assert np.isnan(fh[-1]) or fh[-1] < 5e-3, why
        assert np.isfinite(r["positions"]).all()
        assert 0.80 < r["phi"] < 0.90
    # the FP64 run reports no mixed-precision error; the mixed run reports its
    # final state's FP32-vs-FP64 pair-term error and its switch step (0 when
    # the max overlap stayed above the switch, 1e-5, to the end)
    assert np.isnan(f["engine_stats"]["pair_force_rel_error"])
    assert np.isfinite(m["engine_stats"]["pair_force_rel_error"])
    assert m["engine_stats"]["fp64_switch_step"] >= 0
    assert abs(m["phi"] - f["phi"]) <= 1e-3
