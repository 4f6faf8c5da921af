"""Graph-mode packings of the 3-D monodisperse N = 2000 packing (phi0 0.08) over 64 seeds against the
reference's distribution on the same seeds (tests/golden/cfg1_seeds.npz):
relaxation to jamming is chaotic, so the graph engine (tree-order FP64
reductions, CUDA libm in the controller) is matched in distribution:
|mean phi_J - reference mean| <= 1e-3, and every packing meets the
reference's convergence gate (max overlap < 5e-4)."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_config1_phiJ_distribution_64_seeds(cuda_device, golden):
    import rcpgenerator_b200 as rb
    g = golden("cfg1_seeds.npz")
    phis, steps, ovs = [], [], []
    for seed in g["seed"].tolist():
        init = rb.initialize_particles({"phi": 0.08, "N": 2000, "Ndim": 3, "box": [1.0, 1.0, 1.0],
                                        "walls": [0, 0, 0], "dist": {"type": "mono", "d": 1.0},
                                        "seed": int(seed)})
        r = rb.run_packing({"positions": init["positions"], "diameters": init["diameters"]},
                           {"box": init["box"], "walls": init["walls"], "neighbor_max": 0,
                            "seed": int(seed)}, as_arrays=True)
        phis.append(r["phi"])
        steps.append(r["steps"])
        ovs.append(r["max_min_dist"])
    phis = np.asarray(phis)
    assert abs(phis.mean() - g["phi"].mean()) <= 1e-3
    assert abs(np.mean(steps) - g["steps"].mean()) <= 0.05 * g["steps"].mean()
    assert (np.asarray(ovs) < 5e-4).all()
