"""Product initializer (host C++, rcpg_initialize_particles) against the
reference's initialize_particles for every distribution family."""

from __future__ import annotations

import numpy as np
import pytest

from tests.golden.make_golden import INIT_CASES


@pytest.mark.parametrize("case", INIT_CASES, ids=[c["name"] for c in INIT_CASES])
def test_initializer_bit_exact(golden, case):
    import rcpgenerator_b200 as rb
    g = golden("initializer.npz")
    cfg = {k: v for k, v in case.items() if k != "name"}
    r = rb.initialize_particles(cfg)
    nm = case["name"]
    assert np.array_equal(np.asarray(r["positions"]), g[nm + "/positions"])
    assert np.array_equal(np.asarray(r["diameters"]), g[nm + "/diameters"])
    assert np.array_equal(np.asarray(r["box"]), g[nm + "/box"])
    assert np.array_equal(np.asarray(r["walls"], dtype=np.int8), g[nm + "/walls"])
    assert r["diameter_scale_factor"] == g[nm + "/scalars"][0]
    assert r["phi_modifier"] == g[nm + "/scalars"][1]


def test_initializer_errors():
    import rcpgenerator_b200 as rb
    with pytest.raises(RuntimeError, match="Ndim must be >=2"):
        rb.initialize_particles({"phi": 0.1, "N": 4, "Ndim": 1})
    with pytest.raises(RuntimeError, match="invalid phi/N"):
        rb.initialize_particles({"phi": 1.5, "N": 4, "Ndim": 2})
    with pytest.raises(ValueError, match="Unsupported distribution"):
        rb.initialize_particles({"phi": 0.1, "N": 4, "Ndim": 2, "dist": {"type": "zipf"}})
    with pytest.raises(RuntimeError, match="custom distribution needs N entries"):
        rb.initialize_particles({"phi": 0.1, "N": 4, "Ndim": 2, "dist": {"type": "custom", "custom": [1.0]}})
