"""rcpgenerator_b200.Packing on the GPU against the reference's own Packing
class (python/rcpgenerator/_wrapper.py:28-628) running the reference engine
at one OpenMP thread (tests/golden/wrapper.json): with engine="exact" every
state after pack / relax / update_* -- positions, diameters, box, walls,
phi_final with the container correction (WRP:309-332), steps, scalars and the
SHA-256 of every history -- and every returned value is identical. The graph
engine converges under the same gate to a nearby phi_final.
"""

from __future__ import annotations

import pytest

from tests import packing_golden as PG

pytestmark = pytest.mark.gpu

G = PG.load()


@pytest.mark.parametrize("name", sorted(G))
def test_packing_exact_engine_reproduces_reference_states(cuda_device, name):
    import rcpgenerator_b200 as rb
    rec = G[name]
    p = rb.Packing(**rec["ctor"], engine="exact")
    assert PG.compact(p.to_dict()) == rec["states"][0]
    for k, (meth, kw) in enumerate(rec["calls"]):
        ret = getattr(p, meth)(**kw)
        if meth in ("pack", "relax"):
            ret = {q: ret[q] for q in ("steps", "phi", "max_min_dist", "force_magnitude")}
        assert PG._plain(ret) == rec["returns"][k + 1], meth
        assert PG.compact(p.to_dict()) == rec["states"][k + 1], meth
        flags = {"initialized": p.initialized, "packed": p.packed, "needs_initialize": p.needs_initialize,
                 "needs_pack": p.needs_pack}
        assert flags == rec["flags"][k + 1], meth


@pytest.mark.parametrize("name", ["bi2d_n64_pack", "disk2d_n80_pack"])
def test_packing_graph_engine_converges(cuda_device, name):
    import rcpgenerator_b200 as rb
    rec = G[name]
    p = rb.Packing(**rec["ctor"])
    p.pack()
    ref = rec["states"][1]["final_result"]
    assert p.packed and not p.needs_pack
    assert p.max_min_dist < 5e-4
    assert abs(p.phi_final - ref["phi_final"]) < 0.02
    assert 0.8 * ref["steps"] < p.steps < 1.25 * ref["steps"]
    assert len(p.phi_history) == p.steps
