"""The stateful API (rcpgenerator_b200.Packing) against the reference's own
Packing class (python/rcpgenerator/_wrapper.py:28-628), on the host parts that
need no GPU: construction (the initializer), to_dict / from_dict, the state
flags, update_phi / update_box / update_height and argument errors. Every
compared state is the reference object's, recorded by
tests/golden/make_wrapper_golden.py; equality is exact.
"""

from __future__ import annotations

import math

import pytest

from tests import packing_golden as PG

G = PG.load()


@pytest.mark.parametrize("name", sorted(G))
def test_constructor_matches_reference(name):
    import rcpgenerator_b200 as rb
    rec = G[name]
    p = rb.Packing(**rec["ctor"])
    assert PG.compact(p.to_dict()) == rec["states"][0]
    assert {"initialized": p.initialized, "packed": p.packed, "needs_initialize": p.needs_initialize,
            "needs_pack": p.needs_pack} == rec["flags"][0]


@pytest.mark.parametrize("name", sorted(G))
def test_attribute_writes_move_state_flags_like_reference(name):
    import rcpgenerator_b200 as rb
    rec = G[name]
    q = rb.Packing(**rec["ctor"])
    q.seed = 17
    f1 = {"initialized": q.initialized, "packed": q.packed, "needs_initialize": q.needs_initialize,
          "needs_pack": q.needs_pack}
    q.phi = rec["ctor"]["phi"] * 1.5
    f2 = {"initialized": q.initialized, "packed": q.packed, "needs_initialize": q.needs_initialize,
          "needs_pack": q.needs_pack}
    assert [f1, f2] == rec["flags_after_seed_then_phi"]


def test_realized_state_updates_match_reference():
    """update_phi / update_box / update_height applied to the reference's own
    states (restored with from_dict) give the reference's next states and
    return values."""
    import rcpgenerator_b200 as rb
    rec = G["mono3d_n64_relax"]
    for k, (meth, kw) in enumerate(rec["calls"]):
        if not meth.startswith("update_"):
            continue
        p = rb.Packing.from_dict(PG.expand(rec["states"][k]))
        ret = getattr(p, meth)(**kw)
        assert PG._plain(ret) == rec["returns"][k + 1], meth
        assert PG.compact(p.to_dict()) == rec["states"][k + 1], meth


@pytest.mark.parametrize("name", sorted(G))
def test_from_dict_round_trip(name):
    import rcpgenerator_b200 as rb
    for st in G[name]["states"]:
        p = rb.Packing.from_dict(PG.expand(st))
        q = rb.Packing.from_dict(p.to_dict())
        assert PG.compact(q.to_dict()) == PG.compact(p.to_dict())
        assert PG.compact(p.copy().to_dict()) == PG.compact(p.to_dict())


def test_container_fraction_and_argument_errors():
    import rcpgenerator_b200 as rb
    from rcpgenerator_b200._wrapper import _container_fraction
    assert _container_fraction([-3, -1, -1]) == math.pi / 6.0
    assert _container_fraction([-2, -1]) == math.pi / 4.0
    assert _container_fraction([0, 0]) == 1.0
    rec = G["bi2d_n64_pack"]
    p = rb.Packing(**rec["ctor"])
    with pytest.raises(ValueError):
        p.relax(0)
    with pytest.raises(ValueError):
        p.relax(10, fix_diameter=True, target_phi=0.5)
    with pytest.raises(ValueError):
        p.update_box([1.0])
    with pytest.raises(ValueError):
        p.update_phi(-1.0)
    with pytest.raises(TypeError):
        rb.Packing(N=10, Ndim=2, box=[1.0, 1.0], bogus=1)
    with pytest.raises(NotImplementedError):
        p.render()
