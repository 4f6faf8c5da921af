"""The engine's own per-particle arithmetic (rcpg_core.h), controller
(rcpg_schedule.h) and setup (rcpg_setup.cpp), run on the CPU by the host
emulation, against complete reference packings (tests/golden/packs.npz)."""

from __future__ import annotations

import hashlib

import numpy as np
import pytest

HIST = ("phi_history", "force_history", "energy_history", "max_overlap_history", "mu_history",
        "alpha_history")
FAST = ["n4_2d", "n16_2d", "n64_3d_bi", "n64_2d_walls_500", "n128_3d_sphere_3000",
        "n200_2d_disk_2500", "n300_4d_1500", "n64_3d_fix_diameter", "n100_2d_mu",
        "n60_2d_fix_height_wall", "n600_3d_powerlaw10_sphere_1500", "n80_2d_no_reorder"]


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def case_options(g, case):
    """Run options the golden packing was made with (PackingRunOptions keys)."""
    pre = f"{case}/opt/"
    return {k[len(pre):]: g[k][()] for k in g.files if k.startswith(pre)}


def check_pack(r, g, case):
    sc = g[f"{case}/scalars"]
    assert r["steps"] == int(sc[0])
    assert r["phi"] == sc[1]
    assert r["max_min_dist"] == sc[2]
    assert r["force_magnitude"] == sc[3] or (np.isnan(r["force_magnitude"]) and np.isnan(sc[3]))
    assert np.array_equal(r["positions"], g[f"{case}/positions"])
    assert np.array_equal(r["diameters"], g[f"{case}/diameters"])
    assert np.array_equal(np.asarray(r["particle_origin"], dtype=np.uint64), g[f"{case}/particle_origin"])
    for h in HIST:
        assert digest(np.asarray(r[h], dtype=np.float64)) == str(g[f"{case}/{h}_sha256"]), h
    assert digest(np.asarray(r["mu_flag_history"], dtype=np.int8)) == str(g[f"{case}/mu_flag_history_sha256"])


@pytest.mark.parametrize("case", FAST)
def test_emulation_reproduces_reference_pack(hostemu, golden, case):
    g = golden("packs.npz")
    o = case_options(g, case)
    r = hostemu.run(g[f"{case}/input_positions"], g[f"{case}/input_diameters"], g[f"{case}/box_in"],
                    g[f"{case}/walls_in"], max_steps=int(g[f"{case}/max_steps"]),
                    reorder=int(o.get("reorder_interval", 2000)), fix_height=bool(g[f"{case}/fix_height"]),
                    mu=float(o["mu"]) if "mu" in o else None, fix_diameter=bool(o.get("fix_diameter", False)))
    check_pack(r, g, case)
