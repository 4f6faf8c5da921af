"""Golden outputs of the reference's stateful API, rcpgenerator.Packing
(python/rcpgenerator/_wrapper.py:28-628), on the reference engine.

Runs in a container that holds the reference tree. The reference package's
__init__ imports its matplotlib renderer, so _wrapper.py is loaded on its own
into a stand-in package whose _rcpgenerator is the reference's compiled module
(oracle/_ref, built from its sources by oracle/Makefile) and whose render
module is a stub; the Packing class itself runs unmodified.

Records, per scenario, the reference object's to_dict() after each call
(construction, pack, relax, update_phi, update_box, update_height; each
history as its length and SHA-256), the values those calls return, and its
state flags, as JSON in tests/golden/wrapper.json.

Usage:  python tests/golden/make_wrapper_golden.py /path/to/RCPGenerator
"""

from __future__ import annotations

import importlib.util
import json
import os
import subprocess
import sys
import types
from pathlib import Path

REPO = Path(__file__).resolve().parents[2]
OUT = Path(__file__).resolve().parent / "wrapper.json"
REF_DIR = REPO / "oracle" / "_ref"

SCENARIOS = {
    # periodic 2-D bidisperse, packed to the convergence gate
    "bi2d_n64_pack": {"ctor": dict(phi=0.1, N=64, Ndim=2, box=[1.0, 1.0], walls=[0, 0], seed=5,
                                   dist={"type": "bidisperse", "d1": 1.0, "d2": 1.4, "p": 0.5}),
                      "calls": [["pack", {}]]},
    # a disk container (walls[0] = -2): phi_final and phi_history against the disk
    "disk2d_n80_pack": {"ctor": dict(phi=0.1, N=80, Ndim=2, box=[1.0, 1.0], walls=[-2, 0], seed=4,
                                     dist={"type": "mono", "d": 1.0}),
                        "calls": [["pack", {}]]},
    # relax options and the realized-state updates
    "mono3d_n64_relax": {"ctor": dict(phi=0.2, N=64, Ndim=3, box=[1.0, 1.0, 1.0], walls=[0, 0, 0], seed=6,
                                      dist={"type": "mono", "d": 1.0}),
                         "calls": [["relax", {"n_steps": 300, "mu": 1e-3}],
                                   ["update_phi", {"target_phi": 0.3}],
                                   ["relax", {"n_steps": 200, "fix_diameter": True}],
                                   ["update_box", {"box": [1.2, 1.0, 0.9]}],
                                   ["update_height", {"height": 1.1}]]},
    "sphere3d_n100_target": {"ctor": dict(phi=0.1, N=100, Ndim=3, box=[1.0, 1.0, 1.0], walls=[-3, 0, 0],
                                          seed=9, dist={"type": "flat", "d_min": 0.5, "d_max": 1.5}),
                             "calls": [["relax", {"n_steps": 2500, "target_phi": 0.45}]]},
}


def _load_reference_wrapper(ref_root: Path):
    sys.path.insert(0, str(REF_DIR))
    for k in list(os.environ):
        if k.startswith("RCP_"):
            del os.environ[k]
    import _rcpgenerator  # noqa: E402  (the reference's compiled module)

    _rcpgenerator.set_num_threads(1)
    pkg = types.ModuleType("refpkg")
    pkg.__path__ = []
    sys.modules["refpkg"] = pkg
    sys.modules["refpkg._rcpgenerator"] = _rcpgenerator
    render = types.ModuleType("refpkg.render")

    def _no_render(*a, **k):
        raise RuntimeError("rendering is not recorded")

    render.animate_packing_2d = _no_render
    render.render_packing = _no_render
    sys.modules["refpkg.render"] = render
    src = ref_root / "python_code" / "python" / "python" / "rcpgenerator" / "_wrapper.py"
    spec = importlib.util.spec_from_file_location("refpkg._wrapper", src)
    mod = importlib.util.module_from_spec(spec)
    sys.modules["refpkg._wrapper"] = mod
    spec.loader.exec_module(mod)
    return mod.Packing


def compact(d: dict) -> dict:
    """to_dict() with each history list replaced by its length and the SHA-256
    of its float64 bytes (the states are compared exactly either way)."""
    import hashlib

    import numpy as np

    d = json.loads(json.dumps(d))
    for k in ("phi_history", "force_history", "energy_history"):
        h = d["final_result"].get(k, [])
        d["final_result"][k] = {"len": len(h), "sha256": hashlib.sha256(
            np.ascontiguousarray(np.asarray(h, dtype=np.float64)).tobytes()).hexdigest()}
    return d


def _flags(p) -> dict:
    return {"initialized": p.initialized, "packed": p.packed, "needs_initialize": p.needs_initialize,
            "needs_pack": p.needs_pack}


def main(ref_root: str) -> None:
    subprocess.run(["make", "-C", str(REPO / "oracle"), "PY=" + sys.executable,
                    "REF_ROOT=" + str(Path(ref_root) / "python_code" / "python")], check=True)
    Packing = _load_reference_wrapper(Path(ref_root))
    out = {}
    for name, sc in SCENARIOS.items():
        p = Packing(**sc["ctor"])
        rec = {"ctor": sc["ctor"], "calls": sc["calls"], "states": [compact(p.to_dict())], "flags": [_flags(p)],
               "returns": [None]}
        for meth, kw in sc["calls"]:
            ret = getattr(p, meth)(**kw)
            if meth in ("pack", "relax"):
                ret = {k: ret[k] for k in ("steps", "phi", "max_min_dist", "force_magnitude")}
            rec["states"].append(compact(p.to_dict()))
            rec["flags"].append(_flags(p))
            rec["returns"].append(ret)
        # attribute writes move the flags (WRP:128-138)
        q = Packing(**sc["ctor"])
        q.seed = 17
        f_pack = _flags(q)
        q.phi = sc["ctor"]["phi"] * 1.5
        rec["flags_after_seed_then_phi"] = [f_pack, _flags(q)]
        out[name] = rec
        print(name, [r["steps"] if isinstance(r, dict) else r for r in rec["returns"]])
    OUT.write_text(json.dumps(out))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_wrapper_golden.py /path/to/RCPGenerator")
    main(sys.argv[1])
