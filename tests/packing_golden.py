"""Helpers of the Packing tests: the reference's recorded Packing states
(tests/golden/wrapper.json, tests/golden/make_wrapper_golden.py) and the same
compact form of this package's Packing.to_dict()."""

from __future__ import annotations

import hashlib
import json
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden" / "wrapper.json"


def load() -> dict:
    return json.loads(GOLDEN.read_text())


def _plain(v):
    """NumPy arrays and scalars -> the JSON types the reference returns."""
    return json.loads(json.dumps(v, default=lambda o: o.tolist() if hasattr(o, "tolist") else o))


def compact(d: dict) -> dict:
    """to_dict() with each history replaced by its length and SHA-256, and the
    engine selector (a keyword this package adds) dropped from pack_config."""
    d = _plain(d)
    d["pack_config"].pop("engine", None)
    for k in ("phi_history", "force_history", "energy_history"):
        h = d["final_result"].get(k, [])
        d["final_result"][k] = {"len": len(h), "sha256": hashlib.sha256(
            np.ascontiguousarray(np.asarray(h, dtype=np.float64)).tobytes()).hexdigest()}
    return d


def expand(state: dict) -> dict:
    """A recorded state as from_dict() input (histories dropped)."""
    s = json.loads(json.dumps(state))
    for k in ("phi_history", "force_history", "energy_history"):
        s["final_result"][k] = []
    return s
