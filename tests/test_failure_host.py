"""Argument errors of run_packing need no GPU and carry the reference's types
and texts (ENG:4440, :4446: std::runtime_error -> RuntimeError), checked
against the reference's compiled module where it is built (oracle/_ref)."""

from __future__ import annotations

import os
import sys
from pathlib import Path

import pytest

REF = Path(__file__).resolve().parents[1] / "oracle" / "_ref"
INP = {"positions": [[0.1, 0.1], [0.5, 0.5]], "diameters": [0.1, 0.1]}
CASES = [({"box": [1.0, 1.0], "walls": [0, 0, 0]}, "Error: --walls expects Ndim entries"),
         ({"box": [1.0, 1.0, 1.0], "walls": [0, 0]}, "Error: --box length mismatch")]


@pytest.mark.parametrize("cfg,text", CASES)
def test_argument_errors_match_reference(cfg, text):
    import rcpgenerator_b200 as rb
    with pytest.raises(RuntimeError) as ei:
        rb.run_packing(INP, cfg)
    assert str(ei.value) == text
    if any(REF.glob("_rcpgenerator*.so")):
        sys.path.insert(0, str(REF))
        for k in list(os.environ):
            if k.startswith("RCP_"):
                del os.environ[k]
        import _rcpgenerator as ref
        with pytest.raises(RuntimeError) as er:
            ref.run_packing(INP, dict(cfg, neighbor_max=0, seed=0))
        assert str(er.value) == text


def test_size_mismatch_is_value_error():
    import rcpgenerator_b200 as rb
    with pytest.raises(ValueError):
        rb.run_packing({"positions": [[0.1, 0.1], [0.5, 0.5]], "diameters": [0.1]}, {"box": [1.0, 1.0]})
