"""Host logic of the learned warm start on the CPU: descriptors, training
targets, the growth-rung rule, and the engine's growth_steps option in the
host emulation of exact mode (the rung ends at the given step, the schedule
after it is the reference's)."""

from __future__ import annotations

import math

import numpy as np
import pytest

from rcpgenerator_b200 import warmstart as W


def test_descriptors():
    d = np.array([1.0, 1.0, 1.4, 1.4])
    x = W.descriptors(d, 3, [0, 0, 0])
    assert x.shape == (11,)
    assert W.descriptors(d, 3, [0, 0, 0], with_n=True)[11] == pytest.approx(math.log(4.0))
    r = d / d.mean()
    for k in range(1, 9):
        assert x[k - 1] == pytest.approx(math.log(np.mean(r ** k)) / k, rel=1e-14, abs=1e-15)
    assert x[0] == pytest.approx(0.0, abs=1e-15)  # first moment of d/<d> is 1
    assert tuple(x[8:]) == (3.0, 0.0, 0.0)
    assert tuple(W.descriptors(d, 2, [1, 0])[8:]) == (2.0, 1.0, 0.0)
    assert tuple(W.descriptors(d, 3, [-3, -1, -1])[8:]) == (3.0, 0.0, 1.0)
    # scale-free: the moments of d/<d> do not see the units
    np.testing.assert_allclose(W.descriptors(d * 7.0, 3), W.descriptors(d, 3), rtol=1e-13, atol=1e-15)


def test_targets_and_knots():
    assert W.KNOT_STEPS[0] == 250 and W.KNOT_STEPS[-1] == 45255 and len(W.KNOT_STEPS) == 16
    ph = np.linspace(0.3, 0.64, 3000)
    t = W.targets({"phi_history": ph, "phi": 0.64})
    assert t[0] == 0.64
    assert t[1] == pytest.approx(ph[249] / 0.64)
    assert t[-1] == pytest.approx(ph[-1] / 0.64)  # knots past the run take its last phi


def test_reference_growth_steps():
    assert W.reference_growth_steps(400, 3) == int(6000 + 9 * math.sqrt(1200))
    assert W.reference_growth_steps(100_000, 3) == 10929
    assert W.reference_growth_steps(1, 2) == 6012


class _Fake(W.WarmStart):
    def __init__(self, **kw):  # no network: only the rule
        self.eps = kw.get("eps", 2e-3)
        self.margin = kw.get("margin", 1.5)
        self.min_steps = kw.get("min_steps", 1500)


def test_growth_rule():
    ws = _Fake()
    pred = np.concatenate([[0.64], np.linspace(0.9, 1.0, 16)])
    # first knot at 1 - eps: ratio 0.998 is reached at knot 15 (index of linspace >= 0.998)
    k = int(np.nonzero(np.linspace(0.9, 1.0, 16) >= 1 - 2e-3)[0][0])
    g = ws.growth_steps_from_prediction(pred, 100_000, 3)
    assert g == min(max(int(round(1.5 * W.KNOT_STEPS[k])), 1500), W.reference_growth_steps(100_000, 3))
    # a curve that never reaches 1 - eps keeps the reference's deadline
    assert ws.growth_steps_from_prediction(np.concatenate([[0.6], np.full(16, 0.9)]), 400, 3) == \
        W.reference_growth_steps(400, 3)
    # early saturation is clamped to min_steps
    assert ws.growth_steps_from_prediction(np.concatenate([[0.6], np.ones(16)]), 400, 3) == 1500


class _EchoNet:
    """Stands in for the device network: returns its standardised input."""
    widths = (3, 4, 3)

    def forward(self, Xn):
        return np.asarray(Xn, dtype=np.float32)


def test_inputs_held_inside_the_training_range():
    ws = W.WarmStart(_EchoNet(), np.zeros(3), np.ones(3), np.zeros(3), np.ones(3),
                     x_lo=np.array([0.0, -1.0, 2.0]), x_hi=np.array([1.0, 1.0, 5.0]))
    P = ws.predict(np.array([[0.5, -3.0, 9.0], [2.0, 0.25, 3.0]]))
    np.testing.assert_array_equal(P, [[0.5, -1.0, 5.0], [1.0, 0.25, 3.0]])
    # a model without a recorded range sees the raw inputs
    ws2 = W.WarmStart(_EchoNet(), np.zeros(3), np.ones(3), np.zeros(3), np.ones(3))
    np.testing.assert_array_equal(ws2.predict([[9.0, 9.0, 9.0]]), [[9.0, 9.0, 9.0]])


def test_shipped_model_records_its_training_range():
    z = np.load(W.MODEL_PATH)
    assert "x_lo" in z.files and z["x_lo"].shape == z["x_mean"].shape == z["x_hi"].shape
    assert np.all(z["x_lo"] <= z["x_mean"]) and np.all(z["x_mean"] <= z["x_hi"])
    # log N is the last input: trained on N in [64, 16384]
    assert math.exp(z["x_lo"][-1]) >= 64 - 1e-6 and math.exp(z["x_hi"][-1]) <= 16384 + 1e-6
    assert float(z["margin"]) == 2.0


def test_training_rows_hold_out_the_benchmark_sample():
    from rcpgenerator_b200.train_warmstart import training_rows
    keep = training_rows(np.arange(4096), 8)
    assert keep.sum() == 3584 and not keep[::8].any() and keep[1::8].all()
    assert training_rows(np.arange(5), 0).all()


def test_growth_steps_option_in_the_host_emulation(golden):
    """growth_steps = 1500 ends the rung at step 1501 (mu_flag 1 -> 0), the
    default keeps the reference's deadline; everything before is identical."""
    from tests import hostemu_lib
    g = golden("packs.npz")
    case = "n16_2d"
    H = hostemu_lib.load()
    args = (g[f"{case}/input_positions"], g[f"{case}/input_diameters"], g[f"{case}/box_in"],
            g[f"{case}/walls_in"])
    a = H.run(*args)
    b = H.run(*args, growth_steps=1500)
    fa, fb = a["mu_flag_history"], b["mu_flag_history"]
    assert fb[1499] == 1 and fb[1500] == 0
    dl = W.reference_growth_steps(16, 2)
    assert fa[dl - 1] == 1 and fa[dl] == 0
    np.testing.assert_array_equal(a["phi_history"][:1500], b["phi_history"][:1500])
    assert b["steps"] < a["steps"]
