"""The warm-start network's CPU oracle (oracle/mlp_oracle.py), pinned on the CPU:
its gradient against central finite differences, its BF16 rounding against
torch's float32 -> bfloat16 conversion, and its Adam step against torch.optim.Adam."""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import mlp_oracle as mo  # noqa: E402

WIDTHS = (5, 7, 6, 3)


def _setup(seed=0, B=9):
    rng = np.random.default_rng(seed)
    n = mo.param_count(WIDTHS)
    p = rng.normal(0.0, 0.5, n)
    X = rng.normal(size=(B, WIDTHS[0]))
    T = rng.normal(size=(B, WIDTHS[-1]))
    w = rng.uniform(0.5, 2.0, WIDTHS[-1])
    return p, X, T, w


def test_param_layout():
    n = mo.param_count(WIDTHS)
    assert n == 5 * 7 + 7 + 7 * 6 + 6 + 6 * 3 + 3
    p = np.arange(n, dtype=np.float64)
    (W0, b0), (W1, b1), (W2, b2) = mo.unpack(p, WIDTHS)
    assert W0.shape == (7, 5) and W0[0, 0] == 0 and b0[0] == 35
    assert W1[0, 0] == 42 and b2[-1] == n - 1


@pytest.mark.parametrize("seed", [0, 1])
def test_gradient_matches_finite_differences(seed):
    p, X, T, w = _setup(seed)
    loss, g = mo.loss_and_grad(p, WIDTHS, X, T, w)
    h = 1e-6
    fd = np.empty_like(p)
    for k in range(p.size):
        e = np.zeros_like(p)
        e[k] = h
        fd[k] = (mo.loss_and_grad(p + e, WIDTHS, X, T, w)[0] - mo.loss_and_grad(p - e, WIDTHS, X, T, w)[0]) / (2 * h)
    assert loss > 0
    np.testing.assert_allclose(g, fd, rtol=1e-6, atol=1e-9)


def test_bf16_round_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.normal(size=4096) * 10.0 ** rng.integers(-20, 20, 4096),
                        [0.0, -0.0, 1.0, 1.00390625, 1.01171875, 3.0e38, -1e-40]]).astype(np.float32)
    ref = torch.from_numpy(x).to(torch.bfloat16).to(torch.float64).numpy()
    np.testing.assert_array_equal(mo.bf16_round(x), ref)


def test_adam_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(4)
    p0 = rng.normal(size=20)
    grads = [rng.normal(size=20) for _ in range(5)]
    t = torch.tensor(p0.copy(), dtype=torch.float64, requires_grad=True)
    opt = torch.optim.Adam([t], lr=1e-2, betas=(0.9, 0.999), eps=1e-8)
    p, m, v = p0.copy(), np.zeros(20), np.zeros(20)
    for s, g in enumerate(grads, 1):
        opt.zero_grad()
        t.grad = torch.tensor(g)
        opt.step()
        p, m, v = mo.adam(p, m, v, g, 1e-2, s)
    np.testing.assert_allclose(p, t.detach().numpy(), rtol=1e-12, atol=1e-14)


def test_bf16_emulation_is_close_to_fp64():
    p, X, T, w = _setup(5, B=64)
    _, g64 = mo.loss_and_grad(p, WIDTHS, X, T, w)
    _, g16 = mo.loss_and_grad(p, WIDTHS, X, T, w, bf16=True)
    assert np.linalg.norm(g16 - g64) / np.linalg.norm(g64) < 3e-2


def test_mlp_abi_sizes_on_the_host():
    """Parameter count and workspace size of the C ABI (host functions) agree
    with the oracle's layout; invalid widths give 0."""
    import ctypes as C
    from rcpgenerator_b200 import _native as N
    w = (C.c_int32 * 5)(11, 256, 256, 256, 17)
    assert N.lib.rcpg_mlp_param_count(w, 4) == mo.param_count((11, 256, 256, 256, 17)) == 139025
    ws = N.lib.rcpg_mlp_workspace_bytes(w, 4, 256)
    # activations (BF16) + pre-activations (FP32) + gradient scratch + loss terms
    need = 256 * (2 * (11 + 3 * 256 + 17) + 4 * (3 * 256 + 17) + 8 * 256 + 4 * 17)
    assert need <= ws <= need + 256 * 16
    assert N.lib.rcpg_mlp_param_count((C.c_int32 * 3)(4, 0, 2), 2) == 0
    assert N.lib.rcpg_mlp_workspace_bytes(w, 4, 0) == 0
