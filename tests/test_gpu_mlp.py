"""The warm-start network's CUDA kernels (csrc/rcpg_mlp.cu, through the C ABI)
against the CPU oracle oracle/mlp_oracle.py, which rounds to BF16 exactly
where the kernels store BF16 and computes in FP64 otherwise. The remaining
differences come from the tensor cores' FP32 accumulation (their summation
order and internal alignment, about 1e-6 relative on a pre-activation) and
from the BF16 roundings those differences flip (2^-8 relative each, on about
one stored value in a thousand), which compound over the three hidden
layers: relative tolerances of 1e-3 on the output and 5e-3 on each layer's
gradient norm."""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import mlp_oracle as mo  # noqa: E402

pytestmark = pytest.mark.gpu

WIDTHS = (11, 256, 256, 256, 17)


def _net(seed=0, widths=WIDTHS):
    from rcpgenerator_b200.warmstart import Network
    return Network(widths=widths, seed=seed)


def _data(seed, B, widths=WIDTHS):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(B, widths[0])).astype(np.float32)
    T = rng.normal(size=(B, widths[-1])).astype(np.float32)
    w = rng.uniform(0.5, 4.0, widths[-1]).astype(np.float32)
    return X, T, w


def _blocks(v, widths):
    out, off = [], 0
    for l in range(len(widths) - 1):
        n = widths[l + 1] * widths[l] + widths[l + 1]
        out.append(v[off:off + n])
        off += n
    return out


@pytest.mark.parametrize("B", [1, 37, 256])
def test_forward_matches_oracle(cuda_device, B):
    net = _net(1)
    X, _, _ = _data(2, B)
    Y = net.forward(X)
    Yo, _, _ = mo.forward(net.params(), WIDTHS, X, bf16=True)
    assert Y.shape == (B, WIDTHS[-1])
    assert np.linalg.norm(Y - Yo) <= 1e-3 * np.linalg.norm(Yo)


@pytest.mark.parametrize("K,O,B", [(11, 17, 5), (256, 256, 70), (100, 3, 129)])
def test_tensor_core_gemm_exact_on_small_integers(cuda_device, K, O, B):
    """A one-layer network (no activation) on small integers: every product
    and partial sum is exact in BF16 / FP32, so the forward GEMM, the weight
    gradient GEMM and the bias gradient must match NumPy exactly; this pins
    the fragment layout of the tensor-core tiles and the tile edges."""
    from rcpgenerator_b200.warmstart import Network
    rng = np.random.default_rng(K * 1000 + O + B)
    W = rng.integers(-3, 4, size=(O, K)).astype(np.float64)
    X = rng.integers(-3, 4, size=(B, K)).astype(np.float32)
    net = Network(widths=(K, O), params=np.concatenate([W.ravel(), np.zeros(O)]))
    Y = net.forward(X)
    np.testing.assert_array_equal(Y, X.astype(np.float64) @ W.T)
    # dL/dz = 2 (Y - T) / (B O) with (Y - T) small integers and B O a power of two
    Bp, Op = 32, 16
    W2 = rng.integers(-3, 4, size=(Op, K)).astype(np.float64)
    X2 = rng.integers(-3, 4, size=(Bp, K)).astype(np.float32)
    d = rng.integers(-3, 4, size=(Bp, Op)).astype(np.float64)
    T2 = (X2.astype(np.float64) @ W2.T - d).astype(np.float32)
    net2 = Network(widths=(K, Op), params=np.concatenate([W2.ravel(), np.zeros(Op)]))
    net2.train_step(X2, T2, 0.0, update=False)
    g = net2.grad.cpu().numpy().astype(np.float64)
    dz = 2.0 * d / (Bp * Op)
    np.testing.assert_array_equal(g[:Op * K].reshape(Op, K), dz.T @ X2.astype(np.float64))
    np.testing.assert_array_equal(g[Op * K:], dz.sum(axis=0))


@pytest.mark.parametrize("widths,B", [(WIDTHS, 64), ((5, 19, 33, 3), 45), ((11, 256, 17), 300)])
def test_gradient_matches_oracle(cuda_device, widths, B):
    net = _net(3, widths)
    X, T, w = _data(4, B, widths)
    loss = float(net.train_step(X, T, 0.0, w, update=False))
    g = net.grad.cpu().numpy().astype(np.float64)
    lo, go = mo.loss_and_grad(net.params(), widths, X, T, w, bf16=True)
    assert abs(loss - lo) <= 1e-4 * lo
    for gb, ob in zip(_blocks(g, widths), _blocks(go, widths)):
        assert np.linalg.norm(gb - ob) <= 5e-3 * np.linalg.norm(ob) + 1e-12


def test_adam_step_matches_oracle(cuda_device):
    net = _net(5)
    X, T, w = _data(6, 64)
    p0 = net.params()
    m = np.zeros_like(p0)
    v = np.zeros_like(p0)
    p = p0.copy()
    for s in range(1, 4):
        _, g = mo.loss_and_grad(net.params(), WIDTHS, X, T, w, bf16=True)
        net.train_step(X, T, 1e-3, w)
        p, m, v = mo.adam(p, m, v, net.grad.cpu().numpy().astype(np.float64), 1e-3, s)
        # the kernel's update of the FP32 master copy, from its own gradient
        assert np.abs(net.params() - p).max() <= 1e-6 * np.abs(p).max()
        # and its gradient from the oracle's
        gk = net.grad.cpu().numpy().astype(np.float64)
        assert np.linalg.norm(gk - g) <= 5e-3 * np.linalg.norm(g)
        p = net.params()
    # the BF16 copy is the rounded master copy
    w16 = net.w16.float().cpu().numpy().astype(np.float64)
    np.testing.assert_array_equal(w16, mo.bf16_round(net.params()))


def test_training_fits_a_smooth_map(cuda_device):
    """Adam on the kernels fits y = sin(x . a) (17 outputs) well below the
    variance of the targets."""
    from rcpgenerator_b200.warmstart import WarmStart
    rng = np.random.default_rng(7)
    X = rng.normal(size=(2048, 11))
    A = rng.normal(size=(11, 17)) * 0.3
    Y = np.sin(X @ A) + 0.1 * (X[:, :1] ** 2)
    ws = WarmStart.fit(X, Y, epochs=60, batch=256, lr=2e-3, seed=1, phi_weight=1.0)
    loss = ws.meta["train_loss"]
    assert loss[-1] < 0.05 * loss[0]
    P = ws.predict(X[:256])
    assert np.mean((P - Y[:256]) ** 2) < 0.05 * np.var(Y)


def test_errors_are_loud(cuda_device):
    from rcpgenerator_b200 import _native as N
    import ctypes as C
    w = (C.c_int32 * 3)(4, 8, 2)
    err = N.errbuf()
    rc = N.lib.rcpg_mlp_forward(w, 2, 4, None, None, None, None, None, 0, None, err, len(err))
    assert rc == N.RCPG_EINVAL and b"bad arguments" in err.value
