"""CPU oracle of the learned warm start's network -- TEST INFRASTRUCTURE ONLY.

The warm-start MLP has no counterpart in the reference (its Packing API has no
learned component), so this file is the checker written for this project: a
NumPy FP64 restatement of the CUDA kernels in rcpgenerator_b200/csrc/rcpg_mlp.cu
(forward, mean-squared-error loss, backward, Adam). It is pinned by finite
differences (tests/test_mlp_oracle.py), not by reference outputs.

With ``bf16=True`` it rounds what the kernels store in BF16 (weights, the
input, every activation and every pre-activation gradient) to BF16, round to
nearest even, and keeps everything else in FP64, so the CUDA gradients differ
from it only by FP32 accumulation order and the rare BF16 tie that order flips.

Parameter layout (shared with the kernels): for layer l, W_l [w[l+1] x w[l]]
row-major, then b_l [w[l+1]], concatenated over the layers.
"""

from __future__ import annotations

import math

import numpy as np

_erf = np.vectorize(math.erf, otypes=[np.float64])


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.ascontiguousarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    nan = np.isnan(f)
    out = r.astype(np.uint32).view(np.float32).astype(np.float64)
    out[nan] = np.nan
    return out


def param_count(widths) -> int:
    return int(sum(widths[l + 1] * widths[l] + widths[l + 1] for l in range(len(widths) - 1)))


def unpack(params: np.ndarray, widths):
    """[(W_l, b_l)] views of the packed parameter vector."""
    out, off = [], 0
    for l in range(len(widths) - 1):
        i, o = widths[l], widths[l + 1]
        W = params[off:off + o * i].reshape(o, i)
        off += o * i
        b = params[off:off + o]
        off += o
        out.append((W, b))
    return out


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def forward(params, widths, X, bf16=False):
    """Returns (Y, acts, zs): acts[l] is layer l's input, zs[l] its pre-activation."""
    rnd = bf16_round if bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    layers = unpack(np.asarray(params, dtype=np.float64), widths)
    a = rnd(X)
    acts, zs = [a], []
    for l, (W, b) in enumerate(layers):
        z = a @ rnd(W).T + b
        zs.append(z)
        a = rnd(gelu(z)) if l + 1 < len(layers) else z
        acts.append(a)
    return zs[-1], acts, zs


def loss_and_grad(params, widths, X, T, out_weight=None, bf16=False):
    """MSE loss sum(w (Y - T)^2) / (B * O) and its gradient w.r.t. the packed
    parameters, as rcpg_mlp_train_step computes them."""
    rnd = bf16_round if bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    params = np.asarray(params, dtype=np.float64)
    Y, acts, zs = forward(params, widths, X, bf16)
    B, O = Y.shape
    w = np.ones(O) if out_weight is None else np.asarray(out_weight, dtype=np.float64)
    d = Y - np.asarray(T, dtype=np.float64)
    loss = float((w * d * d).sum() / (B * O))
    dz = rnd(2.0 * w * d / (B * O))
    layers = unpack(params, widths)
    grads = []
    for l in range(len(layers) - 1, -1, -1):
        W, _ = layers[l]
        gW = dz.T @ acts[l]
        gb = dz.sum(axis=0)
        grads.append(np.concatenate([gW.ravel(), gb]))
        if l > 0:
            da = dz @ rnd(W)
            dz = rnd(da * gelu_grad(zs[l - 1]))
    return loss, np.concatenate(grads[::-1])


def adam(params, m, v, g, lr, step, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update (the kernel's formula), FP64; returns new (params, m, v)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    c1 = 1 - b1 ** step
    c2 = 1 - b2 ** step
    return params - lr * (m / c1) / (np.sqrt(v / c2) + eps), m, v
