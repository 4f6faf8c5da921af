"""Learned warm start of the packing engine (no counterpart in the reference).

A small network maps a packing's size-distribution descriptors to its
predicted jamming fraction phi_J and its growth curve, and the warm start
shortens the growth rung of the reference's schedule (mu_flag = 1, the first
6000 + 9 sqrt(N ndim) steps, rcp_generator.cpp:5834-5931) to the step at which
the predicted curve has reached phi_J. The rest of the run -- mu decay,
oscillation, and the unchanged overlap / force convergence gate -- is the
plain method's, so every warm-started packing still ends by the engine's
own criterion; the time saved is in the rung, whose length also sets the
oscillation period that follows it.

Network: inputs are the first 8 moments of d/<d> (as log(m_k)/k), Ndim, a
hard-wall flag, a container flag and log N (12 values, standardised; a model
trained without log N takes the first 11); 3 hidden layers
of 256 GELU units; 17 outputs: phi_J and the growth curve phi(t_k)/phi_J at 16
knots t_k = 250 * 2^(k/2) steps (k = 0..15, 250 to 45,255 steps). Weights are
BF16 with FP32 master copies and FP32 accumulation; training and inference run
on the GPU in the kernels of csrc/rcpg_mlp.cu through the C ABI
(rcpg_mlp_forward / rcpg_mlp_train_step). PyTorch holds the device memory.

Training data: packings run by the batch engine from the plain method, drawn
like the batched workload (N log-uniform, Ndim in {2, 3, 4}, mono / bidisperse
/ log-normal diameters, periodic boxes at phi 0.10).
"""

from __future__ import annotations

import ctypes as C
import math
from pathlib import Path
from typing import Any

import numpy as np

from . import _native as N
from ._api import initialize_particles, run_packing_batch

WIDTHS = (12, 256, 256, 256, 17)
KNOT_STEPS = np.round(250.0 * 2.0 ** (np.arange(16) / 2.0)).astype(np.int64)
N_FEATURES = WIDTHS[0]
MODEL_PATH = Path(__file__).resolve().parent / "warmstart_model.npz"


# ---- descriptors and targets ---------------------------------------------------

def descriptors(diameters, ndim: int, walls=(), with_n: bool = False) -> np.ndarray:
    """The network's raw inputs for one packing: log(m_k)/k for the moments
    m_k = <(d/<d>)^k>, k = 1..8; Ndim; 1.0 if any hard wall (walls[k] > 0);
    1.0 if a container (walls[0] < 0); with ``with_n`` also log N (12 values,
    else 11)."""
    d = np.asarray(diameters, dtype=np.float64)
    r = d / d.mean()
    mom = [math.log(float(np.mean(r ** k))) / k for k in range(1, 9)]
    w = np.asarray(walls, dtype=np.int64).ravel()
    hard = float(np.any(w > 0)) if w.size else 0.0
    cont = float(w[0] < 0) if w.size else 0.0
    extra = [math.log(float(d.size))] if with_n else []
    return np.asarray(mom + [float(ndim), hard, cont] + extra, dtype=np.float64)


def reference_growth_steps(N: int, ndim: int) -> int:
    """The reference's growth-rung deadline max(1500, 6000 + 9 sqrt(N ndim))
    (rcp_generator.cpp:4713-4737)."""
    return int(max(1500.0, 2.0 * 4000.0 + 9.0 * math.sqrt(float(N) * float(ndim)) - 2000.0))


def targets(result: dict) -> np.ndarray:
    """17 training targets of a finished plain packing: phi_J (the final phi)
    and phi(t_k) / phi_J at the knots (the last phi where the run ended
    earlier)."""
    ph = np.asarray(result["phi_history"], dtype=np.float64)
    phi_j = float(result["phi"])
    idx = np.minimum(KNOT_STEPS, len(ph)) - 1
    return np.concatenate([[phi_j], ph[idx] / phi_j])


# ---- the network on the device ----------------------------------------------------

def _torch():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("rcpgenerator_b200.warmstart: the network runs on CUDA only (no CPU path)")
    return torch


class Network:
    """The MLP's parameters on the GPU and its kernels' entry points."""

    def __init__(self, widths=WIDTHS, seed: int = 0, device: int = 0, params: np.ndarray | None = None):
        torch = _torch()
        self.widths = tuple(int(w) for w in widths)
        self.layers = len(self.widths) - 1
        self._w = (C.c_int32 * len(self.widths))(*self.widths)
        self.device = torch.device("cuda", device)
        n = int(N.lib.rcpg_mlp_param_count(self._w, self.layers))
        if params is None:
            rng = np.random.default_rng(seed)
            parts = []
            for l in range(self.layers):
                i, o = self.widths[l], self.widths[l + 1]
                parts.append(rng.normal(0.0, math.sqrt(2.0 / i), o * i))
                parts.append(np.zeros(o))
            params = np.concatenate(parts)
        params = np.asarray(params, dtype=np.float32)
        if params.size != n:
            raise ValueError(f"expected {n} parameters, got {params.size}")
        self.w32 = torch.from_numpy(params.copy()).to(self.device)
        self.w16 = torch.empty(n, dtype=torch.bfloat16, device=self.device)
        self.m = torch.zeros(n, dtype=torch.float32, device=self.device)
        self.v = torch.zeros(n, dtype=torch.float32, device=self.device)
        self.grad = torch.zeros(n, dtype=torch.float32, device=self.device)
        self.step = 0
        self._ws = None
        self._ws_batch = 0
        self._sync_bf16()

    @property
    def n_params(self) -> int:
        return int(self.w32.numel())

    def _stream(self):
        torch = _torch()
        return C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def _sync_bf16(self) -> None:
        rc = N.lib.rcpg_mlp_to_bf16(self.n_params, C.c_void_p(self.w32.data_ptr()),
                                    C.c_void_p(self.w16.data_ptr()), self._stream())
        if rc != N.RCPG_OK:
            raise N.NativeError(rc, "rcpgenerator_b200: rcpg_mlp_to_bf16 failed")

    def _workspace(self, batch: int):
        torch = _torch()
        if self._ws is None or batch > self._ws_batch:
            nb = int(N.lib.rcpg_mlp_workspace_bytes(self._w, self.layers, batch))
            self._ws = torch.empty(nb, dtype=torch.uint8, device=self.device)
            self._ws_batch = batch
        return self._ws

    def _dev(self, a):
        torch = _torch()
        if isinstance(a, torch.Tensor):
            return a.to(device=self.device, dtype=torch.float32).contiguous()
        return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(self.device)

    def forward(self, X) -> np.ndarray:
        torch = _torch()
        X = self._dev(X)
        B = int(X.shape[0])
        Y = torch.empty((B, self.widths[-1]), dtype=torch.float32, device=self.device)
        ws = self._workspace(B)
        err = N.errbuf()
        rc = N.lib.rcpg_mlp_forward(self._w, self.layers, B, C.c_void_p(self.w16.data_ptr()),
                                    C.c_void_p(self.w32.data_ptr()), C.c_void_p(X.data_ptr()),
                                    C.c_void_p(Y.data_ptr()), C.c_void_p(ws.data_ptr()), ws.numel(),
                                    self._stream(), err, len(err))
        N.raise_for(rc, err)
        return Y.cpu().numpy()

    def train_step(self, X, T, lr: float, out_weight=None, update: bool = True):
        """One step of the MSE loss; returns the loss (a device scalar) and
        leaves dL/dparams in ``self.grad``. ``update`` False computes the
        gradient only."""
        torch = _torch()
        X, T = self._dev(X), self._dev(T)
        B = int(X.shape[0])
        ow = None if out_weight is None else self._dev(out_weight)
        terms = torch.empty((B, self.widths[-1]), dtype=torch.float32, device=self.device)
        ws = self._workspace(B)
        if update:
            self.step += 1
        err = N.errbuf()
        rc = N.lib.rcpg_mlp_train_step(
            self._w, self.layers, B, C.c_void_p(self.w32.data_ptr()), C.c_void_p(self.w16.data_ptr()),
            C.c_void_p(self.m.data_ptr()) if update else None,
            C.c_void_p(self.v.data_ptr()) if update else None,
            C.c_void_p(self.grad.data_ptr()), C.c_void_p(X.data_ptr()), C.c_void_p(T.data_ptr()),
            C.c_void_p(ow.data_ptr()) if ow is not None else None, float(lr if update else 0.0),
            max(self.step, 1), C.c_void_p(terms.data_ptr()), C.c_void_p(ws.data_ptr()), ws.numel(),
            self._stream(), err, len(err))
        N.raise_for(rc, err)
        return terms.sum() / terms.numel()

    def params(self) -> np.ndarray:
        return self.w32.cpu().numpy().astype(np.float64)


# ---- the warm start ----------------------------------------------------------------

class WarmStart:
    """Trained network + the rule that turns its prediction into a growth-rung
    length: the first knot at which the predicted phi(t)/phi_J reaches
    1 - ``eps``, times ``margin``, kept within [``min_steps``, the reference's
    deadline]. Inputs are held inside the range of the training set
    (``x_lo``, ``x_hi``) before the network sees them: a packing larger than
    any trained on is predicted as the largest trained size, instead of by
    extrapolating the network in log N."""

    def __init__(self, net: Network, x_mean, x_std, y_mean, y_std, eps: float = 2e-3,
                 margin: float = 2.0, min_steps: int = 1500, meta: dict | None = None,
                 x_lo=None, x_hi=None):
        self.net = net
        self.x_mean = np.asarray(x_mean, dtype=np.float64)
        self.x_std = np.asarray(x_std, dtype=np.float64)
        self.x_lo = None if x_lo is None else np.asarray(x_lo, dtype=np.float64)
        self.x_hi = None if x_hi is None else np.asarray(x_hi, dtype=np.float64)
        self.y_mean = np.asarray(y_mean, dtype=np.float64)
        self.y_std = np.asarray(y_std, dtype=np.float64)
        self.eps = float(eps)
        self.margin = float(margin)
        self.min_steps = int(min_steps)
        self.meta = dict(meta or {})

    # training
    @classmethod
    def fit(cls, X, Y, epochs: int = 400, batch: int = 256, lr: float = 1e-3, seed: int = 0,
            device: int = 0, phi_weight: float = 4.0, **kw) -> "WarmStart":
        """Trains a fresh network on raw descriptors X [n x 11] and targets
        Y [n x 17] with the GPU kernels (Adam, cosine learning rate)."""
        X = np.asarray(X, dtype=np.float64)
        Y = np.asarray(Y, dtype=np.float64)
        xm, xs = X.mean(0), X.std(0)
        xs = np.where(xs > 1e-9, xs, 1.0)
        ym, ys = Y.mean(0), Y.std(0)
        ys = np.where(ys > 1e-9, ys, 1.0)
        net = Network(widths=(X.shape[1],) + tuple(WIDTHS[1:]), seed=seed, device=device)
        Xn = net._dev((X - xm) / xs)
        Yn = net._dev((Y - ym) / ys)
        ow = np.ones(Y.shape[1])
        ow[0] = phi_weight
        ow = net._dev(ow)
        rng = np.random.default_rng(seed)
        n = X.shape[0]
        bs = min(batch, n)
        per_epoch = max(1, n // bs)
        total = epochs * per_epoch
        losses = []
        torch = _torch()
        for e in range(epochs):
            perm = torch.from_numpy(rng.permutation(n)).to(net.device)
            acc = None
            for b in range(per_epoch):
                idx = perm[b * bs:(b + 1) * bs]
                t = net.step / max(total - 1, 1)
                lr_t = lr * 0.5 * (1.0 + math.cos(math.pi * min(t, 1.0)))
                loss = net.train_step(Xn[idx], Yn[idx], max(lr_t, 1e-6), ow)
                acc = loss if acc is None else acc + loss
            losses.append(float(acc) / per_epoch)
        ws = cls(net, xm, xs, ym, ys, x_lo=X.min(0), x_hi=X.max(0), **kw)
        ws.meta.update(train_loss=losses, n_train=int(n), epochs=int(epochs), batch=int(bs), lr=float(lr))
        return ws

    # inference
    def predict(self, X) -> np.ndarray:
        """Raw descriptors [n x 11] -> [n x 17] (phi_J, 16 knot ratios)."""
        X = np.atleast_2d(np.asarray(X, dtype=np.float64))
        if self.x_lo is not None:
            X = np.clip(X, self.x_lo, self.x_hi)
        Yn = self.net.forward((X - self.x_mean) / self.x_std)
        return Yn.astype(np.float64) * self.y_std + self.y_mean

    def growth_steps_from_prediction(self, pred: np.ndarray, N: int, ndim: int) -> int:
        ref = reference_growth_steps(N, ndim)
        ratios = np.asarray(pred[1:17])
        hit = np.nonzero(ratios >= 1.0 - self.eps)[0]
        if hit.size == 0:
            return ref
        g = int(round(self.margin * float(KNOT_STEPS[hit[0]])))
        return int(min(max(g, self.min_steps), ref))

    def plan(self, items: list) -> tuple[np.ndarray, np.ndarray]:
        """For [(input, config), ...]: predicted phi_J and growth-rung lengths."""
        with_n = self.net.widths[0] > 11
        X = np.stack([descriptors(inp["diameters"], np.asarray(inp["positions"]).shape[1],
                                  cfg.get("walls", []), with_n) for inp, cfg in items])
        P = self.predict(X)
        gs = np.asarray([self.growth_steps_from_prediction(P[k], len(items[k][0]["diameters"]),
                                                           np.asarray(items[k][0]["positions"]).shape[1])
                         for k in range(len(items))], dtype=np.uint64)
        return P[:, 0], gs

    def options(self, input: dict, config: dict) -> dict:
        """Run options of a warm-started run_packing_observed call."""
        _, gs = self.plan([(input, config)])
        return {"growth_steps": int(gs[0])}

    def run_batch(self, items: list, options: dict | None = None, concurrency: int = 0) -> tuple[list, np.ndarray]:
        """run_packing_batch with each packing's growth rung set by the
        network; returns (results, predicted phi_J)."""
        phi_pred, gs = self.plan(items)
        return run_packing_batch(items, options, concurrency, growth_steps=gs), phi_pred

    # persistence
    def save(self, path) -> None:
        np.savez_compressed(
            path, params=self.net.params().astype(np.float32), widths=np.asarray(self.net.widths),
            x_mean=self.x_mean, x_std=self.x_std, y_mean=self.y_mean, y_std=self.y_std,
            **({} if self.x_lo is None else {"x_lo": self.x_lo, "x_hi": self.x_hi}),
            eps=self.eps, margin=self.margin, min_steps=self.min_steps,
            meta=np.asarray(repr({k: v for k, v in self.meta.items() if k != "train_loss"})))

    @classmethod
    def load(cls, path=MODEL_PATH, device: int = 0) -> "WarmStart":
        z = np.load(path, allow_pickle=False)
        net = Network(widths=tuple(z["widths"].tolist()), device=device, params=z["params"])
        lo_hi = {"x_lo": z["x_lo"], "x_hi": z["x_hi"]} if "x_lo" in z.files else {}
        return cls(net, z["x_mean"], z["x_std"], z["y_mean"], z["y_std"], float(z["eps"]),
                   float(z["margin"]), int(z["min_steps"]), {"saved": str(z["meta"])}, **lo_hi)


# ---- data --------------------------------------------------------------------------

def draw_packing(seed: int, n_range=(64, 16384), ndims=(2, 3, 4), phi: float = 0.10) -> tuple[dict, dict]:
    """One packing drawn like the batched workload: N log-uniform on n_range,
    ndim from ndims, diameters mono (d=1), bidisperse 50:50 with ratio uniform
    on [1.1, 3.0], or log-normal with std/mean uniform on [0.1, 0.6] truncated
    to [0.2, 5] x mean; periodic unit box at initial phi ``phi``."""
    rng = np.random.default_rng(seed)
    n = int(round(math.exp(rng.uniform(math.log(n_range[0]), math.log(n_range[1])))))
    nd = int(rng.choice(list(ndims)))
    kind = int(rng.integers(3))
    if kind == 0:
        dist: dict[str, Any] = {"type": "mono", "d": 1.0}
    elif kind == 1:
        dist = {"type": "bidisperse", "d1": 1.0, "d2": float(rng.uniform(1.1, 3.0)), "p": 0.5}
    else:
        cv = rng.uniform(0.1, 0.6)
        s2 = math.log1p(cv * cv)
        d = rng.lognormal(-0.5 * s2, math.sqrt(s2), size=4 * n)
        d = d[(d >= 0.2) & (d <= 5.0)][:n]
        dist = {"type": "custom", "custom": d.tolist()}
    init = initialize_particles({"phi": phi, "N": n, "Ndim": nd, "box": [1.0] * nd,
                                 "walls": [0] * nd, "dist": dist, "seed": seed})
    return ({"positions": np.asarray(init["positions"]), "diameters": np.asarray(init["diameters"])},
            {"box": init["box"], "walls": init["walls"], "neighbor_max": 0, "seed": seed})


def draw_evaluation_packing(seed: int, N: int = 100_000, phi: float = 0.10) -> tuple[dict, dict]:
    """A held-out 3-D packing: bidisperse 50:50 with ratio uniform on [1.1, 3.0]
    or log-normal with std/mean uniform on [0.1, 0.6] (truncated to [0.2, 5] x
    mean), periodic unit box at initial phi ``phi``."""
    rng = np.random.default_rng(10_000_000 + seed)
    if rng.integers(2) == 0:
        dist: dict[str, Any] = {"type": "bidisperse", "d1": 1.0, "d2": float(rng.uniform(1.1, 3.0)), "p": 0.5}
    else:
        cv = rng.uniform(0.1, 0.6)
        s2 = math.log1p(cv * cv)
        d = rng.lognormal(-0.5 * s2, math.sqrt(s2), size=4 * N)
        d = d[(d >= 0.2) & (d <= 5.0)][:N]
        dist = {"type": "custom", "custom": d.tolist()}
    init = initialize_particles({"phi": phi, "N": N, "Ndim": 3, "box": [1.0] * 3,
                                 "walls": [0] * 3, "dist": dist, "seed": seed})
    return ({"positions": np.asarray(init["positions"]), "diameters": np.asarray(init["diameters"])},
            {"box": init["box"], "walls": init["walls"], "neighbor_max": 0, "seed": seed})


def generate_training_set(count: int, seed0: int = 0, n_range=(64, 16384), options: dict | None = None,
                          concurrency: int = 0, chunk: int = 1024) -> tuple[np.ndarray, np.ndarray]:
    """Runs ``count`` plain packings (draw_packing, seeds seed0..) in the batch
    engine and returns their descriptors X [count x 12] (with log N) and
    targets Y [count x 17]."""
    X, Y = [], []
    for s0 in range(seed0, seed0 + count, chunk):
        items = [draw_packing(s, n_range) for s in range(s0, min(s0 + chunk, seed0 + count))]
        res = run_packing_batch(items, options, concurrency)
        for (inp, cfg), r in zip(items, res):
            X.append(descriptors(inp["diameters"], np.asarray(inp["positions"]).shape[1], cfg["walls"], True))
            Y.append(targets(r))
    return np.asarray(X), np.asarray(Y)


def evaluate(ws: WarmStart, items: list, options: dict | None = None, concurrency: int = 0,
             plain_options: dict | None = None, plain: tuple | None = None) -> dict:
    """Runs ``items`` plain and warm-started (same seeds, same batch call
    shape) and compares: packings/hour of each (host wall clock around the
    batch call), steps, phi_J per packing, and the network's phi_J error.
    ``plain_options`` (default: ``options``) are the plain runs' options, e.g.
    FP64 pair arithmetic for the plain method against mixed-precision
    warm-started runs. ``plain``: (results, seconds) of the plain runs of an
    earlier evaluate() of the same items (its "plain_runs" entry), reused
    instead of running them again."""
    import time

    plain_opts = options if plain_options is None else plain_options
    if plain is None:
        t0 = time.perf_counter()
        plain_res = run_packing_batch(items, plain_opts, concurrency)
        plain_s = time.perf_counter() - t0
    else:
        plain_res, plain_s = plain
    t1 = time.perf_counter()
    warm, phi_pred = ws.run_batch(items, options, concurrency)
    warm_s = time.perf_counter() - t1
    plain = plain_res
    _, gs = ws.plan(items)
    pj = np.asarray([r["phi"] for r in plain])
    wj = np.asarray([r["phi"] for r in warm])
    ps = np.asarray([r["steps"] for r in plain], dtype=np.float64)
    wsteps = np.asarray([r["steps"] for r in warm], dtype=np.float64)
    n = len(items)
    return {
        "packings": n,
        "plain_packings_per_hour": n / plain_s * 3600.0,
        "warm_packings_per_hour": n / warm_s * 3600.0,
        "plain_mean_steps": float(ps.mean()),
        "warm_mean_steps": float(wsteps.mean()),
        "growth_steps_mean": float(np.mean(gs)),
        "reference_growth_steps_mean": float(np.mean([reference_growth_steps(len(i["diameters"]),
                                                                             np.asarray(i["positions"]).shape[1])
                                                      for i, _ in items])),
        "phi_plain_mean": float(pj.mean()),
        "phi_warm_mean": float(wj.mean()),
        "delta_phi_mean": float(wj.mean() - pj.mean()),
        "delta_phi_abs_mean": float(np.abs(wj - pj).mean()),
        "phi_pred_mae": float(np.abs(phi_pred - pj).mean()),
        "phi_pred_bias": float((phi_pred - pj).mean()),
        "delta_phi_abs_max": float(np.abs(wj - pj).max()),
        "max_overlap_warm": float(max(r["max_min_dist"] for r in warm)),
        "max_overlap_plain": float(max(r["max_min_dist"] for r in plain)),
        "plain_pair_precision": str((plain_opts or {}).get("pair_precision", "f64")),
        "warm_pair_precision": str((options or {}).get("pair_precision", "f64")),
        "margin": float(ws.margin),
        "plain_runs": (plain, plain_s),  # for further evaluations of the same items
    }
