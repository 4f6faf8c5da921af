"""Trains the learned warm start on the GPU and writes the model file.

    python -m rcpgenerator_b200.train_warmstart --count 4096 --out rcpgenerator_b200/warmstart_model.npz

Generates ``count`` plain packings with the batch engine (draw_packing: N
log-uniform on [--n-min, --n-max], Ndim in {2, 3, 4}, mono / bidisperse /
log-normal diameters) or takes them from ``--data`` (for instance the plain
runs of ``bench.py --workload batch --save-training``, leaving out every
``--exclude-stride``-th seed), trains the network with the project's BF16 kernels,
evaluates it on held-out packings (draw_evaluation_packing: 3-D, N = --eval-n)
plain against warm-started, and prints one JSON line with the figures.
"""

from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import warmstart as W


def training_rows(seeds, stride: int) -> np.ndarray:
    """Rows of a saved training set that train the network: every packing
    whose seed is not a multiple of ``stride`` (those are the batch
    benchmark's sample, held out); all rows when ``stride`` <= 0."""
    seeds = np.asarray(seeds, dtype=np.int64)
    return np.ones(seeds.shape, dtype=bool) if stride <= 0 else (seeds % stride) != 0


def main(argv=None) -> dict:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--count", type=int, default=4096)
    ap.add_argument("--seed0", type=int, default=0)
    ap.add_argument("--n-min", type=int, default=64)
    ap.add_argument("--n-max", type=int, default=16384)
    ap.add_argument("--epochs", type=int, default=300)
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--eps", type=float, default=2e-3)
    ap.add_argument("--margin", type=float, default=2.0)
    ap.add_argument("--pair-precision", default="mixed", choices=("f64", "mixed"))
    ap.add_argument("--data", default=None, help="reuse a saved training set (.npz with X, Y)")
    ap.add_argument("--save-data", default=None)
    ap.add_argument("--out", default=str(W.MODEL_PATH))
    ap.add_argument("--eval-count", type=int, default=16)
    ap.add_argument("--eval-n", type=int, default=100_000)
    ap.add_argument("--eval-seed0", type=int, default=0, help="first seed of the held-out evaluation packings")
    ap.add_argument("--eval-concurrency", type=int, default=8)
    ap.add_argument("--eval-margins", default="", help="extra comma-separated margins to evaluate")
    ap.add_argument("--eval-plain-precision", default=None, choices=("f64", "mixed"),
                    help="pair precision of the evaluation's plain runs (default: --pair-precision)")
    ap.add_argument("--exclude-stride", type=int, default=0,
                    help="with --data holding seeds: leave out of training every packing whose seed is a "
                         "multiple of this stride (held out for the batch benchmark's sample)")
    ap.add_argument("--eval-only", action="store_true", help="evaluate the model file --out without training")
    a = ap.parse_args(argv)
    opts = {"pair_precision": a.pair_precision}
    plain_opts = {"pair_precision": a.eval_plain_precision or a.pair_precision}
    if a.eval_only:
        ws = W.WarmStart.load(a.out)
        items = [W.draw_evaluation_packing(s, a.eval_n) for s in range(a.eval_seed0, a.eval_seed0 + a.eval_count)]
        ev = W.evaluate(ws, items, opts, a.eval_concurrency, plain_opts)
        plain_runs = ev.pop("plain_runs")
        out = {"model": str(a.out), "eval": ev}
        out["eval"]["N"] = a.eval_n
        # other rung margins on the same plain runs
        for m in [float(x) for x in a.eval_margins.split(",") if x]:
            ws.margin = m
            e2 = W.evaluate(ws, items, opts, a.eval_concurrency, plain_opts, plain=plain_runs)
            e2.pop("plain_runs")
            out[f"eval_margin_{m:g}"] = e2
        print(json.dumps(out))
        return out
    t0 = time.perf_counter()
    held = 0
    if a.data:
        z = np.load(a.data)
        X, Y = z["X"], z["Y"]
        if a.exclude_stride > 0 and "seeds" in z.files:
            keep = training_rows(z["seeds"], a.exclude_stride)
            held = int((~keep).sum())
            X, Y = X[keep], Y[keep]
    else:
        X, Y = W.generate_training_set(a.count, a.seed0, (a.n_min, a.n_max), opts)
        if a.save_data:
            np.savez_compressed(a.save_data, X=X, Y=Y)
    t1 = time.perf_counter()
    ws = W.WarmStart.fit(X, Y, epochs=a.epochs, batch=a.batch, lr=a.lr, eps=a.eps, margin=a.margin)
    t2 = time.perf_counter()
    ws.meta.update(data=(f"{len(X)} plain packings of {a.data}" if a.data else
                         f"{len(X)} plain packings, N log-uniform [{a.n_min}, {a.n_max}], seeds {a.seed0}.."),
                   pair_precision=a.pair_precision)
    ws.save(a.out)
    # fit on the training set (phi_J)
    P = ws.predict(X)
    out = {"train_packings": int(len(X)), "held_out_of_data": held, "generate_s": t1 - t0, "train_s": t2 - t1,
           "train_loss_first": ws.meta["train_loss"][0], "train_loss_last": ws.meta["train_loss"][-1],
           "train_phi_mae": float(np.abs(P[:, 0] - Y[:, 0]).mean()),
           "train_phi_std": float(Y[:, 0].std())}
    if a.eval_count > 0:
        items = [W.draw_evaluation_packing(s, a.eval_n) for s in range(a.eval_seed0, a.eval_seed0 + a.eval_count)]
        ev = W.evaluate(ws, items, opts, a.eval_concurrency, plain_opts)
        plain_runs = ev.pop("plain_runs")
        out["eval"] = ev
        out["eval"]["N"] = a.eval_n
        for m in [float(x) for x in a.eval_margins.split(",") if x]:
            ws.margin = m
            e2 = W.evaluate(ws, items, opts, a.eval_concurrency, plain_opts, plain=plain_runs)
            e2.pop("plain_runs")
            out[f"eval_margin_{m:g}"] = e2
        ws.margin = a.margin
    print(json.dumps(out))
    return out


if __name__ == "__main__":
    main()
