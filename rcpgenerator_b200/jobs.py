"""Packing jobs of the reference's analysis package (rcptools) on the batch
engine, and its pair-overlap diagnostics on the GPU.

The reference runs a study as a list of job dicts, one process per core,
each job building one `Packing` from a diameter list and packing it
(rcptools/jobs.py:34-134 run_one_custom_packing, :265-371 run_packing_job,
:392-418 run_jobs). Here the same job dicts go to the GPU together:
`run_jobs` prepares every packing on the host exactly as
`run_one_custom_packing` does, runs all of them in one `run_packing_batch`
call (optionally warm-started), and returns the reference's result rows.
`overlap_report` (rcptools/overlap.py:7-113) runs on the GPU
(`rcpg_overlap_report`); `engine_max_overlap` and `phi_corrected` are the
reference's one-liners (jobs.py:346-360, overlap.py:116-127).
"""

from __future__ import annotations

import ctypes as C
import math
import traceback
from typing import Any

import numpy as np

from . import _native as N
from ._api import run_packing_batch
from ._wrapper import Packing


# ---- diagnostics ------------------------------------------------------------------

def phi_corrected(phi, max_overlap, Ndim):
    """phi * (1 - max_overlap)^Ndim: the packing fraction after the uniform
    contraction that clears every overlap (overlap.py:116-127)."""
    return float(phi) * (1.0 - float(max_overlap)) ** int(Ndim)


def engine_max_overlap(packing):
    """The engine's final max fractional overlap (packing.max_min_dist), the
    quantity overlap_report's max_overlap measures (jobs.py:346-360)."""
    v = getattr(packing, "max_min_dist", None)
    return float(v) if v is not None else 0.0


def _state_of(packing):
    pos = None
    for attr in ("positions", "points", "x", "coords"):
        if hasattr(packing, attr):
            pos = np.asarray(getattr(packing, attr), dtype=np.float64)
            break
    if pos is None:
        raise AttributeError("packing has no positions/points/x/coords attribute")
    D = np.asarray(packing.diameters, dtype=np.float64)
    box = None
    for attr in ("box", "L", "box_size"):
        if hasattr(packing, attr):
            b = np.asarray(getattr(packing, attr), dtype=np.float64)
            box = (b[1::2] - b[0::2]) if b.size == 2 * pos.shape[1] else b
            break
    return pos, D, box


def overlap_report(packing, frac_def="sum", verbose=False, device: int = 0):
    """Distribution of fractional overlaps over all overlapping pairs, with
    the keys and conventions of the reference's overlap_report; computed by
    the GPU kernel. Pairs come sorted by (i, j)."""
    pos, D, box = _state_of(packing)
    n = int(pos.shape[0]) if pos.ndim == 2 else 0
    ndim = int(pos.shape[1]) if pos.ndim == 2 else 0
    empty = {"n_overlapping": 0, "n_candidate_pairs": 0, "fractions_min": np.array([]),
             "fractions_sum": np.array([]), "max_overlap": 0.0, "mean_overlap": 0.0,
             "X_shrink_to_clear": 0.0, "ndim": ndim, "pairs": np.zeros((0, 2), int)}
    if n == 0 or D.size == 0:
        return empty
    pos = np.ascontiguousarray(pos)
    D = np.ascontiguousarray(D)
    boxp = None
    if box is not None:
        box = np.ascontiguousarray(box, dtype=np.float64)
        boxp = box.ctypes.data_as(N._dp)
    ncand, nov = C.c_uint64(0), C.c_uint64(0)
    cap = 0
    pairs = np.zeros((0, 2), np.uint32)
    fs = fm = np.zeros(0)
    for _ in range(2):  # first call sizes the output
        pairs = np.zeros((max(cap, 1), 2), np.uint32)
        fs = np.zeros(max(cap, 1))
        fm = np.zeros(max(cap, 1))
        err = N.errbuf()
        rc = N.lib.rcpg_overlap_report(n, ndim, pos.ctypes.data_as(N._dp), D.ctypes.data_as(N._dp), boxp,
                                       C.byref(ncand), C.byref(nov), cap,
                                       pairs.ctypes.data_as(N._u32p), fs.ctypes.data_as(N._dp),
                                       fm.ctypes.data_as(N._dp), int(device), err, len(err))
        if rc == N.RCPG_ENOSPC and cap < nov.value:
            cap = int(nov.value)
            continue
        N.raise_for(rc, err)
        break
    m = int(nov.value)
    if m == 0:
        out = dict(empty, n_candidate_pairs=int(ncand.value))
        if verbose:
            print("  no overlapping pairs.")
        return out
    f_sum, f_min = fs[:m], fm[:m]
    out = {
        "n_overlapping": m,
        "n_candidate_pairs": int(ncand.value),
        "fractions_min": f_min,
        "fractions_sum": f_sum,
        "max_overlap": float(f_sum.max()),
        "mean_overlap": float(f_sum.mean()),
        "X_shrink_to_clear": float(f_sum.max()),
        "ndim": ndim,
        "pairs": pairs[:m].astype(np.int64),
    }
    if verbose:
        rep = f_min if frac_def == "min" else f_sum
        label = "overlap / min(r_i,r_j)" if frac_def == "min" else "overlap / (r_i+r_j)"
        print(f"N = {n}, candidate close-pairs = {out['n_candidate_pairs']}, overlapping = {m}")
        q = np.quantile(rep, [0.5, 0.9, 0.99, 1.0])
        print(f"fractional overlap ({label}): median {q[0]:.2e}, p90 {q[1]:.2e}, p99 {q[2]:.2e}, max {q[3]:.2e}")
    return out


# ---- single packings (run_one_custom_packing) --------------------------------------

def _volume(diameters, ndim):
    r = np.asarray(diameters, dtype=float) / 2.0
    if ndim == 2:
        return float(np.sum(np.pi * r ** 2))
    if ndim == 3:
        return float(np.sum((4.0 / 3.0) * np.pi * r ** 3))
    return float(np.sum(np.pi ** (ndim / 2.0) / math.gamma(ndim / 2.0 + 1.0) * r ** ndim))


def prepare_custom_packing(diameters, *, seed=123, Ndim=2, phi_init=0.5, initializer_phi=0.11, box=None,
                           walls=None, neighbor_max=0, fix_height=False, size_ratio_hint=None,
                           reorder_interval=None, verbose=False, engine="graph") -> Packing:
    """The Packing that run_one_custom_packing packs (jobs.py:34-134): a
    dilute monodisperse initialisation at `initializer_phi`, then the given
    diameters (finite, at least 1e-12) scaled to `phi_init` -- not packed."""
    d = np.asarray(diameters, dtype=float)
    d = d[np.isfinite(d)]
    d = np.maximum(d, 1e-12)
    n = len(d)
    box = [1.0] * Ndim if box is None else list(box)
    walls = [0] * Ndim if walls is None else list(walls)
    p = Packing(phi=float(initializer_phi), N=n, Ndim=Ndim, box=box, walls=walls, fix_height=fix_height,
                dist={"type": "mono", "d": 1.0}, neighbor_max=max(0, int(neighbor_max)), seed=int(seed),
                verbose=verbose, engine=engine)
    p.initialize()
    box_vol = float(np.prod(np.asarray(p.box, dtype=float)))
    cur = _volume(d, Ndim) / box_vol
    if cur <= 0:
        raise ValueError("Current custom-diameter phi is non-positive.")
    scale = (float(phi_init) / cur) ** (1.0 / Ndim)
    p.diameters = (d * scale).tolist()
    p.phi = float(phi_init)
    object.__setattr__(p, "_initialized", True)
    object.__setattr__(p, "_needs_initialize", False)
    object.__setattr__(p, "_packed", False)
    object.__setattr__(p, "_needs_pack", True)
    return p


def run_one_custom_packing(diameters, *, reorder_interval=None, verbose=False, **kw) -> Packing:
    """run_one_custom_packing (jobs.py:34-134) on this engine."""
    p = prepare_custom_packing(diameters, verbose=verbose, **kw)
    if reorder_interval is None:
        p.pack()
    else:
        p._execute_packing(verbose=verbose, progress_interval=1000, capture_trajectory=False,
                           trajectory_interval=0, options={"reorder_interval": int(reorder_interval)})
    return p


# ---- job rows (run_packing_job / run_jobs) -----------------------------------------

def _prescreen_reject(D, ndim, phi_target, threshold):
    """Geometric pre-screen of jobs.py:137-143: reject when the largest
    diameter exceeds L_min / threshold, L_min the box side at phi_target."""
    V = _volume(D, ndim)
    L_min = (V / float(phi_target)) ** (1.0 / float(ndim))
    dmax = float(np.max(D)) if len(D) else 0.0
    return (dmax > L_min / float(threshold)), dmax, L_min


def _safe_phi(packing) -> float:
    """phi recomputed from positions, diameters and box (relative to a curved
    container's volume), 0.0 on any sanity failure: non-finite values,
    non-positive diameters or box, a particle outside the box by more than
    1e-6 of its largest side (rcptools/_helpers.py:30-77)."""
    try:
        pos, D, box = _state_of(packing)
    except AttributeError:
        return 0.0
    if pos.size == 0 or pos.ndim != 2 or D.size != pos.shape[0] or box is None:
        return 0.0
    ndim = pos.shape[1]
    box = np.atleast_1d(box).astype(float)
    if box.size == 1:
        box = np.full(ndim, float(box.item()))
    if box.size != ndim:
        return 0.0
    if not np.all(np.isfinite(pos)) or not np.all(np.isfinite(D)) or np.any(D <= 0):
        return 0.0
    tol = 1e-6 * np.max(box)
    if np.any(pos < -tol) or np.any(pos > box + tol) or np.any(box <= 0):
        return 0.0
    w = getattr(packing, "walls", None)
    t = -int(w[0]) if (w is not None and len(w) and int(w[0]) < 0) else 0
    cf = (math.pi ** (t / 2.0) / math.gamma(t / 2.0 + 1.0) * (0.5 ** t)) if t >= 2 else 1.0
    vb = float(np.prod(box))
    return _volume(D, ndim) / vb / cf if vb > 0 else 0.0


def _row(job, seed, packing=None, error=None, rejected=False, D=None):
    base = {"candidate": job.get("candidate"), "seed": seed, "generation": job.get("generation"),
            "stage": job.get("stage"), "theta": job.get("theta")}
    if error is not None:
        return dict(base, success=False, rejected=False, error=error, phi=None, phi_rcp=None, phi_corr=None,
                    max_overlap=None, mean_overlap=None, n_overlapping=None, steps=None, force_magnitude=None,
                    max_min_dist=None, Dmin=None, Dmax=None, D_ratio=None, packing_path=None)
    if rejected:
        return dict(base, success=True, rejected=True, phi=0.0, phi_rcp=0.0, phi_corr=0.0, max_overlap=0.0,
                    mean_overlap=0.0, n_overlapping=0, steps=None, force_magnitude=None, max_min_dist=None,
                    Dmin=float(D.min()) if len(D) else None, Dmax=float(D.max()) if len(D) else None,
                    D_ratio=float(D.max() / D.min()) if len(D) and D.min() > 0 else None, packing_path=None)
    d_final = np.asarray(packing.diameters, dtype=float)
    phi = _safe_phi(packing)
    mo = engine_max_overlap(packing)
    ndim = int(job["Ndim"])
    return dict(base, success=True, rejected=False, error=None, phi=float(phi),
                phi_rcp=float(packing.phi_final if packing.phi_final is not None else packing.phi),
                phi_corr=float(phi_corrected(phi, mo, ndim)), max_overlap=float(mo), mean_overlap=None,
                n_overlapping=None, steps=int(packing.steps) if packing.steps is not None else None,
                force_magnitude=float(packing.force_magnitude) if packing.force_magnitude is not None else None,
                max_min_dist=float(packing.max_min_dist) if packing.max_min_dist is not None else None,
                Dmin=float(d_final.min()) if len(d_final) else None,
                Dmax=float(d_final.max()) if len(d_final) else None,
                D_ratio=float(d_final.max() / d_final.min()) if len(d_final) else None, packing_path=None)


def _prepare_job(job):
    """(seed, D, Packing or None, row or None) of one job: the shuffle and the
    pre-screen of run_packing_job (jobs.py:268-300), then the packing."""
    seed = int(job["seed"])
    # a copy: the caller's job keeps its diameters (the reference's workers
    # shuffle a pickled copy)
    D = np.array(job["diameters"], dtype=float)
    np.random.default_rng(seed).shuffle(D)
    ndim = int(job["Ndim"])
    ps = job.get("prescreen", {}) or {}
    if ps.get("enabled", False):
        reject, _, _ = _prescreen_reject(D, ndim, ps.get("phi_target", 0.85), ps.get("threshold", 2.5))
        if reject:
            return seed, D, None, _row(job, seed, rejected=True, D=D)
    p = prepare_custom_packing(D, seed=seed, Ndim=ndim, phi_init=float(job["phi_init"]),
                               initializer_phi=float(job["initializer_phi"]), box=job.get("box"),
                               walls=job.get("walls"), neighbor_max=int(job.get("neighbor_max", 0)),
                               fix_height=bool(job.get("fix_height", False)),
                               size_ratio_hint=job.get("size_ratio_hint"))
    return seed, D, p, None


def run_packing_job(job) -> dict:
    """run_packing_job (jobs.py:265-371): one job, one packing, one row."""
    seed = job.get("seed")
    try:
        seed, D, p, row = _prepare_job(job)
        if row is not None:
            return row
        p.pack()
        return _row(job, seed, packing=p)
    except Exception as e:  # the reference reports failures as rows
        r = _row(job, seed, error=repr(e))
        r["traceback"] = traceback.format_exc()
        return r


def run_jobs(jobs, config: dict | None = None) -> list[dict]:
    """run_jobs (jobs.py:392-418) on the GPU: every accepted job's packing in
    one run_packing_batch call (config["gpu_concurrency"], default 0: the
    automatic persistent / streams split), rows in job order.
    config["warm_start"] = a WarmStart sets each packing's growth rung."""
    config = dict(config or {})
    jobs = list(jobs)
    rows: list[Any] = [None] * len(jobs)
    prepared = []
    for k, job in enumerate(jobs):
        try:
            seed, D, p, row = _prepare_job(job)
        except Exception as e:
            rows[k] = dict(_row(job, job.get("seed"), error=repr(e)), traceback=traceback.format_exc())
            continue
        if row is not None:
            rows[k] = row
        else:
            prepared.append((k, seed, p))
    if prepared:
        items = []
        for _, _, p in prepared:
            cfg = p._collect_pack_config()
            cfg["pair_precision"] = config.get("pair_precision", "f64")
            items.append(({"positions": np.asarray(p.positions, dtype=float),
                           "diameters": np.asarray(p.diameters, dtype=float)}, cfg))
        conc = int(config.get("gpu_concurrency", 0))
        ws = config.get("warm_start")
        try:
            if ws is not None:
                results, _ = ws.run_batch(items, {}, conc)
            else:
                results = run_packing_batch(items, {}, conc, as_arrays=True)
            for (k, seed, p), r in zip(prepared, results):
                p._apply_packing_result({key: (v.tolist() if isinstance(v, np.ndarray) else v)
                                         for key, v in r.items()})
                rows[k] = _row(jobs[k], seed, packing=p)
        except Exception:
            # one failure fails the batch call: fall back to one packing per job for the rows
            for k, seed, p in prepared:
                rows[k] = run_packing_job(jobs[k])
    return rows
