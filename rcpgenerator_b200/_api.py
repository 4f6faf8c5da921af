"""Module-level API mirroring the reference binding ``_rcpgenerator``.

Same functions, dict keys, defaults and error types as the pybind11 module of
the reference (python_code/python/src/bindings/module.cpp:200-296):
``initialize_particles(config)``, ``run_packing(input, config)``,
``run_packing_observed(input, config, progress_interval, capture_positions,
trajectory_interval, callback, options)``, ``set_num_threads`` /
``get_num_threads``. Inputs may be nested lists (as the reference takes them)
or NumPy arrays; results are nested lists like the reference's unless
``as_arrays=True`` is passed, which returns NumPy arrays without the O(N)
Python-object conversion.

Engine selection (not in the reference): ``config["engine"]`` is ``"graph"``
(default: GPU-resident controller, CUDA-graph replay) or ``"exact"`` (host
controller, reductions in the reference's one-thread order), and
``config["device"]`` picks the CUDA device.
"""

from __future__ import annotations

import ctypes as C
from typing import Any, Callable

import numpy as np

from . import _native as N

_dp = C.POINTER(C.c_double)
_i8p = C.POINTER(C.c_int8)

_num_threads = 1

_DIST_DEFAULTS = dict(
    type="mono", d=1.0, mu=1.0, sigma=0.2, mu1=1.0, sigma1=0.2, mu2=2.0, sigma2=0.3, p=0.5,
    d1=1.0, d2=2.0, d_min=0.5, d_max=1.5, exponent=-2.5, scale=1.0, shape=2.0,
)


def set_num_threads(n: int) -> None:
    """Kept for API compatibility (module.cpp:203-215). The GPU engine has no
    OpenMP team; the value is recorded and returned by get_num_threads."""
    global _num_threads
    if int(n) < 1:
        raise ValueError("num_threads must be >= 1")
    _num_threads = int(n)


def get_num_threads() -> int:
    return _num_threads


def _f64(a: Any) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _as_ptr(a: np.ndarray, t=_dp):
    return a.ctypes.data_as(t)


def initialize_particles(config: dict) -> dict:
    """initialize_particles (initialize_particles.cpp:399-474; module.cpp:228-234)."""
    phi = float(config.get("phi", 0.05))
    n = int(config.get("N", 0))
    ndim = int(config.get("Ndim", 0))
    box = _f64(config.get("box", []))
    walls = np.ascontiguousarray(np.asarray(config.get("walls", []), dtype=np.int8))
    fix_height = bool(config.get("fix_height", False))
    seed = int(config.get("seed", 0))
    dist_in = dict(config.get("dist", {}))
    dist = dict(_DIST_DEFAULTS)
    dist.update(dist_in)
    custom = _f64(dist.get("custom", []))
    dd = N.Distribution()
    dd.type = str(dist["type"]).encode()
    for k in ("d", "mu", "sigma", "mu1", "sigma1", "mu2", "sigma2", "p", "d1", "d2", "d_min",
              "d_max", "exponent", "scale", "shape"):
        setattr(dd, k, float(dist[k]))
    dd.custom = _as_ptr(custom) if custom.size else None
    dd.custom_len = int(custom.size)
    nd_out = max(ndim, 0)
    pos = np.zeros(max(n, 0) * nd_out, dtype=np.float64)
    dia = np.zeros(max(n, 0), dtype=np.float64)
    box_out = np.zeros(max(nd_out, 1), dtype=np.float64)
    walls_out = np.zeros(max(nd_out, 1), dtype=np.int8)
    sf = C.c_double()
    pm = C.c_double()
    err = N.errbuf()
    rc = N.lib.rcpg_initialize_particles(
        phi, max(n, 0), ndim,
        _as_ptr(box) if box.size else None, int(box.size),
        _as_ptr(walls, _i8p) if walls.size else None, int(walls.size),
        int(fix_height), C.byref(dd), seed & 0xFFFFFFFFFFFFFFFF,
        _as_ptr(pos), _as_ptr(dia), _as_ptr(box_out), _as_ptr(walls_out, _i8p),
        C.byref(sf), C.byref(pm), err, len(err),
    )
    if rc == N.RCPG_EINVAL:
        raise ValueError(err.value.decode())
    if rc != N.RCPG_OK:
        raise RuntimeError(err.value.decode())
    return {
        "positions": pos.reshape(n, ndim).tolist(),
        "diameters": dia.tolist(),
        "box": box_out[:ndim].tolist(),
        "walls": [int(w) for w in walls_out[:ndim]],
        "diameter_scale_factor": sf.value,
        "phi_modifier": pm.value,
    }


class _Inputs:
    """Keeps the NumPy buffers alive while the C structs point at them."""

    def __init__(self, inp: dict, config: dict, options: dict | None):
        pos = inp.get("positions", [])
        self.positions = _f64(pos)
        n = int(self.positions.shape[0]) if self.positions.ndim == 2 else 0
        ndim = int(self.positions.shape[1]) if self.positions.ndim == 2 else 0
        self.diameters = _f64(inp.get("diameters", []))
        self.box = _f64(config.get("box", []))
        self.walls = np.ascontiguousarray(np.asarray(config.get("walls", []), dtype=np.int8))
        pi = N.PackingInput()
        pi.N = n
        pi.ndim = ndim
        pi.positions = _as_ptr(self.positions) if self.positions.size else None
        pi.diameters = _as_ptr(self.diameters) if self.diameters.size else None
        pi.box = _as_ptr(self.box) if self.box.size else None
        pi.box_len = int(self.box.size)
        pi.walls = _as_ptr(self.walls, _i8p) if self.walls.size else None
        pi.walls_len = int(self.walls.size)
        pi.neighbor_max = int(config.get("neighbor_max", 0)) & 0xFFFFFFFF
        pi.seed = int(config.get("seed", 0)) & 0xFFFFFFFF
        pi.fix_height = int(bool(config.get("fix_height", False)))
        self.pi = pi
        if n == 0 or ndim == 0:
            raise RuntimeError("rcpgenerator_b200: empty packing input")
        if self.diameters.size != n:
            raise ValueError("diameters must have one entry per particle")
        ro = N.RunOptions()
        N.lib.rcpg_default_options(C.byref(ro))
        opts = dict(options or {})
        if "max_steps" in opts:
            ro.max_steps = int(opts["max_steps"])
        if "fix_diameter" in opts:
            ro.fix_diameter = int(bool(opts["fix_diameter"]))
        if "reorder_interval" in opts:
            ro.reorder_interval = int(opts["reorder_interval"])
        if "mu" in opts:
            ro.has_mu_override = 1
            ro.mu_override = float(opts["mu"])
        if "target_phi" in opts:
            ro.has_target_phi = 1
            ro.target_phi = float(opts["target_phi"])
        if "initial_phi_target" in opts:
            ro.has_initial_phi_target = 1
            ro.initial_phi_target = float(opts["initial_phi_target"])
        if "growth_steps" in opts:
            ro.growth_steps = int(opts["growth_steps"])
        engine = str(config.get("engine", opts.get("engine", "graph")))
        if engine not in ("graph", "exact"):
            raise ValueError(f"unknown engine {engine!r} (expected 'graph' or 'exact')")
        ro.exact = 1 if engine == "exact" else 0
        ro.device = int(config.get("device", opts.get("device", 0)))
        ro.graph_steps = int(config.get("graph_steps", opts.get("graph_steps", 32)))
        prec = str(config.get("pair_precision", opts.get("pair_precision", "f64")))
        if prec not in ("f64", "mixed"):
            raise ValueError(f"unknown pair_precision {prec!r} (expected 'f64' or 'mixed')")
        ro.pair_precision = 1 if prec == "mixed" else 0
        ro.mixed_switch = float(config.get("mixed_switch", opts.get("mixed_switch", 1e-5)))
        self.ro = ro


def _arr(ptr, n: int, dtype) -> np.ndarray:
    if n == 0 or not ptr:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)


def result_to_dict(r: N.Result, as_arrays: bool = False) -> dict:
    """PackingResult -> the reference's result dict (module.cpp:154-184)."""
    n, nd, s = int(r.N), int(r.ndim), int(r.steps)
    pos = _arr(r.positions, n * nd, np.float64).reshape(n, nd)
    out: dict[str, Any] = {
        "positions": pos,
        "diameters": _arr(r.diameters, n, np.float64),
        "box": _arr(r.box, nd, np.float64),
        "walls": _arr(r.walls, nd, np.int8),
        "phi_history": _arr(r.phi_history, s, np.float64),
        "force_history": _arr(r.force_history, s, np.float64),
        "energy_history": _arr(r.energy_history, s, np.float64),
        "max_overlap_history": _arr(r.max_overlap_history, s, np.float64),
        "mu_history": _arr(r.mu_history, s, np.float64),
        "alpha_history": _arr(r.alpha_history, s, np.float64),
        "mu_flag_history": _arr(r.mu_flag_history, s, np.int8),
        "particle_origin": _arr(r.particle_origin, n, np.uint64),
    }
    if not as_arrays:
        out = {k: v.tolist() for k, v in out.items()}
    out.update(
        {
            # research-only fields of the reference (RCP_PP_WINDOW / spike log), always empty here
            "pp_F_sq_sum": [], "pp_F_sign_flips": [], "pp_pos_range_max": [],
            "pp_contact_sum": [], "pp_signflip_resets": [], "pp_window_steps": 0,
            "spike_log": [], "reorder_log": [],
            "steps": s,
            "phi": float(r.phi),
            "max_min_dist": float(r.max_min_dist),
            "force_magnitude": float(r.force_magnitude),
        }
    )
    out["engine_stats"] = {
        "pair_builds": int(r.pair_builds),
        "row_capacity": int(r.row_capacity),
        "kernel_launches": int(r.kernel_launches),
        "fp64_switch_step": int(r.fp64_switch_step),
        "pair_energy_rel_error": float(r.pair_energy_rel_error),
        "pair_force_rel_error": float(r.pair_force_rel_error),
    }
    return out


def _trace_to_dict(r: N.Result, captured: bool) -> dict:
    t = int(r.trace_len)
    n, nd = int(r.N), int(r.ndim)
    tr = {
        "steps": _arr(r.trace_steps, t, np.uint64).tolist(),
        "positions": [],
        "diameters": [],
        "phi": _arr(r.trace_phi, t, np.float64).tolist(),
        "force": _arr(r.trace_force, t, np.float64).tolist(),
        "energy": _arr(r.trace_energy, t, np.float64).tolist(),
        "max_min_dist": _arr(r.trace_max_min_dist, t, np.float64).tolist(),
    }
    if captured and t and r.trace_positions:
        p = _arr(r.trace_positions, t * n * nd, np.float64).reshape(t, n, nd)
        d = _arr(r.trace_diameters, t * n, np.float64).reshape(t, n)
        tr["positions"] = p.tolist()
        tr["diameters"] = d.tolist()
    return tr


def _run(inp: dict, config: dict, options: dict | None, progress_interval: int,
         capture_positions: bool, trajectory_interval: int, callback: Callable | None,
         as_arrays: bool) -> tuple[dict, dict]:
    ins = _Inputs(inp, config, options)
    n, nd = ins.pi.N, ins.pi.ndim
    cb_error: list[BaseException] = []

    def _obs(op, posp, _user):
        if callback is None or cb_error:
            return
        o = op.contents
        upd = {
            "step": int(o.step), "phi": o.phi, "force_magnitude": o.force_magnitude,
            "energy": o.energy, "max_min_dist": o.max_min_dist,
        }
        if posp:
            upd["positions"] = np.ctypeslib.as_array(posp, shape=(n * nd,)).reshape(n, nd).tolist()
        try:
            callback(upd)
        except BaseException as e:  # re-raised after the run
            cb_error.append(e)

    cfn = N.OBSERVER(_obs) if callback is not None else N.OBSERVER()
    res = C.POINTER(N.Result)()
    err = N.errbuf()
    rc = N.lib.rcpg_run_packing(
        C.byref(ins.pi), C.byref(ins.ro), int(progress_interval), int(bool(capture_positions)),
        int(trajectory_interval), cfn, None, C.byref(res), err, len(err),
    )
    N.raise_for(rc, err)
    try:
        if cb_error:
            raise cb_error[0]
        out = result_to_dict(res.contents, as_arrays=as_arrays)
        tr = _trace_to_dict(res.contents, bool(capture_positions))
    finally:
        N.lib.rcpg_result_free(res)
    return out, tr


def run_packing(input: dict, config: dict, as_arrays: bool = False) -> dict:
    """run_packing (rcp_generator.cpp:4336-4341; module.cpp:236-245)."""
    out, _ = _run(input, config, None, 0, False, 0, None, as_arrays)
    return out


def run_packing_observed(input: dict, config: dict, progress_interval: int = 0,
                         capture_positions: bool = False, trajectory_interval: int = 0,
                         callback: Callable | None = None, options: dict | None = None,
                         as_arrays: bool = False) -> dict:
    """run_packing_observed (module.cpp:247-296): {"result": ..., "trace": ...}."""
    out, tr = _run(input, config, options or {}, progress_interval, capture_positions,
                   trajectory_interval, callback, as_arrays)
    return {"result": out, "trace": tr}


def run_packing_batch(items: list, options: dict | None = None, concurrency: int = 0,
                      as_arrays: bool = True, growth_steps=None) -> list[dict]:
    """Many independent packings, ``items`` = [(input, config), ...] as for
    run_packing; the run options (``options`` plus the engine keys ``engine``,
    ``pair_precision``, ``device``, ... of the first config) are shared.
    ``concurrency`` < 0 runs them in the persistent batch engine (one launch
    per ndim, each thread block running whole packings); 0 sends the cheap
    ones there and the others to 32 ordinary engines on CUDA streams at the
    same time; k > 0 runs k ordinary engines at a time on their own streams
    (the reference runs one process per core, rcptools/jobs.py:392-401).
    ``growth_steps`` (optional, one int per item, 0 = the reference's deadline)
    sets each packing's growth-rung length, as a warm start does.
    Returns the result dicts in input order; a failed packing raises after all
    have run, naming its index."""
    items = list(items)
    if not items:
        return []
    ins = [_Inputs(inp, cfg, options) for inp, cfg in items]
    arr = (N.PackingInput * len(ins))(*[x.pi for x in ins])
    res = (C.POINTER(N.Result) * len(ins))()
    status = (C.c_int32 * len(ins))()
    err = N.errbuf()
    if growth_steps is None:
        rc = N.lib.rcpg_run_batch(arr, len(ins), C.byref(ins[0].ro), int(concurrency), res, status,
                                  err, len(err))
    else:
        gs = np.ascontiguousarray(np.asarray(growth_steps, dtype=np.uint64))
        if gs.shape != (len(ins),):
            raise ValueError("growth_steps needs one entry per packing")
        rc = N.lib.rcpg_run_batch_growth(arr, len(ins), C.byref(ins[0].ro),
                                         gs.ctypes.data_as(N._u64p), int(concurrency), res, status,
                                         err, len(err))
    try:
        N.raise_for(rc, err)
        return [result_to_dict(r.contents, as_arrays=as_arrays) for r in res]
    finally:
        for r in res:
            if r:
                N.lib.rcpg_result_free(r)


def batch_tuning(ndim: int, device: int = 0, pair_precision: str = "f64") -> dict:
    """The persistent batch kernel's autotuned launch shape for packings of
    `ndim` (tuned on first use): blocks per SM and the packing-steps per second
    measured at 1 and 2 blocks per SM."""
    b = C.c_int32(0)
    r = (C.c_double * 2)()
    err = N.errbuf()
    rc = N.lib.rcpg_batch_tuning(int(ndim), int(device), 1 if pair_precision == "mixed" else 0, C.byref(b), r,
                                 err, len(err))
    N.raise_for(rc, err)
    return {"blocks_per_sm": int(b.value), "steps_per_s": [float(r[0]), float(r[1])]}


class PackingEngine:
    """One packing advanced in slices of steps (rcpg_engine_* of the C ABI).

    Used by the benchmark and by callers that interleave their own work
    between steps; ``advance(k)`` runs at most k more steps of the same loop
    run_packing executes.
    """

    def __init__(self, input: dict, config: dict, options: dict | None = None, stream: int = 0):
        self._ins = _Inputs(input, config, options)
        self._h = C.c_void_p()
        err = N.errbuf()
        rc = N.lib.rcpg_engine_create(C.byref(self._ins.pi), C.byref(self._ins.ro),
                                      C.c_void_p(stream or None), C.byref(self._h), err, len(err))
        N.raise_for(rc, err)

    def advance(self, steps: int = 0) -> bool:
        fin = C.c_int32()
        err = N.errbuf()
        rc = N.lib.rcpg_engine_advance(self._h, int(steps), C.byref(fin), err, len(err))
        N.raise_for(rc, err)
        return bool(fin.value)

    @property
    def steps(self) -> int:
        return int(N.lib.rcpg_engine_steps(self._h))

    @property
    def kernel_launches(self) -> int:
        return int(N.lib.rcpg_engine_kernel_launches(self._h))

    def result(self, as_arrays: bool = True) -> dict:
        res = C.POINTER(N.Result)()
        err = N.errbuf()
        rc = N.lib.rcpg_engine_result(self._h, C.byref(res), err, len(err))
        N.raise_for(rc, err)
        try:
            return result_to_dict(res.contents, as_arrays=as_arrays)
        finally:
            N.lib.rcpg_result_free(res)

    def profile_pair_kernel(self, reps: int = 20) -> dict:
        """Mean launch time of the pair-force kernel on the current state and
        its algorithmic bytes per launch (CUDA events on the engine stream)."""
        ms, b, row = C.c_double(), C.c_double(), C.c_double()
        err = N.errbuf()
        rc = N.lib.rcpg_engine_profile_pair_kernel(self._h, int(reps), C.byref(ms), C.byref(b),
                                                   C.byref(row), err, len(err))
        N.raise_for(rc, err)
        return {"avg_ms": ms.value, "alg_bytes": b.value, "mean_row": row.value}

    def profile_build_kernel(self, reps: int = 10) -> dict:
        """Mean launch time of the neighbour build's search kernel (graph mode:
        the tiled build with the forces fused) on full rebuilds of the current
        state, and its algorithmic bytes per launch."""
        ms, b = C.c_double(), C.c_double()
        err = N.errbuf()
        rc = N.lib.rcpg_engine_profile_build_kernel(self._h, int(reps), C.byref(ms), C.byref(b),
                                                    err, len(err))
        N.raise_for(rc, err)
        return {"avg_ms": ms.value, "alg_bytes": b.value}

    def close(self) -> None:
        if self._h:
            N.lib.rcpg_engine_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
