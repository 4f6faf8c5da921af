"""Throughput of the packing engine on the 2-D bidisperse N = 1M packing.

Workload (one replica per GPU, independent packings, no collective):
2-D bidisperse disks, N = 1,000,000, diameters 1.0 : 1.4 at 50:50 number
fraction, periodic unit square, initial phi 0.30, seed 123 (+ rank), placed by
the engine's initializer (a bit-exact restatement of the reference's
initialize_particles). One step = one ADAM step of Packing.pack()'s loop:
refresh trigger, neighbour rebuild when triggered, forces + reductions,
controller, ADAM + position update. Steps are timed from the start of the
run (the heavy-overlap early phase the reference is timed on).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Prints one JSON line (rank 0).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "packings/hour and ADAM steps/sec vs plain GPU engine at equal phi_J error"
UNIT = "ADAM steps/s"
WORKLOAD = dict(phi=0.30, N=1_000_000, Ndim=2, box=[1.0, 1.0], walls=[0, 0],
                dist={"type": "bidisperse", "d1": 1.0, "d2": 1.4, "p": 0.5}, seed=123)
PEAKS = REPO / "MEASURED_PEAKS.json"
# DRAM bytes (read + write) per algorithmic byte of k_forces from one ncu capture
# (profiles/k_forces_bidisperse2d_n3e5_mixed.md: 23.2 MB for 20.26 MB at N = 300k);
# the N = 1M launch is too large to capture with the full metric set
FORCES_TRAFFIC_PER_ALG_BYTE = 23.2 / 20.26
# the same for the cell-unit build with fused forces, k_cells<2, mixed>
# (profiles/k_cells_bidisperse2d_n3e5_mixed.md: 12.3 MB for 22.7 MB at N = 300k; the rows and
# forces it writes are still in L2 when the launch ends)
BUILD_TRAFFIC_PER_ALG_BYTE = 12.3 / 22.7


def workload_name(n: int) -> str:
    return f"bidisperse2d_N{n:.0e}_phi0.30_seed123".replace("e+0", "e")


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def hbm_peak():
    try:
        p = json.loads(PEAKS.read_text())
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.flush()
        rows = [r.split(",") for r in Path(self.out.name).read_text().strip().splitlines() if r.strip()]
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [c.strip() for c in r]
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
            except (ValueError, IndexError):
                continue
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_input(rank: int):
    import rcpgenerator_b200 as rb
    cfg = dict(WORKLOAD)
    cfg["seed"] = WORKLOAD["seed"] + rank
    init = rb.initialize_particles(cfg)
    pos = np.ascontiguousarray(init["positions"], dtype=np.float64)
    dia = np.ascontiguousarray(init["diameters"], dtype=np.float64)
    return pos, dia, init


def reference_sample(pos, dia, box, walls, warmup: int, steps: int, threads: int):
    """The reference engine (oracle/_ref, compiled from the reference sources)
    on the same input, run to step warmup + steps and timed by its own
    observer callback from the end of step `warmup` (>= 1) to the end of step
    warmup + steps: the same window as the GPU arm's."""
    ref = reference_module()
    if ref is None:
        return None, "reference build oracle/_ref missing"
    ref.set_num_threads(threads)
    stamps = {}

    def cb(update):
        stamps[int(update["step"])] = time.perf_counter()

    w = max(1, warmup)
    t0 = time.perf_counter()
    ref.run_packing_observed({"positions": pos.tolist(), "diameters": dia.tolist()},
                             {"box": box, "walls": walls, "neighbor_max": 0, "seed": 0},
                             1, False, 0, cb, {"max_steps": w + steps})
    t1 = time.perf_counter()
    if w not in stamps or w + steps not in stamps:
        return None, "reference produced no step timings"
    per = (stamps[w + steps] - stamps[w]) / steps
    return {"steps_per_s": 1.0 / per, "timed_steps": steps, "first": w + 1, "last": w + steps,
            "wall_s": t1 - t0}, None


# ---- batched workload: many independent small packings (packings/hour) ----
BATCH_METRIC = "packings/hour"


def batch_instances(seeds):
    """Independent packings drawn like the batched workload: N log-uniform on
    [64, 16384], ndim from {2, 3, 4}, diameters mono (d=1), bidisperse 50:50
    with ratio uniform on [1.1, 3.0], or log-normal with std/mean uniform on
    [0.1, 0.6] truncated to [0.2, 5] x mean; periodic unit boxes at phi 0.10;
    one packing per seed (rcpgenerator_b200.warmstart.draw_packing)."""
    from rcpgenerator_b200.warmstart import draw_packing
    return [draw_packing(int(s)) for s in seeds]


def _ref_capped(args_):
    """One capped reference packing in a worker process (one OpenMP thread)."""
    pos, dia, box, walls, cap = args_
    sys.path.insert(0, str(REPO / "oracle" / "_ref"))
    for k in list(os.environ):
        if k.startswith("RCP_"):
            del os.environ[k]
    import _rcpgenerator as ref
    ref.set_num_threads(1)
    t0 = time.perf_counter()
    r = ref.run_packing_observed({"positions": pos.tolist(), "diameters": dia.tolist()},
                                 {"box": box, "walls": walls, "neighbor_max": 0, "seed": 0},
                                 0, False, 0, None, {"max_steps": cap})["result"]
    return len(pos) * int(r["steps"]), time.perf_counter() - t0


def reference_batch_rate(items, cap: int, procs: int):
    """Reference particle-steps/s per core on capped runs of the same packings,
    one process per core (the reference's own throughput pattern)."""
    import multiprocessing as mp
    if not any((REPO / "oracle" / "_ref").glob("_rcpgenerator*.so")):
        return None
    work = [(i["positions"], i["diameters"], c["box"], c["walls"], cap) for i, c in items]
    with mp.get_context("spawn").Pool(procs) as pool:
        res = pool.map(_ref_capped, work)
    ps = sum(r[0] for r in res)
    t = sum(r[1] for r in res)
    return ps / t


def run_batch_workload(args) -> int:
    import rcpgenerator_b200 as rb
    rank, world, local = dist_env()
    # a stratified sample of the generator's seeds 0..4095 (every stride-th),
    # the ranks taking interleaved seeds
    stride = args.batch_stride or max(1, 4096 // max(1, args.batch_count * world))
    seeds = [(k * world + rank) * stride for k in range(args.batch_count)]
    items = batch_instances(seeds)
    run_opts = {"pair_precision": args.pair_precision, "device": local}
    for _, c in items:
        c.update({"pair_precision": args.pair_precision, "device": local})
    # warm-up: load the kernels and the pools
    rb.run_packing_batch(items[:2], {"max_steps": 50}, concurrency=args.concurrency)
    t0 = time.perf_counter()
    # the one-at-a-time sample: every k-th packing, so that it spans the size range
    single_stride = max(1, len(items) // max(1, args.batch_single))
    single = rb.run_packing_batch(items[::single_stride][: args.batch_single], run_opts, concurrency=1)
    t1 = time.perf_counter()
    res = rb.run_packing_batch(items, run_opts, concurrency=args.concurrency)
    t2 = time.perf_counter()
    ps = sum(len(i["positions"]) * r["steps"] for (i, _), r in zip(items, res))
    steps = [r["steps"] for r in res]
    if args.save_training:
        # the plain runs as warm-start training data (descriptors with log N, targets, seeds)
        from rcpgenerator_b200 import warmstart as W
        X = np.stack([W.descriptors(i["diameters"], np.asarray(i["positions"]).shape[1], c["walls"], True)
                      for i, c in items])
        Y = np.stack([W.targets(r) for r in res])
        np.savez_compressed(args.save_training, X=X, Y=Y, seeds=np.asarray(seeds, dtype=np.int64))
    value = len(items) / (t2 - t1) * 3600.0
    single_value = len(single) / (t1 - t0) * 3600.0
    warm = None
    if not args.no_warm_start:
        from rcpgenerator_b200 import warmstart as W
        if Path(args.warm_start_model).exists():
            ws = W.WarmStart.load(args.warm_start_model, device=local)
            t3 = time.perf_counter()
            wres, phi_pred = ws.run_batch(items, run_opts, concurrency=args.concurrency)
            t4 = time.perf_counter()
            pj = np.asarray([r["phi"] for r in res])
            wj = np.asarray([r["phi"] for r in wres])
            warm = {"value": len(items) / (t4 - t3) * 3600.0, "unit": BATCH_METRIC,
                    "vs_plain_engine": len(items) / (t4 - t3) * 3600.0 / single_value,
                    "vs_batched_plain": (t2 - t1) / (t4 - t3),
                    "mean_steps": float(np.mean([r["steps"] for r in wres])),
                    "delta_phi_J_mean": float(wj.mean() - pj.mean()),
                    "delta_phi_J_abs_mean": float(np.abs(wj - pj).mean()),
                    "phi_J_pred_mae": float(np.abs(phi_pred - pj).mean()),
                    "max_overlap": float(max(r["max_min_dist"] for r in wres)),
                    "model": str(Path(args.warm_start_model).name),
                    "note": "the same packings with the network's growth-rung lengths (inference inside "
                            "the timed region); phi_J compared packing by packing with the batched plain run"}
    cpu = None
    if not args.no_cpu_baseline and rank == 0:
        procs = os.cpu_count() or 1
        sample = items[: min(len(items), procs)]
        rate = reference_batch_rate(sample, args.cpu_cap_steps, procs)
        if rate:
            mean_ps = ps / len(items)  # particle-steps per packing, from the engine's own runs
            cpu = {"value": procs * 3600.0 * rate / mean_ps, "unit": BATCH_METRIC, "cores": procs,
                   "kind": "reference",
                   "sample": f"{len(sample)} of the packings capped at {args.cpu_cap_steps} steps, one "
                             f"process per core: {rate:.3g} particle-steps/s per core, scaled by the "
                             f"engine's mean {mean_ps:.3g} particle-steps per packing"}
    line = {
        "metric": BATCH_METRIC, "value": value, "unit": BATCH_METRIC, "n_gpus": world,
        "steps": int(sum(steps)), "warmup": 1, "ms_per_step": (t2 - t1) * 1e3 / max(sum(steps), 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 state, f32 pair terms" if args.pair_precision == "mixed" else "f64",
        "data": "synthetic",
        "config": {"workload": f"batch{len(items)}_N64-16384_ndim234_phi0.10", "packings": len(items),
                   "seeds": f"{seeds[0]}, {seeds[1] if len(seeds) > 1 else ''}, ... every {stride * world}-th of 0..4095",
                   "concurrency": args.concurrency,
                   "engine": {0: "persistent batch kernel for the small packings + engines on 32 streams"}.get(
                       args.concurrency, "persistent batch kernel" if args.concurrency < 0 else "graph engines on streams"),
                   "pair_precision": args.pair_precision, "particle_steps": ps,
                   "mean_steps": float(np.mean(steps)), "parallelism": f"replicas{world}",
                   "timing": "host wall clock around run_packing_batch (inputs on the host, results back)"},
        "plain_engine": {"value": single_value, "unit": BATCH_METRIC, "packings": len(single),
                         "note": "the same engine one packing at a time (concurrency 1), every "
                                 f"{single_stride}-th packing of the batch"},
        "cpu_baseline": cpu,
        "e2e": {"value": value, "unit": BATCH_METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                "note": "the timed region is already end to end (host arrays in, result dicts out)"},
        "warm_start": warm,
    }
    if rank == 0:
        print(json.dumps(line))
    return 0


def run_one_packing(args) -> int:
    """ADAM steps/s of one packing of the batched workload's generator (seed
    --seed), graph engine: 300 untimed steps, then --steps timed (host wall
    clock around PackingEngine.advance, which ends in a device sync). For
    profiling the engines that run a batch's large packings."""
    import rcpgenerator_b200 as rb
    from rcpgenerator_b200.warmstart import draw_packing
    rank, _, local = dist_env()
    inp, cfg = draw_packing(args.seed)
    cfg.update({"pair_precision": args.pair_precision, "device": local})
    eng = rb.PackingEngine(inp, cfg, {})
    eng.advance(300)
    steps = max(args.steps, 1) * 10
    t0 = time.perf_counter()
    eng.advance(steps)
    dt = time.perf_counter() - t0
    done = eng.steps - 300
    n, nd = inp["positions"].shape
    if rank == 0:
        print(json.dumps({"metric": "ADAM steps/s", "value": done / dt, "unit": "ADAM steps/s",
                          "steps": done, "config": {"workload": f"batch_generator_seed{args.seed}_{nd}d_N{n}",
                                                    "pair_precision": args.pair_precision}}))
    eng.close()
    return 0


def bench_config(n: int, warmup: int, steps: int) -> dict:
    """The workload as both arms name it (identical dict in both lines)."""
    return {"workload": workload_name(n), "N": n, "Ndim": 2,
            "dist": "bidisperse 1.0:1.4 at 50:50", "init_phi": 0.30, "box": "periodic unit square",
            "seed": WORKLOAD["seed"], "window": f"ADAM steps {warmup + 1}..{warmup + steps} of pack() from "
                                                 f"the start (early phase, a rebuild every step)",
            "l2": "inputs larger than L2 (~150 MB touched per step)"}


def reference_module():
    """The reference engine compiled from its own sources (oracle/_ref), with a
    clean RCP_* environment; None when it was not built."""
    ref_dir = REPO / "oracle" / "_ref"
    if not any(ref_dir.glob("_rcpgenerator*.so")):
        return None
    if str(ref_dir) not in sys.path:
        sys.path.insert(0, str(ref_dir))
    for k in list(os.environ):
        if k.startswith("RCP_"):
            del os.environ[k]
    import _rcpgenerator as ref
    return ref


def run_reference_arm(args):
    """The reference's own CPU engine on the same workload: its own
    initializer (same seed, the input this project's initializer reproduces
    bit for bit) and its run_packing_observed, timed per step by its own
    observer on all host threads. Nothing of this project is imported."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    ref = reference_module()
    if ref is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref missing"}))
        return 0
    cfg = dict(WORKLOAD)
    init = ref.initialize_particles(cfg)
    pos = np.asarray(init["positions"], dtype=np.float64)
    dia = np.asarray(init["diameters"], dtype=np.float64)
    threads = os.cpu_count() or 1
    s, why = reference_sample(pos, dia, init["box"], init["walls"], args.warmup, args.steps, threads)
    if s is None:
        print(json.dumps({"impl": "reference", "unavailable": why}))
        return 0
    v = s["steps_per_s"]
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": bench_config(WORKLOAD["N"], args.warmup, args.steps),
        "engine": "reference C++/OpenMP run_packing_observed (oracle/_ref, portable build), "
                  "input from its own initialize_particles",
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"steps {s['first']}..{s['last']} of the packing (observer timestamps), "
                                   f"setup excluded"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def growth_deadline(n: int, nd: int) -> int:
    """Last step of the growth rung (mu_flag = 1) on the reference's schedule:
    6000 + 9 sqrt(N d), at least 1500 (ENG:4713-4737)."""
    return max(1500, int(6000 + 9 * (n * nd) ** 0.5))


def timed_window(eng, stream, steps: int, clocks=None):
    """K steps of an engine timed with CUDA events on its stream."""
    import torch
    torch.cuda.synchronize()
    l0, s0 = eng.kernel_launches, eng.steps
    if clocks is not None:
        clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    eng.advance(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop() if clocks is not None else None
    return e0.elapsed_time(e1), eng.steps - s0, eng.kernel_launches - l0, clk


def late_phase(rb, pos, dia, init, precision, local, steps):
    """ADAM steps/s after the growth rung: the engine is advanced untimed past
    the rung's last step, then `steps` steps are timed (the phase where most
    steps skip the rebuild and the pair kernel dominates)."""
    import torch
    stream = torch.cuda.Stream()
    eng = rb.PackingEngine({"positions": pos, "diameters": dia},
                           {"box": init["box"], "walls": init["walls"], "device": local,
                            "pair_precision": precision}, {}, stream=stream.cuda_stream)
    n, nd = pos.shape
    start = growth_deadline(n, nd) + 200
    eng.advance(start)
    b0 = eng.result(as_arrays=True)["engine_stats"]["pair_builds"]
    ms, done, launches, _ = timed_window(eng, stream, steps)
    res = eng.result(as_arrays=True)
    prof = eng.profile_pair_kernel(reps=20)
    eng.close()
    return {"value": done / (ms / 1e3), "unit": UNIT, "steps": done, "ms_per_step": ms / max(done, 1),
            "window": f"steps {start + 1}..{start + done}", "pair_builds_in_window":
            int(res["engine_stats"]["pair_builds"] - b0),
            "fp64_switch_step": int(res["engine_stats"]["fp64_switch_step"]),
            "max_overlap_at_end": float(res["max_overlap_history"][-1]) if len(res["max_overlap_history"]) else None,
            "gpu_launches": int(launches)}, prof


def roofline_of(prof, peak, peak_kind, kernel, traffic_per_byte):
    achieved = prof["alg_bytes"] / (prof["avg_ms"] / 1e3) / 1e9
    out = {"bound": "hbm", "kernel": kernel, "achieved": achieved, "peak": peak, "unit": "GB/s",
           "frac": achieved / peak, "peak_kind": peak_kind,
           "traffic": prof["alg_bytes"] * traffic_per_byte,
           "traffic_note": "ncu DRAM bytes per algorithmic byte of a smaller capture (profiles/), scaled",
           "alg_bytes_per_launch": prof["alg_bytes"], "avg_launch_ms": prof["avg_ms"]}
    if "mean_row" in prof:
        out["mean_row"] = prof["mean_row"]
    return out


def batch_summary(args, local):
    """packings/hour of the batched workload on a sample of its generator
    (seeds 0..count-1): the batch engine plain and warm-started, the same
    engine one packing at a time, and the reference estimate."""
    ns = argparse.Namespace(**vars(args))
    ns.batch_count = args.bench_batch
    buf = []
    import contextlib
    import io
    with contextlib.redirect_stdout(io.StringIO()) as out:
        run_batch_workload(ns)
    for line in out.getvalue().splitlines():
        if line.startswith("{"):
            buf.append(json.loads(line))
    if not buf:
        return None
    b = buf[-1]
    return {"metric": BATCH_METRIC, "value": b["value"], "unit": BATCH_METRIC,
            "packings": b["config"]["packings"], "workload": b["config"]["workload"],
            "engine": b["config"]["engine"], "mean_steps": b["config"]["mean_steps"],
            "pair_precision": b["config"]["pair_precision"], "timing": b["config"]["timing"],
            "plain_engine": b["plain_engine"], "warm_start": b["warm_start"],
            "cpu_baseline": b["cpu_baseline"]}


def run_single(args) -> int:
    """The default line: ADAM steps/s of the N = 1M packing."""
    import torch
    import torch.distributed as dist
    import rcpgenerator_b200 as rb

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    pos, dia, init = make_input(rank)
    n, nd = pos.shape
    run_cfg = {"box": init["box"], "walls": init["walls"], "device": local,
               "pair_precision": args.pair_precision}

    def early(precision, clocks=None):
        stream = torch.cuda.Stream()
        cfg = dict(run_cfg, pair_precision=precision)
        eng = rb.PackingEngine({"positions": pos, "diameters": dia}, cfg, {}, stream=stream.cuda_stream)
        eng.advance(args.warmup)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        return eng, timed_window(eng, stream, args.steps, clocks)

    # the headline window: early phase, the workload's stated (mixed) precision
    clocks = ClockSampler(local)
    eng, (ms, done_steps, launches, clk) = early(args.pair_precision, clocks)
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    bprof = eng.profile_build_kernel(reps=10)
    # without the late-phase windows the pair kernel is timed on this state
    prof = None if not args.no_late else eng.profile_pair_kernel(reps=20)
    res = eng.result(as_arrays=True)
    eng.close()
    # the same window in FP64 pair arithmetic
    other = "f64" if args.pair_precision == "mixed" else "mixed"
    eng2, (ms2, done2, _, _) = early(other)
    eng2.close()
    late = {}
    if not args.no_late:
        for prec in (args.pair_precision, other):
            late[prec], p = late_phase(rb, pos, dia, init, prec, local, args.late_steps)
            if prec == args.pair_precision:
                prof = p

    # end to end through the public API: host buffers in, results out
    torch.cuda.synchronize()
    e2e_steps, t_e2e = 0, 0.0
    if not args.no_e2e:
        t0 = time.perf_counter()
        r2 = rb.run_packing_observed({"positions": pos, "diameters": dia}, run_cfg,
                                     0, False, 0, None, {"max_steps": args.steps}, as_arrays=True)["result"]
        t_e2e = time.perf_counter() - t0
        e2e_steps = int(r2["steps"])

    batch = None
    if not args.no_batch and rank == 0:
        batch = batch_summary(args, local)

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return 0
    value = world * done_steps / (ms / 1e3)
    peak, peak_kind = hbm_peak()
    cpu = None
    if not args.no_cpu_baseline:
        s, why = reference_sample(pos, dia, init["box"], init["walls"], 1, args.cpu_sample_steps,
                                  os.cpu_count() or 1)
        if s is not None:
            cpu = {"value": s["steps_per_s"], "unit": UNIT, "cores": os.cpu_count(),
                   "kind": "reference",
                   "sample": f"steps {s['first']}..{s['last']} of the same packing on the reference "
                             f"engine (oracle/_ref), all host threads"}
        else:
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                   "sample": why}
    dtype = {"mixed": "f64 state, f32 pair terms", "f64": "f64"}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": done_steps,
        "warmup": args.warmup, "ms_per_step": ms / max(done_steps, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": dtype[args.pair_precision],
        "data": "synthetic",
        "config": bench_config(n, args.warmup, args.steps),
        "engine": {"mode": "graph (CUDA-graph step loop, controller on the GPU)",
                   "pair_precision": args.pair_precision,
                   "fp64_switch_step": int(res["engine_stats"]["fp64_switch_step"]),
                   "parallelism": f"replicas{world}",
                   "pair_builds": int(res["engine_stats"]["pair_builds"]),
                   "row_capacity": int(res["engine_stats"]["row_capacity"])},
        # the same window with the other pair precision (FP64 is the reference's precision)
        "other_precision": {"pair_precision": other, "dtype": dtype[other],
                            "value": done2 / (ms2 / 1e3), "unit": UNIT, "ms_per_step": ms2 / max(done2, 1)},
        "late_phase": late or None,
        # the step's dominant kernel in this window: every step rebuilds its
        # rows, and the tiled build computes that step's forces in the same pass
        "roofline": roofline_of(bprof, peak, peak_kind, "k_cells (cell-unit neighbour build + fused forces)",
                                BUILD_TRAFFIC_PER_ALG_BYTE),
        # the pair kernel of the steps without a rebuild (the reference's 81 % kernel),
        # on the state after the growth rung
        "roofline_pair_kernel": (roofline_of(prof, peak, peak_kind, "k_forces (pair energy/gradient, full rows)",
                                             FORCES_TRAFFIC_PER_ALG_BYTE) if prof else None),
        "cpu_baseline": cpu,
        "e2e": None if args.no_e2e else {"value": e2e_steps / t_e2e, "unit": UNIT,
                "h2d_bytes_per_step": int((n * (nd + 1) * 8) / max(e2e_steps, 1)),
                "d2h_bytes_per_step": int((n * (nd + 2) * 8 + e2e_steps * 6 * 8) / max(e2e_steps, 1)),
                "note": "run_packing_observed(max_steps=K) from host NumPy arrays: setup, K steps, results"},
        "batch": batch,
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


JAM_CONFIGS = {
    # the N = 1M 2-D bidisperse packing of the default line
    2: dict(phi=0.30, N=1_000_000, Ndim=2, box=[1.0, 1.0], walls=[0, 0],
            dist={"type": "bidisperse", "d1": 1.0, "d2": 1.4, "p": 0.5}, seed=123),
    # 3-D power law d^-3 on [0.1, 1] (size ratio 10) in a spherical container, N = 2M
    3: dict(phi=0.20, N=2_000_000, Ndim=3, box=[1.0, 1.0, 1.0], walls=[-3, 0, 0],
            dist={"type": "powerlaw", "d_min": 0.1, "d_max": 1.0, "exponent": -3.0}, seed=123),
}


def run_jam(args) -> int:
    """One packing run to the reference's convergence gate (pack()) in mixed
    and in FP64 pair precision: phi_J, steps, final max overlap, wall time and
    the mixed run's differences from the FP64 run."""
    import rcpgenerator_b200 as rb
    rank, _, local = dist_env()
    cfg = dict(JAM_CONFIGS[args.jam_config])
    if args.n != WORKLOAD["N"]:
        cfg["N"] = args.n
    t0 = time.perf_counter()
    init = rb.initialize_particles(cfg)
    t_init = time.perf_counter() - t0
    inp = {"positions": np.ascontiguousarray(init["positions"]),
           "diameters": np.ascontiguousarray(init["diameters"])}
    out = {"workload": f"config{args.jam_config}", "N": cfg["N"], "Ndim": cfg["Ndim"], "dist": cfg["dist"]["type"],
           "walls": cfg["walls"], "init_phi": cfg["phi"], "initializer_s": t_init}
    runs = {}
    for prec in ("mixed", "f64"):
        t0 = time.perf_counter()
        r = rb.run_packing_observed(inp, {"box": init["box"], "walls": init["walls"], "device": local,
                                          "pair_precision": prec}, 0, False, 0, None,
                                    {"max_steps": args.jam_max_steps}, as_arrays=True)["result"]
        dt = time.perf_counter() - t0
        st = r["engine_stats"]
        runs[prec] = r
        out[prec] = {"phi_J": float(r["phi"]), "steps": int(r["steps"]), "max_overlap": float(r["max_min_dist"]),
                     "force_magnitude": float(r["force_magnitude"]), "wall_s": dt, "steps_per_s": r["steps"] / dt,
                     "converged": bool(r["steps"] < args.jam_max_steps),
                     "pair_builds": int(st["pair_builds"]), "fp64_switch_step": int(st["fp64_switch_step"]),
                     "pair_energy_rel_error": float(st["pair_energy_rel_error"]),
                     "pair_force_rel_error": float(st["pair_force_rel_error"])}
    a, b = runs["mixed"], runs["f64"]
    out["mixed_vs_f64"] = {"delta_phi_J": float(a["phi"] - b["phi"]),
                           "delta_steps": int(a["steps"] - b["steps"]),
                           "delta_final_energy": float(a["energy_history"][-1] - b["energy_history"][-1])}
    if rank == 0:
        print(json.dumps(out))
    return 0


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cpu-sample-steps", type=int, default=12)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--no-late", action="store_true", help="skip the late-phase windows")
    ap.add_argument("--late-steps", type=int, default=2000)
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-workload sub-object")
    ap.add_argument("--bench-batch", type=int, default=512, help="packings in the default line's batch sample")
    ap.add_argument("--no-warm-start", action="store_true", help="batch workload: skip the warm-started arm")
    ap.add_argument("--warm-start-model", default=str(REPO / "rcpgenerator_b200" / "warmstart_model.npz"))
    ap.add_argument("--pair-precision", default="mixed", choices=["mixed", "f64"],
                    help="pair arithmetic: mixed = FP32 pair terms while the max overlap >= 1e-5 "
                         "(the workload's stated precision), f64 = FP64 throughout")
    ap.add_argument("--n", type=int, default=WORKLOAD["N"], help="particles (smaller cases for profiling)")
    ap.add_argument("--workload", default="single", choices=["single", "batch", "one", "jam"],
                    help="single: ADAM steps/s of one N=1M packing; batch: packings/hour of many small ones; "
                         "one: ADAM steps/s of packing --seed of the batch generator (profiling); "
                         "jam: one packing of --jam-config run to convergence in mixed and FP64 precision")
    ap.add_argument("--jam-config", type=int, default=2, choices=[2, 3])
    ap.add_argument("--jam-max-steps", type=int, default=400_000,
                    help="jam workload: step cap of each run (a run that reaches it did not converge)")
    ap.add_argument("--seed", type=int, default=4, help="one: generator seed (4: 4-D, N = 11,948)")
    ap.add_argument("--batch-count", type=int, default=128)
    ap.add_argument("--batch-stride", type=int, default=0,
                    help="batch: generator seeds k * stride (0: 4096 // count, a stratified sample of "
                         "seeds 0..4095)")
    ap.add_argument("--batch-single", type=int, default=8, help="packings timed one at a time")
    ap.add_argument("--save-training", default=None,
                    help="batch workload: write the plain runs' warm-start descriptors, targets and seeds (.npz)")
    ap.add_argument("--concurrency", type=int, default=0,
                    help="-1: persistent batch kernel; 0: persistent for small packings + 32 streams; k: k streams")
    ap.add_argument("--cpu-cap-steps", type=int, default=300)
    args = ap.parse_args()
    WORKLOAD["N"] = args.n
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "batch":
        return run_batch_workload(args)
    if args.workload == "one":
        return run_one_packing(args)
    if args.workload == "jam":
        return run_jam(args)
    return run_single(args)


if __name__ == "__main__":
    sys.exit(main())
