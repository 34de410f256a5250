"""Benchmark of the B200 r²HPDHG engine on the 1M x 1.5M random LP and the other workloads below.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload random1m|random10k|staircase8760|batch720x64|batch720x64f|batch10kx64f|serve48]
                    [--precision fp64|mixed] [--reductions exact|fast]
                    [--iterations L | --full]

One STEP is one cold solve of the seeded LP: setup (structure, scaling, ‖Ã‖₂), at most L = 640
r²HPDHG iterations (10 checks) and the finish (unscaling, KKT, z = c − Aᵀy, in-process check).
The metric is r²HPDHG iterations per second, whole job, over the K steps. Both arms run exactly
this step on the same LP (engine level, no presolve) and print the same `config`; the
reference's CPU engine takes about 12 s per step on the 1M LP, so L is what both can time.
`--full` drops the cap: a step is a complete solve to 1e-8 KKT and the metric is solves/s.

value: model resident in HBM before the timed region (ps26119_solve_lp_device), timed with CUDA
events on the solve's stream, max over ranks. e2e: the same steps through the reference-facing
C API (ps26119_solve_lp_ex, presolve and in-process check on) from pinned host buffers, the
model's host-to-device copy and the x, y, z device-to-host copy inside the timed region.
After the timed steps a single-GPU run adds (outside the timed region): `cpu_baseline`, one
step of the reference CPU engine; `reference_gpu`, the same step through the reference's own
CUDA backend built for sm_100a on this GPU; `time_to_tol`, measured wall-clock solves to 1e-8
through the C API (the 10k random LP in fp64 and mixed, the T = 8760 staircase LP in mixed),
the first also through the reference's CUDA backend.

torchrun (N > 1): every rank solves its own replica (a single LP does not shard; no collective
on the data path): weak scaling.

--impl reference: the reference's own CPU engine (built from its sources into oracle/_ref) on
all host threads through ps26119::solve, each step the same capped cold solve, timed on the
host clock; a single-GPU run adds its measured time to 1e-8 on the 10k random LP.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(ROOT, "ps26119-solver_b200"), os.path.join(ROOT, "oracle")]

WORKLOADS = {
    "random1m": {"desc": "random equality LP m=1,000,000 n=1,500,000 nnz=6,000,000 (6/row, N(0,1)), seed 1",
                 "kind": "random", "m": 1_000_000},
    "random10k": {"desc": "random equality LP m=10,000 n=15,000 nnz=60,000 (6/row, N(0,1)), seed 1",
                  "kind": "random", "m": 10_000},
    "staircase8760": {"desc": "staircase planning LP T=8760 (429,240 x 525,600), seed 1", "kind": "staircase",
                      "T": 8760},
    "batch720x64": {"desc": "64 scenarios (b, c x lognormal(0, 0.1)) of the staircase LP T=720 "
                            "(35,280 x 43,200, 126,024 nnz), seed 1", "kind": "batch", "T": 720, "K": 64},
    "batch720x64f": {"desc": "64 feasible scenarios of the staircase LP T=720 (35,280 x 43,200, 126,024 nnz): "
                             "interior point, slacks and c x lognormal(0, 0.1), seed 1", "kind": "batch", "T": 720,
                     "K": 64, "feasible": True},
    "batch10kx64f": {"desc": "64 feasible scenarios of the random equality LP m=10,000 n=15,000 (60,000 nnz): "
                             "x0, c x lognormal(0, 0.1), b = A x', seed 1", "kind": "batch", "base": "random",
                     "m": 10_000, "K": 64, "feasible": True},
    "serve48": {"desc": "48 LP requests from the random-LP generator, m log-uniform in [1e3, 2e4] (n = 1.5m, "
                        "6 nnz/row), Poisson arrivals, each solved to 1e-8 (a bounded sample of the "
                        "2,000-request stream with m up to 2e5), seed 1", "kind": "serve", "N": 48,
                "m_lo": 1_000, "m_hi": 20_000, "slots": 16},
}
# DRAM bytes per iteration (both fused kernels: dram__bytes_read.sum + dram__bytes_write.sum of
# one launch each) from the ncu capture summarised in the named profile.
NCU_TRAFFIC = {("random1m", "fp64"): (146.08e6 + 5.14e6) + (120.07e6 + 3.59e6)}
NCU_TRAFFIC_SOURCE = {("random1m", "fp64"): "profiles/k_slab_fed_random1m.md"}
# Measured to-tolerance solves a default single-LP run adds after its timed steps.
TIME_TO_TOL = [("random10k", "fp64"), ("random10k", "mixed"), ("staircase8760", "mixed")]


def make_lp(name):
    from ps26119 import generators as g
    w = WORKLOADS[name]
    random = w["kind"] == "random" or w.get("base") == "random"
    return g.random_lp(w["m"], seed=1) if random else g.staircase_lp(w["T"], seed=1)


def make_scenarios(name, lp):
    from ps26119 import generators as g
    make = g.feasible_scenarios if WORKLOADS[name].get("feasible") else g.scenarios
    return make(lp, WORKLOADS[name]["K"], sigma=0.1, seed=1)


def make_requests(name):
    from ps26119 import generators as g
    w = WORKLOADS[name]
    rng = np.random.default_rng(1)
    ms = np.exp(rng.uniform(np.log(w["m_lo"]), np.log(w["m_hi"]), w["N"])).astype(int)
    return [g.random_lp(int(m), seed=1000 + k) for k, m in enumerate(ms)]


def run_serve(args, rank, world, local):
    """The request loop (ps26119_server_*): one step = one stream of N requests arriving as a
    Poisson process, admitted by slots and HBM budget, each solved to 1e-8 (mixed precision with
    its fp64 polish, or fp64). value = served solves/s over the stream (first submission to last
    completion); latency = completion − submission. The sequential baseline is a sample of the
    same requests solved one at a time in plain fp64 through ps26119_solve_lp_ex; the arrival
    rate is slots × that sequential rate, so the device stays saturated."""
    import torch
    import ps26119
    torch.cuda.set_device(local)
    w = WORKLOADS[args.workload]
    reqs = make_requests(args.workload)
    N, slots = len(reqs), args.serve_slots or w["slots"]

    def alone(lp, precision="fp64"):
        return ps26119.solve_lp(lp.c, (lp.col_start, lp.row_index, lp.value), lp.row_lower, lp.row_upper,
                                lp.col_lower, lp.col_upper, sense=lp.sense, offset=lp.offset, algorithm="r2hpdhg",
                                precision=precision)

    alone(min(reqs, key=lambda lp: lp.num_rows))  # warm-up: first-call costs stay out
    S = min(N, args.serve_sample)
    # a size-stratified sample: every (N/S)-th request in order of size, so that the sequential
    # mean stands for the whole stream
    by_size = sorted(range(N), key=lambda k: reqs[k].num_rows)
    sample = [reqs[by_size[(2 * j + 1) * N // (2 * S)]] for j in range(S)]
    seq = []
    for lp in sample:
        t0 = time.perf_counter()
        r = alone(lp)
        seq.append(time.perf_counter() - t0)
        if r.status != ps26119.OPTIMAL:
            raise RuntimeError(f"sequential solve ended {r.status_name}")
    t_seq = max_over_ranks(float(np.mean(seq)), world)
    rate = world * slots / t_seq
    due = np.cumsum(np.random.default_rng(2).exponential(1.0 / rate, N))
    # several GPUs: every rank serves its share of the stream (longest first to the least-loaded
    # rank, by nonzeros), at the requests' own arrival times; no data crosses GPUs
    from ps26119 import shard
    mine = shard.assign(N, world, [lp.nnz for lp in reqs])[rank]
    steps = []
    with clock_sampler(local) as clocks:
        for _ in range(args.steps):
            barrier(world)
            t_create = time.perf_counter()  # the server's clock (request times) starts here
            with ps26119.Server(slots=slots, grouped=not args.serve_solo) as srv:
                t0 = time.perf_counter()
                ids = []
                for k in mine:
                    pause = due[k] - (time.perf_counter() - t0)
                    if pause > 0:
                        time.sleep(pause)
                    ids.append(srv.submit(reqs[k], precision=args.precision))
                out = [srv.result(i) for i in ids]
            bad = [f"{r.status_name} ({r.message})" for r, _ in out if r.status != ps26119.OPTIMAL or r.check != "PASS"]
            if bad:
                raise RuntimeError(f"{len(bad)} served solves failed, e.g. {bad[:3]}")
            sub = np.array([t[0] for _, t in out])
            fin = np.array([t[2] for _, t in out])
            start = np.array([t[1] for _, t in out])
            span = max_over_ranks(float(fin.max() - (t0 - t_create)) if len(out) else 0.0, world)
            got = shard.gather({k: (float(f - b), float(f - a), r.iterations)
                                for k, (r, _), b, a, f in zip(mine, out, sub, start, fin)}, world)
            steps.append((span, np.array([got[k][0] for k in range(N)]), [got[k][2] for k in range(N)],
                          np.array([got[k][1] for k in range(N)])))
    sec = float(np.mean([s[0] for s in steps]))
    lat = np.concatenate([s[1] for s in steps])
    svc = np.concatenate([s[3] for s in steps])
    value = N / sec
    h2d = sum(lp.nnz * 12 + (lp.num_cols + 1) * 4 + lp.num_cols * 24 + lp.num_rows * 16 for lp in reqs)
    d2h = sum(lp.num_cols * 16 + lp.num_rows * 8 for lp in reqs)
    unit = "solves/s"
    return {
        "metric": f"served LP solves/s on {args.workload} ({args.precision}, p50/p99 latency)", "value": value,
        "unit": unit, "n_gpus": world, "steps": args.steps, "warmup": 1, "ms_per_step": sec * 1e3,
        "higher_is_better": True, "scaling": "strong" if world > 1 else "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32+f64", "data": "synthetic (seeded generator)",
        "config": {"workload": w["desc"], "requests": N, "slots": slots, "precision": args.precision,
                   "tolerance": 1e-8, "arrival_rate_per_s": rate, "rows": [int(lp.num_rows) for lp in reqs],
                   "entry": "ps26119_server_submit / ps26119_server_poll (host arrays)",
                   "engines": "each request's own kernels" if args.serve_solo else
                              "grouped: one launch per half-step over every running request",
                   "cuda_device_max_connections": os.environ.get("CUDA_DEVICE_MAX_CONNECTIONS"),
                   "parallelism": f"requests sharded over {world} GPUs" if world > 1 else "1 GPU",
                   "l2": "many small LPs: L2-resident, latency-bound"},
        "latency_ms": {"p50": float(np.percentile(lat, 50) * 1e3), "p99": float(np.percentile(lat, 99) * 1e3),
                       "mean": float(lat.mean() * 1e3), "note": "submission to completion (queueing included)"},
        "service_ms": {"p50": float(np.percentile(svc, 50) * 1e3), "p99": float(np.percentile(svc, 99) * 1e3),
                       "note": "admission to completion"},
        "sequential_fp64": {"solves_per_s": 1.0 / t_seq, "speedup": value * t_seq / world,
                            "speedup_note": "per GPU: served solves/s / GPUs x the sequential solve time",
                            "sample": f"{S} of the requests (stratified by size) solved one at a time, plain "
                                      "fp64, ps26119_solve_lp_ex"},
        "iterations": steps[-1][2],
        "gpu_launches": None,
        "clocks": clocks.summary(),
        "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "note": "the server takes host arrays: every request's copies are inside the stream's time"},
    }


def cpu_model():
    """The host CPU's model name (for the CPU baseline's record), or None."""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def hbm_peak():
    """The measured HBM copy bandwidth (GB/s) and its source; the pool's earlier measurement,
    6,650 GB/s, when the measured file is absent."""
    try:
        peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))).get("hbm_gbs")
    except (OSError, ValueError):
        peak = None
    return (peak, "measured") if peak else (6650.0, "fallback")


def roofline_batch(lp, args, sec, results):
    """Kernel roofline of the batch's SpMM kernels (CUDA events over their launches in every
    epoch) against the measured HBM copy peak, and the whole-step figure beside it. Finished
    scenarios leave the lockstep batch (their slots are compacted away), so a lockstep iteration
    moves Ã and Ãᵀ once plus the vectors of the slots still running: over the last step,
    its_max·(2·nnz·(s_v + 4) + 4(m + n)) + Σ_k its_k·s_w·(9n + 7m) bytes, its_k being scenario
    k's iterations. Mixed precision is counted at 4-byte values and vectors throughout (its
    final fp64 stretch moves more), so its figure is a lower bound."""
    peak, peak_src = hbm_peak()
    res, st = results[-1]
    m, n, nnz = lp.num_rows, lp.num_cols, lp.nnz
    s_v = s_w = 4 if args.precision == "mixed" else 8
    its = [r.iterations for r in res]
    total = max(its) * (2 * nnz * (s_v + 4) + 4 * (m + n)) + sum(its) * s_w * (9 * n + 7 * m)
    bpi = total / max(1, max(its))
    kern_ms = st["spmv_kernel_ms"]
    pairs = max(1, st["spmv_kernel_launches"] // 2)
    out = {"bound": "hbm", "unit": "GB/s", "peak": peak, "peak_source": f"{peak_src} (MEASURED_PEAKS.json hbm_gbs)",
           "algorithmic_bytes": bpi, "traffic": None,
           "unit_of_work": "one lockstep iteration of the running slots: the two fused SpMM+update kernels "
                           "(algorithmic_bytes: the mean over the last step's lockstep iterations)",
           "achieved_whole_step": total * len(results) / sec / 1e9 if len(results) == args.steps else None,
           "note": "achieved: algorithmic bytes / live kernel time, last step; achieved_whole_step: every step's "
                   "bytes / step wall time"}
    if kern_ms > 0:
        out.update({"achieved": total / (kern_ms * 1e-3) / 1e9, "kernel_us_per_iteration": 1e3 * kern_ms / pairs})
        out["frac"] = out["achieved"] / peak
    return out


def run_batch(args, rank, world, local):
    """The shared-matrix batch (ps26119_solve_batch): one step = one batch solve of K scenarios
    from host arrays (the batch entry point takes host memory, so value and e2e are the same
    call); unit = scenario-iterations/s (or scenario solves/s with --full)."""
    import torch
    import ps26119
    torch.cuda.set_device(local)
    lp = make_lp(args.workload)
    scen_all = make_scenarios(args.workload, lp)
    # several GPUs: the scenarios are sharded over the ranks (each solves its share as one batch;
    # no data crosses GPUs), so the whole job is the same K scenarios: strong scaling
    from ps26119 import shard
    scen = [scen_all[k] for k in shard.assign(len(scen_all), world)[rank]]
    K = len(scen_all)
    limit = 0 if args.full else args.iterations
    A = (lp.col_start, lp.row_index, lp.value)

    def step():
        res = ps26119.solve_batch(lp.c, A, lp.row_lower, lp.row_upper, lp.col_lower, lp.col_upper, scenarios=scen,
                                  sense=lp.sense, offset=lp.offset, iteration_limit=limit, precision=args.precision)
        bad = [r.status_name for r in res if r.status_name not in ("Optimal", "IterationLimit")]
        if bad or (args.full and any(r.status_name != "Optimal" for r in res)):
            raise RuntimeError(f"batch ended {set(r.status_name for r in res)}")
        return res, ps26119.last_stats()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    results = []
    with clock_sampler(local) as clocks:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            results.append(step())
        torch.cuda.synchronize()
        sec = time.perf_counter() - t0
    sec = max_over_ranks(sec, world)
    res, st = results[-1]
    scen_its = sum_over_ranks(float(sum(r.iterations for r in res)), world)
    units = K * args.steps if args.full else scen_its * args.steps
    value = units / sec
    m, n, nnz = lp.num_rows, lp.num_cols, lp.nnz
    bpi = 2 * nnz * 12 + 4 * (m + n) + K * 8 * (9 * n + 7 * m)  # per lockstep iteration, all K slots
    unit = "scenario solves/s" if args.full else "scenario-iterations/s"
    its = max(r.iterations for r in res)
    line = {
        "metric": f"batched r2HPDHG on {args.workload} ({unit})", "value": value, "unit": unit, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "strong" if world > 1 else "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32+f64", "data": "synthetic (seeded generator)",
        "config": {"workload": WORKLOADS[args.workload]["desc"], "m": m, "n": n, "nnz": nnz, "scenarios": K,
                   "precision": args.precision,
                   "tolerance": 1e-8, "iteration_cap": limit or None, "entry": "ps26119_solve_batch (host arrays)",
                   "iterations_per_step": its, "parallelism": f"scenarios sharded over {world} GPUs" if world > 1 else "1 GPU",
                   "l2": f"inputs larger than L2: {bpi / 1e6:.0f} MB streamed per lockstep iteration"},
        "roofline": roofline_batch(lp, args, sec, results),
        "gpu_launches": int(sum(s["kernel_launches"] for _, s in results)),
        "clocks": clocks.summary(),
        "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": nnz * 12 + (n + 1) * 4 + K * 8 * (3 * n + 2 * m),
                "d2h_bytes_per_step": K * 8 * (2 * n + m), "note": "the batch entry point takes host arrays"},
    }
    if args.full:
        line["scenarios_optimal"] = sum(r.status_name == "Optimal" for r in res)
        line["iterations"] = {"max": its, "median": float(np.median([r.iterations for r in res]))}
        line["sequential_fp64"] = sequential_sample(args, lp, scen, value / world)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import reference
        cores = os.cpu_count() or 1
        if reference.available():
            t0 = time.perf_counter()
            w = reference.batch(lp, scen, threads=0, iteration_limit=args.cpu_sample_iterations)
            rs = time.perf_counter() - t0
            rits = max(x["iterations"] for x in w)
            line["cpu_baseline"] = {"value": K * rits / rs, "unit": "scenario-iterations/s", "cores": cores,
                                    "cpu_model": cpu_model(),
                                    "kind": "reference",
                                    "sample": f"reference solve_batch ({cores} threads), {rits} lockstep iterations "
                                              f"of {K} scenarios incl. setup in {rs:.1f} s"}
    return line


def sequential_sample(args, lp, scen, batched_rate):
    """Scenarios solved one at a time to 1e-8 in plain fp64 through the single-LP engine on the
    same GPU (ps26119_solve_lp_engine, no presolve): a sample of args.serve_sample scenarios,
    evenly spaced; the batch's speed-up is its solves/s times the mean sequential solve time."""
    import ps26119
    S = max(1, min(len(scen), args.serve_sample))
    pick = [scen[(2 * j + 1) * len(scen) // (2 * S)] for j in range(S)]
    times, its = [], []
    for sc in pick:
        t0 = time.perf_counter()
        r = ps26119.solve_lp(sc["obj"], (lp.col_start, lp.row_index, lp.value), sc["row_lower"], sc["row_upper"],
                             lp.col_lower, lp.col_upper, sense=lp.sense, offset=lp.offset, algorithm="r2hpdhg",
                             precision="fp64", engine={"presolve": False}, time_limit=1800)
        times.append(time.perf_counter() - t0)
        its.append(r.iterations)
        if r.status != ps26119.OPTIMAL:
            return {"note": f"sequential solve ended {r.status_name}: {r.message}"}
    t_seq = float(np.mean(times))
    return {"solves_per_s": 1.0 / t_seq, "speedup": batched_rate * t_seq, "iterations": its,
            "sample": f"{S} of the {len(scen)} scenarios (evenly spaced), each solved alone to 1e-8 in plain fp64, "
                      "ps26119_solve_lp_engine without presolve, same GPU"}


def bytes_per_iteration(m, n, nnz, s_v, s_w):
    """Algorithmic bytes of one r²HPDHG iteration: Ã and Ãᵀ streamed once (values + int32 column
    indices), int32 row pointers, and the vectors 9n + 7m in the working precision."""
    return 2 * nnz * (s_v + 4) + 4 * (m + n) + s_w * (9 * n + 7 * m)


class NvmlClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled every 200 ms during the timed region,
    in-process through NVML. Only clocks and reasons are queried: a full nvidia-smi query (power
    included) every 200 ms was measured to slow the engine's per-check synchronisations."""

    NAMES = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
             ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
             ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
             ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, gpu_index):
        import pynvml
        self.nv = pynvml
        pynvml.nvmlInit()
        count = pynvml.nvmlDeviceGetCount()
        self.h = pynvml.nvmlDeviceGetHandleByIndex(0 if count == 1 else gpu_index)
        self.samples = []
        self.stop = threading.Event()

    def _loop(self):
        nv = self.nv
        get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        while not self.stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                mx = nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM)
                self.samples.append((sm, mx, get_reasons(self.h)))
            except Exception:  # noqa: BLE001 - a failed query is just a missing sample
                pass
            self.stop.wait(0.2)

    def __enter__(self):
        self.thread = threading.Thread(target=self._loop, daemon=True)
        self.thread.start()
        return self

    def __exit__(self, *exc):
        self.stop.set()
        self.thread.join(timeout=5)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["not sampled"], "samples": 0}
        reasons = set()
        for _, _, bits in self.samples:
            for name, attr in self.NAMES:
                if bits & getattr(self.nv, attr, 0):
                    reasons.add(name)
        return {"sm_mhz": float(np.median([s[0] for s in self.samples])),
                "sm_max_mhz": float(max(s[1] for s in self.samples)), "reasons": sorted(reasons),
                "samples": len(self.samples), "source": "nvml"}


def clock_sampler(gpu_index):
    """NVML when it loads, else nvidia-smi."""
    try:
        return NvmlClockSampler(gpu_index)
    except Exception:  # noqa: BLE001 - no NVML: fall back to the nvidia-smi process
        return ClockSampler(gpu_index)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = str(gpu_index)
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", self.gpu], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for k, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(k)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["not sampled"], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=900))
    return rank, world, local


def max_over_ranks(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def metric_name(args):
    w = args.workload
    if args.full:
        return f"time-to-1e-8 KKT on {w} ({args.precision}) as solves/s"
    return f"r2HPDHG iterations/s on {w} ({args.precision}), cold solves capped at {args.iterations} iterations"


def shared_config(args, lp, world):
    """The `config` both arms print: the workload and what one step does, nothing arm-specific."""
    m, n, nnz = lp.num_rows, lp.num_cols, lp.nnz
    s = 4 if args.precision == "mixed" else 8
    return {"workload": WORKLOADS[args.workload]["desc"], "m": m, "n": n, "nnz": nnz, "tolerance": 1e-8,
            "precision": args.precision, "iteration_cap": None if args.full else args.iterations,
            "presolve": False, "parallelism": f"replicas x{world}",
            "l2": f"inputs larger than L2: {bytes_per_iteration(m, n, nnz, s, s) / 1e6:.0f} MB streamed per iteration"}


def run_ours(args, rank, world, local):
    import torch
    import ps26119
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    lp = make_lp(args.workload)
    m, n, nnz = lp.num_rows, lp.num_cols, lp.nnz
    t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=dev)
    arrs = [t(lp.c, torch.float64), t(lp.col_lower, torch.float64), t(lp.col_upper, torch.float64),
            t(lp.row_lower, torch.float64), t(lp.row_upper, torch.float64), t(lp.col_start, torch.int32),
            t(lp.row_index, torch.int32), t(lp.value, torch.float64)]
    ptrs = [a.data_ptr() for a in arrs]
    x = torch.empty(n, dtype=torch.float64, device=dev)
    y = torch.empty(m, dtype=torch.float64, device=dev)
    z = torch.empty(n, dtype=torch.float64, device=dev)
    stream = torch.cuda.Stream(device=dev)
    limit = 0 if args.full else args.iterations
    engine = {"presolve": False, "exact": args.reductions == "exact"}

    def step():
        r = ps26119.solve_lp_device(m, n, lp.sense, lp.offset, ptrs, precision=args.precision,
                                    iteration_limit=limit, engine=engine,
                                    out=(x.data_ptr(), y.data_ptr(), z.data_ptr()), stream=stream.cuda_stream)
        want = ps26119.OPTIMAL if args.full else (ps26119.OPTIMAL, ps26119.ITERATION_LIMIT)
        if (r.status != want) if args.full else (r.status not in want):
            raise RuntimeError(f"solve ended {r.status_name}: {r.message}")
        return r, ps26119.last_stats()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    results = []
    with clock_sampler(local) as clocks:
        torch.cuda.synchronize()
        evs[0].record(stream)
        for k in range(args.steps):
            results.append(step())
            evs[k + 1].record(stream)
        torch.cuda.synchronize()
    ms = max_over_ranks(evs[0].elapsed_time(evs[-1]), world)
    step_ms = [evs[k].elapsed_time(evs[k + 1]) for k in range(args.steps)]
    barrier(world)
    r, st = results[-1]
    iters = int(sum(rr.iterations for rr, _ in results))
    units = args.steps if args.full else iters
    value = world * units / (ms / 1e3)
    s_v = s_w = 4 if args.precision == "mixed" else 8
    bpi = bytes_per_iteration(m, n, nnz, s_v, s_w)
    kern_ms = sum(s["spmv_kernel_ms"] for _, s in results)
    kern_pairs = max(1, sum(s["spmv_kernel_launches"] for _, s in results) // 2)
    iter_ms = kern_ms / kern_pairs
    peak, peak_src = hbm_peak()
    achieved = bpi / (iter_ms * 1e-3) / 1e9
    line = {
        "metric": metric_name(args), "value": value, "unit": "solves/s" if args.full else "iterations/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32+f64", "data": "synthetic (seeded generator)",
        "config": shared_config(args, lp, world),
        "entry": "ps26119_solve_lp_device (model resident in HBM, engine level, no presolve)",
        "reductions": args.reductions,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": NCU_TRAFFIC.get((args.workload, args.precision)),
                     "traffic_source": NCU_TRAFFIC_SOURCE.get((args.workload, args.precision)),
                     "peak_source": f"{peak_src} (MEASURED_PEAKS.json hbm_gbs)",
                     "unit_of_work": "one r2HPDHG iteration: the two fused SpMV+update kernels",
                     "algorithmic_bytes": bpi, "kernel_us_per_iteration": iter_ms * 1e3,
                     "timing": "CUDA events recorded inside the epoch graphs on the solve's stream, all timed steps"},
        "step_ms": step_ms,
        "step_engine_ms": [1e3 * rr.seconds for rr, _ in results],
        "gpu_launches": int(sum(s["kernel_launches"] for _, s in results)),
        "clocks": clocks.summary(),
        "solve": {"status": r.status_name, "iterations": r.iterations, "objective": r.objective,
                  "primal_residual": r.primal_residual, "dual_residual": r.dual_residual, "gap": r.gap,
                  "check": r.check, "setup_s": st["setup_seconds"], "loop_s": st["loop_seconds"],
                  "finish_s": st["finish_seconds"], "checks": st["checks"], "restarts": st["restarts"],
                  "slab_variants": {"primal": st["slab_variant_primal"], "dual": st["slab_variant_dual"]}},
    }
    g = gather_ceiling(lp.num_rows if args.workload.startswith("random") else None, lp)
    if g:  # the second ceiling: 2·nnz random gathers of x̄ / y per iteration
        achieved_g = 2 * lp.nnz / (iter_ms * 1e-3)
        line["roofline"]["gather"] = {"achieved_gathers_per_s": achieved_g, "peak_gathers_per_s": g["gathers_per_s"],
                                      "frac": achieved_g / g["gathers_per_s"],
                                      "peak_source": "measured live by bench_gather_rate (random 8-byte gathers "
                                                     f"of a {lp.num_cols:,}-element vector resident in L2)"}
    if not args.no_e2e:
        line["e2e"] = run_e2e(args, lp, world, limit)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = reference_sample(args, lp)
    if rank == 0 and world == 1 and not args.no_reference_gpu and not args.full:
        line["reference_gpu"] = reference_gpu_sample(args, lp, value)
    if rank == 0 and world == 1 and not args.no_time_to_tol and not args.full:
        del arrs, x, y, z
        line["time_to_tol"] = time_to_tol_records(args)
    return line


def reference_gpu_sample(args, lp, ours):
    """The reference's own CUDA backend (src/gpu/cuda_backend.cu built for sm_100a, Options::use_gpu)
    on the same LP and cap, same GPU, one untimed warm-up then two timed cold solves (wall clock,
    setup included, as our step)."""
    import reference
    if not reference.available_gpu():
        return {"value": None, "note": "reference CUDA library not built (make -C oracle ref_gpu)"}
    runs = []
    for k in range(3):
        t0 = time.perf_counter()
        s = reference.solve(lp, presolve=False, precision=args.precision, threads=0,
                            iteration_limit=args.iterations, gpu=True)
        sec = time.perf_counter() - t0
        if s.status not in ("IterationLimit", "Optimal"):
            return {"value": None, "note": f"reference GPU solve ended {s.status}: {s.message}"}
        if k:
            runs.append((sec, s))
    wall = sum(r[0] for r in runs)
    its = sum(r[1].iterations for r in runs)
    loop = sum(r[1].seconds - r[1].setup_seconds for r in runs)
    value = its / wall
    return {"value": value, "unit": "iterations/s", "ms_per_step": 1e3 * wall / len(runs),
            "loop_iterations_per_s": its / loop, "setup_s": runs[-1][1].setup_seconds,
            "ms_per_iteration_loop": 1e3 * loop / its, "ours_over_reference_gpu": ours / value,
            "kind": "the reference's CUDA backend (src/gpu/cuda_backend.cu, its k_spmv_subwarp SpMV and "
                    "update kernels) built for sm_100a, driven by its own r2HPDHG loop (host setup and checks)"}


def time_to_tol_records(args, cases=None):
    """Measured time to 1e-8 KKT, one cold call of ps26119_solve_lp_ex each (presolve, the engine,
    the in-process check and the certified bound), wall clock, on the named LPs; the 10k LP also
    through the reference's own CUDA backend on the same GPU. Outside the timed steps.
    `cases`: (workload, precision) pairs, default TIME_TO_TOL."""
    import ps26119
    out = []
    last = None
    for case in cases or TIME_TO_TOL:
        name, precision = case[0], case[1]
        stall = int(case[2]) if len(case) > 2 else 0  # mixed: the precision switch's stall window
        lp = last[1] if last and last[0] == name else make_lp(name)
        last = (name, lp)
        t0 = time.perf_counter()
        r = ps26119.solve_lp(lp.c, (lp.col_start, lp.row_index, lp.value), lp.row_lower, lp.row_upper,
                             lp.col_lower, lp.col_upper, sense=lp.sense, offset=lp.offset, algorithm="r2hpdhg",
                             precision=precision, time_limit=1800,
                             engine={"presolve": True, "mixed_stall_checks": stall} if stall else None)
        sec = time.perf_counter() - t0
        st = ps26119.last_stats()
        rec = {"workload": name, "precision": precision, "seconds": sec, "status": r.status_name,
               "mixed_stall_checks": stall or None,
               "iterations": r.iterations, "switch_iteration": st["switch_iteration"],
               "engine_loop_s": st["loop_seconds"], "objective": r.objective, "certified_bound": r.certified_bound,
               "error_to_certified_bound": abs(r.objective - r.certified_bound) / (1.0 + abs(r.objective)),
               "rel_kkt": max(r.primal_residual, r.dual_residual, r.gap), "check": r.check,
               "entry": "ps26119_solve_lp_ex (presolve, engine, in-process check, certified bound)"}
        if name == "random10k" and precision == "fp64" and not args.no_reference_gpu:
            import reference
            if reference.available_gpu():
                t0 = time.perf_counter()
                s = reference.solve(lp, presolve=True, precision=precision, threads=0, gpu=True, time_limit=900)
                rec["reference_gpu"] = {"seconds": time.perf_counter() - t0, "status": s.status,
                                        "iterations": s.iterations, "objective": s.objective,
                                        "entry": "reference ps26119::solve, use_gpu (its CUDA backend), presolve"}
        out.append(rec)
    return out


def gather_ceiling(m, lp):
    """Runs bench_gather_rate (built by __graft_entry__.build()) for this matrix's shape: random gathers from
    an n-element vector, nnz of them. None when the program is absent or fails."""
    exe = os.path.join(ROOT, "bench_gather_rate")
    if m is None or not os.path.exists(exe):
        return None
    try:
        r = subprocess.run([exe, str(lp.num_cols), str(lp.nnz)], capture_output=True, text=True, timeout=120)
        return json.loads(r.stdout.strip().splitlines()[-1]) if r.returncode == 0 else None
    except (subprocess.SubprocessError, ValueError, IndexError):
        return None


def run_e2e(args, lp, world, limit):
    import torch
    import ps26119
    pin = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), dtype=dt).pin_memory().numpy()
    c, cl, cu = pin(lp.c, torch.float64), pin(lp.col_lower, torch.float64), pin(lp.col_upper, torch.float64)
    rl, ru = pin(lp.row_lower, torch.float64), pin(lp.row_upper, torch.float64)
    cs, ri, v = pin(lp.col_start, torch.int32), pin(lp.row_index, torch.int32), pin(lp.value, torch.float64)
    iters = 0
    if args.warmup > 0:  # one untimed call: first-call costs (host allocations, caches) stay out
        ps26119.solve_lp(c, (cs, ri, v), rl, ru, cl, cu, sense=lp.sense, offset=lp.offset, algorithm="r2hpdhg",
                         precision=args.precision, iteration_limit=limit)
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        r = ps26119.solve_lp(c, (cs, ri, v), rl, ru, cl, cu, sense=lp.sense, offset=lp.offset, algorithm="r2hpdhg",
                             precision=args.precision, iteration_limit=limit)
        if r.status not in (ps26119.OPTIMAL, ps26119.ITERATION_LIMIT):
            raise RuntimeError(f"e2e solve ended {r.status_name}: {r.message}")
        iters += r.iterations
    sec = max_over_ranks(time.perf_counter() - t0, world)
    h2d = lp.nnz * 12 + (lp.num_cols + 1) * 4 + lp.num_cols * 24 + lp.num_rows * 16
    d2h = lp.num_cols * 16 + lp.num_rows * 8
    units = args.e2e_steps if args.full else iters
    return {"value": world * units / sec, "unit": "solves/s" if args.full else "iterations/s",
            "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps": args.e2e_steps,
            "entry": "ps26119_solve_lp_ex (presolve + in-process check)", "ms_per_step": sec * 1e3 / args.e2e_steps,
            "iterations_per_step": iters // max(1, args.e2e_steps), "check": r.check}


def reference_sample(args, lp):
    """The reference CPU engine on this workload: one cold solve with the same iteration cap
    (engine level, no presolve) on all host threads, wall clock (a bounded sample, 10-15 s)."""
    import reference
    cores = os.cpu_count() or 1
    if not reference.available():
        return {"value": None, "unit": "iterations/s", "cores": cores, "cpu_model": cpu_model(), "kind": "reference",
                "sample": "reference library not built"}
    t0 = time.perf_counter()
    s = reference.solve(lp, presolve=False, precision=args.precision, threads=0,
                        iteration_limit=0 if args.full else args.iterations)
    sec = time.perf_counter() - t0
    return {"value": (1.0 if args.full else s.iterations) / sec, "unit": "solves/s" if args.full else "iterations/s",
            "cores": cores, "cpu_model": cpu_model(), "kind": "reference",
            "sample": f"reference ps26119::solve (r2hpdhg, no presolve, {cores} threads): one cold solve of "
                      f"{s.iterations} iterations in {sec:.1f} s (setup {s.setup_seconds:.2f} s)"}


def run_reference(args, rank, world):
    if rank != 0:
        return None
    import reference
    if not reference.available():
        return {"impl": "reference", "unavailable": "reference library oracle/_ref was not built on this machine"}
    if WORKLOADS[args.workload]["kind"] == "serve":
        return {"impl": "reference", "unavailable": "the reference solves the 48 requests to 1e-8 one at a time on "
                "the CPU (about a minute per request); no bounded sample of a latency stream is meaningful"}
    lp = make_lp(args.workload)
    cores = os.cpu_count() or 1
    if WORKLOADS[args.workload]["kind"] == "batch":
        if args.full:
            return {"impl": "reference", "unavailable": "--full batch: the reference CPU batch to 1e-8 takes hours"}
        scen = make_scenarios(args.workload, lp)
        K = len(scen)
        times, its = [], 0
        for i in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            w = reference.batch(lp, scen, threads=0, iteration_limit=args.cpu_sample_iterations)
            sec = time.perf_counter() - t0
            if i >= args.warmup:
                times.append(sec)
                its += K * max(x["iterations"] for x in w)
        value = its / sum(times)
        unit = "scenario-iterations/s"
        sample = (f"reference solve_batch ({cores} threads): {args.cpu_sample_iterations} lockstep iterations of "
                  f"{K} scenarios incl. setup per step")
        return {"metric": f"batched r2HPDHG on {args.workload} ({unit})", "value": value, "unit": unit,
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(times)),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded generator)",
                "config": {"workload": WORKLOADS[args.workload]["desc"], "scenarios": K, "tolerance": 1e-8},
                "impl": "reference",
                "cpu_baseline": {"value": value, "unit": unit, "cores": cores, "cpu_model": cpu_model(), "kind": "reference", "sample": sample},
                "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    # one step = one cold solve of the LP capped at the same iteration count as our arm (setup,
    # iterations, finish), timed on the host clock
    times, its = [], 0
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        s = reference.solve(lp, presolve=False, precision=args.precision, threads=0,
                            iteration_limit=0 if args.full else args.iterations)
        sec = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(sec)
            its += s.iterations
    value = (args.steps if args.full else its) / sum(times)
    unit = "solves/s" if args.full else "iterations/s"
    sample = (f"reference ps26119::solve (r2hpdhg, no presolve, {cores} threads): each step one cold solve "
              f"capped at {args.iterations} iterations, setup {s.setup_seconds:.2f} s of {times[-1]:.1f} s")
    line = {"metric": metric_name(args), "value": value, "unit": unit, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(times)), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
            "data": "synthetic (seeded generator)", "config": shared_config(args, lp, world),
            "entry": "reference ps26119::solve (its CPU engine, all host threads)", "impl": "reference",
            "cpu_baseline": {"value": value, "unit": unit, "cores": cores, "cpu_model": cpu_model(),
                             "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if world == 1 and not args.no_time_to_tol and not args.full:
        lp10 = make_lp("random10k")
        t0 = time.perf_counter()
        r = reference.solve(lp10, presolve=True, precision="fp64", threads=0, time_limit=900)
        line["time_to_tol"] = [{"workload": "random10k", "precision": "fp64", "seconds": time.perf_counter() - t0,
                                "status": r.status, "iterations": r.iterations, "objective": r.objective,
                                "entry": f"reference ps26119::solve (CPU engine, presolve, {cores} threads)"}]
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="random1m")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--reductions", choices=["exact", "fast"], default="fast",
                    help="exact: every sum in the reference's order; fast: fixed-order trees")
    ap.add_argument("--iterations", type=int, default=640, help="iteration cap of one step (both arms)")
    ap.add_argument("--full", action="store_true", help="solve to 1e-8 in every step")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-sample-iterations", type=int, default=256)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true", help="skip the reference CUDA backend's sample")
    ap.add_argument("--no-time-to-tol", action="store_true", help="skip the measured time-to-1e-8 records")
    ap.add_argument("--time-to-tol", default="",
                    help="only the time-to-1e-8 records of these comma-separated workload:precision[:stall] "
                         "cases (e.g. random1m:fp64,random1m:mixed:100; stall = the mixed precision switch's "
                         "stall window in checks, default the reference's 10); no timed steps")
    ap.add_argument("--serve-sample", type=int, default=8, help="requests solved sequentially for the baseline")
    ap.add_argument("--serve-slots", type=int, default=0, help="server slots (0: the workload's)")
    ap.add_argument("--serve-solo", action="store_true",
                    help="each served request launches its own kernels (no grouped launches)")
    args = ap.parse_args()
    if WORKLOADS[args.workload]["kind"] == "serve":
        # one hardware work queue per slot (the default, 8, makes streams beyond 8 share queues);
        # read when the CUDA context is created, so it is set before anything touches CUDA
        os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
    rank, world, local = dist_setup()
    if args.time_to_tol:
        import torch
        torch.cuda.set_device(local)
        cases = [tuple(c.split(":")) for c in args.time_to_tol.split(",")]
        bad = [c for c in cases if len(c) not in (2, 3) or c[0] not in WORKLOADS or c[1] not in ("fp64", "mixed")
               or (len(c) == 3 and not c[2].isdigit())]
        if bad:
            raise SystemExit(f"--time-to-tol: bad case(s) {bad}")
        line = {"time_to_tol": time_to_tol_records(args, cases)} if rank == 0 else None
    elif args.impl == "reference":
        line = run_reference(args, rank, world)
    elif WORKLOADS[args.workload]["kind"] == "batch":
        line = run_batch(args, rank, world, local)
    elif WORKLOADS[args.workload]["kind"] == "serve":
        line = run_serve(args, rank, world, local)
    else:
        line = run_ours(args, rank, world, local)
    if rank == 0 and line is not None:
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
