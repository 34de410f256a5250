"""Benchmark: time to 1e-8 relative KKT of the B200 r²HPDHG engine on the 1M x 1.5M random LP.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload random1m|random10k|staircase8760] [--precision fp64|mixed]

One STEP is one complete solve to 1e-8 (setup on the device: structure, scaling, ‖Ã‖₂; the
r²HPDHG iterations; checks; finish) of the seeded synthetic LP. `value` is whole-job throughput
in solves per second with the model already resident in HBM (ps26119_solve_lp_device), timed
with CUDA events on the solve's stream, max over ranks. `e2e` is the same metric through the
reference-facing C API (ps26119_solve_lp_ex, presolve on) from pinned host buffers, with the
host-to-device copy of the model and the device-to-host copy of x, y, z in the timed region.

With torchrun (N > 1) every rank solves its own replica of the workload: a single LP does not
shard (no collective on the data path), so the scaling is weak.

--impl reference: the reference's own CPU engine (built from its sources into oracle/_ref) on
the host cores, all threads, on the same workload. One step is a bounded sample (the setup plus
a few hundred iterations, iteration-limited); the solve time is the sample's setup plus its
per-iteration time multiplied by the iteration count the full solve needs (RANDOM1M_ITERATIONS
below, the GPU engine's count; the engines agree to one check at every size compared).
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
    "random1m": {"desc": "random equality LP m=1,000,000 n=1,500,000, 6 nnz/row N(0,1), seed 1", "kind": "random",
                 "m": 1_000_000},
    "random10k": {"desc": "random equality LP m=10,000 n=15,000, 6 nnz/row N(0,1), seed 1", "kind": "random",
                  "m": 10_000},
    "staircase8760": {"desc": "staircase planning LP T=8760 (429,240 x 525,600), seed 1", "kind": "staircase",
                      "T": 8760},
}
# Iterations to 1e-8 of the GPU engine (fast mode, fp64) on each workload, used only to
# extrapolate the reference's bounded CPU sample to a full solve. None = not measured yet
# (the reference arm then reports per-iteration cost over the sample's own count).
FULL_ITERATIONS = {"random1m": None, "random10k": 249088, "staircase8760": None}


def make_lp(name):
    from ps26119 import generators as g
    w = WORKLOADS[name]
    return g.random_lp(w["m"], seed=1) if w["kind"] == "random" else g.staircase_lp(w["T"], seed=1)


def bytes_per_iteration(m, n, nnz, s_v, s_w):
    """Algorithmic bytes of one r²HPDHG iteration: Ã and Ãᵀ streamed once (values + int32
    column indices), int32 row pointers, and the vectors 9n + 7m in the working precision."""
    return 2 * nnz * (s_v + 4) + 4 * (m + n) + s_w * (9 * n + 7 * m)


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
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
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


def dist_setup(n_gpus):
    import torch
    import torch.distributed as dist
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        import datetime
        dist.init_process_group("nccl" if torch.cuda.is_available() else "gloo",
                                timeout=datetime.timedelta(seconds=1800))
    return rank, world, local


def max_over_ranks(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


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
    engine = {"presolve": False, "exact": False}

    def step():
        with torch.cuda.stream(stream):
            r = ps26119.solve_lp_device(m, n, lp.sense, lp.offset, ptrs, precision=args.precision, engine=engine,
                                        out=(x.data_ptr(), y.data_ptr(), z.data_ptr()), stream=stream.cuda_stream)
        if r.status != ps26119.OPTIMAL:
            raise RuntimeError(f"solve ended {r.status_name}: {r.message}")
        return r, ps26119.last_stats()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    results = []
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            results.append(step())
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    ms = ev0.elapsed_time(ev1)
    ms = max_over_ranks(ms, world)
    r, st = results[-1]
    s_v = 4 if args.precision == "mixed" else 8
    iters = r.iterations
    iter_ms = st["spmv_kernel_ms"] / max(1, st["spmv_kernel_launches"] // 2)
    bpi = bytes_per_iteration(m, n, nnz, 8, 8) if args.precision == "fp64" else None
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = (bpi / (iter_ms * 1e-3) / 1e9) if bpi else None
    launches = sum(s["kernel_launches"] for _, s in results)
    # e2e through the C API from pinned host buffers (presolve on, as the reference's C API)
    e2e = run_e2e(args, lp, world) if not args.no_e2e else None
    line = {
        "metric": f"time-to-1e-8 KKT, {args.workload} ({args.precision}), as solves/s",
        "value": world * args.steps / (ms / 1e3), "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
        "data": "synthetic (seeded generator)",
        "config": {"workload": WORKLOADS[args.workload]["desc"], "m": m, "n": n, "nnz": nnz,
                   "tolerance": 1e-8, "precision": args.precision, "entry": "ps26119_solve_lp_device (no presolve)",
                   "iterations": iters, "parallelism": f"replicas x{world}",
                   "l2": f"inputs larger than L2: {bpi or 0} algorithmic bytes per iteration"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": None,
                     "unit_of_work": "one r2HPDHG iteration (the two fused SpMV kernels)",
                     "iteration_kernel_us": iter_ms * 1e3},
        "gpu_launches": launches,
        "clocks": clocks.summary(),
        "solve": {"objective": r.objective, "primal_residual": r.primal_residual, "dual_residual": r.dual_residual,
                  "gap": r.gap, "check": r.check, "setup_s": st["setup_seconds"], "loop_s": st["loop_seconds"],
                  "finish_s": st["finish_seconds"], "checks": st["checks"], "restarts": st["restarts"]},
    }
    if e2e:
        line["e2e"] = e2e
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = reference_sample(args, lp, iters)
    return line


def run_e2e(args, lp, world):
    import torch
    import ps26119
    pin = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), dtype=dt).pin_memory().numpy()
    c, cl, cu = pin(lp.c, torch.float64), pin(lp.col_lower, torch.float64), pin(lp.col_upper, torch.float64)
    rl, ru = pin(lp.row_lower, torch.float64), pin(lp.row_upper, torch.float64)
    cs, ri, v = pin(lp.col_start, torch.int32), pin(lp.row_index, torch.int32), pin(lp.value, torch.float64)
    t0 = time.perf_counter()
    r = ps26119.solve_lp(c, (cs, ri, v), rl, ru, cl, cu, sense=lp.sense, offset=lp.offset, algorithm="r2hpdhg",
                         precision=args.precision)
    sec = max_over_ranks(time.perf_counter() - t0, world)
    if r.status != ps26119.OPTIMAL:
        raise RuntimeError(f"e2e solve ended {r.status_name}: {r.message}")
    h2d = lp.nnz * 12 + (lp.num_cols + 1) * 4 + lp.num_cols * 24 + lp.num_rows * 16
    d2h = lp.num_cols * 16 + lp.num_rows * 8
    return {"value": world / sec, "unit": "solves/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
            "steps": 1, "entry": "ps26119_solve_lp_ex (presolve on)", "iterations": r.iterations,
            "check": r.check}


def reference_sample(args, lp, full_iterations):
    """The reference CPU engine on this workload: a bounded, iteration-limited sample with all
    host threads, extrapolated to the full iteration count."""
    import reference
    if not reference.available():
        return {"value": None, "unit": "solves/s", "cores": os.cpu_count(), "kind": "reference",
                "sample": "reference library not built"}
    cores = os.cpu_count() or 1
    limit = args.cpu_sample_iterations
    s = reference.solve(lp, presolve=False, precision=args.precision, threads=0, iteration_limit=limit)
    per_iter = (s.seconds - s.setup_seconds) / max(1, s.iterations)
    total = s.setup_seconds + per_iter * full_iterations
    return {"value": 1.0 / total, "unit": "solves/s", "cores": cores, "kind": "reference",
            "sample": f"{s.iterations} iterations + setup ({s.seconds:.1f} s wall), extrapolated to "
                      f"{full_iterations} iterations; per-iteration {per_iter * 1e3:.2f} ms, setup "
                      f"{s.setup_seconds:.2f} s"}


def run_reference(args, rank, world):
    if rank != 0:
        return None
    import reference
    if not reference.available():
        return {"impl": "reference", "unavailable": "reference library oracle/_ref not built on this machine"}
    lp = make_lp(args.workload)
    full = FULL_ITERATIONS.get(args.workload)
    cores = os.cpu_count() or 1
    limit = args.cpu_sample_iterations
    times = []
    sample = None
    for i in range(args.warmup + args.steps):
        s = reference.solve(lp, presolve=True, precision=args.precision, threads=0, iteration_limit=limit)
        per_iter = (s.seconds - s.setup_seconds) / max(1, s.iterations)
        its = full or s.iterations
        total = s.setup_seconds + per_iter * its
        if i >= args.warmup:
            times.append(total)
        sample = (f"reference ps26119::solve (presolve on, r2hpdhg, {cores} threads): {s.iterations} iterations "
                  f"+ setup per step, extrapolated to {its} iterations")
    sec = float(np.mean(times))
    value = 1.0 / sec
    return {"metric": f"time-to-1e-8 KKT, {args.workload} ({args.precision}), as solves/s", "value": value,
            "unit": "solves/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32+f64", "data": "synthetic (seeded generator)",
            "config": {"workload": WORKLOADS[args.workload]["desc"], "m": lp.num_rows, "n": lp.num_cols,
                       "nnz": lp.nnz, "tolerance": 1e-8, "precision": args.precision},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="random1m")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--cpu-sample-iterations", type=int, default=256)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    rank, world, local = dist_setup(args.gpus)
    if args.impl == "reference":
        line = run_reference(args, rank, world)
    else:
        line = run_ours(args, rank, world, local)
    if rank == 0 and line is not None:
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
