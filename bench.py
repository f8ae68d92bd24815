#!/usr/bin/env python
"""Benchmark of the PDHG hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Default workload (N=1): the single large LP — m = 2,000,000 rows, n = 4,000,000 columns,
40,000,000 nonzeros, column degrees from a Zipf(1.5) law on [2, 5000] rescaled to the
nonzero total, N(0,1) values, rows/bounds/cost as the random LP recipe (seeded synthetic
data). A step is one epoch of 64 PDHG iterations (the reference's check interval) with
its termination/restart check. `value` is PDHG iterations per second of the plain FP64
form, device-resident (inputs in HBM before the timed region); the mixed FP32-SpMV/FP64-
state form is reported beside it. `e2e` times the public one-call API (sp_solve) from
pinned host arrays to the solution back on the host, for K·64 iterations. The matrices
(≥ 1.2 GB) are far larger than the 126 MB L2, so no flush is needed between steps.
On one GPU the line also carries, under `forms`, both forms solved to 1e-6 end to end
(checked by the independent checker), the batched form on the 4096-LP batch and a compact
serving run (48 requests of up to 1e6 nonzeros); `--no-tolerance`, `--no-batch` and
`--no-serve` leave them out.

Other workloads (one JSON line each): transport (2000 x 2000 transportation LP),
batch (the 4096-LP uneven batch, solves/s), serve (Poisson arrivals, p50/p99 latency).

With --gpus N > 1 (launched by torchrun) every rank runs an independent replica of the
workload on its own GPU ("replicas only": the single-GPU path has no exchange step);
times are the max over ranks and `value` sums the ranks' work.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

ITERS_PER_STEP = 64
HBM_FALLBACK_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["powerlaw", "transport", "batch", "serve"], default="powerlaw")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--scale", type=float, default=1.0,
                    help="shrink the power-law LP's m, n and nnz by this factor (profiling runs only)")
    ap.add_argument("--tolerance", type=float, default=1e-6, help="relative KKT target of the to-tolerance solves")
    ap.add_argument("--tolerance-limit-s", type=float, default=300.0, help="time limit of each to-tolerance solve")
    ap.add_argument("--no-tolerance", action="store_true", help="skip the solves to the tolerance")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-form section of the default line")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving section of the default line")
    return ap.parse_args()


# ------------------------------------------------------------------ distributed plumbing

class Dist:
    def __init__(self, n_gpus: int):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist

            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            backend = "nccl"
            try:
                import torch

                torch.cuda.set_device(self.local)
            except Exception:
                backend = "gloo"
            dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
            self.pg = dist
            self.device = f"cuda:{self.local}" if backend == "nccl" else "cpu"

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, v: float) -> float:
        if not self.pg:
            return v
        import torch

        t = torch.tensor([v], dtype=torch.float64, device=self.device)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ------------------------------------------------------------------ clocks during the timed region

class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def settle(self, timeout_s: float = 3.0):
        """Waits until the sampler has written its first line (or `timeout_s`), so that
        starting nvidia-smi does not overlap the work it is sampling."""
        import select

        if not self.proc or not self.proc.stdout:
            return
        r, _, _ = select.select([self.proc.stdout], [], [], timeout_s)
        if r:
            self.proc.stdout.readline()  # a sample taken before the timed work: not kept

    def __exit__(self, *a):
        self.lines = []
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return HBM_FALLBACK_GBS, "fallback"


def profiled_traffic(kernel: str, workload: str, form: str):
    """DRAM bytes per launch of `kernel` on this exact workload and form, from the committed
    ncu summary (a line 'dram_bytes_per_launch <kernel> <workload> <form> <bytes>' in
    profiles/ncu_traffic.txt); None when no capture covers it."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    try:
        for line in open(path):
            f = line.split()
            if len(f) >= 5 and f[0] == "dram_bytes_per_launch" and f[1:4] == [kernel, workload, form]:
                return float(f[4])
    except OSError:
        pass
    return None


# ------------------------------------------------------------------ workloads

POWERLAW = (2_000_000, 4_000_000, 40_000_000)


def powerlaw_shape(scale: float = 1.0):
    return tuple(int(round(v * scale)) for v in POWERLAW)


def powerlaw_lp(seed: int, scale: float = 1.0):
    import saddlepoint_b200 as sp

    m, n, nnz = powerlaw_shape(scale)
    return sp.generate_powerlaw_lp(seed, m, n, nnz, 1.5, 2, 5000)


def workload_key(workload: str, scale: float = 1.0) -> str:
    """The name a profile capture is filed under: the workload at its full-launch size."""
    if workload == "powerlaw":
        m, n, nnz = powerlaw_shape(scale)
        return f"powerlaw_m{m}_n{n}_nnz{nnz}"
    return "transport_2000x2000"


WORKLOAD_DESC = {
    "powerlaw": {"workload": "single large LP, power-law columns", "m": 2_000_000, "n": 4_000_000,
                 "nnz": 40_000_000, "column_degrees": "Zipf(1.5) on [2,5000] rescaled to 40M", "values": "N(0,1)",
                 "iterations_per_step": ITERS_PER_STEP, "l2": "inputs larger than L2 (no flush)"},
    "transport": {"workload": "transportation LP 2000 x 2000", "m": 4000, "n": 4_000_000, "nnz": 8_000_000,
                  "iterations_per_step": ITERS_PER_STEP, "l2": "inputs larger than L2 (no flush)"},
}


def workload_config(args):
    cfg = dict(WORKLOAD_DESC[args.workload], seed=args.seed)
    if args.scale != 1.0:
        m, n, nnz = powerlaw_shape(args.scale)
        cfg.update(scale=args.scale, m=m, n=n, nnz=nnz)
    return cfg


GOLDEN_FULL = os.path.join(ROOT, "tests", "golden", "powerlaw_m2000000_n4000000_nnz40000000_seed1.json")


def oracle_golden(args):
    """The oracle's committed fixture of the default workload (tests/golden/
    make_scale_goldens.py): its FP64 solve at 1e-6 (status, iterations, objective) where the
    oracle ran it to the end; None for other workloads."""
    if args.workload != "powerlaw" or args.scale != 1.0 or args.seed != 1:
        return None
    try:
        with open(GOLDEN_FULL) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


def pinned_copy(lp):
    """The LP's arrays in page-locked host memory (the e2e inputs)."""
    import torch

    import saddlepoint_b200 as sp

    def pin(a, dt):
        t = torch.empty(len(a), dtype=dt, pin_memory=True)
        arr = t.numpy()
        arr[:] = a
        return arr, t

    keep = []
    out = {}
    for k, dt in [("row_ptr", torch.int64), ("col_idx", torch.int32), ("values", torch.float64), ("c", torch.float64),
                  ("lc", torch.float64), ("uc", torch.float64), ("lv", torch.float64), ("uv", torch.float64)]:
        arr, t = pin(getattr(lp, k), dt)
        keep.append(t)
        out[k] = arr
    p = sp.LpProblem(lp.nrows, lp.ncols, out["row_ptr"], out["col_idx"], out["values"], out["c"], out["lc"],
                     out["uc"], out["lv"], out["uv"], lp.c0, lp.maximize, lp.name)
    return p, keep


def time_form(sp, torch, lp, backend, precision, steps, warmup, dist, device):
    """Device-resident iterations/s of one precision on the product's path (each epoch one
    CUDA-graph replay), then per-pass launch times from CUDA events in a separate,
    untimed pass of direct launches; returns a dict of measurements."""
    # tolerances of 0: no check ends the solve, every timed epoch runs its 64 iterations
    params = sp.SolverParams(tolerance=0.0, infeasibility_tolerance=0.0, max_iterations=10**9, precision=precision)
    solver = sp.Solver(lp, params, backend)
    stream = torch.cuda.ExternalStream(backend.stream(), device=f"cuda:{device}")
    solver.run_epochs(warmup)
    solver.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(device) as clk:
        clk.settle()  # the sampler's start-up stays out of the timed region
        dist.barrier()
        torch.cuda.synchronize(device)
        e0.record(stream)
        solver.run_epochs(steps)
        e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize(device)
    ms = e0.elapsed_time(e1)
    ms_max = dist.max(ms)
    done = solver.info().iterations
    if done != (warmup + steps) * ITERS_PER_STEP:
        raise RuntimeError(f"the timed solve stopped early: {done} iterations, status {solver.info().status}")
    # launch times of the two fused passes: events around every 4th P/D launch pair of
    # MID iterations, on the library's stream, over a few more epochs
    solver.set_timing(4)
    solver.run_epochs(max(2, min(steps, 8)))
    solver.sync()
    kern = {}
    for kid, name in ((0, "primal_pass"), (1, "dual_pass")):
        n, tot, bpl = solver.kernel_timing(kid)
        kern[name] = {"launches_timed": n, "avg_ms": tot / max(n, 1), "bytes_per_launch": bpl,
                      "gather_floor_ms": solver.gather_floor(kid, fp32=precision == sp.Precision.Mixed)}
    solver.set_timing(0)
    info = solver.info()
    out = {
        "ms": ms_max, "iters": steps * ITERS_PER_STEP, "kernels": kern, "clocks": clk.summary(),
        "bytes_per_iteration": solver.bytes_per_iteration(), "setup_s": info.setup_time_s,
        "norm_estimate": info.norm_estimate, "engines": solver.engines(), "epoch_kernels": solver.epoch_kernels(),
        "scaled": solver.scaled() if precision == sp.Precision.FP64 else None,
    }
    solver.close()
    return out


def to_tolerance(sp, torch, pinned, backend, precision, device, tol, limit_s):
    """One sp_solve call from pinned host arrays to `tol` relative KKT (upload, scaling,
    power iteration, iterations, solution back), timed with CUDA events on the library's
    stream; the solution is returned for the checker, which runs outside the timing."""
    stream = torch.cuda.ExternalStream(backend.stream(), device=f"cuda:{device}")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    params = sp.SolverParams(tolerance=tol, precision=precision, time_limit=limit_s)
    torch.cuda.synchronize(device)
    t0 = time.time()
    e0.record(stream)
    sol = sp.solve(pinned, params, backend)
    e1.record(stream)
    e1.synchronize()
    return sol, e0.elapsed_time(e1) * 1e-3, time.time() - t0


def checker_report(lp, sol, tol):
    """The independent KKT checker (the oracle's restatement of saddlepoint-check,
    crates/saddlepoint-check/src/lib.rs:62-118) on a GPU answer; never timed."""
    import oracle

    rep = oracle.check(lp, sol.x, sol.y)
    return {"relative_primal": rep.relative_primal, "relative_dual": rep.relative_dual,
            "relative_gap": rep.relative_gap, "max_relative": rep.max_relative(),
            "passes_at": 2.0 * tol, "passed": bool(rep.max_relative() <= 2.0 * tol)}


def run_ours(args):
    import torch

    import saddlepoint_b200 as sp

    dist = Dist(args.gpus)
    device = dist.local
    lp = powerlaw_lp(args.seed, args.scale) if args.workload == "powerlaw" else sp.generate_transport_lp(args.seed)
    wkey = workload_key(args.workload, args.scale)
    backend = sp.CudaBackend(device)
    res = {}
    for prec in (sp.Precision.FP64, sp.Precision.Mixed):
        res[prec] = time_form(sp, torch, lp, backend, prec, args.steps, args.warmup, dist, device)
    f64, mix = res[sp.Precision.FP64], res[sp.Precision.Mixed]
    n = dist.world
    value = n * f64["iters"] / (f64["ms"] * 1e-3)
    mixed_value = n * mix["iters"] / (mix["ms"] * 1e-3)

    peak, peak_kind = measured_peak()

    def roofline(meas, form):
        k = meas["kernels"]
        dom = max(k, key=lambda name: k[name]["avg_ms"])
        d = k[dom]
        achieved = d["bytes_per_launch"] / (d["avg_ms"] * 1e-3) / 1e9 if d["avg_ms"] > 0 else 0.0
        return {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind, "traffic": profiled_traffic(dom, wkey, form),
                "traffic_source": f"profiles/ncu_traffic.txt ({dom} {wkey} {form})",
                "bytes_per_launch": d["bytes_per_launch"], "avg_launch_ms": d["avg_ms"],
                "launches_timed": d["launches_timed"],
                "gather_floor": {"ms": d["gather_floor_ms"], "frac": d["gather_floor_ms"] / d["avg_ms"]
                                 if d["avg_ms"] > 0 else None,
                                 "what": "a kernel doing only this pass's random gathers through its own index "
                                         "stream (no values, no epilogue); frac = its time / the pass's"},
                "timing": "CUDA events on the library's stream around every 4th launch of the pass, in an "
                          "untimed pass of direct launches right after the timed graph replays",
                "other": {name: {"achieved_gbs": k[name]["bytes_per_launch"] / (k[name]["avg_ms"] * 1e-3) / 1e9
                                 if k[name]["avg_ms"] > 0 else None, "avg_launch_ms": k[name]["avg_ms"],
                                 "gather_floor_ms": k[name]["gather_floor_ms"],
                                 "traffic": profiled_traffic(name, wkey, form)}
                          for name in k if name != dom}}

    # e2e: the one-call public API from pinned host memory, K·64 iterations
    pinned, keep = pinned_copy(lp)
    stream = torch.cuda.ExternalStream(backend.stream(), device=f"cuda:{device}")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    iters = args.steps * ITERS_PER_STEP
    dist.barrier()
    torch.cuda.synchronize(device)
    e0.record(stream)
    sol = sp.solve(pinned, sp.SolverParams(tolerance=0.0, infeasibility_tolerance=0.0, max_iterations=iters), backend)
    e1.record(stream)
    e1.synchronize()
    e2e_ms = dist.max(e0.elapsed_time(e1))
    if sol.iterations != iters:
        raise RuntimeError(f"the e2e solve stopped early: {sol.iterations} iterations, status {sol.status.name}")
    h2d = 4 * (lp.nrows + 1) + 4 * lp.nnz + 8 * lp.nnz + 8 * (3 * lp.ncols + 2 * lp.nrows)
    d2h = 8 * (lp.ncols + lp.nrows)
    e2e = {"value": n * iters / (e2e_ms * 1e-3), "unit": "iter/s", "h2d_bytes_per_step": h2d / args.steps,
           "d2h_bytes_per_step": d2h / args.steps, "ms_total": e2e_ms, "iterations": iters,
           "api": f"sp_solve (one call: upload, GPU scaling and transpose, power iteration, {iters} PDHG "
                  "iterations, unscaled solution back)"}

    # to 1e-6 relative KKT in both forms, end to end; checked outside the timing
    # (one GPU only: with N replicas every rank would repeat the same single-GPU solves)
    tol_res = {}
    if not args.no_tolerance and dist.world == 1:
        golden = oracle_golden(args)
        for prec, name in ((sp.Precision.FP64, "fp64"), (sp.Precision.Mixed, "mixed")):
            sol_t, secs, wall = to_tolerance(sp, torch, pinned, backend, prec, device, args.tolerance,
                                             args.tolerance_limit_s)
            secs = dist.max(secs)
            r = {"tolerance": args.tolerance, "status": sol_t.status.name, "iterations": int(sol_t.iterations),
                 "restarts": int(sol_t.restarts), "seconds_e2e": secs, "wall_s": wall,
                 "setup_s": sol_t.setup_time, "solve_s": sol_t.solve_time,
                 "iter_per_s_solve": sol_t.iterations / sol_t.solve_time if sol_t.solve_time > 0 else None,
                 "fp64_from_iteration": int(sol_t.fp64_from_iteration), "objective": sol_t.objective,
                 "dual_objective": sol_t.dual_objective}
            if dist.rank == 0:
                r["checker"] = checker_report(lp, sol_t, args.tolerance)
            if golden and "objective" in golden:  # the oracle's full solve, where it was run to the end
                g_obj = golden["objective"]
                r["oracle_fp64"] = {k: golden[k] for k in ("status", "iterations", "objective", "threads")}
                r["objective_gap_vs_oracle_fp64"] = abs(sol_t.objective - g_obj) / (1.0 + abs(g_obj))
                r["iterations_minus_oracle"] = int(sol_t.iterations) - int(golden["iterations"])
            tol_res[name] = r
            tol_res[name + "_obj"] = sol_t.objective
        o64 = tol_res.pop("fp64_obj")
        omx = tol_res.pop("mixed_obj")
        tol_res["mixed"]["objective_gap_vs_gpu_fp64"] = abs(omx - o64) / (1.0 + abs(o64))

    cpu = None
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(lp, f64["scaled"], f64["norm_estimate"])

    batch = serve = None
    if args.workload == "powerlaw" and args.scale == 1.0 and not args.no_batch and dist.world == 1:
        batch = batch_compact(sp, backend, dist, args.seed)
    if args.workload == "powerlaw" and args.scale == 1.0 and not args.no_serve and dist.world == 1:
        serve = serve_compact(sp, backend, device, args.seed)

    clocks = f64["clocks"]
    line = {
        "metric": "PDHG iter/s (FP64, device-resident)",
        "value": value,
        "unit": "iter/s",
        "n_gpus": n,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": f64["ms"] / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded generators of saddlepoint_b200/csrc/host.cpp)",
        "config": workload_config(args),
        "parallelism": f"replicas x{n}",
        "roofline": roofline(f64, "fp64"),
        "e2e": e2e,
        "gpu_launches": f64["epoch_kernels"] * args.steps,
        "clocks": {k: clocks[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
        "cpu_baseline": cpu,
        "forms": {
            "fp64": {"iter_per_s": value, "ms_per_step": f64["ms"] / args.steps,
                     "gb_per_iteration": f64["bytes_per_iteration"] / 1e9,
                     "hbm_gbs_whole_iteration": f64["bytes_per_iteration"] * value / n / 1e9,
                     "engines": {k: v for k, v in f64["engines"].items() if k.endswith("fp64")},
                     "kernels_per_epoch": f64["epoch_kernels"],
                     "to_tolerance": tol_res.get("fp64")},
            "mixed": {"iter_per_s": mixed_value, "ms_per_step": mix["ms"] / args.steps,
                      "gb_per_iteration": mix["bytes_per_iteration"] / 1e9,
                      "hbm_gbs_whole_iteration": mix["bytes_per_iteration"] * mixed_value / n / 1e9,
                      "roofline": roofline(mix, "mixed"), "clocks": mix["clocks"],
                      "speedup_vs_fp64": mixed_value / value, "engines": mix["engines"],
                      "kernels_per_epoch": mix["epoch_kernels"],
                      "to_tolerance": tol_res.get("mixed"),
                      "note": "iter_per_s runs with tolerances of 0 (every epoch in FP32 SpMV); to_tolerance "
                              "is the solve to 1e-6, which moves the SpMV to FP64 below 1e-5"},
            "batch": batch,
            "serve": serve,
        },
        "setup_s": f64["setup_s"],
    }
    if dist.rank == 0:
        print(json.dumps(line), flush=True)
    backend.close()
    dist.close()


def cpu_baseline(lp, scaled, norm_estimate, iters=ITERS_PER_STEP):
    """The CPU oracle's loop on the same scaled problem (bit-identical to the oracle's own
    ScaledProblem), one epoch of `iters` iterations, all host threads."""
    import oracle

    r = oracle.solve_scaled(lp, scaled, tolerance=1e-12, norm_estimate=norm_estimate, stop_after=iters)
    return {"value": r.iterations / r.solve_time, "unit": "iter/s", "cores": oracle.get_threads(),
            "kind": "port", "sample": f"{r.iterations} PDHG iterations (one epoch incl. its check) of the same "
            f"LP on the C restatement of the reference's CPU backend, {r.solve_time:.2f} s"}


def run_reference(args):
    """The reference's CPU implementation of the path (the C restatement; the Rust
    crate cannot be built here) on this arm's workload, metric and unit. It generates
    the LP with the oracle's own copy of the generators and never loads the CUDA library."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    import oracle

    t0 = time.time()
    m, n, nnz = powerlaw_shape(args.scale)
    lp = oracle.generate_powerlaw_lp(args.seed, m, n, nnz, 1.5, 2, 5000)
    s = oracle.scaled_problem(lp)
    setup_s = time.time() - t0
    # ‖A'‖₂ only sets the step size, not the cost of an iteration: a fixed value keeps
    # the 200 power-iteration SpMVs out of the sample.
    norm = 1.0
    probe = oracle.solve_scaled(lp, s, tolerance=1e-12, norm_estimate=norm, stop_after=2)
    t_it = max(probe.solve_time / 2, 1e-3)
    # steps of `per_step` iterations, run as one continuous loop (checks every 64
    # iterations as in the reference), sized so the timed part stays near two minutes
    per_step = int(max(1, min(ITERS_PER_STEP, 120.0 / max(args.steps, 1) / t_it)))
    oracle.solve_scaled(lp, s, tolerance=1e-12, norm_estimate=norm, stop_after=max(1, args.warmup) * per_step)
    r = oracle.solve_scaled(lp, s, tolerance=1e-12, norm_estimate=norm, stop_after=args.steps * per_step)
    tot_it, tot_s = r.iterations, r.solve_time
    value = tot_it / tot_s
    sample = (f"{args.steps} steps of {per_step} PDHG iterations ({tot_it} in one loop, a check every 64) on the C "
              f"restatement of the reference's CPU backend, {oracle.get_threads()} threads; "
              f"generation (the oracle's copy of the generator) and scaling ({setup_s:.0f} s) untimed")
    line = {
        "impl": "reference", "metric": "PDHG iter/s (FP64, device-resident)", "value": value, "unit": "iter/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot_s / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generators of saddlepoint_b200/csrc/host.cpp)",
        "config": workload_config(args), "parallelism": f"host threads x{oracle.get_threads()}",
        "cpu_baseline": {"value": value, "unit": "iter/s", "cores": oracle.get_threads(), "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def batch_instances(seed: int, count: int):
    """The uneven batch: per instance m log-uniform in [50, 2000], n = 2m, 3-8 nonzeros
    per column, built like the random LP recipe from a per-instance seed."""
    import math

    import numpy as np

    import saddlepoint_b200 as sp

    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        m = int(round(math.exp(rng.uniform(math.log(50), math.log(2000)))))
        out.append(sp.generate_random_lp(seed * 1_000_003 + i, m, 2 * m, (3, 8)))
    return out


def batch_forms(sp, backend, dist, lps, runs, warm=True):
    """Solves/s of the batched persistent kernel on `lps` in both forms (tol 1e-6): an
    untimed first solve, then `runs` timed ones (device time of the launch, max over
    ranks; handed-off stragglers included)."""
    import numpy as np

    count = len(lps)
    out = {}
    for prec, name in ((sp.Precision.FP64, "fp64"), (sp.Precision.Mixed, "mixed")):
        b = sp.BatchSolver(lps, sp.SolverParams(tolerance=1e-6, precision=prec), backend)
        if warm:
            b.solve()
        times = []
        with Clocks(dist.local) as clk:
            clk.settle()
            dist.barrier()
            for _ in range(runs):
                res, t = b.solve()
                times.append(t)
        t_max = dist.max(max(times))
        st = np.array([r.status for r in res])
        its = np.array([r.iterations for r in res])
        handed = [r for r in res if r.handed_off]
        # one persistent-kernel launch, plus the single-LP solves of the handed-off
        # instances: 134 launches per 64-iteration epoch and about 700 for scaling,
        # transpose and power iteration each
        launches = 1 + sum(int(round(r.iterations / 64 * 134)) + 700 for r in handed)
        slowest = int(np.argmax(its))
        out[name] = {"solves_per_s": dist.world * count / t_max, "s_per_batch": t_max,
                     "optimal": int((st == 0).sum()), "not_optimal": int((st != 0).sum()),
                     "iterations_median": float(np.median(its)), "iterations_max": int(its.max()),
                     "slowest_instance": slowest, "slowest_status": int(st[slowest]),
                     "handed_off": len(handed), "handed_off_iterations": [int(r.iterations) for r in handed][:16],
                     "variants": {"lanes": int(sum(r.variant == "lanes" for r in res)),
                                  "tiles": int(sum(r.variant == "tiles" for r in res))},
                     "gpu_launches_per_batch": launches, "clocks": clk.summary()}
        b.close()
        warm = False  # the tuner's calibration and first-launch costs are paid once per device
    return out


def plain_form(sp, backend, lps):
    """The plain form on a sample of the batch: one device-resident sp_solve per instance."""
    t0 = time.time()
    ok = 0
    for lp in lps:
        s = sp.solve(lp, sp.SolverParams(tolerance=1e-6), backend)
        ok += int(s.status == sp.Status.Optimal)
    return {"solves_per_s": len(lps) / (time.time() - t0), "sample": len(lps), "optimal": ok}


def batch_compact(sp, backend, dist, seed):
    """The 4096-LP uneven batch for the default line: one untimed and one timed batch in
    FP64, one timed batch mixed, the plain form on 32 instances, and the ratio."""
    count = 4096
    lps = batch_instances(seed, count)
    forms = batch_forms(sp, backend, dist, lps, runs=1)
    plain = plain_form(sp, backend, lps[:: count // 32])
    return {"workload": "4096 LPs, m log-uniform [50,2000], n=2m, 3-8 nnz/col, tol 1e-6", "fp64": forms["fp64"],
            "mixed": forms["mixed"], "plain_device_solve": plain,
            "batched_over_plain": forms["fp64"]["solves_per_s"] / plain["solves_per_s"],
            "mixed_batched_over_plain": forms["mixed"]["solves_per_s"] / plain["solves_per_s"]}


def run_batch(args):
    """Solves/s of the batched persistent kernel on the 4096-LP uneven batch (tol 1e-6),
    against the plain device-resident form solving instances one at a time."""
    import saddlepoint_b200 as sp

    dist = Dist(args.gpus)
    count = 4096
    lps = batch_instances(args.seed, count)
    backend = sp.CudaBackend(dist.local)
    runs = max(1, min(args.steps, 3))
    forms = batch_forms(sp, backend, dist, lps, runs)
    sample = lps[:: count // 32]
    plain = plain_form(sp, backend, sample)
    cpu = None
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        import oracle

        t0 = time.time()
        k = 0
        for lp in sample[:8]:
            oracle.solve(lp, tolerance=1e-6)
            k += 1
        cpu = {"value": k / (time.time() - t0), "unit": "solves/s", "cores": oracle.get_threads(), "kind": "port",
               "sample": f"{k} instances of the batch solved one after another by the C restatement (serial below "
               "32768 elements, like the reference)"}
    f64 = forms["fp64"]
    line = {
        "metric": "batched solves/s at 1e-6 rel KKT (4096 uneven LPs)", "value": f64["solves_per_s"],
        "unit": "solves/s", "n_gpus": dist.world, "steps": runs, "warmup": 1,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator)",
        "config": {"workload": "4096 LPs, m log-uniform [50,2000], n=2m, 3-8 nnz/col", "tolerance": 1e-6},
        "parallelism": f"replicas x{dist.world}",
        "forms": {"fp64": f64, "mixed": forms["mixed"], "plain_device_solve": plain,
                  "batched_over_plain": f64["solves_per_s"] / plain["solves_per_s"]},
        "cpu_baseline": cpu, "gpu_launches": f64["gpu_launches_per_batch"] * runs,
        "clocks": {k: f64["clocks"][k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
    }
    if dist.rank == 0:
        print(json.dumps(line), flush=True)
    backend.close()
    dist.close()


def serve_requests(seed: int, count: int, max_nnz: float = 1e7):
    """(LP seed, m, n) of each request of the serving workload: nnz log-uniform in
    [1e3, max_nnz], n = nnz/5 columns of 5 entries, m = n/2 rows."""
    import math

    import numpy as np

    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        nnz = math.exp(rng.uniform(math.log(1e3), math.log(max_nnz)))
        n = max(10, int(nnz / 5))
        out.append((seed * 7919 + i, max(5, n // 2), n))
    return out


SERVE_MAX_ITERATIONS = 200_000


def serve_forms(sp, backend, device, seed, nreq, max_nnz):
    """The serving loop under Poisson arrivals (200/s) of `nreq` random LPs, tolerance 1e-6,
    in both precisions: Optimal solves/s, p50/p99 time to solution over the requests that
    reached Optimal, and every other request with its path and error, solved again alone
    (untimed) for comparison."""
    import threading

    import numpy as np

    specs = serve_requests(seed, nreq, max_nnz)
    lps = [sp.generate_random_lp(s, m, n, (5, 5)) for s, m, n in specs]
    gaps = np.random.default_rng(seed + 1).exponential(1.0 / 200.0, size=nreq)
    forms = {}
    for prec in (sp.Precision.FP64, sp.Precision.Mixed):
        params = sp.SolverParams(tolerance=1e-6, max_iterations=SERVE_MAX_ITERATIONS, precision=prec)
        srv = sp.Server(budget_bytes=150e9, max_inflight=8, batch_max_nnz=50_000, params=params, backend=backend)
        results = []

        def collect():
            while len(results) < nreq:
                r = srv.poll(timeout=1.0)
                if r is not None:
                    results.append(r)

        th = threading.Thread(target=collect)
        th.start()
        t0 = time.time()
        with Clocks(device) as clk:
            due = t0
            index = {}
            for i, (lp, g) in enumerate(zip(lps, gaps)):
                due += g
                delay = due - time.time()
                if delay > 0:
                    time.sleep(delay)
                index[srv.submit(lp)] = i
            th.join()
        wall = time.time() - t0
        srv.close()
        # results that are neither Optimal nor the iteration cap, solved again alone (untimed)
        alone = {}
        for r in results:
            if r.status not in (0, 3):
                try:
                    a = sp.solve(lps[index[r.id]], params, backend)
                    alone[r.id] = {"status": int(a.status), "iterations": int(a.iterations)}
                except sp.BackendError as e:
                    alone[r.id] = {"error": str(e)}
        ok = [r for r in results if r.status == 0]
        lat = np.array([r.total_s for r in ok]) if ok else np.array([float("nan")])
        lat_all = np.array([r.total_s for r in results])
        by_path = {}
        for pname in ("slot", "batch"):
            sel = [r for r in ok if r.path == pname]
            if sel:
                t = np.array([r.total_s for r in sel])
                by_path[pname] = {"optimal": len(sel), "p50_s": float(np.percentile(t, 50)),
                                  "p99_s": float(np.percentile(t, 99)),
                                  "iterations_median": float(np.median([r.iterations for r in sel]))}
        name = "fp64" if prec == sp.Precision.FP64 else "mixed"
        forms[name] = {"solves_per_s": len(ok) / wall, "requests_per_s": nreq / wall,
                       "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
                       "latency_over": "requests that reached Optimal (time to 1e-6)",
                       "optimal": len(ok), "not_optimal": nreq - len(ok), "requests": nreq,
                       "not_optimal_requests": sorted(
                           ({"index": index[r.id], "lp_seed": specs[index[r.id]][0], "nrows": specs[index[r.id]][1],
                             "ncols": specs[index[r.id]][2], "status": int(r.status), "iterations": int(r.iterations),
                             "primal_residual": r.primal_residual, "dual_residual": r.dual_residual,
                             "path": r.path, "error": r.error, "message": r.message,
                             "alone": alone.get(r.id)}
                            for r in results if r.status != 0), key=lambda d: d["index"]),
                       "p50_all_s": float(np.percentile(lat_all, 50)),
                       "queue_p50_s": float(np.median([r.queue_s for r in results])), "wall_s": wall,
                       "optimal_by_path": by_path,
                       "clocks": clk.summary()}
    return forms


def serve_compact(sp, backend, device, seed):
    """The serving section of the default line: 48 requests of up to 1e6 nonzeros (the full
    workload, `--workload serve`, goes to 1e7 and takes minutes per form)."""
    forms = serve_forms(sp, backend, device, seed, 48, 1e6)
    return {"workload": "Poisson arrivals 200/s, 48 requests, nnz log-uniform [1e3,1e6], n=nnz/5, m=n/2, tol 1e-6",
            "budget_bytes": 150e9, "max_inflight": 8, "batch_max_nnz": 50_000,
            "max_iterations": SERVE_MAX_ITERATIONS, **forms}


def run_serve(args):
    """The serving loop under Poisson arrivals (λ = 200/s) of random LPs with nnz
    log-uniform in [1e3, 1e7] (n = nnz/5, m = n/2), tolerance 1e-6: p50/p99 time to
    solution and solves/s, FP64 and mixed."""
    import saddlepoint_b200 as sp

    dist = Dist(args.gpus)
    nreq = max(8, min(args.steps, 400))
    backend = sp.CudaBackend(dist.local)
    forms = serve_forms(sp, backend, dist.local, args.seed, nreq, 1e7)
    f64 = forms["fp64"]
    line = {
        "metric": "serving solves/s and p50/p99 time to 1e-6 (Poisson 200/s)", "value": f64["solves_per_s"],
        "unit": "solves/s", "n_gpus": dist.world, "steps": nreq, "warmup": 0, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
        "config": {"workload": "Poisson arrivals 200/s, nnz log-uniform [1e3,1e7], n=nnz/5, m=n/2",
                   "budget_bytes": 150e9, "max_inflight": 8, "batch_max_nnz": 50_000, "requests": nreq,
                   "max_iterations": SERVE_MAX_ITERATIONS},
        "parallelism": f"replicas x{dist.world}",
        "forms": {"fp64": f64, "mixed": forms["mixed"]},
        "p50_s": f64["p50_s"], "p99_s": f64["p99_s"],
        "clocks": {k: f64["clocks"][k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
    }
    if dist.rank == 0:
        print(json.dumps(line), flush=True)
    backend.close()
    dist.close()


def main():
    args = parse()
    if args.impl == "reference":
        if args.workload != "powerlaw":
            print(json.dumps({"impl": "reference", "unavailable": "reference arm is defined for the default workload"}))
            return
        run_reference(args)
        return
    if args.workload in ("powerlaw", "transport"):
        run_ours(args)
    elif args.workload == "batch":
        run_batch(args)
    else:
        run_serve(args)


if __name__ == "__main__":
    main()
