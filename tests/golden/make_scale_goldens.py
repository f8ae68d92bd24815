"""Writes the oracle's answers for the large generated LPs into tests/golden/ as JSON.

    python tests/golden/make_scale_goldens.py [--threads 8] [CASE ...]

The GPU tests of the large-problem engines (tests/test_gpu_scale.py) compare the CUDA
library's solves of these LPs with the oracle's, but the oracle needs minutes to hours
for them, so its answers are computed once on a CPU machine by this script and
committed. Each LP is built by the oracle's copy of the seeded generators (oracle/
sp_gen.c, bit for bit the library's generators), so the script needs neither the CUDA
library nor a GPU. Every fixture records:

  * the LP's shape and a SHA-256 fingerprint of its arrays (tests check that the
    generator still builds the same LP);
  * the oracle's FP64 solve to the case's tolerance: status, iterations, restarts,
    objective, dual objective, ‖A'‖₂ estimate, seconds, threads, and its whole check
    trace (total, restart decision, k after the check, ω, residual);
  * where the case asks for it, the trace of a run stopped after a fixed number of
    iterations (every check of the first 640 iterations, say), written before the full
    solve starts: the oracle needs hours for the full solve of the largest LP, and the
    fixture of the fixed run stands on its own if that solve is cut short.

The oracle's reductions above 32768 elements are chunked by its thread count, so its
results depend (at rounding level) on --threads, which the fixture records.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# name -> (generator, arguments, tolerance, fixed-iteration trace length or 0)
CASES = {
    "powerlaw_m200000_n400000_nnz3000000_seed3": ("powerlaw", (3, 200_000, 400_000, 3_000_000), 1e-6, 640),
    "transport_300x300_seed5": ("transport", (5, 300, 300), 1e-6, 640),
    "transport_2000x2000_seed1": ("transport", (1, 2000, 2000), 1e-6, 640),
    "powerlaw_m2000000_n4000000_nnz40000000_seed1": ("powerlaw", (1, 2_000_000, 4_000_000, 40_000_000), 1e-6, 6400),
}


def fingerprint(lp) -> str:
    """SHA-256 of an LP's arrays (int64 row pointers and column indices, float64 values
    and vectors) in a fixed order."""
    h = hashlib.sha256()
    h.update(np.array([lp.nrows, lp.ncols, len(lp.values)], dtype=np.int64).tobytes())
    h.update(np.ascontiguousarray(lp.row_ptr, dtype=np.int64).tobytes())
    h.update(np.ascontiguousarray(lp.col_idx, dtype=np.int64).tobytes())
    for k in ("values", "c", "lc", "uc", "lv", "uv"):
        h.update(np.ascontiguousarray(getattr(lp, k), dtype=np.float64).tobytes())
    return h.hexdigest()


def build(kind: str, args):
    import oracle

    if kind == "powerlaw":
        return oracle.generate_powerlaw_lp(*args)
    if kind == "transport":
        return oracle.generate_transport_lp(*args)
    return oracle.generate_random_lp(*args)


def trace_rows(trace):
    return [[t["total"], int(t["restarted"]), t["k_after"], t["omega"], t["residual"]] for t in trace]


def make(name: str, threads: int, path: str) -> dict:
    """Writes the fixture to `path`: first with the fixed run alone (so a long full solve
    that is cut short still leaves it), then again with the full solve."""
    import oracle

    kind, args, tol, fixed = CASES[name]
    oracle.set_threads(threads)
    lp = build(kind, args)
    out = {"name": name, "generator": kind, "args": list(args), "nrows": lp.nrows, "ncols": lp.ncols,
           "nnz": lp.nnz, "fingerprint": fingerprint(lp), "tolerance": tol, "threads": oracle.get_threads()}
    if fixed:
        t0 = time.time()
        r = oracle.solve(lp, tolerance=tol, max_iterations=fixed)
        out["fixed"] = {"max_iterations": fixed, "status": r.status, "iterations": r.iterations,
                        "objective": r.objective, "norm_estimate": r.norm_estimate, "seconds": time.time() - t0,
                        "trace": trace_rows(r.trace)}
        with open(path, "w") as f:
            json.dump(out, f, indent=1)
        print(f"{name}: fixed run of {fixed} iterations written", flush=True)
    t0 = time.time()
    r = oracle.solve(lp, tolerance=tol)
    out.update(status=r.status, iterations=r.iterations, restarts=r.restarts, objective=r.objective,
               dual_objective=r.dual_objective, norm_estimate=r.norm_estimate, seconds=time.time() - t0,
               trace=trace_rows(r.trace))
    rep = oracle.check(lp, r.x, r.y)
    out["checker"] = {"relative_primal": rep.relative_primal, "relative_dual": rep.relative_dual,
                      "relative_gap": rep.relative_gap}
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=8)
    ap.add_argument("cases", nargs="*", default=list(CASES))
    a = ap.parse_args()
    for name in a.cases:
        path = os.path.join(HERE, f"{name}.json")
        res = make(name, a.threads, path)
        with open(path, "w") as f:
            json.dump(res, f, indent=1)
        print(f"{name}: {res['status']} in {res['iterations']} iterations, objective {res['objective']:.12g}, "
              f"{res['seconds']:.0f} s -> {path}", flush=True)


if __name__ == "__main__":
    main()
