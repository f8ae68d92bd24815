"""Parity at the sizes where the large-problem engines run.

A problem of 1M+ nonzeros runs its FUSED primal pass on the stream engine and its dual
pass (and the check's) on the SELL copy; smaller ones stay on the tile engine. The tests
here solve LPs of the benchmark's shapes at that size — a power-law LP (200,000 x 400,000,
3M nonzeros), a transportation LP with the benchmark's row structure (300 x 300), the
benchmark's own transportation LP (2000 x 2000, 8M nonzeros) and its 40M-nonzero LP — and
compare with the oracle's answers, which tests/golden/
make_scale_goldens.py computed on a CPU machine and committed (the oracle takes minutes
to hours on these):

  * a fixed run of 640 iterations: every check's restart decision and k equal, ω to 1e-9;
  * the FP64 solve to 1e-6: the oracle's status, iterations within one check interval
    (64), the independent KKT checker at 2e-6 and the objective within 2e-6
    (crates/saddlepoint-cuda/tests/netlib.rs:31-50, README.md:9-11); on the 40M LP the
    oracle's fixture holds the first 6,400 iterations (its full solve takes hours), and the
    full solve's figures where it was run to the end;
  * the mixed form to 1e-6: the status, the checker at 2e-6, the objective within 1e-5 of
    the FP64 oracle's, and the switch to FP64 SpMV taken (or the solve ended at the check
    that would have taken it).

Each fixture carries a fingerprint of its LP's arrays, so a test first checks that the
generator still builds the LP the oracle solved.
"""
import json
import math
import os

import pytest

import oracle
from conftest import GOLDEN

pytestmark = pytest.mark.gpu

TOL = 1e-6
LARGE = {"primal_fp64": "stream", "primal_fp32": "stream", "dual_fp64": "sell", "dual_fp32": "sell"}


def sp():
    import saddlepoint_b200

    return saddlepoint_b200


def golden(name):
    with open(os.path.join(GOLDEN, f"{name}.json")) as f:
        return json.load(f)


def fingerprint(lp):
    import sys

    sys.path.insert(0, GOLDEN)
    from make_scale_goldens import fingerprint as fp

    return fp(lp)


_lps = {}


def case_lp(name):
    if name not in _lps:
        g = golden(name)
        if g["generator"] == "powerlaw":
            lp = sp().generate_powerlaw_lp(*g["args"])
        else:
            lp = sp().generate_transport_lp(*g["args"])
        assert fingerprint(lp) == g["fingerprint"], f"{name}: the generator no longer builds the oracle's LP"
        _lps.clear()  # one large LP held at a time
        _lps[name] = lp
    return _lps[name]


SMALL_CASES = ["powerlaw_m200000_n400000_nnz3000000_seed3", "transport_300x300_seed5", "transport_2000x2000_seed1"]
FULL = "powerlaw_m2000000_n4000000_nnz40000000_seed1"


def engines_env(name):
    """The 300 x 300 transportation case is below the 1M-nonzero size rule: it asks for the
    large-problem engines by name (the stream engine for the primal pass, the SELL copy for
    the dual passes), exactly the assignment the rule gives a large problem."""
    return {"SP_PASS_ENGINE": "large"} if name.startswith("transport_300") else {}


class Env:
    def __init__(self, kv):
        self.kv = kv

    def __enter__(self):
        self.old = {k: os.environ.get(k) for k in self.kv}
        os.environ.update(self.kv)

    def __exit__(self, *a):
        for k, v in self.old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def solve(name, backend, **kw):
    with Env(engines_env(name)):
        s = sp().Solver(case_lp(name), sp().SolverParams(**kw), backend)
        assert s.engines() == LARGE, s.engines()
        sol = s.solve()
        trace = s.trace()
        s.close()
    return sol, trace


@pytest.mark.parametrize("name", SMALL_CASES)
def test_fixed_run_trace_matches_oracle(name, gpu_backend):
    g = golden(name)
    fixed = g["fixed"]
    sol, trace = solve(name, gpu_backend, tolerance=g["tolerance"], max_iterations=fixed["max_iterations"])
    assert sol.status.name == fixed["status"] and sol.iterations == fixed["iterations"]
    assert len(trace) == len(fixed["trace"])
    for a, (total, restarted, k_after, omega, residual) in zip(trace, fixed["trace"]):
        assert a["total"] == total and int(a["restarted"]) == restarted and a["k_after"] == k_after, (a, total)
        assert math.isclose(a["omega"], omega, rel_tol=1e-9), (a["omega"], omega)


@pytest.mark.parametrize("name", SMALL_CASES)
def test_fp64_solve_matches_oracle(name, gpu_backend):
    g = golden(name)
    sol, _ = solve(name, gpu_backend, tolerance=g["tolerance"])
    assert sol.status.name == g["status"]
    assert abs(int(sol.iterations) - int(g["iterations"])) <= 64, (sol.iterations, g["iterations"])
    if g["status"] == "Optimal":
        oracle.check(case_lp(name), sol.x, sol.y).verify(2.0 * TOL)
        err = abs(sol.objective - g["objective"]) / (1.0 + abs(sol.objective) + abs(g["objective"]))
        assert err <= 2.0 * TOL, (sol.objective, g["objective"])


@pytest.mark.parametrize("name", SMALL_CASES)
def test_mixed_solve_matches_fp64_oracle(name, gpu_backend):
    g = golden(name)
    sol, _ = solve(name, gpu_backend, tolerance=g["tolerance"], precision=sp().Precision.Mixed)
    assert sol.status.name == g["status"]
    # The SpMV moves to FP64 at the first check below 1e-5 relative KKT; a solve that is
    # already below 1e-6 at that check ends there without an FP64 iteration (the 2000 x 2000
    # transportation LP does, at the FP64 oracle's own iteration count).
    assert sol.fp64_from_iteration > 0 or sol.iterations == g["iterations"], (sol.fp64_from_iteration, sol.iterations)
    if g["status"] == "Optimal":
        oracle.check(case_lp(name), sol.x, sol.y).verify(2.0 * TOL)
        assert abs(sol.objective - g["objective"]) / (1.0 + abs(g["objective"])) <= 1e-5


def test_benchmark_lp_trace_matches_oracle(gpu_backend):
    """The benchmark's LP (2M x 4M, 40M nonzeros, seed 1): the first 6,400 iterations (100
    checks) take the oracle's restart decisions and k at every check, with ω to 1e-9."""
    g = golden(FULL)
    fixed = g["fixed"]
    s = sp().Solver(case_lp(FULL), sp().SolverParams(tolerance=TOL, max_iterations=fixed["max_iterations"]),
                    gpu_backend)
    assert s.engines() == LARGE
    sol = s.solve()
    trace = s.trace()
    s.close()
    assert sol.status.name == fixed["status"] and sol.iterations == fixed["iterations"]
    assert len(trace) == len(fixed["trace"])
    for a, (total, restarted, k_after, omega, residual) in zip(trace, fixed["trace"]):
        assert a["total"] == total and int(a["restarted"]) == restarted and a["k_after"] == k_after, (a, total)
        assert math.isclose(a["omega"], omega, rel_tol=1e-9), (a["omega"], omega)


def full_solve_reference(g):
    """The oracle's full solve of the LP to 1e-6 when the fixture holds it (it takes the
    oracle several hours on an 8-core machine)."""
    return g if "iterations" in g else None


def test_benchmark_lp_fp64_solve_to_tolerance(gpu_backend):
    """The benchmark's LP solved to 1e-6 in FP64: the independent checker at 2e-6, and the
    oracle's status, iterations (within 64) and objective (within 2e-6) where the fixture
    holds its full solve."""
    g = golden(FULL)
    lp = case_lp(FULL)
    s = sp().Solver(lp, sp().SolverParams(tolerance=TOL), gpu_backend)
    assert s.engines() == LARGE
    sol = s.solve()
    s.close()
    assert sol.status == sp().Status.Optimal
    oracle.check(lp, sol.x, sol.y).verify(2.0 * TOL)
    ref = full_solve_reference(g)
    if ref is not None:
        assert sol.status.name == ref["status"]
        assert abs(int(sol.iterations) - int(ref["iterations"])) <= 64, (sol.iterations, ref["iterations"])
        err = abs(sol.objective - ref["objective"]) / (1.0 + abs(sol.objective) + abs(ref["objective"]))
        assert err <= 2.0 * TOL, (sol.objective, ref["objective"])


def test_benchmark_lp_mixed_solve_to_tolerance(gpu_backend):
    """The mixed form on the benchmark's LP: Optimal at 1e-6 with the checker at 2e-6, the
    switch to FP64 SpMV taken, and the objective within 1e-5 of the FP64 GPU solve's (and of
    the oracle's, where the fixture holds it)."""
    g = golden(FULL)
    lp = case_lp(FULL)
    mixed = sp().solve(lp, sp().SolverParams(tolerance=TOL, precision=sp().Precision.Mixed), gpu_backend)
    assert mixed.status == sp().Status.Optimal and mixed.fp64_from_iteration > 0
    oracle.check(lp, mixed.x, mixed.y).verify(2.0 * TOL)
    fp64 = sp().solve(lp, sp().SolverParams(tolerance=TOL), gpu_backend)
    assert abs(mixed.objective - fp64.objective) / (1.0 + abs(fp64.objective)) <= 1e-5
    ref = full_solve_reference(g)
    if ref is not None:
        assert abs(mixed.objective - ref["objective"]) / (1.0 + abs(ref["objective"])) <= 1e-5
