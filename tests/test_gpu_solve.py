"""End-to-end parity of the GPU solves against the CPU oracle.

Restates crates/saddlepoint-cuda/tests/netlib.rs:31-74: for each instance the GPU and
the CPU reach the same status, the GPU answer passes the independent KKT checker at
2·TOL, and the objectives agree within 2·TOL. In addition the iteration counts must
agree to within one check interval (64), which is the parity the reference claims
between its backends (README.md:9-11), and the scaled problem the GPU builds must equal
the oracle's ScaledProblem bit for bit.
"""
import math

import numpy as np
import pytest

import oracle
from conftest import QUICK, SLOW, TOL, netlib_lp, netlib_reference

pytestmark = pytest.mark.gpu


def sp():
    import saddlepoint_b200

    return saddlepoint_b200


def assert_same_scaled(name, lp, backend):
    s_ref = oracle.scaled_problem(lp)
    solver = sp().Solver(lp, sp().SolverParams(power_iterations=1), backend)
    s_gpu = solver.scaled()
    for part, ref, got in [("a", s_ref.a, s_gpu.a), ("at", s_ref.at, s_gpu.at)]:
        assert np.array_equal(ref[0], got[0]), f"{name} {part} row_ptr"
        assert np.array_equal(ref[1], got[1]), f"{name} {part} col_idx"
        assert np.array_equal(ref[2], got[2]), f"{name} {part} values"
    for k in ("c", "lc", "uc", "lv", "uv", "row_scale", "col_scale"):
        assert np.array_equal(getattr(s_ref, k), getattr(s_gpu, k)), f"{name} {k}"
    assert s_ref.bound_scale == s_gpu.bound_scale and s_ref.obj_scale == s_gpu.obj_scale


@pytest.mark.parametrize("name", QUICK + SLOW)
def test_gpu_scaling_and_transpose_are_bit_exact(name, gpu_backend):
    assert_same_scaled(name, netlib_lp(name), gpu_backend)


def test_gpu_scaling_bit_exact_on_generated_lp(gpu_backend):
    lp = sp().generate_random_lp(11, 500, 1000, (5, 5))
    assert_same_scaled("random", lp, gpu_backend)
    lp = sp().generate_powerlaw_lp(5, 2000, 4000, 40_000)
    assert_same_scaled("powerlaw", lp, gpu_backend)


def compare(name, lp, gpu_sol, ref_sol, tol=TOL, iter_slack=64):
    assert gpu_sol.status.name == ref_sol.status, f"{name}: gpu {gpu_sol.status.name} vs cpu {ref_sol.status}"
    assert abs(int(gpu_sol.iterations) - int(ref_sol.iterations)) <= iter_slack, (
        f"{name}: {gpu_sol.iterations} vs {ref_sol.iterations} iterations")
    if ref_sol.status == "Optimal":
        oracle.check(lp, gpu_sol.x, gpu_sol.y).verify(2.0 * tol)
        err = abs(ref_sol.objective - gpu_sol.objective) / (1.0 + abs(ref_sol.objective) + abs(gpu_sol.objective))
        assert err <= 2.0 * tol, f"{name}: objective cpu {ref_sol.objective} vs gpu {gpu_sol.objective}"


_ref_cache = {}


def reference_solution(name, **kw):
    key = (name, tuple(sorted(kw.items())))
    if key not in _ref_cache:
        _ref_cache[key] = oracle.solve(netlib_lp(name), tolerance=TOL, **kw)
    return _ref_cache[key]


@pytest.mark.parametrize("name", QUICK + SLOW)
def test_netlib_device_solve_matches_cpu(name, gpu_backend):
    lp = netlib_lp(name)
    g = sp().solve(lp, sp().SolverParams(tolerance=TOL), gpu_backend)
    compare(name, lp, g, reference_solution(name))
    status, objective = netlib_reference()[name]
    if status == "optimal":
        assert abs(g.objective - objective) / (1.0 + abs(objective)) <= 1e-5


@pytest.mark.parametrize("name", QUICK)
def test_netlib_stepwise_matches_cpu(name, gpu_backend):
    lp = netlib_lp(name)
    g = sp().solve_stepwise(lp, sp().SolverParams(tolerance=TOL), gpu_backend)
    compare(name, lp, g, reference_solution(name))


@pytest.mark.parametrize("name", QUICK)
def test_netlib_step_implied_termination(name, gpu_backend):
    lp = netlib_lp(name)
    g = sp().solve(lp, sp().SolverParams(tolerance=TOL, termination=sp().Termination.StepImplied), gpu_backend)
    ref = reference_solution(name, termination=1)
    assert g.status.name == ref.status
    assert abs(int(g.iterations) - int(ref.iterations)) <= 64
    if ref.status == "Optimal":
        oracle.check(lp, g.x, g.y).verify(100.0 * TOL)


@pytest.mark.parametrize("name", ["afiro", "adlittle", "israel", "sctest", "woodinfe"])
def test_restart_trace_matches_cpu(name, gpu_backend):
    """Check by check, the device controller takes the oracle's restart decisions."""
    lp = netlib_lp(name)
    solver = sp().Solver(lp, sp().SolverParams(tolerance=TOL), gpu_backend)
    g = solver.solve()
    ref = reference_solution(name)
    tg = solver.trace()
    tr = ref.trace
    assert len(tg) == len(tr) and g.iterations == ref.iterations
    for a, b in zip(tg, tr):
        assert a["total"] == b["total"] and a["restarted"] == b["restarted"] and a["k_after"] == b["k_after"]
        assert math.isclose(a["omega"], b["omega"], rel_tol=1e-9)
        # r² is a difference of the metric's terms, so its rounding error is relative to
        # those terms, not to r: compare loosely (the decisions above are compared exactly)
        assert math.isclose(a["residual"], b["residual"], rel_tol=1e-6, abs_tol=1e-300)


def tiny():
    inf = math.inf
    rp, ci, v = oracle.from_triplets(2, 2, [0, 0, 1, 1], [0, 1, 0, 1], [1.0, 2.0, 3.0, 1.0])
    return sp().LpProblem(2, 2, rp, ci, v, np.array([-1.0, -1.0]), np.array([-inf, -inf]), np.array([4.0, 6.0]),
                          np.zeros(2), np.array([inf, inf]))


def test_solves_tiny_lp_on_gpu(gpu_backend):
    s = sp().solve(tiny(), sp().SolverParams(tolerance=1e-8), gpu_backend)
    assert s.status == sp().Status.Optimal
    assert abs(s.objective + 2.8) < 1e-6
    assert abs(s.x[0] - 1.6) < 1e-5 and abs(s.x[1] - 1.2) < 1e-5


def test_detects_infeasibility_on_gpu(gpu_backend):
    inf = math.inf
    p = tiny()
    p.nrows = 1
    p.row_ptr, p.col_idx, p.values = oracle.from_triplets(1, 2, [0, 0], [0, 1], [1.0, 1.0])
    p.lc, p.uc, p.uv = np.array([5.0]), np.array([inf]), np.array([1.0, 1.0])
    assert sp().solve(p, None, gpu_backend).status == sp().Status.PrimalInfeasible
    q = tiny()
    q.nrows = 1
    q.row_ptr, q.col_idx, q.values = oracle.from_triplets(1, 2, [0, 0], [0, 1], [1.0, -1.0])
    q.lc, q.uc = np.array([-inf]), np.array([1.0])
    assert sp().solve(q, None, gpu_backend).status == sp().Status.DualInfeasible


def test_invalid_problem_is_rejected(gpu_backend):
    p = tiny()
    p.lv = np.array([1.0, 0.0])
    p.uv = np.array([0.0, 1.0])  # crossed bounds (problem.rs:179-181)
    with pytest.raises(sp().SolveError) as e:
        sp().solve(p, None, gpu_backend)
    assert e.value.code == 6


def test_random_lp_matches_cpu_at_1e4(gpu_backend):
    """500 x 1000, 5 nonzeros per column at distinct rows, N(0,1) values, tolerance 1e-4."""
    lp = sp().generate_random_lp(2024, 500, 1000, (5, 5))
    ref = oracle.solve(lp, tolerance=1e-4)
    g = sp().solve(lp, sp().SolverParams(tolerance=1e-4), gpu_backend)
    compare("random", lp, g, ref, tol=1e-4)


def test_device_solve_is_deterministic(gpu_backend):
    lp = netlib_lp("israel")
    a = sp().solve(lp, sp().SolverParams(tolerance=TOL), gpu_backend)
    b = sp().solve(lp, sp().SolverParams(tolerance=TOL), gpu_backend)
    assert a.iterations == b.iterations
    assert np.array_equal(a.x, b.x) and np.array_equal(a.y, b.y)


@pytest.mark.parametrize("name", ["afiro", "israel", "shell", "standata", "etamacro"])
def test_mixed_precision_reaches_tolerance(name, gpu_backend):
    """Mixed form: FP32 SpMV until the relative KKT error is below 1e-5, then FP64; the answer
    must pass the checker at the same tolerance and its objective must be within 1e-5 relative
    of the FP64 oracle's."""
    lp = netlib_lp(name)
    g = sp().solve(lp, sp().SolverParams(tolerance=TOL, precision=sp().Precision.Mixed), gpu_backend)
    ref = reference_solution(name)
    assert g.status.name == ref.status
    if ref.status == "Optimal":
        oracle.check(lp, g.x, g.y).verify(2.0 * TOL)
        assert abs(g.objective - ref.objective) / (1.0 + abs(ref.objective)) <= 1e-5


@pytest.mark.parametrize("name", ["afiro", "adlittle", "israel"])
def test_netlib_read_by_the_library_solves_like_the_oracle(name, gpu_backend):
    """The product path end to end: sp.read_mps on the fixture file, then sp.solve."""
    from conftest import NETLIB

    lp = sp().read_mps(f"{NETLIB}/{name}.mps.gz")
    g = sp().solve(lp, sp().SolverParams(tolerance=TOL), gpu_backend)
    compare(name, netlib_lp(name), g, reference_solution(name))


@pytest.mark.parametrize("name", ["afiro", "israel", "shell", "25fv47", "80bau3b"])
def test_norm_estimate_matches_oracle(name, gpu_backend):
    """Solver::estimate_norm (solver.rs:215-242): the device power iteration gives the
    oracle's ‖A'‖₂ estimate to 1e-12 relative."""
    lp = netlib_lp(name)
    s = oracle.scaled_problem(lp)
    ref = oracle.solve_scaled(lp, s, tolerance=TOL, stop_after=1)
    g = sp().Solver(lp, sp().SolverParams(tolerance=TOL), gpu_backend).info()
    assert math.isclose(g.norm_estimate, ref.norm_estimate, rel_tol=1e-12), (g.norm_estimate, ref.norm_estimate)


def test_norm_estimate_matches_oracle_on_powerlaw_lp(gpu_backend):
    lp = sp().generate_powerlaw_lp(5, 20_000, 40_000, 400_000)
    s = oracle.scaled_problem(lp)
    ref = oracle.solve_scaled(lp, s, tolerance=TOL, stop_after=1)
    g = sp().Solver(lp, sp().SolverParams(tolerance=TOL), gpu_backend).info()
    assert math.isclose(g.norm_estimate, ref.norm_estimate, rel_tol=1e-12), (g.norm_estimate, ref.norm_estimate)


def test_collapsed_power_iteration_is_a_numerical_error(gpu_backend):
    """A'v = 0 for the power iteration's start vector (one row, +1 and -1 on columns 0 and
    7, whose start entries are equal): the reference returns SolveError::Numerical
    ("power iteration collapsed", solver.rs:229-231); so do the oracle and the GPU."""
    inf = math.inf
    rp, ci, v = oracle.from_triplets(1, 8, [0, 0], [0, 7], [1.0, -1.0])
    lp = sp().LpProblem(1, 8, rp, ci, v, np.linspace(-1.0, 1.0, 8), np.array([-inf]), np.array([1.0]), np.zeros(8),
                        np.full(8, 10.0))
    with pytest.raises(RuntimeError, match="numerical"):
        oracle.solve(lp, tolerance=TOL)
    for solve in (sp().solve, sp().solve_stepwise):
        with pytest.raises(sp().SolveError) as e:
            solve(lp, sp().SolverParams(tolerance=TOL), gpu_backend)
        assert e.value.code == 5, e.value
