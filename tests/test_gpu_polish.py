"""Warm starts of the device-resident solve and feasibility polishing (both without a
counterpart in the reference, whose solve starts at 0; cuPDLPx, which its benchmark compares
against, polishes, bench/README.md:1-6)."""
import numpy as np
import pytest

import oracle
from conftest import netlib_lp

pytestmark = pytest.mark.gpu


def sp():
    import saddlepoint_b200

    return saddlepoint_b200


def test_warm_start_from_zeros_is_the_cold_solve(gpu_backend):
    lp = netlib_lp("israel")
    s = sp().Solver(lp, sp().SolverParams(tolerance=1e-6), gpu_backend)
    cold = s.solve()
    s.warm_start(np.zeros(lp.ncols), np.zeros(lp.nrows))
    warm = s.solve()
    assert warm.iterations == cold.iterations and np.array_equal(warm.x, cold.x) and np.array_equal(warm.y, cold.y)


@pytest.mark.parametrize("name", ["afiro", "israel", "sctest", "adlittle"])
def test_warm_start_from_a_solution_converges_at_once(name, gpu_backend):
    lp = netlib_lp(name)
    first = sp().solve(lp, sp().SolverParams(tolerance=1e-7), gpu_backend)
    s = sp().Solver(lp, sp().SolverParams(tolerance=1e-6), gpu_backend)
    s.warm_start(first.x, first.y)
    again = s.solve()
    assert again.status == sp().Status.Optimal and again.iterations <= 128, again.iterations
    oracle.check(lp, again.x, again.y).verify(2e-6)


@pytest.mark.parametrize("name", ["afiro", "adlittle", "israel", "sctest", "scrs8", "25fv47"])
def test_polish_tightens_feasibility(name, gpu_backend):
    """A 1e-4 answer polished at 1e-9: its primal and dual violations fall below 1e-8 of the
    checker's scales, and its objective gap stays of the order of the original one (the
    polishing steps are as long as the original residuals)."""
    lp = netlib_lp(name)
    rough = sp().solve(lp, sp().SolverParams(tolerance=1e-4), gpu_backend)
    before = oracle.check(lp, rough.x, rough.y)
    x, y, its = sp().polish(lp, rough.x, rough.y, 1e-9, backend=gpu_backend)
    after = oracle.check(lp, x, y)
    assert after.relative_primal <= 1e-8 and after.relative_dual <= 1e-8, (after.relative_primal, after.relative_dual)
    assert after.relative_gap <= 100 * max(before.relative_gap, 1e-6), (before.relative_gap, after.relative_gap)
    assert its[0] > 0 or before.relative_primal <= 1e-8
