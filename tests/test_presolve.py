"""Presolve and postsolve (host code, no GPU): the reductions on planted structure, the
statuses presolve proves on its own, and round trips in which the oracle solves the
reduced LP and the postsolved answer passes the independent KKT checker on the original
LP with the original's objective."""
import math

import numpy as np
import pytest

import oracle
import saddlepoint_b200 as sp
from conftest import QUICK, SLOW, netlib_lp, netlib_reference

INF = math.inf


def planted(seed=4):
    """A random LP with extra structure: 3 empty rows (feasible), 4 singleton rows (one an
    equality, one tightening both bounds), 3 fixed columns, and 4 empty columns whose costs
    point at a finite bound or are zero."""
    base = oracle.generate_random_lp(seed, 120, 240, (3, 6))
    m0, n0 = base.nrows, base.ncols
    rng = np.random.default_rng(seed)
    rows, cols, vals = [], [], []
    for i in range(m0):
        for k in range(base.row_ptr[i], base.row_ptr[i + 1]):
            rows.append(i)
            cols.append(int(base.col_idx[k]))
            vals.append(float(base.values[k]))
    # every row an inequality with room around the generator's x0 in [0, 1]^n, so the
    # fixed values and implied bounds below keep the LP feasible
    lc = [lo - 5.0 if lo == hi else lo for lo, hi in zip(base.lc, base.uc)]
    uc = [hi + 5.0 for hi in base.uc]
    lv, uv, c = list(base.lv), list(base.uv), list(base.c)
    # empty rows
    for lo, hi in ((-1.0, 1.0), (0.0, 0.0), (-INF, 3.0)):
        lc.append(lo)
        uc.append(hi)
    # singleton rows on columns 5, 17, 40, 41 (the base LP's bounds are 0 <= x <= 10)
    for j, a, lo, hi in ((5, 2.0, 1.0, 30.0), (17, -0.5, -0.4, -0.1), (40, 3.0, 1.5, 1.5), (41, 1.0, -INF, 2.5)):
        rows.append(len(lc))
        cols.append(j)
        vals.append(a)
        lc.append(lo)
        uc.append(hi)
    # fixed columns: 3 existing ones
    for j in (2, 9, 100):
        lv[j] = uv[j] = float(rng.uniform(0, 1))
    # empty columns
    for cj, lo, hi in ((1.5, -2.0, 4.0), (-0.7, 0.0, 9.0), (0.0, 1.0, 5.0), (0.0, -3.0, -1.0)):
        c.append(cj)
        lv.append(lo)
        uv.append(hi)
    m, n = len(lc), len(c)
    rp, ci, v = oracle.from_triplets(m, n, rows, cols, vals)
    return oracle.OracleLp(m, n, rp, ci, v, np.array(c), np.array(lc), np.array(uc), np.array(lv), np.array(uv),
                           c0=0.25)


def round_trip(lp, tol=1e-7):
    pre = sp.presolve(lp)
    assert pre.status is None
    r = oracle.solve(pre.reduced, tolerance=tol)
    assert r.status == "Optimal"
    x, y = pre.postsolve(r.x, r.y)
    ref = oracle.solve(lp, tolerance=tol)
    return pre, r, x, y, ref


def test_planted_reductions_and_round_trip():
    lp = planted()
    pre, r, x, y, ref = round_trip(lp)
    assert pre.counts == {"empty_rows": 3, "singleton_rows": 4, "fixed_cols": 4, "empty_cols": 4}
    # the equality singleton row fixes column 40 (1.5 / 3), so four columns are fixed
    assert pre.reduced.ncols == lp.ncols - 8 and pre.reduced.nrows == lp.nrows - 7
    assert x[40] == 0.5 and x[2] == lp.lv[2] and x[240] == -2.0 and x[241] == 9.0 and x[242] == 1.0 and x[243] == -1.0
    rep = oracle.check(lp, x, y)
    rep.verify(1e-6)
    assert abs(rep.primal_objective - ref.objective) <= 1e-6 * (1.0 + abs(ref.objective))
    # the reduced problem's objective constant carries the removed columns' costs
    assert abs(r.objective - ref.objective) <= 1e-6 * (1.0 + abs(ref.objective))


def test_presolve_proves_primal_infeasibility():
    lp = planted()
    lp.lc = lp.lc.copy()
    lp.lc[lp.nrows - 7] = 1.0  # the first empty row now needs 0 >= 1
    assert sp.presolve(lp).status == sp.Status.PrimalInfeasible
    lp = planted()
    lp.uc = lp.uc.copy()
    lp.uc[lp.nrows - 4] = -2.0  # singleton row 2 x_5 in [1, -2]
    assert sp.presolve(lp).status == sp.Status.PrimalInfeasible


def test_presolve_proves_dual_infeasibility():
    lp = planted()
    lp.uv = lp.uv.copy()
    lp.uv[lp.ncols - 3] = INF  # an empty column with cost -0.7 and no upper bound
    assert sp.presolve(lp).status == sp.Status.DualInfeasible


def test_everything_fixed_is_solved_by_presolve():
    rp, ci, v = oracle.from_triplets(2, 3, [0, 0, 1], [0, 1, 2], [1.0, 2.0, -1.0])
    lp = oracle.OracleLp(2, 3, rp, ci, v, np.array([1.0, -1.0, 2.0]), np.array([-INF, -5.0]), np.array([10.0, 5.0]),
                         np.array([1.0, 2.0, 3.0]), np.array([1.0, 2.0, 3.0]), c0=1.0)
    pre = sp.presolve(lp)
    assert pre.status == sp.Status.Optimal and pre.reduced.ncols == 0
    x, y = pre.postsolve(np.zeros(0), np.zeros(0))
    assert np.array_equal(x, [1.0, 2.0, 3.0]) and np.array_equal(y, [0.0, 0.0])
    oracle.check(lp, x, y).verify(1e-12)


@pytest.mark.parametrize("name", QUICK + SLOW)
def test_netlib_round_trip(name):
    """Every Netlib LP of the reference's regression through presolve, the oracle on the
    reduced LP at 1e-7, and postsolve: the reference's status (woodinfe's infeasibility is
    proved by presolve itself), the original LP's checker at 2e-6 and HiGHS's objective
    within 1e-5 (crates/saddlepoint-cpu/tests/netlib.rs:43-72)."""
    lp = netlib_lp(name)
    status, objective = netlib_reference()[name]
    pre = sp.presolve(lp)
    if pre.status is not None:
        assert status == "infeasible" and pre.status == sp.Status.PrimalInfeasible, (name, pre.status)
        return
    r = oracle.solve(pre.reduced, tolerance=1e-7)
    if status != "optimal":
        assert r.status == "PrimalInfeasible", (name, r.status)
        return
    assert r.status == "Optimal"
    x, y = pre.postsolve(r.x, r.y)
    rep = oracle.check(lp, x, y)
    rep.verify(2e-6)
    assert abs(rep.primal_objective - objective) <= 1e-5 * (1.0 + abs(objective))
