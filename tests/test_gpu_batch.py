"""The batched persistent kernel and the serving loop against the oracle and against
themselves: every instance's answer passes the independent checker at the tolerance and
matches the oracle's status, iterations (within the reference's check granularity
wherever one lane sums a row) and objective; and a result is the same bits whether
its LP is solved alone or in a mix."""
import math

import numpy as np
import pytest

import oracle
from conftest import netlib_lp

pytestmark = pytest.mark.gpu

TOL = 1e-6


def sp():
    import saddlepoint_b200

    return saddlepoint_b200


def uneven(seed, count, mmin=50, mmax=400):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        m = int(round(math.exp(rng.uniform(math.log(mmin), math.log(mmax)))))
        out.append(sp().generate_random_lp(seed * 1000 + i, m, 2 * m, (3, 8)))
    return out


@pytest.fixture(scope="module")
def batch_lps():
    return uneven(17, 24)


def test_batch_matches_oracle(batch_lps, gpu_backend):
    b = sp().BatchSolver(batch_lps, sp().SolverParams(tolerance=TOL), gpu_backend)
    res, elapsed = b.solve()
    assert elapsed > 0
    for i, (lp, r) in enumerate(zip(batch_lps, res)):
        ref = oracle.solve(lp, tolerance=TOL)
        assert sp().Status(r.status).name == ref.status, (i, r.status, ref.status)
        x, y = b.solution(i)
        oracle.check(lp, x, y).verify(2 * TOL)
        rel = abs(r.objective - ref.objective) / (1 + abs(r.objective) + abs(ref.objective))
        assert rel <= 2 * TOL
        if r.lanes_a == 1 and r.lanes_t == 1:
            assert abs(r.iterations - ref.iterations) <= 64
        else:
            assert abs(r.iterations - ref.iterations) <= max(64, 0.05 * ref.iterations)


def test_batch_instance_alone_equals_in_mix(batch_lps, gpu_backend):
    mix = sp().BatchSolver(batch_lps, sp().SolverParams(tolerance=TOL), gpu_backend)
    res_mix, _ = mix.solve()
    for i in (0, 7, 23):
        alone = sp().BatchSolver([batch_lps[i]], sp().SolverParams(tolerance=TOL), gpu_backend)
        res_alone, _ = alone.solve()
        assert res_alone[0].iterations == res_mix[i].iterations
        assert res_alone[0].objective == res_mix[i].objective
        xa, ya = alone.solution(0)
        xm, ym = mix.solution(i)
        assert np.array_equal(xa, xm) and np.array_equal(ya, ym)


@pytest.mark.parametrize("variant", ["tiles", "lanes"])
def test_batch_variants_match_oracle(variant, batch_lps, gpu_backend, monkeypatch):
    monkeypatch.setenv("SP_BATCH_VARIANT", variant)
    b = sp().BatchSolver(batch_lps[:10], sp().SolverParams(tolerance=TOL), gpu_backend)
    res, _ = b.solve()
    for i, (lp, r) in enumerate(zip(batch_lps[:10], res)):
        assert r.variant == variant
        ref = oracle.solve(lp, tolerance=TOL)
        assert sp().Status(r.status).name == ref.status
        x, y = b.solution(i)
        oracle.check(lp, x, y).verify(2 * TOL)


def test_batch_tile_variant_equals_the_solo_device_solve(batch_lps, gpu_backend, monkeypatch):
    """The tile variant drives the single-LP solve's own passes, tiles and reductions from
    inside one CTA, so each instance's answer is the solo sp_solve's, bit for bit."""
    monkeypatch.setenv("SP_BATCH_VARIANT", "tiles")
    lps = batch_lps[:8] + [netlib_lp("afiro"), netlib_lp("adlittle")]
    b = sp().BatchSolver(lps, sp().SolverParams(tolerance=TOL), gpu_backend)
    res, _ = b.solve()
    for i, lp in enumerate(lps):
        solo = sp().solve(lp, sp().SolverParams(tolerance=TOL), gpu_backend)
        x, y = b.solution(i)
        assert res[i].iterations == solo.iterations, (i, res[i].iterations, solo.iterations)
        assert np.array_equal(x, solo.x) and np.array_equal(y, solo.y), i


def test_batch_hand_off_gives_the_solo_device_solve(batch_lps, gpu_backend, monkeypatch):
    """An instance the kernel stops for the hand-off (still running after the queue has
    drained) is solved again from the start by sp_solve: its result is the solo solve's,
    bit for bit. With a hand-off delay of zero every instance but the first to finish is a
    straggler: the grid has one CTA per instance, and the first CTA to finish drains the
    queue."""
    monkeypatch.setenv("SP_BATCH_HANDOFF_S", "1e-9")
    lps = batch_lps[:5] + [netlib_lp("afiro"), netlib_lp("adlittle")]
    params = sp().SolverParams(tolerance=TOL)
    b = sp().BatchSolver(lps, params, gpu_backend)
    res, elapsed = b.solve()
    assert elapsed > 0
    assert sum(r.handed_off for r in res) >= len(lps) - 1
    for i, (lp, r) in enumerate(zip(lps, res)):
        x, y = b.solution(i)
        if not r.handed_off:
            oracle.check(lp, x, y).verify(2 * TOL)
            continue
        solo = sp().solve(lp, params, gpu_backend)
        assert r.iterations == solo.iterations, (i, r.iterations, solo.iterations)
        assert r.objective == solo.objective and r.status == int(solo.status)
        assert np.array_equal(x, solo.x) and np.array_equal(y, solo.y), i


def test_batch_without_stragglers_hands_off_nothing(batch_lps, gpu_backend):
    b = sp().BatchSolver(batch_lps[:8], sp().SolverParams(tolerance=TOL), gpu_backend)
    res, _ = b.solve()
    assert not any(r.handed_off for r in res)


def test_batch_repeat_is_identical(batch_lps, gpu_backend):
    b = sp().BatchSolver(batch_lps[:6], sp().SolverParams(tolerance=TOL), gpu_backend)
    r1, _ = b.solve()
    x1 = [b.solution(i) for i in range(6)]
    r2, _ = b.solve()
    for i in range(6):
        assert r1[i].iterations == r2[i].iterations
        x2 = b.solution(i)
        assert np.array_equal(x1[i][0], x2[0]) and np.array_equal(x1[i][1], x2[1])


def test_batch_netlib_and_infeasible(gpu_backend):
    names = ["afiro", "sctest", "adlittle", "woodinfe", "forest6"]
    lps = [netlib_lp(n) for n in names]
    b = sp().BatchSolver(lps, sp().SolverParams(tolerance=TOL), gpu_backend)
    res, _ = b.solve()
    for name, lp, r in zip(names, lps, res):
        ref = oracle.solve(lp, tolerance=TOL)
        assert sp().Status(r.status).name == ref.status, name
        if ref.status == "Optimal":
            x, y = b.solution(names.index(name))
            oracle.check(lp, x, y).verify(2 * TOL)


def test_batch_mixed_precision(batch_lps, gpu_backend):
    b = sp().BatchSolver(batch_lps[:8], sp().SolverParams(tolerance=TOL, precision=sp().Precision.Mixed),
                         gpu_backend)
    res, _ = b.solve()
    for i, (lp, r) in enumerate(zip(batch_lps[:8], res)):
        assert r.status == 0, (i, r.status)
        x, y = b.solution(i)
        oracle.check(lp, x, y).verify(2 * TOL)


def test_server_results_match_solo_solves(gpu_backend):
    small = uneven(5, 6, 50, 150)
    large = [sp().generate_random_lp(900 + i, 3000, 6000, (5, 5)) for i in range(3)]
    lps = small + large
    srv = sp().Server(budget_bytes=2e9, max_inflight=2, batch_max_nnz=5000,
                      params=sp().SolverParams(tolerance=TOL), backend=gpu_backend)
    ids = [srv.submit(lp) for lp in lps]
    got = {}
    while len(got) < len(lps):
        r = srv.poll(timeout=60.0)
        assert r is not None, "server stalled"
        got[r.id] = r
    srv.close()
    for rid, lp in zip(ids, lps):
        r = got[rid]
        assert r.status == 0
        assert r.total_s >= r.solve_s >= 0 and r.queue_s >= 0
        oracle.check(lp, r.x, r.y).verify(2 * TOL)
        if lp.nnz <= 5000:  # batch path: the same bits as a batch of one
            alone = sp().BatchSolver([lp], sp().SolverParams(tolerance=TOL), gpu_backend)
            res, _ = alone.solve()
            xa, ya = alone.solution(0)
            assert res[0].iterations == r.iterations and np.array_equal(xa, r.x) and np.array_equal(ya, r.y)
        else:  # slot path: the same bits as a solo device-resident solve
            solo = sp().solve(lp, sp().SolverParams(tolerance=TOL), gpu_backend)
            assert solo.iterations == r.iterations and np.array_equal(solo.x, r.x) and np.array_equal(solo.y, r.y)


def test_server_admits_within_budget(gpu_backend):
    """A budget that fits one request at a time still serves every request, in order."""
    lps = [sp().generate_random_lp(40 + i, 2000, 4000, (5, 5)) for i in range(3)]
    fp = sp().Server.footprint(2000, 4000, 20000)
    srv = sp().Server(budget_bytes=1.5 * fp, max_inflight=3, batch_max_nnz=0,
                      params=sp().SolverParams(tolerance=TOL), backend=gpu_backend)
    for lp in lps:
        srv.submit(lp)
    rs = [srv.poll(timeout=60.0) for _ in lps]
    srv.close()
    assert all(r is not None and r.status == 0 for r in rs)
    assert [r.id for r in rs] == [1, 2, 3]
    # admitted one after another: each waits for the previous to finish
    assert rs[1].queue_s >= rs[0].solve_s * 0.5 and rs[2].queue_s >= rs[1].queue_s


def test_server_under_load_matches_solo_solves(gpu_backend):
    """Twelve requests of 0.2M-3M nonzeros (the larger ones on the stream and SELL engines)
    on eight concurrent slots, their set-ups and epochs overlapping and their device memory
    handed back and forth through the stream-ordered pool: every result has the bits of the
    same LP solved alone."""
    rng = np.random.default_rng(17)
    lps = []
    for i in range(12):
        n = int(np.exp(rng.uniform(np.log(4e4), np.log(6e5))))
        lps.append(sp().generate_random_lp(700 + i, n // 2, n, (5, 5)))
    params = sp().SolverParams(tolerance=TOL, max_iterations=1280)
    srv = sp().Server(budget_bytes=100e9, max_inflight=8, batch_max_nnz=0, params=params, backend=gpu_backend)
    ids = [srv.submit(lp) for lp in lps]
    got = {}
    while len(got) < len(lps):
        r = srv.poll(timeout=120.0)
        assert r is not None, "server stalled"
        got[r.id] = r
    srv.close()
    for rid, lp in zip(ids, lps):
        r = got[rid]
        solo = sp().solve(lp, params, gpu_backend)
        assert r.error == 0, r.message
        assert r.status == int(solo.status) and r.iterations == solo.iterations
        assert np.array_equal(r.x, solo.x) and np.array_equal(r.y, solo.y)


def _with_nan_bound(lp):
    bad = sp().LpProblem.from_any(lp)
    bad.lv = np.array(bad.lv, dtype=np.float64, copy=True)
    bad.lv[0] = math.nan
    return bad


def test_invalid_problems_are_refused_before_any_solve(batch_lps, gpu_backend):
    """Every entry point validates as Solver::new does (solver.rs:155): sp_solve and the
    stepwise solve fail with SP_ERR_PROBLEM and the reference's message, a batch names the
    instance, and the server refuses the request at submit while it keeps serving others."""
    bad = _with_nan_bound(batch_lps[1])
    params = sp().SolverParams(tolerance=TOL)
    for run in (sp().solve, sp().solve_stepwise):
        with pytest.raises(sp().SolveError) as e:
            run(bad, params, gpu_backend)
        assert e.value.code == 6 and str(e.value).endswith("variable 0 is NaN")
    with pytest.raises(sp().SolveError) as e:
        sp().BatchSolver([batch_lps[0], bad], params, gpu_backend)
    assert e.value.code == 6 and str(e.value).endswith("instance 1: variable 0 is NaN")
    srv = sp().Server(budget_bytes=2e9, max_inflight=1, batch_max_nnz=0, params=params, backend=gpu_backend)
    try:
        with pytest.raises(sp().SolveError) as e:
            srv.submit(bad)
        assert e.value.code == 6
        rid = srv.submit(batch_lps[0])
        r = srv.poll(timeout=60.0)
        assert r is not None and r.id == rid and r.error == 0 and r.status == 0
    finally:
        srv.close()
