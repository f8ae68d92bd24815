"""The warp-specialized stream engine of the MID passes against the tile engine.

Both engines compute every row sum with the same products in the same order, so a
solve gives the same bits whichever engine runs the MID iterations
(SP_PASS_ENGINE=stream, read when a solver is created, selects the stream engine;
SP_STREAM_GATHER its gatherer form). The matrices cover what the pipeline handles
specially: many tiles per CTA (the slots wrap), rows longer than a tile (the
CTA-wide path), warp rows, runs of empty rows (tiles with no nonzeros) and
16-byte-unaligned tile starts.
"""
import os

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

VARIANTS = ["ldg4", "ldg4deep", "ldg8b16", "cp4", "ldg8deep", "ldg6deep", "ldg4b16deep", "ldg4pair", "ldg6pair"]


def sp():
    import saddlepoint_b200

    return saddlepoint_b200


def solve_with(engine, lp, params, backend, variant="ldg4"):
    old = {k: os.environ.get(k) for k in ("SP_PASS_ENGINE", "SP_STREAM_GATHER")}
    os.environ["SP_PASS_ENGINE"] = engine
    os.environ["SP_STREAM_GATHER"] = variant
    try:
        return sp().solve(lp, params, backend)
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v


def ragged_lp(seed=3, m=3000, n=6000, empty_rows=700, empty_cols=700):
    """A feasible LP with a dense row (n - empty_cols entries), a dense column
    (m - empty_rows entries), runs of empty rows and columns, and otherwise 1-9
    entries per column."""
    rng = np.random.default_rng(seed)
    live_rows = np.arange(empty_rows, m)
    trip = []
    for j in range(n):
        if empty_rows <= j < empty_rows + empty_cols:
            continue
        if j == n - 1:
            rows = set(live_rows.tolist())  # dense column
        else:
            rows = set(rng.choice(live_rows, size=int(rng.integers(1, 10)), replace=False).tolist())
        rows.add(m - 1)  # dense row: every nonempty column
        for i in sorted(rows):
            trip.append((i, j, float(rng.uniform(-2, 2)) or 1.0))
    trip.sort()
    rp = np.zeros(m + 1, dtype=np.int64)
    for i, _, _ in trip:
        rp[i + 1] += 1
    rp = np.cumsum(rp)
    ci = np.array([t[1] for t in trip], dtype=np.int32)
    va = np.array([t[2] for t in trip], dtype=np.float64)
    x0 = rng.uniform(0, 1, n)
    ax = np.array([np.dot(va[rp[i]:rp[i + 1]], x0[ci[rp[i]:rp[i + 1]]]) for i in range(m)])
    lc = np.where(rng.uniform(size=m) < 0.5, ax, -np.inf)
    uc = ax.copy()
    lc[:empty_rows] = -1.0
    uc[:empty_rows] = 1.0
    c = rng.uniform(0.1, 1.0, n)
    return sp().LpProblem(m, n, rp, ci, va, c, lc, uc, np.zeros(n), np.full(n, 10.0), name="ragged")


def fixed_iterations(iters, precision=None):
    kw = {"tolerance": 0.0, "max_iterations": iters}
    if precision is not None:
        kw["precision"] = precision
    return sp().SolverParams(**kw)


def assert_identical(a, b):
    assert a.iterations == b.iterations and a.restarts == b.restarts
    assert np.array_equal(a.x, b.x) and np.array_equal(a.y, b.y)
    assert a.objective == b.objective or (np.isnan(a.objective) and np.isnan(b.objective))


@pytest.fixture(scope="module")
def powerlaw_lp():
    # about 1900 tiles per pass: every CTA of the persistent grid takes a dozen
    return sp().generate_powerlaw_lp(7, 200_000, 400_000, 3_000_000, 1.5, 2, 5000)


@pytest.mark.parametrize("variant", VARIANTS)
def test_stream_engine_equals_tile_engine(variant, powerlaw_lp, gpu_backend):
    params = fixed_iterations(320)
    assert_identical(solve_with("stream", powerlaw_lp, params, gpu_backend, variant),
                     solve_with("tiles", powerlaw_lp, params, gpu_backend))


def test_sell_path_equals_tile_engine(powerlaw_lp, gpu_backend):
    """SP_PASS_ENGINE=sell: every MID pass on its SELL copy (warp rows from CSR)."""
    params = fixed_iterations(320)
    assert_identical(solve_with("sell", powerlaw_lp, params, gpu_backend),
                     solve_with("tiles", powerlaw_lp, params, gpu_backend))
    params = fixed_iterations(320, sp().Precision.Mixed)
    assert_identical(solve_with("sell", powerlaw_lp, params, gpu_backend),
                     solve_with("tiles", powerlaw_lp, params, gpu_backend))


def test_sell_path_on_two_streams_equals_tile_engine(gpu_backend):
    """A pass over 4M+ nonzeros runs its SELL warp rows and windows as two launches on two
    streams (smaller passes in one launch): the same bits either way."""
    lp = sp().generate_powerlaw_lp(3, 300_000, 600_000, 5_000_000, 1.5, 2, 1500)
    for precision in (None, sp().Precision.Mixed):
        params = fixed_iterations(192, precision)
        assert_identical(solve_with("sell", lp, params, gpu_backend), solve_with("tiles", lp, params, gpu_backend))


def test_sell_path_with_warp_rows_and_empty_rows(gpu_backend):
    # dense row of 1500 and dense column of 1800 entries (warp rows, no row beyond a tile),
    # empty rows and columns, ragged slices
    lp = ragged_lp(seed=11, m=2500, n=1800, empty_rows=700, empty_cols=300)
    params = fixed_iterations(256)
    assert_identical(solve_with("sell", lp, params, gpu_backend), solve_with("tiles", lp, params, gpu_backend))


def test_stream_engine_mixed_form_equals_tile_engine(powerlaw_lp, gpu_backend):
    params = fixed_iterations(320, sp().Precision.Mixed)
    assert_identical(solve_with("stream", powerlaw_lp, params, gpu_backend),
                     solve_with("tiles", powerlaw_lp, params, gpu_backend))


def test_stream_engine_long_rows_and_empty_tiles(gpu_backend):
    lp = ragged_lp()
    params = fixed_iterations(256)
    for variant in ("ldg4deep", "cp4"):
        assert_identical(solve_with("stream", lp, params, gpu_backend, variant),
                         solve_with("tiles", lp, params, gpu_backend))


def test_stream_engine_solve_of_ragged_lp_matches_oracle(gpu_backend):
    lp = ragged_lp(seed=5, m=1500, n=3000, empty_rows=600, empty_cols=300)
    ref = oracle.solve(lp, tolerance=1e-4)
    g = solve_with("stream", lp, sp().SolverParams(tolerance=1e-4), gpu_backend)
    assert g.status.name == ref.status
    assert abs(int(g.iterations) - int(ref.iterations)) <= 64
    if ref.status == "Optimal":
        oracle.check(lp, g.x, g.y).verify(2e-4)


def test_stream_engine_stall_path_reports_and_leaves_the_context_usable(powerlaw_lp, gpu_backend):
    """The stream engine's bounded waits, exercised without a fault: with the test knob
    SP_TEST_STREAM_WITHHOLD (read when a solver is created) the loader never issues the
    copies of one tile and every wait gives up after 100 µs, so the CTA that owns that
    tile takes its stall path (no copy is in flight, nothing faults). The solve must end
    with SP_ERR_CUDA and the stall message, and the next solve on the same context must
    give a clean solve's bits."""
    params = fixed_iterations(192)
    clean = solve_with("stream", powerlaw_lp, params, gpu_backend)
    os.environ["SP_TEST_STREAM_WITHHOLD"] = "0"
    try:
        with pytest.raises(sp().SolveError) as e:
            solve_with("stream", powerlaw_lp, params, gpu_backend)
    finally:
        del os.environ["SP_TEST_STREAM_WITHHOLD"]
    assert e.value.code == 1 and "did not complete within its wait limit" in str(e.value)
    assert_identical(solve_with("stream", powerlaw_lp, params, gpu_backend), clean)


def test_gather_floor_is_below_the_pass_time(powerlaw_lp, gpu_backend):
    """sp_solver_gather_floor times a kernel doing only a pass's gathers; the fused pass does
    those gathers and more, so its launch takes longer than the floor."""
    s = sp().Solver(powerlaw_lp, fixed_iterations(10**9), gpu_backend)
    s.run_epochs(2)
    s.set_timing(1)
    s.run_epochs(2)
    s.sync()
    for kid in (0, 1):
        n, tot, _ = s.kernel_timing(kid)
        floor = s.gather_floor(kid)
        assert n > 0 and 0.0 < floor < tot / n, (kid, floor, tot / n)
    s.close()
