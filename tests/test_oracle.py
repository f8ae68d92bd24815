"""Pins the CPU oracle to the reference's own tests and fixtures (no GPU).

Each test restates a reference test: crates/saddlepoint-cpu/src/lib.rs:296-326,
crates/saddlepoint-check/src/lib.rs:143-161, crates/saddlepoint-core/src/scaling.rs:224-279,
crates/saddlepoint-core/src/solver.rs:486-504, crates/saddlepoint-io/src/lib.rs:328-380,
crates/saddlepoint-cpu/tests/netlib.rs:43-110 and the HiGHS objectives of data/netlib/reference.csv.
"""
import hashlib
import math
import os

import numpy as np
import pytest

import oracle
from conftest import KNOWN_HARD, NETLIB, QUICK, SLOW, TOL, netlib_bytes, netlib_lp, netlib_reference

INF = math.inf


def tiny():
    """min -x - y s.t. x + 2y ≤ 4, 3x + y ≤ 6, x, y ≥ 0 (crates/saddlepoint-cpu/src/lib.rs:280-294)."""
    rp, ci, v = oracle.from_triplets(2, 2, [0, 0, 1, 1], [0, 1, 0, 1], [1.0, 2.0, 3.0, 1.0])
    return oracle.OracleLp(2, 2, rp, ci, v, np.array([-1.0, -1.0]), np.array([-INF, -INF]), np.array([4.0, 6.0]),
                           np.array([0.0, 0.0]), np.array([INF, INF]))


def test_solves_tiny_lp():
    s = oracle.solve(tiny(), tolerance=1e-8)
    assert s.status == "Optimal"
    assert abs(s.objective + 2.8) < 1e-6
    assert abs(s.x[0] - 1.6) < 1e-5 and abs(s.x[1] - 1.2) < 1e-5


def test_detects_primal_infeasibility():
    p = tiny()
    p.row_ptr, p.col_idx, p.values = oracle.from_triplets(1, 2, [0, 0], [0, 1], [1.0, 1.0])
    p.nrows = 1
    p.lc, p.uc, p.uv = np.array([5.0]), np.array([INF]), np.array([1.0, 1.0])
    assert oracle.solve(p).status == "PrimalInfeasible"


def test_detects_dual_infeasibility():
    p = tiny()
    p.row_ptr, p.col_idx, p.values = oracle.from_triplets(1, 2, [0, 0], [0, 1], [1.0, -1.0])
    p.nrows = 1
    p.lc, p.uc = np.array([-INF]), np.array([1.0])
    assert oracle.solve(p).status == "DualInfeasible"


def test_checker_accepts_known_optimum():
    r = oracle.check(tiny(), [1.6, 1.2], [-0.4, -0.2])
    r.verify(1e-12)
    assert abs(r.primal_objective + 2.8) < 1e-12


def test_checker_rejects_suboptimal_point():
    with pytest.raises(AssertionError):
        oracle.check(tiny(), [1.0, 1.0], [-0.4, -0.2]).verify(1e-6)


def test_checker_rejects_wrong_dual_sign():
    assert oracle.check(tiny(), [1.6, 1.2], [0.4, 0.2]).relative_dual > 0.1


def sample():
    """scaling.rs:207-222."""
    rp, ci, v = oracle.from_triplets(2, 3, [0, 0, 1, 1], [0, 1, 1, 2], [100.0, 0.5, 3.0, -0.01])
    return oracle.OracleLp(2, 3, rp, ci, v, np.array([1.0, -2.0, 30.0]), np.array([1.0, -INF]),
                           np.array([1.0, 4.0]), np.array([0.0, -1.0, -INF]), np.array([INF, 2.0, 5.0]))


def test_scaled_matrix_is_r_a_c():
    p = sample()
    s = oracle.scaled_problem(p)
    for i in range(2):
        for k in range(p.row_ptr[i], p.row_ptr[i + 1]):
            j = p.col_idx[k]
            assert s.a[1][k] == j
            expected = p.values[k] * s.row_scale[i] * s.col_scale[j]
            assert abs(expected - s.a[2][k]) <= 1e-14 * abs(expected)


def test_unscaling_round_trips_feasibility_and_objective():
    p = sample()
    s = oracle.scaled_problem(p)
    x = np.array([0.01, 0.3, -2.0])
    xs = x / s.col_scale * s.bound_scale
    back = xs * s.col_scale / s.bound_scale
    assert np.all(np.abs(back - x) < 1e-14)
    assert abs(float(p.c @ x) - float(s.c @ xs) * s.objective_factor()) < 1e-12
    ax = np.array([sum(p.values[k] * x[p.col_idx[k]] for k in range(p.row_ptr[i], p.row_ptr[i + 1])) for i in range(2)])
    asx = np.array([sum(s.a[2][k] * xs[s.a[1][k]] for k in range(s.a[0][i], s.a[0][i + 1])) for i in range(2)])
    f = s.primal_residual_factors()
    assert np.all(np.abs(ax - asx * f) < 1e-12)


def test_ruiz_equilibrates_rows_and_columns():
    params = oracle.default_scaling()
    params.geometric_mean_passes = 0
    params.ruiz_iterations = 30
    params.pock_chambolle_enabled = 0
    params.bound_objective_rescaling = 0
    s = oracle.scaled_problem(sample(), params)
    v = np.abs(s.a[2])
    rmax = [v[s.a[0][i]:s.a[0][i + 1]].max() for i in range(2)]
    cmax = [v[s.at[0][j]:s.at[0][j + 1]].max() for j in range(3)]
    assert all(abs(x - 1.0) < 1e-3 for x in rmax + cmax)


def test_pid_moves_weight_toward_displacement_ratio():
    p = oracle.default_params()
    pid = oracle.PidState(1.0)
    w = pid.update(p, 1.0, 1e-2, 1.0, 1e-3, 1e-3)
    assert abs(math.log(w) - math.log(100.0)) < 0.1


def test_pid_safeguard_restores_best_weight():
    p = oracle.default_params()
    pid = oracle.PidState(1.0)
    best = pid.update(p, 1.0, 1.0, 4.0, 1e-3, 1e-3)
    pid.update(p, best, 1.0, 9.0, 1e-3, 1e-1)
    assert pid.update(p, 7.0, 1e-20, 1.0, 1e-3, 1e-3) == best
    assert pid.integral == 0.0


MPS_SAMPLE = b"""NAME          TESTLP
OBJSENSE
    MAX
ROWS
 N  COST
 L  LIM1
 G  LIM2
 E  MYEQN
 E  R4
COLUMNS
    X1        COST         1.0   LIM1         1.0
    X1        LIM2         1.0
    MARKER    'MARKER'     'INTORG'
    X2        COST         2.0   LIM1         1.0
    X2        MYEQN       -1.0
    MARKER    'MARKER'     'INTEND'
    X3        COST        -1.0   MYEQN        1.0
    X3        R4           1.0
RHS
    RHS       COST        -3.5
    RHS       LIM1         4.0   LIM2         1.0
    RHS       MYEQN        7.0   R4           2.0
RANGES
    RNG       LIM1         2.5   R4          -1.0
BOUNDS
 UP BND       X1           4.0
 MI BND       X2
 UP BND       X2           1.0
 FR BND       X3
ENDATA
"""


def test_mps_parses_all_sections():
    """io/src/lib.rs:361-375."""
    p = oracle.read_mps(MPS_SAMPLE)
    assert p.maximize
    assert list(p.c) == [-1.0, -2.0, 1.0]
    assert p.c0 == -3.5
    assert list(p.lc) == [1.5, 1.0, 7.0, 1.0]
    assert list(p.uc) == [4.0, INF, 7.0, 2.0]
    assert list(p.lv) == [0.0, -INF, -INF]
    assert list(p.uv) == [4.0, 1.0, INF]
    assert p.nnz == 6
    assert list(p.col_idx[p.row_ptr[2]:p.row_ptr[3]]) == [1, 2]
    assert list(p.values[p.row_ptr[2]:p.row_ptr[3]]) == [-1.0, 1.0]
    assert oracle.validate(p)


def test_mps_rejects_unknown_rows():
    """io/src/lib.rs:377-381: the error names line 5."""
    with pytest.raises(ValueError, match=r"^line 5:"):
        oracle.read_mps(b"NAME X\nROWS\n N obj\nCOLUMNS\n    x  nope  1\nENDATA\n")


def test_from_triplets_sums_duplicates_and_drops_zeros():
    """CsrMatrix::from_triplets (problem.rs:33-77): columns sorted, duplicates summed, zeros dropped."""
    rp, ci, v = oracle.from_triplets(3, 4, [2, 0, 0, 2, 1, 2], [3, 1, 1, 0, 2, 3], [1.0, 2.0, 3.0, 4.0, 5.0, -1.0])
    assert list(rp) == [0, 1, 2, 3]
    assert list(ci) == [1, 2, 0]
    assert list(v) == [5.0, 5.0, 4.0]


def test_from_triplets_sums_each_pair_in_input_order():
    """The stated rule for repeated (row, column) pairs (problem.rs sorts each row with
    sort_unstable_by_key, which leaves their order open): a stable sort, so each pair's
    values are summed in input order — the rule the GPU builder (sp_csr_from_triplets) is
    held to. Checked against a plain restatement on random triplets with many repeats."""
    rng = np.random.default_rng(3)
    for trial in range(20):
        m, n, k = int(rng.integers(1, 30)), int(rng.integers(1, 12)), int(rng.integers(0, 400))
        rows = rng.integers(0, m, k)
        cols = rng.integers(0, n, k)
        vals = rng.choice([1e16, -1e16, 1.0, -1.0, 0.5, -0.0, 0.0, 3.25], k)
        want_rp, want_ci, want_v = [0], [], []
        for i in range(m):
            entries = sorted([(int(c), t) for t, (r, c) in enumerate(zip(rows, cols)) if r == i])
            j = 0
            while j < len(entries):
                c, t = entries[j]
                total = vals[t]
                j += 1
                while j < len(entries) and entries[j][0] == c:
                    total = total + vals[entries[j][1]]
                    j += 1
                if total != 0.0:
                    want_ci.append(c)
                    want_v.append(total)
            want_rp.append(len(want_ci))
        rp, ci, v = oracle.from_triplets(m, n, rows, cols, vals)
        assert list(rp) == want_rp and list(ci) == want_ci
        assert np.array_equal(np.asarray(v, dtype=np.float64).view(np.uint64), np.asarray(want_v, dtype=np.float64).view(np.uint64))


def test_transpose_is_stable_counting_sort():
    rp, ci, v = oracle.from_triplets(3, 3, [0, 0, 1, 2, 2], [0, 2, 2, 0, 1], [1.0, 2.0, 3.0, 4.0, 5.0])
    trp, tci, tv = oracle.transpose(3, 3, rp, ci, v)
    assert list(trp) == [0, 2, 3, 5]
    assert list(tci) == [0, 2, 2, 0, 1]
    assert list(tv) == [1.0, 4.0, 5.0, 2.0, 3.0]


def test_fixtures_are_the_reference_data():
    """tests/golden/netlib holds the reference's data/netlib files byte for byte."""
    sums = dict(reversed(line.split("  ")) for line in open(os.path.join(NETLIB, "SHA256SUMS")).read().splitlines())
    for name, digest in sums.items():
        data = netlib_bytes(name[:-4]) if name.endswith(".mps") else open(os.path.join(NETLIB, name), "rb").read()
        assert hashlib.sha256(data).hexdigest() == digest, name


def test_every_instance_is_classified():
    """crates/saddlepoint-cpu/tests/netlib.rs:99-110."""
    on_disk = sorted(f[:-7] for f in os.listdir(NETLIB) if f.endswith(".mps.gz"))
    assert sorted(QUICK + SLOW + KNOWN_HARD) == on_disk


def _run_netlib(name, termination):
    """crates/saddlepoint-cpu/tests/netlib.rs:43-72 on the oracle."""
    p = netlib_lp(name)
    check_tol, obj_tol = (2.0 * TOL, 1e-5) if termination == 0 else (100.0 * TOL, 1e-4)
    s = oracle.solve(p, tolerance=TOL, termination=termination)
    status, objective = netlib_reference()[name]
    if status == "optimal":
        assert s.status == "Optimal", f"{name}: {s.status} after {s.iterations}"
        oracle.check(p, s.x, s.y).verify(check_tol)
        assert abs(s.objective - objective) / (1.0 + abs(objective)) <= obj_tol
    elif status == "infeasible":
        assert s.status == "PrimalInfeasible"


@pytest.mark.parametrize("name", QUICK)
def test_netlib_quick(name):
    _run_netlib(name, 0)


@pytest.mark.parametrize("name", QUICK)
def test_netlib_quick_cupdlpx_termination(name):
    _run_netlib(name, 1)


@pytest.mark.slow
@pytest.mark.parametrize("name", SLOW)
def test_netlib_slow(name):
    _run_netlib(name, 0)



def test_scale_fixtures_match_their_generated_lps():
    """tests/golden/make_scale_goldens.py's fixtures were computed on the LPs the seeded
    generators still build (SHA-256 of the arrays), and the oracle's answers pass its own
    checker at twice the fixture's tolerance."""
    import json
    import sys

    from conftest import GOLDEN

    sys.path.insert(0, GOLDEN)
    from make_scale_goldens import fingerprint

    for name in ("powerlaw_m200000_n400000_nnz3000000_seed3", "transport_300x300_seed5", "transport_2000x2000_seed1"):
        with open(os.path.join(GOLDEN, f"{name}.json")) as f:
            g = json.load(f)
        gen = oracle.generate_powerlaw_lp if g["generator"] == "powerlaw" else oracle.generate_transport_lp
        lp = gen(*g["args"])
        assert (lp.nrows, lp.ncols, lp.nnz) == (g["nrows"], g["ncols"], g["nnz"])
        assert fingerprint(lp) == g["fingerprint"]
        assert g["status"] == "Optimal" and max(g["checker"].values()) <= 2.0 * g["tolerance"]
        assert g["fixed"]["iterations"] == g["fixed"]["max_iterations"] == 640
