"""LpProblem::validate (crates/saddlepoint-core/src/problem.rs:166-194) as the library runs it
before every solve (host code, no GPU): the reference's checks in its order — every
variable's bounds, then every constraint's, then NaN among c and A's values — and its
messages, including over ranges that the library scans on several host threads."""
import math

import numpy as np
import pytest

import oracle
import saddlepoint_b200 as sp

NAN, INF = math.nan, math.inf


def small():
    lp = sp.generate_random_lp(3, 12, 24, (2, 4))
    for k in ("c", "lc", "uc", "lv", "uv", "values"):
        setattr(lp, k, np.array(getattr(lp, k), dtype=np.float64, copy=True))
    return lp


def message(lp):
    with pytest.raises(sp.SolveError) as e:
        sp.validate(lp)
    assert e.value.code == 6  # SP_ERR_PROBLEM
    return str(e.value).split(": ", 1)[1]


def test_a_valid_problem_passes():
    sp.validate(small())


@pytest.mark.parametrize("edit,expected", [
    (lambda p: p.lv.__setitem__(3, NAN), "variable 3 is NaN"),
    (lambda p: p.uv.__setitem__(3, NAN), "variable 3 is NaN"),
    (lambda p: (p.lv.__setitem__(5, 2.0), p.uv.__setitem__(5, 1.0)), "variable 5 has lower bound 2 above upper bound 1"),
    (lambda p: (p.lc.__setitem__(2, 1.5), p.uc.__setitem__(2, -0.25)),
     "constraint 2 has lower bound 1.5 above upper bound -0.25"),
    (lambda p: p.lc.__setitem__(0, NAN), "constraint 0 is NaN"),
    (lambda p: p.c.__setitem__(4, NAN), "coefficient 4 is NaN"),
    (lambda p: p.values.__setitem__(7, NAN), "coefficient 31 is NaN"),  # numbered after the 24 costs
    (lambda p: (p.lv.__setitem__(1, INF), p.uv.__setitem__(1, 5.0)), "variable 1 has lower bound inf above upper bound 5"),
    (lambda p: (p.lv.__setitem__(1, 1e20), p.uv.__setitem__(1, 1e-7)),
     "variable 1 has lower bound 100000000000000000000 above upper bound 0.0000001"),
])
def test_each_failure_has_the_reference_message(edit, expected):
    lp = small()
    edit(lp)
    assert message(lp) == expected
    assert not oracle.validate(lp) and oracle.validate_message(lp) == expected


def test_the_reference_order_decides_between_failures():
    lp = small()
    lp.c[0] = NAN
    lp.lc[9], lp.uc[9] = 1.0, 0.0
    assert message(lp) == "constraint 9 has lower bound 1 above upper bound 0"  # bounds before coefficients
    lp.lv[7] = NAN
    assert message(lp) == "variable 7 is NaN"  # variables before constraints
    lp.lv[3], lp.uv[3] = 4.0, 3.0
    assert message(lp) == "variable 3 has lower bound 4 above upper bound 3"  # the first column with either


def big(n):
    """One row of two entries over n columns (n large enough that the scans are split)."""
    rp = np.array([0, 2], dtype=np.int64)
    ci = np.array([0, 1], dtype=np.int32)
    return sp.LpProblem(1, n, rp, ci, np.array([1.0, 1.0]), np.zeros(n), np.array([-1.0]), np.array([1.0]),
                        np.zeros(n), np.ones(n))


def test_the_first_failure_wins_across_the_split_scans():
    n = 2_000_000
    lp = big(n)
    sp.validate(lp)
    lp.lv[1_900_000], lp.uv[1_900_000] = 3.0, 2.0
    lp.uv[1_200_000] = NAN
    lp.c[5] = NAN
    assert message(lp) == "variable 1200000 is NaN" == oracle.validate_message(lp)
    lp.uv[1_200_000] = 1.0
    assert message(lp) == "variable 1900000 has lower bound 3 above upper bound 2"
    lp.lv[1_900_000] = 0.0
    assert message(lp) == "coefficient 5 is NaN"
    lp.c[5] = 0.0
    lp.values[1] = NAN
    assert message(lp) == f"coefficient {n + 1} is NaN" == oracle.validate_message(lp)


def test_agrees_with_the_oracle_on_random_faults():
    """The oracle restates the reference's checks and messages (oracle.validate_message):
    the same verdict and the same text on LPs with up to two random faults."""
    rng = np.random.default_rng(9)
    for _ in range(200):
        lp = small()
        for _ in range(int(rng.integers(0, 4))):
            k = ("c", "lc", "uc", "lv", "uv", "values")[int(rng.integers(0, 6))]
            v = getattr(lp, k)
            v[int(rng.integers(0, len(v)))] = (NAN, -5.0, 5.0, INF, -INF)[int(rng.integers(0, 5))]
        expected = oracle.validate_message(lp)
        if not expected:
            assert oracle.validate(lp)
            sp.validate(lp)
        else:
            assert message(lp) == expected


def test_problems_without_rows_or_columns():
    """Empty ranges validate (the reference's loops simply do not run); a NaN bound on the one
    column of a row-less problem is still found."""
    empty_rows = sp.LpProblem(0, 3, np.array([0], dtype=np.int64), np.zeros(0, dtype=np.int32), np.zeros(0),
                              np.ones(3), np.zeros(0), np.zeros(0), np.zeros(3), np.ones(3))
    sp.validate(empty_rows)
    empty_cols = sp.LpProblem(2, 0, np.array([0, 0, 0], dtype=np.int64), np.zeros(0, dtype=np.int32), np.zeros(0),
                              np.zeros(0), np.array([-1.0, -INF]), np.array([1.0, 0.0]), np.zeros(0), np.zeros(0))
    sp.validate(empty_cols)
    one = sp.LpProblem(0, 1, np.array([0], dtype=np.int64), np.zeros(0, dtype=np.int32), np.zeros(0),
                       np.ones(1), np.zeros(0), np.zeros(0), np.array([NAN]), np.ones(1))
    assert message(one) == "variable 0 is NaN"


@pytest.mark.parametrize("field,length,expected", [
    ("c", 5, "c has length 5, expected 24"),
    ("lv", 30, "lv has length 30, expected 24"),
    ("uc", 0, "uc has length 0, expected 12"),
    ("row_ptr", 12, "A has length 12, expected 13"),
])
def test_array_lengths_are_checked_before_the_library_sees_them(field, length, expected):
    """The C ABI takes lengths from nrows, ncols and the row pointers; the Python layer checks
    the arrays' own lengths first, in the reference's order and words (problem.rs:168-177),
    so a short array is an error and never an out-of-bounds read."""
    lp = small()
    v = getattr(lp, field)
    setattr(lp, field, np.resize(v, length) if length else v[:0])
    assert message(lp) == expected
    with pytest.raises(sp.SolveError):
        sp.presolve(lp)


def test_matrix_structure_is_checked_after_the_reference_checks():
    """Row pointers from 0 to nnz and never decreasing, column indices in range: the C ABI
    checks what the reference's CsrMatrix keeps by construction (SP_ERR_INVALID), so a bad
    index is an error instead of a read outside a vector on the GPU."""
    lp = small()
    lp.col_idx = np.array(lp.col_idx, dtype=np.int32, copy=True)
    lp.col_idx[5] = lp.ncols
    with pytest.raises(sp.SolveError) as e:
        sp.validate(lp)
    assert e.value.code == 2 and str(e.value).endswith(f"A's column index {lp.ncols} at entry 5 is out of range for 24 columns")
    lp.lv[0] = NAN  # the reference's checks come first
    assert message(lp) == "variable 0 is NaN"
    lp = small()
    lp.row_ptr = np.array(lp.row_ptr, dtype=np.int64, copy=True)
    lp.row_ptr[3], lp.row_ptr[4] = lp.row_ptr[4], lp.row_ptr[3]
    with pytest.raises(sp.SolveError) as e:
        sp.validate(lp)
    assert e.value.code == 2 and "row pointers decrease after row" in str(e.value)
