"""CsrMatrix::from_triplets (crates/saddlepoint-core/src/problem.rs:33-77) on the GPU
(sp_csr_from_triplets) against the oracle's host restatement: the same CSR, bit for bit,
on triplets with repeated (row, column) pairs in scrambled order, runs that cancel to an
exact zero or to -0.0, empty rows and columns; and the reference's out-of-range rejection."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def sp():
    import saddlepoint_b200

    return saddlepoint_b200


def same_bits(a, b):
    return a.dtype == b.dtype and a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def check(m, n, rows, cols, vals, backend):
    rp, ci, v = sp().csr_from_triplets(m, n, rows, cols, vals, backend)
    orp, oci, ov = oracle.from_triplets(m, n, rows, cols, vals)
    assert np.array_equal(rp, np.asarray(orp, dtype=np.int64))
    assert np.array_equal(ci, np.asarray(oci, dtype=np.int32))
    assert same_bits(v, np.asarray(ov, dtype=np.float64))
    return rp, ci, v


def test_duplicates_cancellations_and_empty_rows(gpu_backend):
    rng = np.random.default_rng(5)
    m, n, k = 3000, 2000, 200_000
    rows = rng.integers(0, m // 2, k)  # the upper half of the rows stays empty
    cols = rng.integers(0, 40, k)      # few columns per row: many repeated pairs
    vals = rng.choice([1.5, -1.5, 0.25, 1e-300, -1e-300, 3.0, -0.0, 1e16, -1e16, 1.0], k)
    rp, ci, v = check(m, n, rows, cols, vals, gpu_backend)
    assert rp[-1] < k and (v != 0.0).all()
    assert (np.diff(rp)[m // 2:] == 0).all()


def test_sums_whose_order_matters(gpu_backend):
    # per (row, column) in input order: (1e16 - 1e16) + 1 = 1 is kept; (1e16 + 1) - 1e16 = 0
    # is dropped; -0.0 + 0.0 = 0.0 is dropped. Any other order of the additions differs.
    rows = np.array([1, 0, 2, 0, 1, 0, 1, 2])
    cols = np.array([3, 5, 1, 5, 3, 5, 3, 1])
    vals = np.array([1e16, 1e16, -0.0, -1e16, 1.0, 1.0, -1e16, 0.0])
    rp, ci, v = check(3, 6, rows, cols, vals, gpu_backend)
    assert list(rp) == [0, 1, 1, 1] and list(ci) == [5] and list(v) == [1.0]


def test_large_random_matrix(gpu_backend):
    rng = np.random.default_rng(11)
    m, n, k = 200_000, 300_000, 3_000_000
    rows = rng.integers(0, m, k)
    cols = rng.integers(0, n, k)
    vals = rng.standard_normal(k)
    check(m, n, rows, cols, vals, gpu_backend)


def test_empty_and_out_of_range(gpu_backend):
    rp, ci, v = sp().csr_from_triplets(4, 3, [], [], [], gpu_backend)
    assert list(rp) == [0, 0, 0, 0, 0] and len(ci) == 0 and len(v) == 0
    with pytest.raises(sp().BackendError):
        sp().csr_from_triplets(4, 3, [0, 4], [0, 1], [1.0, 2.0], gpu_backend)
    with pytest.raises(sp().BackendError):
        sp().csr_from_triplets(4, 3, [0, 1], [0, -1], [1.0, 2.0], gpu_backend)
