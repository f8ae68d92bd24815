"""The C-ABI boundary, checked without a GPU: the library loads, it exports every
entry point include/saddlepoint_b200.h declares, the parameter defaults are the
reference's (crates/saddlepoint-core/src/solver.rs:70-93, scaling.rs:25-34), the
no-GPU path is an error (never a CPU fallback), and the host-side generators are
deterministic and have the shapes their recipes state."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import saddlepoint_b200 as sp
from saddlepoint_b200 import _lib as L

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "saddlepoint_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sp_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_entry_point():
    lib = sp.library()
    names = declared_functions()
    assert len(names) >= 50
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the ctypes table covers the same set
    assert sorted(n for n, _, _ in L.SIGNATURES) == names


def test_defaults_are_the_reference_defaults():
    p = L.Params()
    sp.library().sp_solver_params_default(C.byref(p))
    assert (p.tolerance, p.infeasibility_tolerance, p.max_iterations, p.check_every) == (1e-6, 1e-8, 1_000_000, 64)
    assert (p.step_size_factor, p.reflection) == (0.998, 1.0)
    assert (p.restart_sufficient, p.restart_necessary, p.restart_artificial) == (0.2, 0.5, 0.36)
    assert (p.pid_kp, p.pid_ki, p.pid_kd, p.pid_discount) == (0.99, 0.01, 0.0, 0.3)
    assert p.power_iterations == 200
    assert (p.geometric_mean_passes, p.ruiz_iterations, p.pock_chambolle_enabled, p.pock_chambolle_alpha) == (12, 10, 1, 1.0)
    assert p.bound_objective_rescaling == 1 and p.termination == 0 and p.precision == 0
    assert p.mixed_switch_tolerance == 1e-5
    # and the Python mirror carries the same values
    q = sp.SolverParams().to_c()
    for name, _ in L.Params._fields_:
        assert getattr(q, name) == getattr(p, name), name


def test_no_gpu_is_an_error_not_a_fallback():
    try:
        import torch

        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    with pytest.raises(sp.BackendError) as e:
        sp.CudaBackend(0)
    assert e.value.code == 4
    with pytest.raises(sp.BackendError):
        sp.solve(sp.generate_random_lp(1, 10, 20, (2, 3)))


def test_random_generator_is_deterministic_and_shaped():
    a = sp.generate_random_lp(2024, 500, 1000, (5, 5))
    b = sp.generate_random_lp(2024, 500, 1000, (5, 5))
    c = sp.generate_random_lp(2025, 500, 1000, (5, 5))
    assert (a.nrows, a.ncols, a.nnz) == (500, 1000, 5000)
    for k in ("row_ptr", "col_idx", "values", "c", "lc", "uc", "lv", "uv"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
    assert not np.array_equal(a.values, c.values)
    # columns sorted within rows, 5 distinct rows per column
    for i in range(a.nrows):
        row = a.col_idx[a.row_ptr[i]:a.row_ptr[i + 1]]
        assert np.all(np.diff(row) > 0)
    assert np.all(np.bincount(a.col_idx, minlength=a.ncols) == 5)
    assert np.all(a.lc[:250] == a.uc[:250]) and np.all(np.isneginf(a.lc[250:]))
    assert np.all(a.lv == 0.0) and np.all(a.uv == 10.0)
    assert np.all(np.abs(a.c) <= 1.0)
    assert abs(a.values.mean()) < 0.1 and abs(a.values.std() - 1.0) < 0.1


def test_powerlaw_generator_hits_its_target():
    p = sp.generate_powerlaw_lp(5, 20_000, 40_000, 400_000, 1.5, 2, 5000)
    assert p.nnz == 400_000
    deg = np.bincount(p.col_idx, minlength=p.ncols)
    assert deg.min() >= 2 and deg.max() <= 5000
    assert deg.max() > 20 * np.median(deg)  # a heavy tail


def test_transport_generator_balances_supply_and_demand():
    p = sp.generate_transport_lp(3, 40, 50)
    assert (p.nrows, p.ncols, p.nnz) == (90, 2000, 4000)
    assert np.all(np.bincount(p.col_idx, minlength=p.ncols) == 2)
    assert p.lc[:40].sum() == p.lc[40:].sum()
    assert np.all(p.lc == p.uc) and np.all(np.isposinf(p.uv))
    assert set(np.unique(p.c)).issubset(set(range(1, 101)))


def test_server_footprint_grows_with_size():
    f1 = sp.Server.footprint(1000, 2000, 10_000)
    f2 = sp.Server.footprint(100_000, 200_000, 1_000_000)
    assert 0 < f1 < f2
    assert sp.Server.footprint(10, 20, 100, 1) > sp.Server.footprint(10, 20, 100, 0)


@pytest.mark.parametrize("kind,args", [
    ("random", (3, 50, 100, (3, 8))), ("random", (11, 500, 1000, (5, 5))), ("random", (7, 2000, 4000, (1, 40))),
    ("powerlaw", (5, 2000, 4000, 40_000)), ("powerlaw", (3, 20_000, 40_000, 400_000)),
    ("powerlaw", (1, 200, 400, 20_000)), ("transport", (1, 30, 40)), ("transport", (5, 300, 300)),
])
def test_generators_equal_the_oracle_copy(kind, args):
    """The library's seeded generators (host code) and the oracle's C copy build the same
    arrays bit for bit; the oracle's copy is what the CPU-side benchmark arm and the
    fixture script use, so they never load the library."""
    import oracle

    ours = getattr(sp, f"generate_{kind}_lp")(*args)
    ref = getattr(oracle, f"generate_{kind}_lp")(*args)
    assert (ours.nrows, ours.ncols, ours.nnz) == (ref.nrows, ref.ncols, ref.nnz)
    assert np.array_equal(ours.row_ptr, ref.row_ptr)
    assert np.array_equal(ours.col_idx.astype(np.int64), ref.col_idx)
    for k in ("values", "c", "lc", "uc", "lv", "uv"):
        assert np.array_equal(getattr(ours, k), getattr(ref, k)), k
