"""CPU oracle for the PDHG path — TEST INFRASTRUCTURE ONLY.

ctypes binding of ``oracle/_build/libsp_oracle.so``, a plain-C restatement of
the reference saddlepoint's CPU path (``crates/saddlepoint-core``,
``crates/saddlepoint-cpu``, ``crates/saddlepoint-check``,
``crates/saddlepoint-io``). Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg may import this module, and only as the checker
(or the timed CPU baseline): the CUDA library never calls it.

Problems are passed as any object with the attributes ``nrows, ncols, row_ptr,
col_idx, values, c, c0, lc, uc, lv, uv, maximize`` (numpy arrays for the
vectors), which ``OracleLp`` and ``saddlepoint_b200.LpProblem`` both have.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libsp_oracle.so")

i64 = C.c_int64
u64 = C.c_uint64
dbl = C.c_double
PD = C.POINTER(C.c_double)
PI64 = C.POINTER(C.c_int64)


class Csr(C.Structure):
    _fields_ = [("nrows", i64), ("ncols", i64), ("nnz", i64), ("row_ptr", PI64), ("col_idx", PI64), ("values", PD)]


class Lp(C.Structure):
    _fields_ = [("a", Csr), ("c", PD), ("lc", PD), ("uc", PD), ("lv", PD), ("uv", PD), ("c0", dbl), ("maximize", C.c_int)]


class ScalingParams(C.Structure):
    _fields_ = [
        ("geometric_mean_passes", i64),
        ("ruiz_iterations", i64),
        ("pock_chambolle_enabled", C.c_int),
        ("pock_chambolle_alpha", dbl),
        ("bound_objective_rescaling", C.c_int),
    ]


class ScaledC(C.Structure):
    _fields_ = [
        ("a", Csr), ("at", Csr), ("c", PD), ("lc", PD), ("uc", PD), ("lv", PD), ("uv", PD),
        ("row_scale", PD), ("col_scale", PD), ("bound_scale", dbl), ("obj_scale", dbl),
    ]


class SolverParams(C.Structure):
    _fields_ = [
        ("tolerance", dbl), ("infeasibility_tolerance", dbl), ("max_iterations", u64), ("time_limit_s", dbl),
        ("check_every", u64), ("step_size_factor", dbl), ("reflection", dbl),
        ("restart_sufficient", dbl), ("restart_necessary", dbl), ("restart_artificial", dbl),
        ("pid_kp", dbl), ("pid_ki", dbl), ("pid_kd", dbl), ("pid_discount", dbl),
        ("power_iterations", u64), ("scaling", ScalingParams), ("termination", C.c_int),
    ]


class CheckRecord(C.Structure):
    _fields_ = [
        ("total", u64), ("k_after", u64), ("residual", dbl), ("omega", dbl), ("primal_obj", dbl),
        ("dual_obj", dbl), ("primal_res", dbl), ("dual_res", dbl), ("restarted", C.c_int),
    ]


class Solution(C.Structure):
    _fields_ = [
        ("status", C.c_int), ("x", PD), ("y", PD), ("objective", dbl), ("dual_objective", dbl),
        ("primal_residual", dbl), ("dual_residual", dbl), ("gap", dbl), ("iterations", u64), ("restarts", u64),
        ("solve_time_s", dbl), ("norm_estimate", dbl), ("trace", C.POINTER(CheckRecord)), ("trace_len", i64),
    ]


class KktReport(C.Structure):
    _fields_ = [
        ("primal_objective", dbl), ("dual_objective", dbl), ("constraint_violation", dbl),
        ("bound_violation", dbl), ("dual_violation", dbl), ("relative_primal", dbl),
        ("relative_dual", dbl), ("relative_gap", dbl),
    ]

    def max_relative(self) -> float:
        return max(self.relative_primal, self.relative_dual, self.relative_gap)

    def verify(self, tol: float) -> None:
        if not self.max_relative() <= tol:
            raise AssertionError(
                f"KKT check failed at tol {tol:e}: primal {self.relative_primal:.3e}, "
                f"dual {self.relative_dual:.3e}, gap {self.relative_gap:.3e}"
            )


class CpuProblem(C.Structure):
    _fields_ = [
        ("a", C.POINTER(Csr)), ("at", C.POINTER(Csr)), ("c", PD), ("lc", PD), ("uc", PD), ("lv", PD), ("uv", PD),
        ("primal_factor", PD), ("dual_factor", PD),
    ]


class PrimalStats(C.Structure):
    _fields_ = [("residual_sq", dbl), ("objective", dbl)]


class DualStats(C.Structure):
    _fields_ = [("residual_sq", dbl), ("objective", dbl)]


class RayStats(C.Structure):
    _fields_ = [("objective", dbl), ("violation_sq", dbl), ("norm_sq", dbl)]


class GenParams(C.Structure):
    _fields_ = [
        ("kind", C.c_int), ("seed", u64), ("nrows", i64), ("ncols", i64), ("nnz_per_col_min", i64),
        ("nnz_per_col_max", i64), ("target_nnz", i64), ("zipf_s", dbl), ("degree_min", i64), ("degree_max", i64),
        ("supplies", i64), ("demands", i64),
    ]


class Pid(C.Structure):
    _fields_ = [("integral", dbl), ("prev_error", dbl), ("has_prev", C.c_int), ("best_weight", dbl), ("best_balance", dbl)]


STATUS = {0: "Optimal", 1: "PrimalInfeasible", 2: "DualInfeasible", 3: "IterationLimit", 4: "TimeLimit"}

_lib = None


def build(force: bool = False) -> str:
    """Compiles the oracle with its Makefile (gcc); returns the library path."""
    if force or not os.path.exists(_LIB_PATH) or _stale():
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def _stale() -> bool:
    t = os.path.getmtime(_LIB_PATH)
    return any(os.path.getmtime(os.path.join(_HERE, f)) > t for f in ("sp_oracle.c", "sp_mps.c", "sp_gen.c", "sp_oracle.h"))


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        L = _lib
        L.or_solve.argtypes = [C.POINTER(Lp), C.POINTER(SolverParams), C.POINTER(Solution)]
        L.or_solution_free.argtypes = [C.POINTER(Solution)]
        L.or_solver_params_default.argtypes = [C.POINTER(SolverParams)]
        L.or_check.argtypes = [C.POINTER(Lp), PD, PD, C.POINTER(KktReport)]
        L.or_read_mps.argtypes = [C.c_char_p, C.c_size_t, C.POINTER(Lp), PI64, C.c_char_p, C.c_size_t]
        L.or_lp_free.argtypes = [C.POINTER(Lp)]
        L.or_csr_from_triplets.argtypes = [i64, i64, i64, PI64, PI64, PD, C.POINTER(Csr)]
        L.or_csr_transpose.argtypes = [C.POINTER(Csr), C.POINTER(Csr)]
        L.or_csr_free.argtypes = [C.POINTER(Csr)]
        L.or_scaled_new.argtypes = [C.POINTER(Lp), C.POINTER(ScalingParams), C.POINTER(ScaledC)]
        L.or_scaled_free.argtypes = [C.POINTER(ScaledC)]
        L.or_scaling_params_default.argtypes = [C.POINTER(ScalingParams)]
        L.or_cpu_load.argtypes = [C.POINTER(ScaledC), C.POINTER(CpuProblem)]
        L.or_cpu_free.argtypes = [C.POINTER(CpuProblem)]
        for name in ("or_cpu_spmv", "or_cpu_spmv_t"):
            getattr(L, name).argtypes = [C.POINTER(CpuProblem), PD, PD]
        L.or_cpu_primal_step.argtypes = [C.POINTER(CpuProblem), PD, PD, dbl, PD, PD]
        L.or_cpu_dual_step.argtypes = [C.POINTER(CpuProblem), PD, PD, dbl, PD]
        L.or_cpu_halpern_step.argtypes = [PD, PD, PD, dbl, dbl, i64]
        L.or_cpu_distance_sq.argtypes = [PD, PD, i64]
        L.or_cpu_distance_sq.restype = dbl
        L.or_cpu_sub.argtypes = [PD, PD, PD, i64]
        L.or_cpu_norm_sq.argtypes = [PD, i64]
        L.or_cpu_norm_sq.restype = dbl
        L.or_cpu_dot.argtypes = [PD, PD, i64]
        L.or_cpu_dot.restype = dbl
        L.or_cpu_scale.argtypes = [PD, dbl, i64]
        L.or_cpu_primal_stats.argtypes = [C.POINTER(CpuProblem), PD, PD]
        L.or_cpu_primal_stats.restype = PrimalStats
        L.or_cpu_dual_stats.argtypes = [C.POINTER(CpuProblem), PD, PD]
        L.or_cpu_dual_stats.restype = DualStats
        L.or_cpu_step_dual_residual_sq.argtypes = [C.POINTER(CpuProblem), PD, PD, PD, PD, dbl]
        L.or_cpu_step_dual_residual_sq.restype = dbl
        L.or_cpu_primal_ray_stats.argtypes = [C.POINTER(CpuProblem), PD, PD]
        L.or_cpu_primal_ray_stats.restype = RayStats
        L.or_cpu_dual_ray_stats.argtypes = [C.POINTER(CpuProblem), PD, PD]
        L.or_cpu_dual_ray_stats.restype = RayStats
        L.or_pid_init.argtypes = [C.POINTER(Pid), dbl]
        L.or_pid_update.argtypes = [C.POINTER(Pid), C.POINTER(SolverParams), dbl, dbl, dbl, dbl, dbl]
        L.or_pid_update.restype = dbl
        L.or_set_threads.argtypes = [C.c_int]
        L.or_get_threads.restype = C.c_int
        L.or_lp_validate.argtypes = [C.POINTER(Lp)]
        L.or_lp_validate_at.argtypes = [C.POINTER(Lp), C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int64)]
        L.or_generate.argtypes = [C.POINTER(GenParams), C.POINTER(Lp)]
    return _lib


def set_threads(n: int) -> None:
    lib().or_set_threads(int(n))


def get_threads() -> int:
    return int(lib().or_get_threads())


# ---------------------------------------------------------------- helpers

def _pd(a: np.ndarray):
    return a.ctypes.data_as(PD)


def _pi(a: np.ndarray):
    return a.ctypes.data_as(PI64)


def _f64(v) -> np.ndarray:
    return np.ascontiguousarray(v, dtype=np.float64)


def _i64(v) -> np.ndarray:
    return np.ascontiguousarray(v, dtype=np.int64)


def _arr(ptr, n, dtype=np.float64) -> np.ndarray:
    if n == 0:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)


@dataclass
class OracleLp:
    """The reference's LpProblem (crates/saddlepoint-core/src/problem.rs:129-145) as numpy arrays."""

    nrows: int
    ncols: int
    row_ptr: np.ndarray
    col_idx: np.ndarray
    values: np.ndarray
    c: np.ndarray
    lc: np.ndarray
    uc: np.ndarray
    lv: np.ndarray
    uv: np.ndarray
    c0: float = 0.0
    maximize: bool = False
    name: str = ""

    @property
    def nnz(self) -> int:
        return int(self.values.shape[0])


class _LpView:
    """Keeps numpy buffers alive while a C view of an LP is in use."""

    def __init__(self, p):
        self.rp = _i64(p.row_ptr)
        self.ci = _i64(p.col_idx)
        self.v = _f64(p.values)
        self.vecs = [_f64(getattr(p, k)) for k in ("c", "lc", "uc", "lv", "uv")]
        c, lc, uc, lv, uv = self.vecs
        self.s = Lp()
        self.s.a = Csr(int(p.nrows), int(p.ncols), int(self.v.shape[0]), _pi(self.rp), _pi(self.ci), _pd(self.v))
        self.s.c, self.s.lc, self.s.uc, self.s.lv, self.s.uv = _pd(c), _pd(lc), _pd(uc), _pd(lv), _pd(uv)
        self.s.c0 = float(p.c0)
        self.s.maximize = int(bool(p.maximize))


def _csr_to_np(c: Csr):
    return (_arr(c.row_ptr, c.nrows + 1, np.int64), _arr(c.col_idx, c.nnz, np.int64), _arr(c.values, c.nnz))


def read_mps(text: bytes, name: str = "") -> OracleLp:
    """read_mps (crates/saddlepoint-io/src/lib.rs:59-309). Raises ValueError('line N: msg')."""
    L = lib()
    lp = Lp()
    line = i64(0)
    err = C.create_string_buffer(256)
    rc = L.or_read_mps(text, len(text), C.byref(lp), C.byref(line), err, 256)
    if rc != 0:
        raise ValueError(f"line {line.value}: {err.value.decode()}")
    m, n = lp.a.nrows, lp.a.ncols
    rp, ci, v = _csr_to_np(lp.a)
    out = OracleLp(
        nrows=m, ncols=n, row_ptr=rp, col_idx=ci, values=v, c=_arr(lp.c, n), lc=_arr(lp.lc, m),
        uc=_arr(lp.uc, m), lv=_arr(lp.lv, n), uv=_arr(lp.uv, n), c0=lp.c0, maximize=bool(lp.maximize), name=name,
    )
    L.or_lp_free(C.byref(lp))
    return out


def _take(lp: Lp, name: str) -> OracleLp:
    m, n = lp.a.nrows, lp.a.ncols
    rp, ci, v = _csr_to_np(lp.a)
    out = OracleLp(
        nrows=m, ncols=n, row_ptr=rp, col_idx=ci, values=v, c=_arr(lp.c, n), lc=_arr(lp.lc, m),
        uc=_arr(lp.uc, m), lv=_arr(lp.lv, n), uv=_arr(lp.uv, n), c0=lp.c0, maximize=bool(lp.maximize), name=name,
    )
    lib().or_lp_free(C.byref(lp))
    return out


def _generate(g: GenParams, name: str) -> OracleLp:
    lp = Lp()
    rc = lib().or_generate(C.byref(g), C.byref(lp))
    if rc != 0:
        raise ValueError(f"generator rejected its parameters ({rc})")
    return _take(lp, name)


def generate_random_lp(seed: int, nrows: int, ncols: int, nnz_per_col=(5, 5)) -> OracleLp:
    """The random LP recipe (the CUDA library's generate_random_lp, the same arrays)."""
    g = GenParams(kind=0, seed=seed, nrows=nrows, ncols=ncols, nnz_per_col_min=nnz_per_col[0],
                  nnz_per_col_max=nnz_per_col[1])
    return _generate(g, f"random_{nrows}x{ncols}_s{seed}")


def generate_powerlaw_lp(seed: int, nrows: int, ncols: int, target_nnz: int, zipf_s: float = 1.5,
                         degree_min: int = 2, degree_max: int = 5000) -> OracleLp:
    """Power-law column degrees (the CUDA library's generate_powerlaw_lp, the same arrays)."""
    g = GenParams(kind=1, seed=seed, nrows=nrows, ncols=ncols, target_nnz=target_nnz, zipf_s=zipf_s,
                  degree_min=degree_min, degree_max=degree_max)
    return _generate(g, f"powerlaw_{nrows}x{ncols}_{target_nnz}_s{seed}")


def generate_transport_lp(seed: int, supplies: int = 2000, demands: int = 2000) -> OracleLp:
    """Transportation LP (the CUDA library's generate_transport_lp, the same arrays)."""
    g = GenParams(kind=2, seed=seed, supplies=supplies, demands=demands)
    return _generate(g, f"transport_{supplies}x{demands}_s{seed}")


def from_triplets(nrows: int, ncols: int, rows, cols, vals):
    """CsrMatrix::from_triplets (problem.rs:33-77) -> (row_ptr, col_idx, values)."""
    L = lib()
    r, c, v = _i64(rows), _i64(cols), _f64(vals)
    out = Csr()
    rc = L.or_csr_from_triplets(nrows, ncols, len(v), _pi(r), _pi(c), _pd(v), C.byref(out))
    if rc != 0:
        raise ValueError("triplet out of range")
    res = _csr_to_np(out)
    L.or_csr_free(C.byref(out))
    return res


def transpose(nrows: int, ncols: int, row_ptr, col_idx, values):
    """CsrMatrix::transpose (problem.rs:88-109) -> (row_ptr, col_idx, values)."""
    L = lib()
    rp, ci, v = _i64(row_ptr), _i64(col_idx), _f64(values)
    a = Csr(nrows, ncols, len(v), _pi(rp), _pi(ci), _pd(v))
    out = Csr()
    L.or_csr_transpose(C.byref(a), C.byref(out))
    res = _csr_to_np(out)
    L.or_csr_free(C.byref(out))
    return res


def default_scaling() -> ScalingParams:
    s = ScalingParams()
    lib().or_scaling_params_default(C.byref(s))
    return s


def default_params(**kw) -> SolverParams:
    p = SolverParams()
    lib().or_solver_params_default(C.byref(p))
    for k, v in kw.items():
        if k == "termination" and isinstance(v, str):
            v = {"projected": 0, "step_implied": 1, "cupdlpx": 1}[v]
        setattr(p, k, v)
    return p


@dataclass
class Scaled:
    """ScaledProblem (crates/saddlepoint-core/src/scaling.rs:36-50) as numpy arrays."""

    a: tuple
    at: tuple
    c: np.ndarray
    lc: np.ndarray
    uc: np.ndarray
    lv: np.ndarray
    uv: np.ndarray
    row_scale: np.ndarray
    col_scale: np.ndarray
    bound_scale: float
    obj_scale: float
    nrows: int = 0
    ncols: int = 0

    def primal_residual_factors(self):
        return 1.0 / (self.row_scale * self.bound_scale)

    def dual_residual_factors(self):
        return 1.0 / (self.col_scale * self.obj_scale)

    def objective_factor(self):
        return 1.0 / (self.bound_scale * self.obj_scale)


def scaled_problem(p, params: ScalingParams | None = None) -> Scaled:
    """ScaledProblem::new (scaling.rs:53-103)."""
    L = lib()
    view = _LpView(p)
    sp = params if params is not None else default_scaling()
    cs = ScaledC()
    L.or_scaled_new(C.byref(view.s), C.byref(sp), C.byref(cs))
    m, n = int(p.nrows), int(p.ncols)
    res = Scaled(
        a=_csr_to_np(cs.a), at=_csr_to_np(cs.at), c=_arr(cs.c, n), lc=_arr(cs.lc, m), uc=_arr(cs.uc, m),
        lv=_arr(cs.lv, n), uv=_arr(cs.uv, n), row_scale=_arr(cs.row_scale, m), col_scale=_arr(cs.col_scale, n),
        bound_scale=cs.bound_scale, obj_scale=cs.obj_scale, nrows=m, ncols=n,
    )
    L.or_scaled_free(C.byref(cs))
    return res


@dataclass
class OracleSolution:
    """Solution (solver.rs:104-121) plus the per-check trace."""

    status: str
    x: np.ndarray
    y: np.ndarray
    objective: float
    dual_objective: float
    primal_residual: float
    dual_residual: float
    gap: float
    iterations: int
    restarts: int
    solve_time: float
    norm_estimate: float
    trace: list = field(default_factory=list)


def solve(p, params: SolverParams | None = None, **kw) -> OracleSolution:
    """solve (solver.rs:154-157) on the CPU oracle. Raises RuntimeError on a SolveError."""
    L = lib()
    view = _LpView(p)
    prm = params if params is not None else default_params(**kw)
    sol = Solution()
    rc = L.or_solve(C.byref(view.s), C.byref(prm), C.byref(sol))
    if rc != 0:
        raise RuntimeError({-1: "invalid problem", -2: "numerical breakdown", -3: "allocation"}.get(rc, str(rc)))
    m, n = int(p.nrows), int(p.ncols)
    trace = [
        dict(total=int(r.total), k_after=int(r.k_after), residual=r.residual, omega=r.omega,
             primal_obj=r.primal_obj, dual_obj=r.dual_obj, primal_res=r.primal_res, dual_res=r.dual_res,
             restarted=bool(r.restarted))
        for r in (sol.trace[i] for i in range(sol.trace_len))
    ]
    out = OracleSolution(
        status=STATUS[sol.status], x=_arr(sol.x, n), y=_arr(sol.y, m), objective=sol.objective,
        dual_objective=sol.dual_objective, primal_residual=sol.primal_residual, dual_residual=sol.dual_residual,
        gap=sol.gap, iterations=int(sol.iterations), restarts=int(sol.restarts), solve_time=sol.solve_time_s,
        norm_estimate=sol.norm_estimate, trace=trace,
    )
    L.or_solution_free(C.byref(sol))
    return out


def solve_scaled(p, s, params: SolverParams | None = None, norm_estimate: float = 0.0, stop_after: int = 0,
                 **kw) -> OracleSolution:
    """Solver::run (solver.rs:311-438) on a given ScaledProblem ``s`` (any object with the
    attributes of ``Scaled``); ``norm_estimate`` > 0 replaces estimate_norm; ``stop_after`` > 0
    ends the loop after that many iterations without forcing a check. Used to time the loop
    alone on a large problem without the serial scaling passes."""
    L = lib()
    L.or_solve_scaled.argtypes = [C.POINTER(Lp), C.POINTER(ScaledC), C.POINTER(SolverParams), dbl, u64,
                                  C.POINTER(Solution)]
    view = _LpView(p)
    m, n = int(p.nrows), int(p.ncols)
    keep = [_i64(s.a[0]), _i64(s.a[1]), _f64(s.a[2]), _i64(s.at[0]), _i64(s.at[1]), _f64(s.at[2])]
    vecs = [_f64(v) for v in (s.c, s.lc, s.uc, s.lv, s.uv, s.row_scale, s.col_scale)]
    cs = ScaledC()
    cs.a = Csr(m, n, len(keep[2]), _pi(keep[0]), _pi(keep[1]), _pd(keep[2]))
    cs.at = Csr(n, m, len(keep[5]), _pi(keep[3]), _pi(keep[4]), _pd(keep[5]))
    cs.c, cs.lc, cs.uc, cs.lv, cs.uv, cs.row_scale, cs.col_scale = [_pd(v) for v in vecs]
    cs.bound_scale, cs.obj_scale = float(s.bound_scale), float(s.obj_scale)
    prm = params if params is not None else default_params(**kw)
    sol = Solution()
    rc = L.or_solve_scaled(C.byref(view.s), C.byref(cs), C.byref(prm), float(norm_estimate), int(stop_after),
                           C.byref(sol))
    if rc != 0:
        raise RuntimeError(f"oracle solve failed ({rc})")
    out = OracleSolution(
        status=STATUS[sol.status], x=_arr(sol.x, n), y=_arr(sol.y, m), objective=sol.objective,
        dual_objective=sol.dual_objective, primal_residual=sol.primal_residual, dual_residual=sol.dual_residual,
        gap=sol.gap, iterations=int(sol.iterations), restarts=int(sol.restarts), solve_time=sol.solve_time_s,
        norm_estimate=sol.norm_estimate,
    )
    L.or_solution_free(C.byref(sol))
    return out


def check(p, x, y) -> KktReport:
    """saddlepoint_check::check (crates/saddlepoint-check/src/lib.rs:62-118)."""
    L = lib()
    view = _LpView(p)
    xx, yy = _f64(x), _f64(y)
    r = KktReport()
    L.or_check(C.byref(view.s), _pd(xx), _pd(yy), C.byref(r))
    return r


def validate(p) -> bool:
    return lib().or_lp_validate(C.byref(_LpView(p).s)) == 0


def validate_message(p) -> str:
    """LpProblem::validate's error text (problem.rs:148-154, 166-194) for the first failure, ""
    when the problem is valid; numbers as Rust's `{}` prints an f64 (shortest round trip,
    never an exponent)."""
    import numpy as np

    what, kind, index = C.c_int(), C.c_int(), C.c_int64()
    if lib().or_lp_validate_at(C.byref(_LpView(p).s), C.byref(what), C.byref(kind), C.byref(index)) == 0:
        return ""
    name = ("variable", "constraint", "coefficient")[what.value]
    i = index.value
    if kind.value == 1:
        return f"{name} {i} is NaN"
    lo, hi = (p.lv, p.uv) if what.value == 0 else (p.lc, p.uc)

    def num(v):
        return np.format_float_positional(float(v), trim="-")

    return f"{name} {i} has lower bound {num(lo[i])} above upper bound {num(hi[i])}"


class CpuBackend:
    """The reference CpuBackend (crates/saddlepoint-cpu/src/lib.rs:101-260) over numpy vectors.

    ``load`` takes a ``Scaled``; every method mirrors the trait method of the same name.
    """

    def __init__(self):
        self.L = lib()

    class Problem:
        pass

    def load(self, s: Scaled):
        P = CpuBackend.Problem()
        P.keep = [_i64(s.a[0]), _i64(s.a[1]), _f64(s.a[2]), _i64(s.at[0]), _i64(s.at[1]), _f64(s.at[2])]
        k = P.keep
        P.a = Csr(s.nrows, s.ncols, len(k[2]), _pi(k[0]), _pi(k[1]), _pd(k[2]))
        P.at = Csr(s.ncols, s.nrows, len(k[5]), _pi(k[3]), _pi(k[4]), _pd(k[5]))
        P.vecs = [_f64(v) for v in (s.c, s.lc, s.uc, s.lv, s.uv)]
        P.pf = _f64(s.primal_residual_factors())
        P.df = _f64(s.dual_residual_factors())
        P.c = CpuProblem(C.pointer(P.a), C.pointer(P.at), *[_pd(v) for v in P.vecs], _pd(P.pf), _pd(P.df))
        P.m, P.n = s.nrows, s.ncols
        return P

    def spmv(self, P, x):
        out = np.empty(P.m)
        self.L.or_cpu_spmv(C.byref(P.c), _pd(_f64(x)), _pd(out))
        return out

    def spmv_t(self, P, y):
        out = np.empty(P.n)
        self.L.or_cpu_spmv_t(C.byref(P.c), _pd(_f64(y)), _pd(out))
        return out

    def primal_step(self, P, x, aty, tau):
        xt, xb = np.empty(P.n), np.empty(P.n)
        self.L.or_cpu_primal_step(C.byref(P.c), _pd(_f64(x)), _pd(_f64(aty)), tau, _pd(xt), _pd(xb))
        return xt, xb

    def dual_step(self, P, y, ax_bar, sigma):
        yt = np.empty(P.m)
        self.L.or_cpu_dual_step(C.byref(P.c), _pd(_f64(y)), _pd(_f64(ax_bar)), sigma, _pd(yt))
        return yt

    def halpern_step(self, z, z_t, anchor, w, rho):
        out = _f64(z).copy()
        self.L.or_cpu_halpern_step(_pd(out), _pd(_f64(z_t)), _pd(_f64(anchor)), w, rho, len(out))
        return out

    def distance_sq(self, a, b):
        a, b = _f64(a), _f64(b)
        return self.L.or_cpu_distance_sq(_pd(a), _pd(b), len(a))

    def sub(self, a, b):
        a, b = _f64(a), _f64(b)
        out = np.empty(len(a))
        self.L.or_cpu_sub(_pd(a), _pd(b), _pd(out), len(a))
        return out

    def norm_sq(self, v):
        v = _f64(v)
        return self.L.or_cpu_norm_sq(_pd(v), len(v))

    def dot(self, a, b):
        a, b = _f64(a), _f64(b)
        return self.L.or_cpu_dot(_pd(a), _pd(b), len(a))

    def scale(self, v, alpha):
        out = _f64(v).copy()
        self.L.or_cpu_scale(_pd(out), alpha, len(out))
        return out

    def primal_stats(self, P, x, ax):
        r = self.L.or_cpu_primal_stats(C.byref(P.c), _pd(_f64(x)), _pd(_f64(ax)))
        return r.residual_sq, r.objective

    def dual_stats(self, P, y, aty):
        r = self.L.or_cpu_dual_stats(C.byref(P.c), _pd(_f64(y)), _pd(_f64(aty)))
        return r.residual_sq, r.objective

    def step_dual_residual_sq(self, P, x, x_t, aty, aty_t, tau):
        return self.L.or_cpu_step_dual_residual_sq(
            C.byref(P.c), _pd(_f64(x)), _pd(_f64(x_t)), _pd(_f64(aty)), _pd(_f64(aty_t)), tau
        )

    def primal_ray_stats(self, P, dx, adx):
        r = self.L.or_cpu_primal_ray_stats(C.byref(P.c), _pd(_f64(dx)), _pd(_f64(adx)))
        return r.objective, r.violation_sq, r.norm_sq

    def dual_ray_stats(self, P, dy, atdy):
        r = self.L.or_cpu_dual_ray_stats(C.byref(P.c), _pd(_f64(dy)), _pd(_f64(atdy)))
        return r.objective, r.violation_sq, r.norm_sq


class PidState:
    """PidState (solver.rs:445-480), for its unit tests."""

    def __init__(self, omega: float):
        self.s = Pid()
        lib().or_pid_init(C.byref(self.s), omega)

    def update(self, params: SolverParams, omega, dx, dy, rel_primal, rel_dual) -> float:
        return lib().or_pid_update(C.byref(self.s), C.byref(params), omega, dx, dy, rel_primal, rel_dual)

    @property
    def integral(self):
        return self.s.integral
