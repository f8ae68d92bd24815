"""saddlepoint_b200 — a B200 (sm_100a) backend for saddlepoint's restarted reflected-Halpern PDHG.

Host-side mirror of the reference's Rust API over the C ABI of
``include/saddlepoint_b200.h``:

* ``CudaBackend`` — the fused ``Backend`` trait (crates/saddlepoint-core/src/backend.rs:43-137),
  one method per trait method, each a call into the CUDA library;
* ``LpProblem``, ``SolverParams``, ``Solution``, ``Status``, ``Termination`` — the
  reference's types (crates/saddlepoint-core/src/{problem,solver}.rs);
* ``solve()`` — the device-resident solve (scaling, power iteration, PDHG epochs in
  CUDA graphs, restarts/PID/termination on the device), FP64 or mixed precision;
* ``solve_stepwise()`` — the reference's loop driven over the trait entry points;
* ``Solver`` — a reusable device-resident solver for repeated runs and timing;
* ``BatchSolver`` and ``Server`` — the batched and serving forms;
* ``generate_*`` — the seeded synthetic LP generators.

Everything computes on the GPU; nothing here falls back to the CPU.
"""
from __future__ import annotations

import ctypes as C
import enum
import os
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _lib as L

__all__ = [
    "BackendError", "SolveError", "Status", "Termination", "Precision", "LpProblem", "ScaledProblem",
    "SolverParams", "Solution", "CudaBackend", "Solver", "solve", "solve_stepwise", "BatchSolver", "Server",
    "generate_random_lp", "generate_powerlaw_lp", "generate_transport_lp", "library", "read_mps", "MpsError",
    "csr_from_triplets", "presolve", "Presolved", "solve_presolved", "polish", "validate",
]


class BackendError(RuntimeError):
    """An error from the CUDA library (CudaError in crates/saddlepoint-cuda/src/backend.rs:27-40)."""

    def __init__(self, code: int, message: str = ""):
        self.code = code
        super().__init__(f"{L.ERRORS.get(code, 'error')} ({code}){': ' + message if message else ''}")


class SolveError(BackendError):
    """SolveError (crates/saddlepoint-core/src/solver.rs:123-131): Problem, Numerical or Backend."""


class Status(enum.IntEnum):  # solver.rs:95-102
    Optimal = 0
    PrimalInfeasible = 1
    DualInfeasible = 2
    IterationLimit = 3
    TimeLimit = 4


class Termination(enum.IntEnum):  # solver.rs:56-68
    Projected = 0
    StepImplied = 1


class Precision(enum.IntEnum):
    FP64 = 0
    Mixed = 1


def library():
    return L.load()


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _pd(a: np.ndarray):
    return a.ctypes.data_as(L.PD)


@dataclass
class LpProblem:
    """LpProblem (crates/saddlepoint-core/src/problem.rs:129-145): min cᵀx + c0 s.t. lc ≤ Ax ≤ uc, lv ≤ x ≤ uv."""

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
        return int(len(self.values))

    @classmethod
    def from_any(cls, p) -> "LpProblem":
        if isinstance(p, cls):
            return p
        return cls(int(p.nrows), int(p.ncols), p.row_ptr, p.col_idx, p.values, p.c, p.lc, p.uc, p.lv, p.uv,
                   float(p.c0), bool(p.maximize), getattr(p, "name", ""))

    def objective(self, x) -> float:  # problem.rs:198-201
        v = float(np.dot(self.c, x)) + self.c0
        return -v if self.maximize else v


class _LpView:
    """Keeps the arrays of an LpProblem alive while C holds pointers to them. The C ABI takes
    the lengths from nrows, ncols and the row pointers, so the arrays' own lengths are
    checked here first, as LpProblem::validate checks them (problem.rs:168-177): SolveError
    (SP_ERR_PROBLEM) "c has length 5, expected 24" and the like, before any pointer is handed
    over."""

    def __init__(self, p: LpProblem):
        m, n = int(p.nrows), int(p.ncols)
        for what, v, want in (("c", p.c, n), ("lv", p.lv, n), ("uv", p.uv, n), ("lc", p.lc, m), ("uc", p.uc, m)):
            if len(v) != want:
                raise SolveError(L.SP_ERR_PROBLEM, f"{what} has length {len(v)}, expected {want}")
        if len(p.row_ptr) != m + 1 or len(p.col_idx) != len(p.values):
            raise SolveError(L.SP_ERR_PROBLEM, f"A has length {len(p.row_ptr)}, expected {m + 1}")
        self.rp = np.ascontiguousarray(p.row_ptr, dtype=np.int64)
        self.ci = np.ascontiguousarray(p.col_idx, dtype=np.int32)
        self.v = _f64(p.values)
        self.vecs = [_f64(getattr(p, k)) for k in ("c", "lc", "uc", "lv", "uv")]
        self.s = L.Lp()
        self.s.a = L.Csr(int(p.nrows), int(p.ncols), len(self.v), self.rp.ctypes.data_as(L.PI64),
                         self.ci.ctypes.data_as(L.PI32), _pd(self.v))
        self.s.c, self.s.lc, self.s.uc, self.s.lv, self.s.uv = [_pd(v) for v in self.vecs]
        self.s.c0 = float(p.c0)
        self.s.maximize = int(bool(p.maximize))


@dataclass
class SolverParams:
    """SolverParams (solver.rs:24-52) and ScalingParams (scaling.rs:14-34), with the reference's defaults."""

    tolerance: float = 1e-6
    infeasibility_tolerance: float = 1e-8
    max_iterations: int = 1_000_000
    time_limit: Optional[float] = None
    check_every: int = 64
    step_size_factor: float = 0.998
    reflection: float = 1.0
    restart_sufficient: float = 0.2
    restart_necessary: float = 0.5
    restart_artificial: float = 0.36
    pid_kp: float = 0.99
    pid_ki: float = 0.01
    pid_kd: float = 0.0
    pid_discount: float = 0.3
    power_iterations: int = 200
    geometric_mean_passes: int = 12
    ruiz_iterations: int = 10
    pock_chambolle_alpha: Optional[float] = 1.0
    bound_objective_rescaling: bool = True
    log_every_checks: int = 0
    termination: Termination = Termination.Projected
    precision: Precision = Precision.FP64
    mixed_switch_tolerance: float = 1e-5

    def to_c(self) -> L.Params:
        p = L.Params()
        library().sp_solver_params_default(C.byref(p))
        for k in ("tolerance", "infeasibility_tolerance", "max_iterations", "check_every", "step_size_factor",
                  "reflection", "restart_sufficient", "restart_necessary", "restart_artificial", "pid_kp", "pid_ki",
                  "pid_kd", "pid_discount", "power_iterations", "geometric_mean_passes", "ruiz_iterations",
                  "log_every_checks", "mixed_switch_tolerance"):
            setattr(p, k, getattr(self, k))
        p.time_limit_s = float(self.time_limit) if self.time_limit else 0.0
        p.pock_chambolle_enabled = int(self.pock_chambolle_alpha is not None)
        p.pock_chambolle_alpha = float(self.pock_chambolle_alpha or 0.0)
        p.bound_objective_rescaling = int(self.bound_objective_rescaling)
        p.termination = int(self.termination)
        p.precision = int(self.precision)
        return p


@dataclass
class Solution:
    """Solution (solver.rs:104-121), plus setup time, ‖A'‖₂ and the mixed form's switch point."""

    status: Status
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
    setup_time: float = 0.0
    norm_estimate: float = 0.0
    fp64_from_iteration: int = 0
    trace: list = field(default_factory=list)


def _solution(info: L.Info, x, y) -> Solution:
    return Solution(Status(info.status), x, y, info.objective, info.dual_objective, info.primal_residual,
                    info.dual_residual, info.gap, int(info.iterations), int(info.restarts), info.solve_time_s,
                    info.setup_time_s, info.norm_estimate, int(info.fp64_from_iteration))


@dataclass
class PrimalStats:  # backend.rs:14-20
    residual_sq: float
    objective: float


@dataclass
class DualStats:  # backend.rs:22-29
    residual_sq: float
    objective: float


@dataclass
class RayStats:  # backend.rs:31-41
    objective: float
    violation_sq: float
    norm_sq: float


@dataclass
class ScaledProblem:
    """ScaledProblem (crates/saddlepoint-core/src/scaling.rs:36-50) as host arrays."""

    nrows: int
    ncols: int
    a: tuple  # (row_ptr, col_idx, values)
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

    def primal_residual_factors(self):  # scaling.rs:123-126
        return 1.0 / (self.row_scale * self.bound_scale)

    def dual_residual_factors(self):  # scaling.rs:128-131
        return 1.0 / (self.col_scale * self.obj_scale)

    def objective_factor(self):  # scaling.rs:134-136
        return 1.0 / (self.bound_scale * self.obj_scale)

    def unscale_primal(self, xs):  # scaling.rs:114-116
        return xs * self.col_scale / self.bound_scale

    def unscale_dual(self, ys):  # scaling.rs:119-121
        return ys * self.row_scale / self.obj_scale


class _Handle:
    """A native object that belongs to a backend's context. The backend keeps a weak
    reference to each, so closing the backend frees its objects first and a handle
    never outlives the context it was made on."""

    _free = ""

    def _attach(self, backend: "CudaBackend", handle):
        self.backend, self.h = backend, handle
        backend._children.add(self)

    def close(self):
        h = getattr(self, "h", None)
        if h:
            self.h = None
            getattr(library(), self._free)(h)

    def __del__(self):
        self.close()


class Vector(_Handle):
    """A device vector owned by the backend (Backend::Vector)."""

    _free = "sp_vec_free"

    def __init__(self, backend: "CudaBackend", handle, n: int):
        self.n = n
        self._attach(backend, handle)

    def __len__(self):
        return self.n


class Problem(_Handle):
    """The scaled problem on the device (Backend::Problem)."""

    _free = "sp_problem_free"

    def __init__(self, backend: "CudaBackend", handle, m: int, n: int):
        self.m, self.n = m, n
        self._attach(backend, handle)


class CudaBackend:
    """The Backend trait on a B200 (crates/saddlepoint-core/src/backend.rs:43-137).

    ``CudaBackend(0)`` raises ``BackendError`` (code 4, unavailable) when there is no
    GPU, like ``CudaBackend::new`` returns ``Err`` (crates/saddlepoint-cuda/src/backend.rs:129-140).
    """

    def __init__(self, ordinal: int = 0):
        import weakref

        lib = library()
        h = C.c_void_p()
        rc = lib.sp_ctx_create(ordinal, C.byref(h))
        if rc != L.SP_OK:
            raise BackendError(rc, f"no usable CUDA device {ordinal}")
        self.lib, self.h = lib, h
        self._children = weakref.WeakSet()

    def close(self):
        if getattr(self, "h", None):
            for child in list(self._children):
                child.close()
            self.lib.sp_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _check(self, rc: int, cls=BackendError):
        if rc != L.SP_OK:
            raise cls(rc, self.lib.sp_ctx_last_error(self.h).decode())

    def name(self) -> str:
        buf = C.create_string_buffer(256)
        self._check(self.lib.sp_ctx_name(self.h, buf, 256))
        return buf.value.decode()

    def stream(self) -> int:
        return int(self.lib.sp_ctx_stream(self.h) or 0)

    # ---- Backend::load / upload / download / copy
    def load(self, s: ScaledProblem) -> Problem:
        arp, aci, av = (np.ascontiguousarray(s.a[0], np.int64), np.ascontiguousarray(s.a[1], np.int32), _f64(s.a[2]))
        trp, tci, tv = (np.ascontiguousarray(s.at[0], np.int64), np.ascontiguousarray(s.at[1], np.int32),
                        _f64(s.at[2]))
        A = L.Csr(s.nrows, s.ncols, len(av), arp.ctypes.data_as(L.PI64), aci.ctypes.data_as(L.PI32), _pd(av))
        AT = L.Csr(s.ncols, s.nrows, len(tv), trp.ctypes.data_as(L.PI64), tci.ctypes.data_as(L.PI32), _pd(tv))
        vecs = [_f64(v) for v in (s.c, s.lc, s.uc, s.lv, s.uv, s.primal_residual_factors(), s.dual_residual_factors())]
        h = C.c_void_p()
        self._check(self.lib.sp_problem_load(self.h, C.byref(A), C.byref(AT), *[_pd(v) for v in vecs], C.byref(h)))
        return Problem(self, h, s.nrows, s.ncols)

    def upload(self, data) -> Vector:
        d = _f64(data)
        h = C.c_void_p()
        self._check(self.lib.sp_vec_upload(self.h, _pd(d), len(d), C.byref(h)))
        return Vector(self, h, len(d))

    def download(self, v: Vector) -> np.ndarray:
        out = np.empty(v.n)
        self._check(self.lib.sp_vec_download(self.h, v.h, _pd(out), v.n))
        return out

    def copy(self, src: Vector, dst: Vector) -> None:
        self._check(self.lib.sp_vec_copy(self.h, src.h, dst.h))

    # ---- SpMV and steps
    def spmv(self, p: Problem, x: Vector, out: Vector) -> None:
        self._check(self.lib.sp_spmv(self.h, p.h, x.h, out.h))

    def spmv_t(self, p: Problem, y: Vector, out: Vector) -> None:
        self._check(self.lib.sp_spmv_t(self.h, p.h, y.h, out.h))

    def primal_step(self, p, x, aty, tau, x_t, x_bar) -> None:
        self._check(self.lib.sp_primal_step(self.h, p.h, x.h, aty.h, tau, x_t.h, x_bar.h))

    def dual_step(self, p, y, ax_bar, sigma, y_t) -> None:
        self._check(self.lib.sp_dual_step(self.h, p.h, y.h, ax_bar.h, sigma, y_t.h))

    def halpern_step(self, z, z_t, anchor, w, rho) -> None:
        self._check(self.lib.sp_halpern_step(self.h, z.h, z_t.h, anchor.h, w, rho))

    # ---- vector helpers
    def distance_sq(self, a, b) -> float:
        r = C.c_double()
        self._check(self.lib.sp_distance_sq(self.h, a.h, b.h, C.byref(r)))
        return r.value

    def sub(self, a, b, out) -> None:
        self._check(self.lib.sp_sub(self.h, a.h, b.h, out.h))

    def norm_sq(self, v) -> float:
        r = C.c_double()
        self._check(self.lib.sp_norm_sq(self.h, v.h, C.byref(r)))
        return r.value

    def dot(self, a, b) -> float:
        r = C.c_double()
        self._check(self.lib.sp_dot(self.h, a.h, b.h, C.byref(r)))
        return r.value

    def scale(self, v, alpha) -> None:
        self._check(self.lib.sp_scale(self.h, v.h, alpha))

    # ---- stats
    def primal_stats(self, p, x, ax) -> PrimalStats:
        r = L.PrimalStatsC()
        self._check(self.lib.sp_primal_stats(self.h, p.h, x.h, ax.h, C.byref(r)))
        return PrimalStats(r.residual_sq, r.objective)

    def dual_stats(self, p, y, aty) -> DualStats:
        r = L.DualStatsC()
        self._check(self.lib.sp_dual_stats(self.h, p.h, y.h, aty.h, C.byref(r)))
        return DualStats(r.residual_sq, r.objective)

    def step_dual_residual_sq(self, p, x, x_t, aty, aty_t, tau) -> float:
        r = C.c_double()
        self._check(self.lib.sp_step_dual_residual_sq(self.h, p.h, x.h, x_t.h, aty.h, aty_t.h, tau, C.byref(r)))
        return r.value

    def primal_ray_stats(self, p, dx, adx) -> RayStats:
        r = L.RayStatsC()
        self._check(self.lib.sp_primal_ray_stats(self.h, p.h, dx.h, adx.h, C.byref(r)))
        return RayStats(r.objective, r.violation_sq, r.norm_sq)

    def dual_ray_stats(self, p, dy, atdy) -> RayStats:
        r = L.RayStatsC()
        self._check(self.lib.sp_dual_ray_stats(self.h, p.h, dy.h, atdy.h, C.byref(r)))
        return RayStats(r.objective, r.violation_sq, r.norm_sq)


_default_backend: Optional[CudaBackend] = None


def _backend(b: Optional[CudaBackend]) -> CudaBackend:
    global _default_backend
    if b is not None:
        return b
    if _default_backend is None:
        _default_backend = CudaBackend(0)
    return _default_backend


class Solver(_Handle):
    """A device-resident solve of one LP (scaling, ‖A'‖₂ and iterates stay on the GPU)."""

    _free = "sp_solver_free"

    def __init__(self, problem, params: Optional[SolverParams] = None, backend: Optional[CudaBackend] = None):
        backend = _backend(backend)
        self.problem = LpProblem.from_any(problem)
        self.params = params or SolverParams()
        view = _LpView(self.problem)
        cp = self.params.to_c()
        h = C.c_void_p()
        self.lib = backend.lib
        backend._check(self.lib.sp_solver_create(backend.h, C.byref(view.s), C.byref(cp), C.byref(h)), SolveError)
        self._attach(backend, h)

    def _c(self, rc):
        self.backend._check(rc, SolveError)

    def reset(self):
        self._c(self.lib.sp_solver_reset(self.h))

    def warm_start(self, x=None, y=None):
        """Reset, then start the next solve from (x, y) in the original space (None: zeros)."""
        xv = None if x is None else _f64(x)
        yv = None if y is None else _f64(y)
        if xv is not None and len(xv) != self.problem.ncols or yv is not None and len(yv) != self.problem.nrows:
            raise ValueError("warm start vectors do not fit the problem")
        self._c(self.lib.sp_solver_warm_start(self.h, None if xv is None else _pd(xv), None if yv is None else _pd(yv)))

    def run_epochs(self, epochs: int):
        self._c(self.lib.sp_solver_run_epochs(self.h, epochs))

    def sync(self):
        self._c(self.lib.sp_solver_sync(self.h))

    def info(self) -> L.Info:
        i = L.Info()
        self._c(self.lib.sp_solver_info(self.h, C.byref(i)))
        return i

    def solve(self) -> Solution:
        info = L.Info()
        self._c(self.lib.sp_solver_solve(self.h, C.byref(info)))
        x, y = self.download()
        return _solution(info, x, y)

    def download(self):
        x, y = np.empty(self.problem.ncols), np.empty(self.problem.nrows)
        self._c(self.lib.sp_solver_download(self.h, _pd(x), _pd(y)))
        return x, y

    def trace(self) -> list:
        n = C.c_int64()
        self._c(self.lib.sp_solver_trace(self.h, None, 0, C.byref(n)))
        buf = (L.CheckRecord * max(n.value, 1))()
        self._c(self.lib.sp_solver_trace(self.h, buf, n.value, C.byref(n)))
        return [dict(total=int(r.total), k_after=int(r.k_after), residual=r.residual, omega=r.omega,
                     primal_obj=r.primal_obj, dual_obj=r.dual_obj, primal_res=r.primal_res, dual_res=r.dual_res,
                     restarted=bool(r.restarted)) for r in buf[: n.value]]

    def set_timing(self, every: int):
        self._c(self.lib.sp_solver_set_timing(self.h, every))

    def kernel_timing(self, kernel_id: int):
        """(launches timed, total ms, algorithmic bytes per launch) of pass 0 (primal) or 1 (dual)."""
        n, ms, b = C.c_int64(), C.c_double(), C.c_double()
        self._c(self.lib.sp_solver_kernel_timing(self.h, kernel_id, C.byref(n), C.byref(ms), C.byref(b)))
        return n.value, ms.value, b.value

    def bytes_per_iteration(self) -> float:
        return float(self.lib.sp_solver_bytes_per_iteration(self.h))

    ENGINES = {0: "tiles", 1: "stream", 2: "sell"}

    def engines(self) -> dict:
        """The engine of each fused pass: {'primal_fp64', 'primal_fp32', 'dual_fp64', 'dual_fp32'}
        -> 'tiles' | 'stream' | 'sell' (the FP32 entries apply to the mixed form)."""
        out = (C.c_int32 * 4)()
        self._c(self.lib.sp_solver_engines(self.h, out))
        keys = ("primal_fp64", "primal_fp32", "dual_fp64", "dual_fp32")
        return {k: self.ENGINES[int(v)] for k, v in zip(keys, out)}

    def gather_floor(self, kernel_id: int, fp32: bool = False, reps: int = 10) -> float:
        """Milliseconds of a kernel doing only pass `kernel_id`'s gathers (0 primal, 1 dual)
        through its own index stream: the floor its random gathers set."""
        ms = C.c_double()
        self._c(self.lib.sp_solver_gather_floor(self.h, kernel_id, int(fp32), reps, C.byref(ms)))
        return ms.value

    def epoch_kernels(self) -> int:
        """Kernel launches in one epoch of check_every iterations (its graph's kernel nodes)."""
        n = C.c_int64()
        self._c(self.lib.sp_solver_epoch_kernels(self.h, C.byref(n)))
        return int(n.value)

    def scaled(self) -> ScaledProblem:
        p = self.problem
        m, n, nnz = p.nrows, p.ncols, p.nnz
        arp, trp = np.empty(m + 1, np.int64), np.empty(n + 1, np.int64)
        aci, tci = np.empty(nnz, np.int32), np.empty(nnz, np.int32)
        av, tv = np.empty(nnz), np.empty(nnz)
        c, lv, uv, cs = np.empty(n), np.empty(n), np.empty(n), np.empty(n)
        lc, uc, rs = np.empty(m), np.empty(m), np.empty(m)
        bs, os_ = C.c_double(), C.c_double()
        self._c(self.lib.sp_solver_scaled(
            self.h, arp.ctypes.data_as(L.PI64), aci.ctypes.data_as(L.PI32), _pd(av), trp.ctypes.data_as(L.PI64),
            tci.ctypes.data_as(L.PI32), _pd(tv), _pd(c), _pd(lc), _pd(uc), _pd(lv), _pd(uv), _pd(rs), _pd(cs),
            C.byref(bs), C.byref(os_)))
        return ScaledProblem(m, n, (arp, aci, av), (trp, tci, tv), c, lc, uc, lv, uv, rs, cs, bs.value, os_.value)


def solve(problem, params: Optional[SolverParams] = None, backend: Optional[CudaBackend] = None) -> Solution:
    """solve() (solver.rs:154-157), device-resident: one call, host arrays in and out."""
    b = _backend(backend)
    p = LpProblem.from_any(problem)
    view = _LpView(p)
    cp = (params or SolverParams()).to_c()
    x, y = np.empty(p.ncols), np.empty(p.nrows)
    info = L.Info()
    b._check(b.lib.sp_solve(b.h, C.byref(view.s), C.byref(cp), _pd(x), _pd(y), C.byref(info)), SolveError)
    return _solution(info, x, y)


def solve_stepwise(problem, params: Optional[SolverParams] = None, backend: Optional[CudaBackend] = None) -> Solution:
    """solve() as the reference's host loop over the trait entry points (solver.rs:311-438)."""
    b = _backend(backend)
    p = LpProblem.from_any(problem)
    view = _LpView(p)
    cp = (params or SolverParams()).to_c()
    x, y = np.empty(p.ncols), np.empty(p.nrows)
    info = L.Info()
    b._check(b.lib.sp_solve_stepwise(b.h, C.byref(view.s), C.byref(cp), _pd(x), _pd(y), C.byref(info)), SolveError)
    return _solution(info, x, y)


# ------------------------------------------------------------------ problem input

class MpsError(ValueError):
    """MpsError::Parse (crates/saddlepoint-io/src/lib.rs:21-27): 'line N: message'."""

    def __init__(self, line: int, msg: str):
        super().__init__(f"line {line}: {msg}")
        self.line, self.msg = line, msg


def validate(problem) -> None:
    """LpProblem::validate (crates/saddlepoint-core/src/problem.rs:166-194) in host code:
    raises SolveError (code SP_ERR_PROBLEM) with the reference's message for the first
    failure in its order; every solve runs the same check first."""
    view = _LpView(LpProblem.from_any(problem))
    buf = C.create_string_buffer(256)
    rc = L.load().sp_problem_validate(C.byref(view.s), buf, 256)
    if rc != L.SP_OK:
        raise SolveError(rc, buf.value.decode())


def read_mps(source, name: str = "") -> LpProblem:
    """read_mps / read_mps_file (crates/saddlepoint-io/src/lib.rs:50-309): MPS text (bytes or
    str) or a path to a .mps file (.mps.gz is decompressed first) to an LpProblem."""
    import gzip

    if isinstance(source, (bytes, bytearray)):
        text = bytes(source)
    elif isinstance(source, str) and ("\n" in source or not os.path.exists(source)):
        text = source.encode()
    else:
        path = os.fspath(source)
        with open(path, "rb") as fh:
            text = fh.read()
        if path.endswith(".gz"):
            text = gzip.decompress(text)
        name = name or os.path.basename(path).split(".")[0]
    lib = library()
    out = L.Lp()
    line = L.i64(0)
    err = C.create_string_buffer(256)
    rc = lib.sp_read_mps(text, len(text), C.byref(out), C.byref(line), err, 256)
    if rc == L.SP_ERR_PARSE:
        raise MpsError(int(line.value), err.value.decode())
    if rc != L.SP_OK:
        raise BackendError(rc, "sp_read_mps failed")
    return _take_lp(out, name)


def csr_from_triplets(nrows: int, ncols: int, rows, cols, vals, backend: "CudaBackend"):
    """CsrMatrix::from_triplets (crates/saddlepoint-core/src/problem.rs:33-77) on the GPU:
    (row_ptr int64, col_idx int32, values float64) of the CSR matrix, bit for bit the host
    rule (runs of one (row, column) summed in input order, exact-zero sums dropped). An
    index out of range raises BackendError (the reference asserts)."""
    r = np.ascontiguousarray(rows, dtype=np.int64)
    c = np.ascontiguousarray(cols, dtype=np.int64)
    v = np.ascontiguousarray(vals, dtype=np.float64)
    if not (len(r) == len(c) == len(v)):
        raise ValueError("rows, cols and vals differ in length")
    out = L.Csr()
    pi = lambda a: a.ctypes.data_as(L.PI64)  # noqa: E731
    backend._check(backend.lib.sp_csr_from_triplets(backend.h, nrows, ncols, len(v), pi(r), pi(c),
                                                    v.ctypes.data_as(L.PD), C.byref(out)))
    nnz = out.nnz

    def arr(ptr, k, dt):
        return np.ctypeslib.as_array(ptr, shape=(k,)).astype(dt, copy=True) if k else np.zeros(0, dt)

    res = (arr(out.row_ptr, nrows + 1, np.int64), arr(out.col_idx, nnz, np.int32), arr(out.values, nnz, np.float64))
    backend.lib.sp_csr_release(C.byref(out))
    return res


# ------------------------------------------------------------------ generators

def _generate(gp: L.GenParams, name: str) -> LpProblem:
    lib = library()
    out = L.Lp()
    rc = lib.sp_generate(C.byref(gp), C.byref(out))
    if rc != L.SP_OK:
        raise BackendError(rc, "generator rejected its parameters")
    return _take_lp(out, name)


def _take_lp(out: L.Lp, name: str) -> LpProblem:
    """Copies a library-owned sp_lp into an LpProblem and releases it."""
    lib = library()
    m, n, nnz = out.a.nrows, out.a.ncols, out.a.nnz

    def arr(ptr, k, dt):
        return np.ctypeslib.as_array(ptr, shape=(k,)).astype(dt, copy=True) if k else np.zeros(0, dt)

    p = LpProblem(m, n, arr(out.a.row_ptr, m + 1, np.int64), arr(out.a.col_idx, nnz, np.int32),
                  arr(out.a.values, nnz, np.float64), arr(out.c, n, np.float64), arr(out.lc, m, np.float64),
                  arr(out.uc, m, np.float64), arr(out.lv, n, np.float64), arr(out.uv, n, np.float64),
                  out.c0, bool(out.maximize), name)
    lib.sp_lp_release(C.byref(out))
    return p


def generate_random_lp(seed: int, nrows: int, ncols: int, nnz_per_col=(5, 5)) -> LpProblem:
    """Random sparse LP: degree uniform in nnz_per_col at distinct uniform rows, N(0,1) values;
    x0 ~ U[0,1]^n, the first nrows/2 rows equalities b = A x0, the rest ≤ A x0 + U[0,1];
    0 ≤ x ≤ 10; c ~ U[-1,1]."""
    g = L.GenParams(kind=0, seed=seed, nrows=nrows, ncols=ncols, nnz_per_col_min=nnz_per_col[0],
                    nnz_per_col_max=nnz_per_col[1])
    return _generate(g, f"random_{nrows}x{ncols}_s{seed}")


def generate_powerlaw_lp(seed: int, nrows: int, ncols: int, target_nnz: int, zipf_s: float = 1.5,
                         degree_min: int = 2, degree_max: int = 5000) -> LpProblem:
    """Random LP whose column degrees follow a truncated Zipf(s) law rescaled to target_nnz."""
    g = L.GenParams(kind=1, seed=seed, nrows=nrows, ncols=ncols, target_nnz=target_nnz, zipf_s=zipf_s,
                    degree_min=degree_min, degree_max=degree_max)
    return _generate(g, f"powerlaw_{nrows}x{ncols}_{target_nnz}_s{seed}")


def generate_transport_lp(seed: int, supplies: int = 2000, demands: int = 2000) -> LpProblem:
    """Transportation LP: supplies × demands arcs, integer supplies/demands, costs U{1..100}."""
    g = L.GenParams(kind=2, seed=seed, supplies=supplies, demands=demands)
    return _generate(g, f"transport_{supplies}x{demands}_s{seed}")


# ------------------------------------------------------------------ polishing

def polish(problem, x, y, tolerance: float = 1e-9, params: Optional[SolverParams] = None,
           backend: Optional[CudaBackend] = None):
    """Feasibility polishing of a solution (x, y) of `problem` on the GPU: two warm-started FP64
    solves bring x to primal and y to dual feasibility within `tolerance`. Returns
    (x, y, (primal iterations, dual iterations))."""
    b = _backend(backend)
    p = LpProblem.from_any(problem)
    view = _LpView(p)
    cp = (params or SolverParams()).to_c()
    xo, yo = _f64(x).copy(), _f64(y).copy()
    if len(xo) != p.ncols or len(yo) != p.nrows:
        raise ValueError("x and y do not fit the problem")
    it = (C.c_uint64 * 2)()
    b._check(b.lib.sp_polish(b.h, C.byref(view.s), C.byref(cp), float(tolerance), _pd(xo), _pd(yo), it), SolveError)
    return xo, yo, (int(it[0]), int(it[1]))


# ------------------------------------------------------------------ presolve

class Presolved:
    """The result of presolve(): the reduced LP to solve (``reduced``), the status presolve
    proved on its own (``status``, None when the reduced LP is to be solved), the rows and
    columns it removed (``counts``), and postsolve()."""

    def __init__(self, problem: LpProblem):
        lib = library()
        self._view = _LpView(problem)
        self.problem = problem
        out = L.Lp()
        h = C.c_void_p()
        st = C.c_int()
        rc = lib.sp_presolve_create(C.byref(self._view.s), C.byref(out), C.byref(h), C.byref(st))
        if rc != L.SP_OK:
            raise BackendError(rc, "presolve rejected the problem")
        self.h = h
        m, n, nnz = out.a.nrows, out.a.ncols, out.a.nnz

        def arr(ptr, k, dt):
            return np.ctypeslib.as_array(ptr, shape=(k,)).astype(dt, copy=True) if k else np.zeros(0, dt)

        self.reduced = LpProblem(m, n, arr(out.a.row_ptr, m + 1, np.int64), arr(out.a.col_idx, nnz, np.int32),
                                 arr(out.a.values, nnz, np.float64), arr(out.c, n, np.float64),
                                 arr(out.lc, m, np.float64), arr(out.uc, m, np.float64), arr(out.lv, n, np.float64),
                                 arr(out.uv, n, np.float64), out.c0, bool(out.maximize), problem.name)
        self.status = None if st.value < 0 else Status(st.value)
        cnt = (C.c_int64 * 4)()
        lib.sp_presolve_counts(h, cnt)
        self.counts = dict(zip(("empty_rows", "singleton_rows", "fixed_cols", "empty_cols"), (int(v) for v in cnt)))

    def postsolve(self, x_red, y_red):
        """(x, y) of the original problem from the reduced problem's solution."""
        xr, yr = _f64(x_red), _f64(y_red)
        x, y = np.empty(self.problem.ncols), np.empty(self.problem.nrows)
        rc = library().sp_presolve_postsolve(self.h, _pd(xr) if len(xr) else None, _pd(yr) if len(yr) else None,
                                             _pd(x), _pd(y))
        if rc != L.SP_OK:
            raise BackendError(rc, "postsolve: the vectors do not fit the reduced problem")
        return x, y

    def close(self):
        if getattr(self, "h", None):
            library().sp_presolve_free(self.h)
            self.h = None

    def __del__(self):
        self.close()


def presolve(problem) -> Presolved:
    """Exact reductions before the solve (empty and singleton rows, fixed and empty columns),
    host code; solve ``.reduced`` and map its answer back with ``.postsolve``."""
    return Presolved(LpProblem.from_any(problem))


def solve_presolved(problem, params: Optional[SolverParams] = None, backend: Optional[CudaBackend] = None) -> Solution:
    """presolve(), the device-resident solve of the reduced LP, postsolve(): the answer in the
    original problem's space (residuals and iteration counts are the reduced solve's)."""
    p = LpProblem.from_any(problem)
    pre = presolve(p)
    try:
        if pre.status is not None:
            x, y = pre.postsolve(np.zeros(0), np.zeros(0)) if pre.status == Status.Optimal else (
                np.zeros(p.ncols), np.zeros(p.nrows))
            obj = p.objective(x)
            return Solution(pre.status, x, y, obj, obj, 0.0, 0.0, 0.0, 0, 0, 0.0)
        s = solve(pre.reduced, params, backend)
        x, y = pre.postsolve(s.x, s.y)
        return Solution(s.status, x, y, s.objective, s.dual_objective, s.primal_residual, s.dual_residual, s.gap,
                        s.iterations, s.restarts, s.solve_time, s.setup_time, s.norm_estimate,
                        s.fp64_from_iteration)
    finally:
        pre.close()


from .batch import BatchSolver, Server  # noqa: E402  (after the core types)
