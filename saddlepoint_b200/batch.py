"""Batched and serving forms (Parts 3 and 4 of the C ABI in include/saddlepoint_b200.h)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from . import _lib as L


def _pkg():
    import saddlepoint_b200

    return saddlepoint_b200


from . import _Handle  # noqa: E402  (the package defines it before importing this module)


class _BatchHandle(_Handle):
    _free = "sp_batch_free"


class _ServerHandle(_Handle):
    _free = "sp_server_destroy"


@dataclass
class BatchResult:
    status: int  # Status value, or negative for a numerical breakdown
    objective: float
    dual_objective: float
    primal_residual: float
    dual_residual: float
    gap: float
    iterations: int
    restarts: int
    lanes_a: int  # lanes per row the tuner picked for A' (0: the staged-tile variant)
    lanes_t: int  # ... and for A'ᵀ
    handed_off: bool = False  # finished by the single-LP solver after outrunning its batch budget

    @property
    def variant(self) -> str:
        return "tiles" if self.lanes_a == 0 and self.lanes_t == 0 else "lanes"


class BatchSolver:
    """Many LPs solved together by one persistent kernel (one CTA per instance at a time).

    ``solve()`` returns one BatchResult per instance and the device time of the launch;
    ``solution(i)`` downloads instance i's x and y in the original space.
    """

    def __init__(self, problems: list, params=None, backend=None):
        sp = _pkg()
        backend = sp._backend(backend)
        self.lib = backend.lib
        self.problems = [sp.LpProblem.from_any(p) for p in problems]
        views = [sp._LpView(p) for p in self.problems]
        arr = (L.Lp * len(views))(*[v.s for v in views])
        cp = (params or sp.SolverParams()).to_c()
        h = C.c_void_p()
        backend._check(self.lib.sp_batch_create(backend.h, arr, len(views), C.byref(cp), C.byref(h)), sp.SolveError)
        self._handle = _BatchHandle()
        self._handle._attach(backend, h)
        self.backend, self.h = backend, h
        self.count = len(self.problems)

    def close(self):
        self._handle.close()
        self.h = None

    def solve(self):
        res = (L.BatchResult * self.count)()
        t = C.c_double()
        self.backend._check(self.lib.sp_batch_solve(self.h, res, C.byref(t)))
        out = [BatchResult(r.status, r.objective, r.dual_objective, r.primal_residual, r.dual_residual, r.gap,
                           int(r.iterations), int(r.restarts), r.lanes_per_row // 100, r.lanes_per_row % 100,
                           bool(r.handed_off))
               for r in res]
        return out, t.value

    def solution(self, i: int):
        p = self.problems[i]
        x, y = np.empty(p.ncols), np.empty(p.nrows)
        self.backend._check(self.lib.sp_batch_download(self.h, i, x.ctypes.data_as(L.PD), y.ctypes.data_as(L.PD)))
        return x, y


@dataclass
class ServerResult:
    id: int
    status: int
    objective: float
    dual_objective: float
    primal_residual: float
    dual_residual: float
    gap: float
    iterations: int
    queue_s: float
    solve_s: float
    total_s: float
    footprint_bytes: int
    x: np.ndarray
    y: np.ndarray
    error: int = 0        # SP_OK, or the SP_ERR_* code of a failed solve
    path: str = "slot"    # "slot" (a device-resident solve) or "batch" (the batched kernel)
    message: str = ""     # the failed solve's error text


class Server:
    """The serving loop: submit LPs as they arrive, poll results as they finish.

    Requests are admitted first come, first served while their HBM footprint fits in
    ``budget_bytes``; large ones run on ``max_inflight`` concurrent solve slots, those
    with at most ``batch_max_nnz`` nonzeros in launches of the batched kernel.
    """

    def __init__(self, budget_bytes: float = 150e9, max_inflight: int = 8, batch_max_nnz: int = 50_000,
                 params=None, backend=None):
        sp = _pkg()
        backend = sp._backend(backend)
        self.lib = backend.lib
        cfg = L.ServerConfig(float(budget_bytes), int(max_inflight), int(batch_max_nnz))
        cp = (params or sp.SolverParams()).to_c()
        h = C.c_void_p()
        backend._check(self.lib.sp_server_create(backend.h, C.byref(cfg), C.byref(cp), C.byref(h)))
        self._handle = _ServerHandle()
        self._handle._attach(backend, h)
        self.backend, self.h = backend, h
        self._shapes = {}

    def submit(self, problem) -> int:
        sp = _pkg()
        p = sp.LpProblem.from_any(problem)
        view = sp._LpView(p)
        rid = C.c_int64()
        self.backend._check(self.lib.sp_server_submit(self.h, C.byref(view.s), C.byref(rid)), sp.SolveError)
        self._shapes[rid.value] = (p.ncols, p.nrows)
        return rid.value

    def poll(self, timeout: Optional[float] = None) -> Optional[ServerResult]:
        r = L.ServerResult()
        got = C.c_int()
        nmax = max((s[0] for s in self._shapes.values()), default=1)
        mmax = max((s[1] for s in self._shapes.values()), default=1)
        x, y = np.empty(max(nmax, 1)), np.empty(max(mmax, 1))
        rc = self.lib.sp_server_poll(self.h, -1.0 if timeout is None else float(timeout), C.byref(r),
                                     x.ctypes.data_as(L.PD), len(x), y.ctypes.data_as(L.PD), len(y), C.byref(got))
        if not got.value:
            return None
        n, m = self._shapes.pop(r.id)
        return ServerResult(r.id, r.status if rc == 0 else -1, r.objective, r.dual_objective, r.primal_residual,
                            r.dual_residual, r.gap, int(r.iterations), r.queue_s, r.solve_s, r.total_s,
                            int(r.footprint_bytes), x[:n].copy(), y[:m].copy(), int(r.error) or rc,
                            "batch" if r.path == 1 else "slot", r.message.decode(errors="replace"))

    def close(self):
        self._handle.close()
        self.h = None

    @staticmethod
    def footprint(nrows: int, ncols: int, nnz: int, precision: int = 0) -> int:
        return int(L.load().sp_server_footprint(nrows, ncols, nnz, precision))
