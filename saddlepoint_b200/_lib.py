"""ctypes declarations of the C ABI in include/saddlepoint_b200.h.

The shared library is the in-tree build ``saddlepoint_b200/_build/libsaddlepoint_b200.so``
(``python -m saddlepoint_b200.build``). There is no fallback: if the library is
missing or does not load, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libsaddlepoint_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "saddlepoint_b200.h")

i32, i64, u64, dbl, cint = C.c_int32, C.c_int64, C.c_uint64, C.c_double, C.c_int
PD = C.POINTER(C.c_double)
PI64 = C.POINTER(C.c_int64)
PI32 = C.POINTER(C.c_int32)
VP = C.c_void_p

SP_OK = 0
SP_ERR_PROBLEM = 6
SP_ERR_PARSE = 8
ERRORS = {
    1: "CUDA error",
    2: "invalid argument",
    3: "problem too large for 32-bit sparse indices",
    4: "CUDA unavailable",
    5: "numerical breakdown",
    6: "invalid problem",
    7: "device error",
    8: "MPS parse error",
}


class Csr(C.Structure):
    _fields_ = [("nrows", i64), ("ncols", i64), ("nnz", i64), ("row_ptr", PI64), ("col_idx", PI32), ("values", PD)]


class Lp(C.Structure):
    _fields_ = [("a", Csr), ("c", PD), ("lc", PD), ("uc", PD), ("lv", PD), ("uv", PD), ("c0", dbl), ("maximize", cint)]


class Params(C.Structure):
    _fields_ = [
        ("tolerance", dbl), ("infeasibility_tolerance", dbl), ("max_iterations", u64), ("time_limit_s", dbl),
        ("check_every", u64), ("step_size_factor", dbl), ("reflection", dbl),
        ("restart_sufficient", dbl), ("restart_necessary", dbl), ("restart_artificial", dbl),
        ("pid_kp", dbl), ("pid_ki", dbl), ("pid_kd", dbl), ("pid_discount", dbl),
        ("power_iterations", u64), ("geometric_mean_passes", u64), ("ruiz_iterations", u64),
        ("pock_chambolle_enabled", cint), ("pock_chambolle_alpha", dbl), ("bound_objective_rescaling", cint),
        ("log_every_checks", u64), ("termination", cint), ("precision", cint), ("mixed_switch_tolerance", dbl),
    ]


class Info(C.Structure):
    _fields_ = [
        ("status", cint), ("objective", dbl), ("dual_objective", dbl), ("primal_residual", dbl),
        ("dual_residual", dbl), ("gap", dbl), ("iterations", u64), ("restarts", u64), ("solve_time_s", dbl),
        ("setup_time_s", dbl), ("norm_estimate", dbl), ("fp64_from_iteration", u64),
    ]


class CheckRecord(C.Structure):
    _fields_ = [
        ("total", u64), ("k_after", u64), ("residual", dbl), ("omega", dbl), ("primal_obj", dbl),
        ("dual_obj", dbl), ("primal_res", dbl), ("dual_res", dbl), ("restarted", cint),
    ]


class PrimalStatsC(C.Structure):
    _fields_ = [("residual_sq", dbl), ("objective", dbl)]


class DualStatsC(C.Structure):
    _fields_ = [("residual_sq", dbl), ("objective", dbl)]


class RayStatsC(C.Structure):
    _fields_ = [("objective", dbl), ("violation_sq", dbl), ("norm_sq", dbl)]


class GenParams(C.Structure):
    _fields_ = [
        ("kind", cint), ("seed", u64), ("nrows", i64), ("ncols", i64), ("nnz_per_col_min", i64),
        ("nnz_per_col_max", i64), ("target_nnz", i64), ("zipf_s", dbl), ("degree_min", i64), ("degree_max", i64),
        ("supplies", i64), ("demands", i64),
    ]


class BatchResult(C.Structure):
    _fields_ = [
        ("status", cint), ("objective", dbl), ("dual_objective", dbl), ("primal_residual", dbl),
        ("dual_residual", dbl), ("gap", dbl), ("iterations", u64), ("restarts", u64), ("lanes_per_row", cint),
        ("handed_off", cint),
    ]


class ServerConfig(C.Structure):
    _fields_ = [("budget_bytes", dbl), ("max_inflight", cint), ("batch_max_nnz", cint)]


class ServerResult(C.Structure):
    _fields_ = [
        ("id", i64), ("status", cint), ("objective", dbl), ("dual_objective", dbl), ("primal_residual", dbl),
        ("dual_residual", dbl), ("gap", dbl), ("iterations", u64), ("queue_s", dbl), ("solve_s", dbl),
        ("total_s", dbl), ("footprint_bytes", i64), ("error", cint), ("path", cint), ("message", C.c_char * 160),
    ]


# (name, restype, argtypes) of every exported entry point.
SIGNATURES = [
    ("sp_ctx_create", cint, [cint, C.POINTER(VP)]),
    ("sp_ctx_destroy", None, [VP]),
    ("sp_ctx_last_error", C.c_char_p, [VP]),
    ("sp_ctx_name", cint, [VP, C.c_char_p, C.c_size_t]),
    ("sp_ctx_stream", VP, [VP]),
    ("sp_problem_load", cint, [VP, C.POINTER(Csr), C.POINTER(Csr), PD, PD, PD, PD, PD, PD, PD, C.POINTER(VP)]),
    ("sp_problem_free", None, [VP]),
    ("sp_vec_upload", cint, [VP, PD, i64, C.POINTER(VP)]),
    ("sp_vec_download", cint, [VP, VP, PD, i64]),
    ("sp_vec_copy", cint, [VP, VP, VP]),
    ("sp_vec_free", None, [VP]),
    ("sp_vec_len", i64, [VP]),
    ("sp_spmv", cint, [VP, VP, VP, VP]),
    ("sp_spmv_t", cint, [VP, VP, VP, VP]),
    ("sp_primal_step", cint, [VP, VP, VP, VP, dbl, VP, VP]),
    ("sp_dual_step", cint, [VP, VP, VP, VP, dbl, VP]),
    ("sp_halpern_step", cint, [VP, VP, VP, VP, dbl, dbl]),
    ("sp_distance_sq", cint, [VP, VP, VP, PD]),
    ("sp_sub", cint, [VP, VP, VP, VP]),
    ("sp_norm_sq", cint, [VP, VP, PD]),
    ("sp_dot", cint, [VP, VP, VP, PD]),
    ("sp_scale", cint, [VP, VP, dbl]),
    ("sp_primal_stats", cint, [VP, VP, VP, VP, C.POINTER(PrimalStatsC)]),
    ("sp_dual_stats", cint, [VP, VP, VP, VP, C.POINTER(DualStatsC)]),
    ("sp_step_dual_residual_sq", cint, [VP, VP, VP, VP, VP, VP, dbl, PD]),
    ("sp_primal_ray_stats", cint, [VP, VP, VP, VP, C.POINTER(RayStatsC)]),
    ("sp_dual_ray_stats", cint, [VP, VP, VP, VP, C.POINTER(RayStatsC)]),
    ("sp_solver_params_default", None, [C.POINTER(Params)]),
    ("sp_solve", cint, [VP, C.POINTER(Lp), C.POINTER(Params), PD, PD, C.POINTER(Info)]),
    ("sp_solve_stepwise", cint, [VP, C.POINTER(Lp), C.POINTER(Params), PD, PD, C.POINTER(Info)]),
    ("sp_solver_create", cint, [VP, C.POINTER(Lp), C.POINTER(Params), C.POINTER(VP)]),
    ("sp_solver_solve", cint, [VP, C.POINTER(Info)]),
    ("sp_solver_reset", cint, [VP]),
    ("sp_solver_warm_start", cint, [VP, PD, PD]),
    ("sp_solver_run_epochs", cint, [VP, u64]),
    ("sp_solver_sync", cint, [VP]),
    ("sp_solver_info", cint, [VP, C.POINTER(Info)]),
    ("sp_solver_download", cint, [VP, PD, PD]),
    ("sp_solver_trace", cint, [VP, C.POINTER(CheckRecord), i64, PI64]),
    ("sp_solver_set_timing", cint, [VP, cint]),
    ("sp_solver_kernel_timing", cint, [VP, cint, PI64, PD, PD]),
    ("sp_solver_bytes_per_iteration", dbl, [VP]),
    ("sp_solver_engines", cint, [VP, C.POINTER(C.c_int32)]),
    ("sp_solver_epoch_kernels", cint, [VP, PI64]),
    ("sp_solver_gather_floor", cint, [VP, cint, cint, cint, PD]),
    ("sp_solver_scaled", cint, [VP, PI64, PI32, PD, PI64, PI32, PD, PD, PD, PD, PD, PD, PD, PD, PD, PD]),
    ("sp_solver_free", None, [VP]),
    ("sp_batch_create", cint, [VP, C.POINTER(Lp), cint, C.POINTER(Params), C.POINTER(VP)]),
    ("sp_batch_solve", cint, [VP, C.POINTER(BatchResult), PD]),
    ("sp_batch_download", cint, [VP, cint, PD, PD]),
    ("sp_batch_free", None, [VP]),
    ("sp_server_create", cint, [VP, C.POINTER(ServerConfig), C.POINTER(Params), C.POINTER(VP)]),
    ("sp_server_submit", cint, [VP, C.POINTER(Lp), PI64]),
    ("sp_server_poll", cint, [VP, dbl, C.POINTER(ServerResult), PD, i64, PD, i64, C.POINTER(cint)]),
    ("sp_server_footprint", i64, [i64, i64, i64, cint]),
    ("sp_server_destroy", None, [VP]),
    ("sp_dot_noalloc", cint, [VP, VP, i64, VP, VP]),
    ("sp_generate", cint, [C.POINTER(GenParams), C.POINTER(Lp)]),
    ("sp_lp_release", None, [C.POINTER(Lp)]),
    ("sp_read_mps", cint, [C.c_char_p, C.c_size_t, C.POINTER(Lp), C.POINTER(i64), C.c_char_p, C.c_size_t]),
    ("sp_problem_validate", cint, [C.POINTER(Lp), C.c_char_p, C.c_size_t]),
    ("sp_csr_from_triplets", cint, [VP, i64, i64, i64, PI64, PI64, PD, C.POINTER(Csr)]),
    ("sp_csr_release", None, [C.POINTER(Csr)]),
    ("sp_polish", cint, [VP, C.POINTER(Lp), C.POINTER(Params), dbl, PD, PD, C.POINTER(u64)]),
    ("sp_presolve_create", cint, [C.POINTER(Lp), C.POINTER(Lp), C.POINTER(VP), C.POINTER(cint)]),
    ("sp_presolve_postsolve", cint, [VP, PD, PD, PD, PD]),
    ("sp_presolve_counts", cint, [VP, PI64]),
    ("sp_presolve_free", None, [VP]),
]

_lib = None


def load(build_if_missing: bool = True):
    """Loads the CUDA library (building it first when it is missing or stale and nvcc exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if build_if_missing:
        try:
            from . import build as _build

            _build.build()
        except (OSError, FileNotFoundError):
            pass  # no nvcc on this machine: use the prebuilt library
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"saddlepoint_b200 CUDA library not built: {LIB_PATH} (run python -m saddlepoint_b200.build)")
    lib = C.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        f = getattr(lib, name)  # a missing symbol is an error: the library and header must agree
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib
