/*
 * saddlepoint_b200.h — C ABI of the B200 (sm_100a) backend for saddlepoint's
 * restarted reflected-Halpern PDHG.
 *
 * Part 1 mirrors the reference's fused `Backend` trait
 * (crates/saddlepoint-core/src/backend.rs:43-137) one entry point per method,
 * so that a Rust shim crate can implement `Backend` by calling these functions.
 * Vectors and problems are opaque handles owned by the
 * library; reductions return their scalars through out-pointers, exactly like
 * the trait returns host `f64`s and stats structs.
 *
 * Part 2 is the performance extension the trait cannot express: the whole
 * solve (scaling passes, power iteration, PDHG epochs, restarts, PID and
 * termination) resident on one GPU, in plain FP64 or mixed FP32-SpMV/FP64-state.
 *
 * Part 3 is the batched form (many LPs, one persistent kernel) and Part 4 the
 * serving loop (continuous batching of arriving LPs under an HBM budget).
 *
 * Every function returns SP_OK (0) or an SP_ERR_* code; the text of the last
 * error on a context is available from sp_ctx_last_error. Infinite bounds are
 * IEEE ±infinity, as in the reference (crates/saddlepoint-core/src/problem.rs:9).
 * Indices: row pointers are int64 on the host and are narrowed to int32 on the
 * device; a problem with 2^31 or more nonzeros is rejected with SP_ERR_TOO_LARGE,
 * as the reference's cuSPARSE backend does (crates/saddlepoint-cuda/src/sparse.rs:60-62).
 */
#ifndef SADDLEPOINT_B200_H
#define SADDLEPOINT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (crates/saddlepoint-cuda/src/backend.rs:27-40; solver.rs:123-131) ---- */
#define SP_OK 0
#define SP_ERR_CUDA 1        /* CudaError::Driver: a CUDA runtime call failed */
#define SP_ERR_INVALID 2     /* bad argument: null handle, length mismatch */
#define SP_ERR_TOO_LARGE 3   /* CudaError::TooLarge: more than 2^31-1 nonzeros */
#define SP_ERR_UNAVAILABLE 4 /* CudaError::Unavailable: no usable device */
#define SP_ERR_NUMERICAL 5   /* SolveError::Numerical */
#define SP_ERR_PROBLEM 6     /* SolveError::Problem: LpProblem::validate failed */
#define SP_ERR_DEVICE 7      /* a kernel reported an error (e.g. a bounded wait ran out) */
#define SP_ERR_PARSE 8       /* MpsError::Parse: malformed MPS text (line and message returned) */

/* ---- Status (crates/saddlepoint-core/src/solver.rs:95-102) ---- */
#define SP_STATUS_OPTIMAL 0
#define SP_STATUS_PRIMAL_INFEASIBLE 1
#define SP_STATUS_DUAL_INFEASIBLE 2
#define SP_STATUS_ITERATION_LIMIT 3
#define SP_STATUS_TIME_LIMIT 4

#define SP_TERMINATION_PROJECTED 0    /* solver.rs:61-62 */
#define SP_TERMINATION_STEP_IMPLIED 1 /* solver.rs:63-67 */
#define SP_PRECISION_FP64 0
#define SP_PRECISION_MIXED 1

typedef struct sp_ctx sp_ctx;
typedef struct sp_problem sp_problem;
typedef struct sp_vec sp_vec;
typedef struct sp_solver sp_solver;
typedef struct sp_batch sp_batch;
typedef struct sp_server sp_server;

/* PrimalStats / DualStats / RayStats (backend.rs:14-41). */
typedef struct { double residual_sq, objective; } sp_primal_stats_t;
typedef struct { double residual_sq, objective; } sp_dual_stats_t;
typedef struct { double objective, violation_sq, norm_sq; } sp_ray_stats_t;

/* A CSR matrix in host memory (CsrMatrix, problem.rs:14-24). */
typedef struct {
    int64_t nrows, ncols, nnz;
    const int64_t *row_ptr; /* nrows + 1 */
    const int32_t *col_idx; /* nnz, sorted within each row */
    const double *values;   /* nnz */
} sp_csr;

/* ========================================================================
 * Part 1 — the Backend trait, one entry point per method.
 * ======================================================================== */

/* CudaBackend::new (crates/saddlepoint-cuda/src/backend.rs:129-158): opens device
 * `ordinal`. Returns SP_ERR_UNAVAILABLE (never aborts) when there is no GPU. */
int sp_ctx_create(int ordinal, sp_ctx **out);
void sp_ctx_destroy(sp_ctx *ctx);
/* Text of the last error on this context ("" if none). */
const char *sp_ctx_last_error(const sp_ctx *ctx);
/* Backend::name (backend.rs:48): "b200 (<device name>)". */
int sp_ctx_name(const sp_ctx *ctx, char *buf, size_t cap);
/* The CUDA stream every call on this context is ordered on (a cudaStream_t). */
void *sp_ctx_stream(sp_ctx *ctx);

/* Backend::load (backend.rs:51; cuda backend.rs:229-248): moves a scaled problem
 * (ScaledProblem, scaling.rs:36-50) onto the device. `at` must be the transpose
 * of `a`; primal_factor has nrows entries and dual_factor ncols entries
 * (ScaledProblem::primal_residual_factors / dual_residual_factors, scaling.rs:123-131). */
int sp_problem_load(sp_ctx *ctx, const sp_csr *a, const sp_csr *at, const double *c, const double *lc,
                    const double *uc, const double *lv, const double *uv, const double *primal_factor,
                    const double *dual_factor, sp_problem **out);
void sp_problem_free(sp_problem *p);

/* Backend::upload / download / copy (backend.rs:53-55). */
int sp_vec_upload(sp_ctx *ctx, const double *data, int64_t len, sp_vec **out);
int sp_vec_download(sp_ctx *ctx, const sp_vec *v, double *out, int64_t len);
int sp_vec_copy(sp_ctx *ctx, const sp_vec *src, sp_vec *dst);
void sp_vec_free(sp_vec *v);
int64_t sp_vec_len(const sp_vec *v);

/* Backend::spmv / spmv_t (backend.rs:57-60): out = A' x, out = A'ᵀ y. */
int sp_spmv(sp_ctx *ctx, const sp_problem *p, const sp_vec *x, sp_vec *out);
int sp_spmv_t(sp_ctx *ctx, const sp_problem *p, const sp_vec *y, sp_vec *out);
/* Backend::primal_step (backend.rs:62-71). */
int sp_primal_step(sp_ctx *ctx, const sp_problem *p, const sp_vec *x, const sp_vec *aty, double tau, sp_vec *x_t,
                   sp_vec *x_bar);
/* Backend::dual_step (backend.rs:73-81). */
int sp_dual_step(sp_ctx *ctx, const sp_problem *p, const sp_vec *y, const sp_vec *ax_bar, double sigma, sp_vec *y_t);
/* Backend::halpern_step (backend.rs:83-92). */
int sp_halpern_step(sp_ctx *ctx, sp_vec *z, const sp_vec *z_t, const sp_vec *anchor, double w, double rho);
/* Backend::distance_sq / sub / norm_sq / dot / scale (backend.rs:94-103). */
int sp_distance_sq(sp_ctx *ctx, const sp_vec *a, const sp_vec *b, double *out);
int sp_sub(sp_ctx *ctx, const sp_vec *a, const sp_vec *b, sp_vec *out);
int sp_norm_sq(sp_ctx *ctx, const sp_vec *v, double *out);
int sp_dot(sp_ctx *ctx, const sp_vec *a, const sp_vec *b, double *out);
int sp_scale(sp_ctx *ctx, sp_vec *v, double alpha);
/* Backend::primal_stats / dual_stats (backend.rs:105-108). */
int sp_primal_stats(sp_ctx *ctx, const sp_problem *p, const sp_vec *x, const sp_vec *ax, sp_primal_stats_t *out);
int sp_dual_stats(sp_ctx *ctx, const sp_problem *p, const sp_vec *y, const sp_vec *aty, sp_dual_stats_t *out);
/* Backend::step_dual_residual_sq (backend.rs:109-121). */
int sp_step_dual_residual_sq(sp_ctx *ctx, const sp_problem *p, const sp_vec *x, const sp_vec *x_t, const sp_vec *aty,
                             const sp_vec *aty_t, double tau, double *out);
/* Backend::primal_ray_stats / dual_ray_stats (backend.rs:123-136). */
int sp_primal_ray_stats(sp_ctx *ctx, const sp_problem *p, const sp_vec *dx, const sp_vec *adx, sp_ray_stats_t *out);
int sp_dual_ray_stats(sp_ctx *ctx, const sp_problem *p, const sp_vec *dy, const sp_vec *atdy, sp_ray_stats_t *out);

/* ========================================================================
 * Part 2 — device-resident solve (extension).
 * ======================================================================== */

/* SolverParams (solver.rs:24-52) + ScalingParams (scaling.rs:14-34), flattened. */
typedef struct {
    double tolerance;               /* 1e-6 */
    double infeasibility_tolerance; /* 1e-8 */
    uint64_t max_iterations;        /* 1,000,000 */
    double time_limit_s;            /* <= 0: none */
    uint64_t check_every;           /* 64 */
    double step_size_factor;        /* 0.998 */
    double reflection;              /* 1.0 */
    double restart_sufficient, restart_necessary, restart_artificial; /* 0.2, 0.5, 0.36 */
    double pid_kp, pid_ki, pid_kd, pid_discount;                      /* 0.99, 0.01, 0, 0.3 */
    uint64_t power_iterations;      /* 200 */
    uint64_t geometric_mean_passes; /* 12 */
    uint64_t ruiz_iterations;       /* 10 */
    int pock_chambolle_enabled;     /* 1 */
    double pock_chambolle_alpha;    /* 1.0 */
    int bound_objective_rescaling;  /* 1 */
    uint64_t log_every_checks;      /* 0 = silent (progress lines go to stderr) */
    int termination;                /* SP_TERMINATION_* */
    int precision;                  /* SP_PRECISION_* */
    double mixed_switch_tolerance;  /* mixed form: go to FP64 SpMV once the relative KKT error is below this (1e-5) */
} sp_solver_params;

void sp_solver_params_default(sp_solver_params *p);

/* An LP in the original space (LpProblem, problem.rs:129-145). c and c0 are
 * already negated for a maximisation problem, as in the reference. */
typedef struct {
    sp_csr a;
    const double *c, *lc, *uc, *lv, *uv;
    double c0;
    int maximize;
} sp_lp;

/* Solution (solver.rs:104-121) without the vectors, plus accounting. */
typedef struct {
    int status;
    double objective, dual_objective, primal_residual, dual_residual, gap;
    uint64_t iterations, restarts;
    double solve_time_s;     /* power iteration + PDHG loop (Solution::solve_time) */
    double setup_time_s;     /* upload, scaling passes, transpose, tile plans */
    double norm_estimate;    /* ‖A'‖₂ from power iteration */
    uint64_t fp64_from_iteration; /* mixed form: first iteration run with FP64 SpMV (0 if never) */
} sp_solution_info;

/* One termination/restart check of the loop (for iteration-level comparisons). */
typedef struct {
    uint64_t total, k_after;
    double residual, omega, primal_obj, dual_obj, primal_res, dual_res;
    int restarted;
} sp_check_record;

/* solve() (solver.rs:154-157) with everything on the device: validates, uploads
 * the LP, runs the scaling passes and the transpose on the GPU, estimates ‖A'‖₂,
 * runs the PDHG loop in CUDA-graph epochs of `check_every` iterations with the
 * restart, PID and termination logic on the device, and downloads x and y in the
 * original space. x has ncols entries, y nrows. */
int sp_solve(sp_ctx *ctx, const sp_lp *lp, const sp_solver_params *params, double *x, double *y,
             sp_solution_info *info);

/* solve() driven from the host over the Part 1 entry points only, with the
 * scaling done on the host: the reference's loop (solver.rs:311-438) step for
 * step, as a Rust host would drive this backend through the trait. */
int sp_solve_stepwise(sp_ctx *ctx, const sp_lp *lp, const sp_solver_params *params, double *x, double *y,
                      sp_solution_info *info);

/* A reusable device-resident solver (for repeated runs and timing). */
int sp_solver_create(sp_ctx *ctx, const sp_lp *lp, const sp_solver_params *params, sp_solver **out);
/* Runs from the current state until a status is reached; fills info. */
int sp_solver_solve(sp_solver *s, sp_solution_info *info);
/* Resets the iterates and counters to the start of a solve (keeps ‖A'‖₂). */
int sp_solver_reset(sp_solver *s);
/* sp_solver_reset, then the next solve starts from (x, y) in the original problem's space
 * (ncols and nrows entries; either may be null for zeros) as iterate and restart anchor,
 * instead of from 0. No counterpart in the reference, whose solve always starts at 0. */
int sp_solver_warm_start(sp_solver *s, const double *x, const double *y);
/* Enqueues `epochs` epochs of check_every iterations without waiting; a converged
 * state turns further epochs into no-ops. */
int sp_solver_run_epochs(sp_solver *s, uint64_t epochs);
int sp_solver_sync(sp_solver *s);
int sp_solver_info(sp_solver *s, sp_solution_info *info);
/* Downloads the current x_t, y_t in the original space. */
int sp_solver_download(sp_solver *s, double *x, double *y);
/* Copies up to `cap` check records; *len receives the number available. */
int sp_solver_trace(sp_solver *s, sp_check_record *out, int64_t cap, int64_t *len);
/* Records CUDA events around every `every`-th launch of each fused kernel (0 = off). */
int sp_solver_set_timing(sp_solver *s, int every);
/* Per fused-kernel timing from the events: id 0 = primal pass (A'ᵀ y + primal
 * epilogue), 1 = dual pass (A' x̄ + dual epilogue). Returns launches timed, total
 * milliseconds and the algorithmic bytes one launch moves. */
int sp_solver_kernel_timing(sp_solver *s, int id, int64_t *launches, double *total_ms, double *bytes_per_launch);
/* Algorithmic bytes of one PDHG iteration in the current precision. */
double sp_solver_bytes_per_iteration(sp_solver *s);
/* Which engine runs each fused pass of the solver (chosen at creation from the
 * problem's size, or SP_PASS_ENGINE): out[0] primal FP64, out[1] primal FP32,
 * out[2] dual FP64, out[3] dual FP32 (the FP32 entries apply to the mixed form). */
enum { SP_ENGINE_TILES = 0, SP_ENGINE_STREAM = 1, SP_ENGINE_SELL = 2 };
int sp_solver_engines(sp_solver *s, int32_t out[4]);
/* The floor a pass's random gathers set: the average time of a kernel that does only
 * those gathers (pass 0 primal: y through A'ᵀ's column indices; 1 dual: x̄ through A''s;
 * fp32 != 0: the mixed form's FP32 vectors), each through the pass's own index stream,
 * over `reps` launches after one warm-up. For reading a pass's time against. */
int sp_solver_gather_floor(sp_solver *s, int pass, int fp32, int reps, double *ms_per_launch);
/* Kernel launches of one epoch of check_every iterations, counted from the
 * kernel nodes of its CUDA graph (the graph is built if it does not exist yet). */
int sp_solver_epoch_kernels(sp_solver *s, int64_t *count);
/* Downloads the scaled problem the solver built on the device (ScaledProblem,
 * scaling.rs:36-50): A' and A'ᵀ in CSR, c', lc', uc', lv', uv', the row and
 * column scales and the two scalar rescalings. Any pointer may be null. */
int sp_solver_scaled(sp_solver *s, int64_t *a_row_ptr, int32_t *a_col_idx, double *a_values, int64_t *at_row_ptr,
                     int32_t *at_col_idx, double *at_values, double *c, double *lc, double *uc, double *lv,
                     double *uv, double *row_scale, double *col_scale, double *bound_scale, double *obj_scale);
void sp_solver_free(sp_solver *s);

/* ========================================================================
 * Part 3 — batched form: many LPs advanced by one persistent kernel.
 * ======================================================================== */

typedef struct {
    int status;
    double objective, dual_objective, primal_residual, dual_residual, gap;
    uint64_t iterations, restarts;
    int lanes_per_row; /* SpMV variant the tuner chose: 0 = staged tiles (the single-LP passes);
                          otherwise lane groups, 100 * (lanes per row of A') + (lanes per row of A'ᵀ) */
    int handed_off;    /* 1: the instance was still running well after every other instance had
                          been started, and was solved again from the start by the single-LP
                          device solver (sp_solve) */
} sp_batch_result;

/* Scales and uploads `count` LPs into one packed arena. An invalid LP (sp_problem_validate)
 * fails the call with SP_ERR_PROBLEM and "instance <i>: <message>". */
int sp_batch_create(sp_ctx *ctx, const sp_lp *lps, int count, const sp_solver_params *params, sp_batch **out);
/* Solves every instance; results[count]. An instance still running in the
 * persistent kernel SP_BATCH_HANDOFF_S seconds (environment, default 2; 0 turns
 * this off) after the last instance was started stops at its next check and is
 * solved again from the start by the single-LP device solver, several such
 * instances at once on their own streams; its result is then exactly sp_solve's.
 * *elapsed_s covers both. */
int sp_batch_solve(sp_batch *b, sp_batch_result *results, double *elapsed_s);
/* x/y of instance i in the original space. */
int sp_batch_download(sp_batch *b, int i, double *x, double *y);
void sp_batch_free(sp_batch *b);

/* ========================================================================
 * Part 4 — serving loop: continuous batching under an HBM budget.
 * ======================================================================== */

typedef struct {
    double budget_bytes; /* HBM admission budget */
    int max_inflight;    /* concurrent solves (CUDA streams) */
    int batch_max_nnz;   /* arrivals at or below this many nonzeros go to the batched kernel */
} sp_server_config;

typedef struct {
    int64_t id;
    int status;
    double objective, dual_objective, primal_residual, dual_residual, gap;
    uint64_t iterations;
    double queue_s, solve_s, total_s; /* waiting for admission, on the device, submit to result */
    int64_t footprint_bytes;
    int error;            /* SP_OK, or the SP_ERR_* code of a failed solve (status is then -1) */
    int path;             /* 0: a solve slot, 1: the batched kernel */
    char message[160];    /* the failed solve's error text */
} sp_server_result;

int sp_server_create(sp_ctx *ctx, const sp_server_config *cfg, const sp_solver_params *params, sp_server **out);
/* Copies the LP; returns at once with a request id. An invalid LP (sp_problem_validate) is
 * refused with SP_ERR_PROBLEM and the message in sp_ctx_last_error of the server's context. */
int sp_server_submit(sp_server *s, const sp_lp *lp, int64_t *id);
/* Waits for the next finished request (timeout_s < 0: wait forever). Returns
 * SP_OK with *got = 1 when a result was written, *got = 0 on timeout. x and y may
 * be null (no solution copied); a non-null x or y with room for fewer than the
 * request's n or m values returns SP_ERR_INVALID with *got = 0 and leaves the
 * result queued for the next poll. */
int sp_server_poll(sp_server *s, double timeout_s, sp_server_result *out, double *x, int64_t xcap, double *y,
                   int64_t ycap, int *got);
/* Footprint the admission control charges for an LP of this shape. */
int64_t sp_server_footprint(int64_t nrows, int64_t ncols, int64_t nnz, int precision);
void sp_server_destroy(sp_server *s);

/* ========================================================================
 * Allocation-free reduction. No counterpart in the reference.
 * ======================================================================== */

/* Maximum length sp_dot_noalloc accepts: its fixed scratch holds one partial sum
 * per 2048 elements, 32768 of them (256 KiB per GPU, held until process exit). */
#define SP_NOALLOC_DOT_MAX_N 67108864LL

/* *result = aᵀb for device arrays a and b of n doubles, enqueued on `stream` (a
 * cudaStream_t; NULL for the default stream); `result` is a device pointer. For
 * callers that cannot allocate device memory where they need the reduction (inside
 * stream capture, under their own pool allocator, in a loop that must not
 * synchronise on cudaMalloc/cudaFree): it allocates nothing and needs no context.
 * Its two-stage reduction keeps its partial sums in a static device array instead;
 * n > SP_NOALLOC_DOT_MAX_N returns SP_ERR_TOO_LARGE and launches nothing. The
 * first call on each device looks up that array's address (cudaGetSymbolAddress);
 * make that first call before any stream capture. All calls share the array, so
 * calls that overlap on the GPU (different streams, no ordering between them)
 * race; calls on one stream are safe. Returns SP_OK or an SP_ERR_* code. */
int sp_dot_noalloc(const double *a, const double *b, int64_t n, double *result, void *stream);

/* ========================================================================
 * Synthetic LP generators (seeded; the recipes are in csrc/host.cpp).
 * ======================================================================== */

#define SP_GEN_RANDOM 0    /* random sparse LP: config-0 style */
#define SP_GEN_POWERLAW 1  /* power-law column degrees */
#define SP_GEN_TRANSPORT 2 /* transportation LP */

typedef struct {
    int kind;
    uint64_t seed;
    int64_t nrows, ncols;
    int64_t nnz_per_col_min, nnz_per_col_max; /* SP_GEN_RANDOM: degree uniform in [min, max] */
    int64_t target_nnz;                       /* SP_GEN_POWERLAW: total nonzeros after rescaling */
    double zipf_s;                            /* SP_GEN_POWERLAW: exponent */
    int64_t degree_min, degree_max;           /* SP_GEN_POWERLAW: truncation of the draw */
    int64_t supplies, demands;                /* SP_GEN_TRANSPORT */
} sp_gen_params;

/* Generated LP with library-owned host arrays; release with sp_lp_release. */
int sp_generate(const sp_gen_params *g, sp_lp *out);
void sp_lp_release(sp_lp *lp);

/* ========================================================================
 * Part 5 — problem input.
 * ======================================================================== */

/* read_mps (crates/saddlepoint-io/src/lib.rs:59-309): free-format MPS text of `len`
 * bytes to an LP with library-owned host arrays (release with sp_lp_release), the
 * matrix built as CsrMatrix::from_triplets builds it (problem.rs:33-77). On malformed
 * text returns SP_ERR_PARSE with the 1-based line in *err_line and the reference's
 * message in err (any of the two may be null). Row and column names are not kept. */
int sp_read_mps(const char *text, size_t len, sp_lp *out, int64_t *err_line, char *err, size_t errlen);

/* LpProblem::validate (crates/saddlepoint-core/src/problem.rs:166-194), host code (no
 * device needed): SP_OK, or SP_ERR_PROBLEM with the reference's message for the first
 * failure in its order — a variable's bounds (NaN, then lower above upper) over all
 * columns, then a constraint's, then a NaN coefficient among c and then A's values
 * (numbered after c) — written into `message` (`cap` bytes; may be null). Then the
 * matrix's structure, which the reference's CsrMatrix keeps by construction: row pointers
 * from 0 to nnz, never decreasing, column indices in [0, ncols) — SP_ERR_INVALID with a
 * message naming the entry. Every solve, batch and server submission runs this check first
 * and fails with the same code and message. */
int sp_problem_validate(const sp_lp *lp, char *message, size_t cap);

/* CsrMatrix::from_triplets (crates/saddlepoint-core/src/problem.rs:33-77) on the GPU of
 * `ctx`, for loading large problems: ntrip (row, column, value) triplets in host memory to
 * a CSR matrix with library-owned host arrays (release with sp_csr_release). Entries are
 * grouped by row, ordered by column within a row, runs of one column summed in input order
 * and exact-zero sums dropped: bit for bit the host rule (and sp_read_mps's). An index out
 * of range returns SP_ERR_INVALID (the reference asserts). */
int sp_csr_from_triplets(sp_ctx *ctx, int64_t nrows, int64_t ncols, int64_t ntrip, const int64_t *rows,
                         const int64_t *cols, const double *vals, sp_csr *out);
void sp_csr_release(sp_csr *m);

/* ========================================================================
 * Part 6 — presolve and feasibility polishing. The reference's path has neither;
 * cuPDLPx, which the reference's benchmark compares against, has both
 * (bench/README.md:1-6).
 * ======================================================================== */

/* Feasibility polishing (as cuPDLPx applies it after a solve), on the GPU of `ctx`: from a
 * solution (x, y) of `lp`, a warm-started FP64 solve of the feasibility problem (the same
 * constraints, zero cost) brings x to primal feasibility within `tolerance` (relative, as the
 * termination test measures it), and a warm-started solve of the problem with every finite
 * bound set to zero (the same dual feasible set, zero dual objective) brings y to dual
 * feasibility within `tolerance`. x and y are overwritten with the polished pair;
 * `iterations` (may be null) receives the two solves' iteration counts. Each solve is capped
 * at params->max_iterations; params may be null for the defaults. */
int sp_polish(sp_ctx *ctx, const sp_lp *lp, const sp_solver_params *params, double tolerance, double *x, double *y,
              uint64_t iterations[2]);

typedef struct sp_presolve sp_presolve;

/* Exact reductions of `lp` (the reference's minimisation form), applied until none
 * applies: empty rows dropped, singleton rows turned into column bounds, fixed columns
 * substituted into the row bounds and the objective constant, empty columns set to the
 * bound their cost points at. `reduced` receives the remaining LP (arrays owned by the
 * presolve object, valid until sp_presolve_free); *status is -1 when the reduced LP is to
 * be solved, SP_STATUS_PRIMAL_INFEASIBLE or SP_STATUS_DUAL_INFEASIBLE when presolve proved
 * it, SP_STATUS_OPTIMAL when no column is left (postsolve with null reduced vectors). */
int sp_presolve_create(const sp_lp *lp, sp_lp *reduced, sp_presolve **out, int *status);
/* Maps the reduced problem's solution (x_red, y_red) back to the original problem's n and
 * m entries: removed columns take their values; removed rows take the duals that make the
 * original KKT conditions hold as the reduced ones do (a singleton row carries the part of
 * its column's reduced cost that the bound it implied absorbs). */
int sp_presolve_postsolve(const sp_presolve *p, const double *x_red, const double *y_red, double *x, double *y);
/* Rows and columns removed: counts[0] empty rows, [1] singleton rows, [2] fixed
 * columns, [3] empty columns. */
int sp_presolve_counts(const sp_presolve *p, int64_t counts[4]);
void sp_presolve_free(sp_presolve *p);

#ifdef __cplusplus
}
#endif
#endif /* SADDLEPOINT_B200_H */
