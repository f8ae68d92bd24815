/*
 * sp_oracle.h — CPU oracle for the restarted reflected-Halpern PDHG path.
 *
 * TEST INFRASTRUCTURE ONLY. This is a plain-C restatement of the reference
 * saddlepoint's CPU path (crates/saddlepoint-core and crates/saddlepoint-cpu)
 * used as the checker for the CUDA library. Only the tests, the smoke check and
 * bench.py's CPU-baseline leg may load it. Nothing in the product links it.
 *
 * Every function cites the reference file:line it restates. Arithmetic follows
 * the reference's operation order: no FMA contraction (build with
 * -ffp-contract=off), sums start from -0.0 where Rust's `Iterator::sum` does,
 * and passes with fewer than 32768 elements run serially, as in
 * crates/saddlepoint-cpu/src/lib.rs:12. Larger passes run on a fixed pool of
 * threads with a fixed chunking (rayon's split is not reproducible; this one is).
 */
#ifndef SP_ORACLE_H
#define SP_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* CsrMatrix (crates/saddlepoint-core/src/problem.rs:14-24). */
typedef struct {
    int64_t nrows, ncols, nnz;
    int64_t *row_ptr; /* nrows + 1 */
    int64_t *col_idx; /* nnz, sorted within each row */
    double *values;   /* nnz */
} or_csr;

/* LpProblem (problem.rs:129-145). */
typedef struct {
    or_csr a;
    double *c, *lc, *uc, *lv, *uv;
    double c0;
    int maximize;
} or_lp;

/* ScalingParams (crates/saddlepoint-core/src/scaling.rs:14-34). */
typedef struct {
    int64_t geometric_mean_passes;
    int64_t ruiz_iterations;
    int pock_chambolle_enabled;
    double pock_chambolle_alpha;
    int bound_objective_rescaling;
} or_scaling_params;

/* ScaledProblem (scaling.rs:36-50). */
typedef struct {
    or_csr a, at;
    double *c, *lc, *uc, *lv, *uv;
    double *row_scale, *col_scale;
    double bound_scale, obj_scale;
} or_scaled;

/* SolverParams (crates/saddlepoint-core/src/solver.rs:24-52). time_limit_s <= 0 means none. */
typedef struct {
    double tolerance;
    double infeasibility_tolerance;
    uint64_t max_iterations;
    double time_limit_s;
    uint64_t check_every;
    double step_size_factor;
    double reflection;
    double restart_sufficient, restart_necessary, restart_artificial;
    double pid_kp, pid_ki, pid_kd, pid_discount;
    uint64_t power_iterations;
    or_scaling_params scaling;
    int termination; /* 0 = Projected, 1 = StepImplied (solver.rs:56-68) */
} or_solver_params;

/* Status (solver.rs:95-102). */
enum { OR_OPTIMAL = 0, OR_PRIMAL_INFEASIBLE = 1, OR_DUAL_INFEASIBLE = 2, OR_ITERATION_LIMIT = 3, OR_TIME_LIMIT = 4 };
/* SolveError (solver.rs:123-131) plus host errors. */
enum { OR_OK = 0, OR_ERR_PROBLEM = -1, OR_ERR_NUMERICAL = -2, OR_ERR_ALLOC = -3, OR_ERR_PARSE = -4 };

/* One restart/termination check of the loop, for iteration-level parity. */
typedef struct {
    uint64_t total, k_after;
    double residual, omega, primal_obj, dual_obj, primal_res, dual_res;
    int restarted;
} or_check_record;

/* Solution (solver.rs:104-121), plus the check trace. */
typedef struct {
    int status;
    double *x, *y;
    double objective, dual_objective, primal_residual, dual_residual, gap;
    uint64_t iterations, restarts;
    double solve_time_s;
    double norm_estimate; /* ‖A'‖₂ as returned by estimate_norm */
    or_check_record *trace;
    int64_t trace_len;
} or_solution;

/* KktReport (crates/saddlepoint-check/src/lib.rs:10-25). */
typedef struct {
    double primal_objective, dual_objective;
    double constraint_violation, bound_violation, dual_violation;
    double relative_primal, relative_dual, relative_gap;
} or_kkt_report;

/* CpuProblem (crates/saddlepoint-cpu/src/lib.rs:25-35). Borrowed pointers. */
typedef struct {
    const or_csr *a, *at;
    const double *c, *lc, *uc, *lv, *uv;
    double *primal_factor, *dual_factor; /* owned */
} or_cpu_problem;

typedef struct { double residual_sq, objective; } or_primal_stats;
typedef struct { double residual_sq, objective; } or_dual_stats;
typedef struct { double objective, violation_sq, norm_sq; } or_ray_stats;

/* ---- thread pool -------------------------------------------------------- */
void or_set_threads(int n);
int or_get_threads(void);

/* ---- CSR (problem.rs:33-126) --------------------------------------------- */
int or_csr_from_triplets(int64_t nrows, int64_t ncols, int64_t ntrip, const int64_t *rows, const int64_t *cols,
                         const double *vals, or_csr *out);
int or_csr_transpose(const or_csr *a, or_csr *out);
void or_csr_mul_vec(const or_csr *a, const double *x, double *out);
void or_csr_scale(or_csr *a, const double *row, const double *col);
void or_csr_free(or_csr *a);
int or_csr_copy(const or_csr *src, or_csr *dst);

/* ---- LP ------------------------------------------------------------------- */
int or_lp_validate(const or_lp *p);
int or_lp_validate_at(const or_lp *p, int *what, int *kind, int64_t *index);
double or_lp_objective(const or_lp *p, const double *x);
void or_lp_free(or_lp *p);

/* ---- scaling (scaling.rs:53-201) ------------------------------------------- */
void or_scaling_params_default(or_scaling_params *p);
int or_scaled_new(const or_lp *p, const or_scaling_params *params, or_scaled *out);
void or_scaled_free(or_scaled *s);
void or_scaled_primal_factors(const or_scaled *s, double *out);
void or_scaled_dual_factors(const or_scaled *s, double *out);
double or_scaled_objective_factor(const or_scaled *s);
void or_scaled_unscale_primal(const or_scaled *s, const double *xs, double *out);
void or_scaled_unscale_dual(const or_scaled *s, const double *ys, double *out);
double or_norm2(const double *v, int64_t n);
double or_finite_bound_norm(const double *lo, const double *hi, int64_t n);

/* ---- CPU backend (crates/saddlepoint-cpu/src/lib.rs:101-260) ---------------- */
int or_cpu_load(const or_scaled *s, or_cpu_problem *out);
void or_cpu_free(or_cpu_problem *p);
void or_cpu_spmv(const or_cpu_problem *p, const double *x, double *out);
void or_cpu_spmv_t(const or_cpu_problem *p, const double *y, double *out);
void or_cpu_primal_step(const or_cpu_problem *p, const double *x, const double *aty, double tau, double *x_t,
                        double *x_bar);
void or_cpu_dual_step(const or_cpu_problem *p, const double *y, const double *ax_bar, double sigma, double *y_t);
void or_cpu_halpern_step(double *z, const double *z_t, const double *anchor, double w, double rho, int64_t n);
double or_cpu_distance_sq(const double *a, const double *b, int64_t n);
void or_cpu_sub(const double *a, const double *b, double *out, int64_t n);
double or_cpu_norm_sq(const double *v, int64_t n);
double or_cpu_dot(const double *a, const double *b, int64_t n);
void or_cpu_scale(double *v, double alpha, int64_t n);
or_primal_stats or_cpu_primal_stats(const or_cpu_problem *p, const double *x, const double *ax);
or_dual_stats or_cpu_dual_stats(const or_cpu_problem *p, const double *y, const double *aty);
double or_cpu_step_dual_residual_sq(const or_cpu_problem *p, const double *x, const double *x_t, const double *aty,
                                    const double *aty_t, double tau);
or_ray_stats or_cpu_primal_ray_stats(const or_cpu_problem *p, const double *dx, const double *adx);
or_ray_stats or_cpu_dual_ray_stats(const or_cpu_problem *p, const double *dy, const double *atdy);

/* ---- solver (solver.rs:154-480) ------------------------------------------- */
void or_solver_params_default(or_solver_params *p);
int or_solve(const or_lp *p, const or_solver_params *params, or_solution *out);
/* Solver::run on a given ScaledProblem (borrowed); norm_override > 0 skips estimate_norm;
 * stop_after > 0 ends the loop after that many iterations without forcing a check. */
int or_solve_scaled(const or_lp *p, const or_scaled *scaled, const or_solver_params *params, double norm_override,
                    uint64_t stop_after, or_solution *out);
void or_solution_free(or_solution *s);
/* PidState::update (solver.rs:459-479), exposed for its unit tests. */
typedef struct { double integral; double prev_error; int has_prev; double best_weight, best_balance; } or_pid;
void or_pid_init(or_pid *pid, double omega);
double or_pid_update(or_pid *pid, const or_solver_params *p, double omega, double dx, double dy, double rel_primal,
                     double rel_dual);

/* ---- checker (crates/saddlepoint-check/src/lib.rs:62-118) -------------------- */
void or_check(const or_lp *p, const double *x, const double *y, or_kkt_report *out);
double or_kkt_max_relative(const or_kkt_report *r);

/* ---- seeded synthetic generators (sp_gen.c) --------------------------------- */
/* kind 0: random LP (nnz_per_col_min..max per column), 1: power-law columns
 * (Zipf(zipf_s) on [degree_min, degree_max] rescaled to target_nnz), 2: transportation
 * LP (supplies x demands). The same draws as the CUDA library's sp_generate. */
typedef struct {
    int kind;
    uint64_t seed;
    int64_t nrows, ncols;
    int64_t nnz_per_col_min, nnz_per_col_max;
    int64_t target_nnz;
    double zipf_s;
    int64_t degree_min, degree_max;
    int64_t supplies, demands;
} or_gen_params;
int or_generate(const or_gen_params *g, or_lp *out);

/* ---- MPS reader (crates/saddlepoint-io/src/lib.rs:59-309) -------------------- */
/* Returns OR_OK or OR_ERR_PARSE with *err_line set (1-based) and err text. */
int or_read_mps(const char *text, size_t len, or_lp *out, int64_t *err_line, char *err, size_t errlen);

#ifdef __cplusplus
}
#endif
#endif
