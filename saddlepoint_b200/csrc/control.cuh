// control.cuh — the decisions the reference's host loop takes at a check
// (crates/saddlepoint-core/src/solver.rs:339-419 and PidState, :445-480), as device
// code shared by the single-LP controller kernel and the batched kernel.
#pragma once

#include "common.cuh"

namespace sp {

// Partial-sum slots of the passes.
constexpr int NP_P = 8;   // primal check pass
constexpr int NP_D = 8;   // dual check pass
constexpr int NP_T = 5;   // A'ᵀ check pass
constexpr int NP_P0 = 1;  // primal pass of a k == 0 iteration
constexpr int NP_D0 = 2;  // dual pass of a k == 0 iteration

// Slot layout of the partial sums a check produces.
//   P[0] Σ(x_t-x)²   P[1] c'ᵀx_t   P[2] atyᵀx_t   P[3] x_tᵀx_t   P[4] xᵀx_t
//   P[5] Σ rv(x_t-x_a)²   P[6] Σ(x_t-x_a)²   P[7] c'ᵀ(x_t-x_a)
//   D[0] Σ(y_t-y)²   D[1] (y_t-y)ᵀA'(x_t-x)   D[2] Σ(excess(A'x_t)·f)²   D[3] Σ bound_term(y_t)
//   D[4] Σ rv(A'(x_t-x_a))²   D[5] Σ forbidden(y_t-y_a)²   D[6] Σ bound_term(y_t-y_a)   D[7] Σ(y_t-y_a)²
//   T[0] Σ(forbidden(c'-A'ᵀy_t)·f)²   T[1] Σ bound_term(c'-A'ᵀy_t)   T[2] step-implied dual residual²
//   T[3] Σ forbidden(-A'ᵀ(y_t-y_a))²   T[4] Σ bound_term(-A'ᵀ(y_t-y_a))

// Sums slot q of a [tiles x NPQ] partial array: each thread adds tiles t, t + NT, ...
// in order, then a fixed tree over the block. The totals are valid in thread 0.
template <int NPQ>
__device__ void sum_slots(const double *part, int tiles, double (&out)[NPQ], double *sh) {
    double v[NPQ];
#pragma unroll
    for (int q = 0; q < NPQ; ++q) v[q] = 0.0;
    for (int t = threadIdx.x; t < tiles; t += NT)
#pragma unroll
        for (int q = 0; q < NPQ; ++q) v[q] += part[t * NPQ + q];
    block_sum<NPQ>(v, sh);
#pragma unroll
    for (int q = 0; q < NPQ; ++q) out[q] = v[q];
}

// fixed_point_residual (solver.rs:275-288) from its three sums.
__device__ __forceinline__ double fixed_point_residual(double eta, double omega, double dx2, double dy2, double cross,
                                                       bool *bad) {
    const double r2 = omega / eta * dx2 + dy2 / (eta * omega) + 2.0 * cross;
    if (!isfinite(r2)) *bad = true;
    return sqrt(fmax(r2, 0.0));
}

// PidState::update (solver.rs:459-479).
__device__ __forceinline__ double pid_update(DevState *st, const DevParams *p, double omega, double dx, double dy,
                                             double rel_primal, double rel_dual) {
    auto sane = [](double v) { return v >= 1e-16 && v <= 1e12; };
    const double ratio = rel_dual / rel_primal;
    if (!sane(dx) || !sane(dy) || !(ratio >= 1e-8 && ratio <= 1e8)) {
        st->pid_integral = 0.0;
        st->pid_has_prev = 0;
        return st->pid_best_weight;
    }
    const double e = log(omega * dx / dy);
    st->pid_integral = p->pid_discount * st->pid_integral + e;
    const double derivative = st->pid_has_prev ? e - st->pid_prev_error : 0.0;
    st->pid_prev_error = e;
    st->pid_has_prev = 1;
    const double next = exp(log(omega) - (p->pid_kp * e + p->pid_ki * st->pid_integral + p->pid_kd * derivative));
    const double balance = fabs(log10(ratio));
    if (balance < st->pid_best_balance) {
        st->pid_best_balance = balance;
        st->pid_best_weight = next;
    }
    return next;
}

// The check iteration whose Halpern counter is kc, after `total` iterations:
// residual, KKT (solver.rs:245-258), convergence (:147-151, :383-385),
// infeasibility (:291-309), iteration limit, restart and PID (:396-419).
// Sets st->done/status, or the restart flag, the next k and ω. *bad is set (and
// st->error) when the iterates are not finite.
__device__ __forceinline__ void check_decide(DevState *st, const DevParams *p, const double *P, const double *D,
                                             const double *T, unsigned long long kc, unsigned long long total,
                                             bool *bad, sp_check_record *rec) {
    const double eta = p->eta, omega = st->omega;
    const double residual = fixed_point_residual(eta, omega, P[0], D[0], D[1], bad);
    if (*bad) {
        st->error = ERR_NUMERICAL_ITERATES;
        st->done = 1;
        return;
    }
    if (kc == 0) st->anchor_residual = residual;
    const double f = p->obj_factor;
    const double primal_obj = P[1] * f + p->c0;
    const double dual_obj = (D[3] + T[1]) * f + p->c0;
    const double primal_res = sqrt(D[2]);
    const double dual_res = sqrt(T[0]);
    const double step_dual = sqrt(T[2]);
    const double tau = eta / omega;
    double test_dual_obj = dual_obj, test_dual_res = dual_res;
    if (p->termination == SP_TERMINATION_STEP_IMPLIED) {  // step_dual_objective (solver.rs:263-271)
        const double lx = P[1] - P[2] + (P[3] - P[4]) / tau;
        test_dual_obj = (D[3] + 0.0 + lx) * f + p->c0;
        test_dual_res = step_dual;
    }
    st->w_last = (double)(kc + 1) / (double)(kc + 2);
    unsigned long long k = kc + 1;
    st->checks += 1;
    st->total = total;
    st->primal_obj = primal_obj;
    st->dual_obj = dual_obj;
    st->primal_res = primal_res;
    st->dual_res = dual_res;
    st->step_dual = step_dual;
    st->step_obj = test_dual_obj;
    st->last_residual = residual;
    st->restart_flag = 0;
    rec->total = total;
    rec->residual = residual;
    rec->primal_obj = primal_obj;
    rec->dual_obj = dual_obj;
    rec->primal_res = primal_res;
    rec->dual_res = dual_res;
    rec->restarted = 0;

    const double eps = p->tolerance;
    const double gap = fabs(primal_obj - test_dual_obj);
    int stop = -1;
    if (primal_res <= eps * (1.0 + p->b_norm) && test_dual_res <= eps * (1.0 + p->c_norm) &&
        gap <= eps * (1.0 + fabs(primal_obj) + fabs(test_dual_obj)))
        stop = SP_STATUS_OPTIMAL;
    if (stop < 0) {
        const double ie = p->infeasibility_tolerance;
        const double d_obj = D[6] + T[4], d_viol = D[5] + T[3], d_norm = D[7];
        const double p_obj = P[7], p_viol = D[4] + P[5], p_norm = P[6];
        if (d_obj > 0.0 && sqrt(d_viol) <= ie * d_obj && d_obj > ie * sqrt(d_norm))
            stop = SP_STATUS_PRIMAL_INFEASIBLE;
        else if (p_obj < 0.0 && sqrt(p_viol) <= -ie * p_obj && -p_obj > ie * sqrt(p_norm))
            stop = SP_STATUS_DUAL_INFEASIBLE;
    }
    if (stop < 0 && total >= p->max_iterations) stop = SP_STATUS_ITERATION_LIMIT;
    if (stop >= 0) {
        st->status = stop;
        st->done = 1;
        st->k = k;
        rec->omega = omega;
        rec->k_after = k;
        return;
    }
    // Mixed form: move the SpMV to FP64 once the relative KKT error is small, or
    // once the FP32 phase stops making progress (it has reached its precision).
    if (p->mixed && !st->fp64) {
        const double rel = fmax(fmax(primal_res / (1.0 + p->b_norm), dual_res / (1.0 + p->c_norm)),
                                fabs(primal_obj - dual_obj) / (1.0 + fabs(primal_obj) + fabs(dual_obj)));
        if (rel < 0.9 * st->mx_best) {
            st->mx_best = rel;
            st->mx_since = 0;
        } else {
            st->mx_since += 1;
        }
        if (rel < p->mixed_switch_tolerance || st->mx_since >= p->mixed_stall_checks) {
            st->fp64 = 1;
            st->fp64_from = total + 1;
        }
    }
    const double r0 = st->anchor_residual;
    const bool restart = residual <= p->restart_sufficient * r0 ||
                         (residual <= p->restart_necessary * r0 && residual > st->prev_residual) ||
                         (double)k >= p->restart_artificial * (double)total;
    st->prev_residual = residual;
    double w = omega;
    if (restart) {
        // distance_sq(x_t, x_anchor) and distance_sq(y_t, y_anchor) are the ray norms.
        const double dx = sqrt(P[6]), dy = sqrt(D[7]);
        w = pid_update(st, p, omega, dx, dy, primal_res / (1.0 + p->b_norm), step_dual / (1.0 + p->c_norm));
        st->omega = w;
        st->restart_flag = 1;
        st->restarts += 1;
        st->prev_residual = INFINITY;
        k = 0;
    }
    st->k = k;
    rec->restarted = restart;
    rec->omega = w;
    rec->k_after = k;
}

}  // namespace sp
