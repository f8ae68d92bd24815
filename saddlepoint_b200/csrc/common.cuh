// common.cuh — shared definitions for the sm_100a PDHG kernels.
//
// The whole library is compiled with --fmad=false: every multiply and add is
// rounded separately, as in the reference's Rust code, so element-wise results
// and short-row SpMV sums are bit-identical to the CPU backend's.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <cstdio>
#include <string>

#include "../../include/saddlepoint_b200.h"

namespace sp {

constexpr int NT = 256;           // threads per CTA of every tile kernel
constexpr int TILE_NNZ = 2048;    // nonzeros staged per tile (8 per thread)
constexpr int TILE_ROWS = 512;    // rows per tile at most
constexpr int SEQ_MAX = 32;       // rows with at most this many entries are summed by one thread, in order
constexpr int RED_BLOCKS = 592;   // 4 CTAs x 148 SMs: grid of the two-stage reductions
constexpr int RED_SLOTS = 8;      // values one reduction call can produce

// A row tile: {first row, end row, first nonzero, end nonzero}.
using Tile = int4;

// ---- the reference's scalar helpers (crates/saddlepoint-cpu/src/lib.rs:70-99, 262-269) ----

// f64::clamp: `if v < lo { lo } else if v > hi { hi } else { v }` (NaN passes through).
__host__ __device__ __forceinline__ double clampd(double v, double lo, double hi) {
    if (v < lo) v = lo;
    if (v > hi) v = hi;
    return v;
}
// excess (lib.rs:70-80): signed distance from v to [lo, hi].
__host__ __device__ __forceinline__ double excess(double v, double lo, double hi) {
    return v < lo ? v - lo : (v > hi ? v - hi : 0.0);
}
// bound_term (lib.rs:82-92): v+ lo - v- hi, skipping infinite bounds.
__host__ __device__ __forceinline__ double bound_term(double v, double lo, double hi) {
    if (v > 0.0 && isfinite(lo)) return v * lo;
    if (v < 0.0 && isfinite(hi)) return v * hi;
    return 0.0;
}
// forbidden (lib.rs:94-99): the part of v whose sign an infinite bound forbids.
__host__ __device__ __forceinline__ double forbidden(double v, double lo, double hi) {
    return ((v > 0.0 && lo == -INFINITY) || (v < 0.0 && hi == INFINITY)) ? v : 0.0;
}
// recession_violation (lib.rs:262-269).
__host__ __device__ __forceinline__ double recession_violation(double v, double lo, double hi) {
    double l = isfinite(lo) ? 0.0 : -INFINITY;
    double h = isfinite(hi) ? 0.0 : INFINITY;
    return excess(v, l, h);
}
// halpern_step element (lib.rs:185): w ((1 + ρ) z_t - ρ z) + (1 - w) anchor.
__host__ __device__ __forceinline__ double halpern(double z, double zt, double anchor, double w, double rho) {
    return w * ((1.0 + rho) * zt - rho * z) + (1.0 - w) * anchor;
}

// ---- warp and block reductions in a fixed order (deterministic) ----

template <class T>
__device__ __forceinline__ T warp_sum_down(T s) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    return s;  // lane 0 holds the sum
}

// Sums K values over the block; thread 0 returns the totals. `sh` needs K * (NT/32) doubles.
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double *sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int W = NT / 32;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double s = warp_sum_down(v[k]);
        if (lane == 0) sh[k * W + warp] = s;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double s = lane < W ? sh[k * W + lane] : 0.0;
            v[k] = warp_sum_down(s);
        }
    }
    __syncthreads();
}

// ---- device-resident solver state (the reference keeps these on the host, solver.rs:311-420) ----

struct DevParams {
    double tolerance, infeasibility_tolerance;
    unsigned long long max_iterations, check_every;
    double reflection, restart_sufficient, restart_necessary, restart_artificial;
    double pid_kp, pid_ki, pid_kd, pid_discount;
    int termination, mixed;
    double mixed_switch_tolerance;
    int mixed_stall_checks;  // checks without a 10 % gain after which the mixed form moves to FP64
    double b_norm, c_norm, c0, obj_factor, eta;
    int bound_objective_rescaling;
};

struct DevState {
    unsigned long long total;  // iterations completed before this epoch
    unsigned long long k;      // Halpern counter at the start of this epoch
    double omega;
    int done, status, error, restart_flag;
    double w_last;             // Halpern weight of the check iteration (for the finish pass)
    int fp64;                  // mixed form: 1 once the SpMV runs in FP64
    int k0_epoch;              // 1 if this epoch started with k == 0
    unsigned long long fp64_from;
    double anchor_residual, prev_residual, last_residual;
    unsigned long long restarts, checks;
    double pid_integral, pid_prev_error;
    int pid_has_prev, pad0;
    double pid_best_weight, pid_best_balance;
    double primal_obj, dual_obj, primal_res, dual_res, step_dual, step_obj;
    // power iteration
    double pi_scale, pi_lambda;
    int pi_done, pi_iters;
    unsigned long long trace_len;
    // mixed form: best relative KKT error of the FP32 phase and checks since it improved
    double mx_best;
    int mx_since;
    int handoff;  // batched form: stopped for the single-LP solver
};

// Mixed form: checks without a 10% gain in the relative KKT error after which the
// FP32 phase is taken to have stalled at its precision and the SpMV moves to FP64.
constexpr int MIXED_STALL_CHECKS = 40;

enum : int { ERR_NONE = 0, ERR_NUMERICAL_POWER = 1, ERR_NUMERICAL_ITERATES = 2, ERR_PIPELINE_STALL = 3 };

// Elements of slack after the last row pointer / nonzero / vector entry of the
// arrays the stream engine stages: a bulk copy rounds its range out to 16 bytes.
constexpr int CSR_PAD = 16;

// ---- host-side error plumbing ----

struct Err {
    int code = SP_OK;
    std::string msg;
};

#define SP_CUDA_TRY(expr)                                                                    \
    do {                                                                                     \
        cudaError_t _e = (expr);                                                             \
        if (_e != cudaSuccess) {                                                             \
            return ::sp::fail(SP_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
        }                                                                                    \
    } while (0)

int fail(int code, const std::string &msg);  // records the error on the current thread's context
void set_current_ctx(sp_ctx *ctx);

// Two timing events, created by init() (checked) and destroyed with the object.
struct EventPair {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int init() {
        SP_CUDA_TRY(cudaEventCreate(&e0));
        SP_CUDA_TRY(cudaEventCreate(&e1));
        return SP_OK;
    }
    ~EventPair() {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
    }
};

}  // namespace sp
