// solver.cu — the device-resident solve: GPU scaling passes and transpose,
// power iteration, PDHG epochs captured as CUDA graphs, and the controller that
// makes the reference's host-side decisions on the device.
//
// Restates crates/saddlepoint-core/src/solver.rs:185-480 (Solver::new, run,
// estimate_norm, kkt, fixed_point_residual, infeasibility, PidState) and
// crates/saddlepoint-core/src/scaling.rs:53-103 (ScaledProblem::new).
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "control.cuh"
#include "internal.cuh"
#include "solver_kernels.cuh"
#include "solver_state.h"

namespace sp {

#define GRID_LOOP(i, n) for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

// ============================================================ controller

struct CtrlArgs {
    const double *partP, *partD, *partT, *partP0, *partD0;
    int nP, nD;  // tiles of A'ᵀ and of A'
    int E;       // iterations in this epoch
    sp_check_record *trace;
    long long trace_cap;
};

// The end of an epoch: the check iteration's decisions (solver.rs:339-419).
__global__ void __launch_bounds__(NT) k_controller(CtrlArgs a, const DevParams *p, DevState *st) {
    __shared__ double sh[NP_P * (NT / 32)];
    if (st->done) return;
    double P[NP_P], D[NP_D], T[NP_T], P0[1], D0[2];
    sum_slots<NP_P>(a.partP, a.nP, P, sh);
    sum_slots<NP_D>(a.partD, a.nD, D, sh);
    sum_slots<NP_T>(a.partT, a.nP, T, sh);
    const bool k0_first = st->k == 0 && a.E >= 2;
    if (k0_first) {
        sum_slots<1>(a.partP0, a.nP, P0, sh);
        sum_slots<2>(a.partD0, a.nD, D0, sh);
    }
    if (threadIdx.x != 0) return;
    bool bad = false;
    if (k0_first) st->anchor_residual = fixed_point_residual(p->eta, st->omega, P0[0], D0[0], D0[1], &bad);
    const unsigned long long kc = st->k + (unsigned long long)(a.E - 1);  // k of the check iteration
    const unsigned long long total = st->total + (unsigned long long)a.E;
    sp_check_record rec;
    check_decide(st, p, P, D, T, kc, total, &bad, &rec);
    if (bad) return;
    if ((long long)st->checks - 1 < a.trace_cap) a.trace[st->checks - 1] = rec;
    st->trace_len = st->checks;
}
// After the check iteration: Halpern step, or the restart's copies (solver.rs:361-362, 411-415).
__global__ void k_finish(SolverPtrs s, int64_t n, int64_t m) {
    const DevState *st = s.st;
    if (st->done) return;
    const double w = st->w_last, rho = s.prm->reflection;
    const int rs = st->restart_flag;
    const bool y32 = s.mixed && !st->fp64;
    GRID_LOOP(j, n) {
        if (rs) {
            const double t = s.xt[j];
            s.xa[j] = t;
            s.x[j] = t;
        } else {
            s.x[j] = halpern(s.x[j], s.xt[j], s.xa[j], w, rho);
        }
    }
    GRID_LOOP(i, m) {
        double v;
        if (rs) {
            v = s.yt[i];
            s.ya[i] = v;
        } else {
            v = halpern(s.y[i], s.yt[i], s.ya[i], w, rho);
        }
        s.y[i] = v;
        if (y32) s.y32[i] = (float)v;
    }
}

// Halpern step of x in the k == 0 iteration that opens an epoch (D did y already).
__global__ void k_halpern_x0(SolverPtrs s, int64_t n) {
    const DevState *st = s.st;
    if (st->done || st->k != 0) return;
    const double w = 1.0 / 2.0, rho = s.prm->reflection;  // (k + 1) / (k + 2) at k = 0
    GRID_LOOP(j, n) { s.x[j] = halpern(s.x[j], s.xt[j], s.xa[j], w, rho); }
}

// ============================================================ power iteration

// start = 1 + 0.01 (j mod 7) (solver.rs:221)
__device__ __forceinline__ double power_start(int64_t j) { return 1.0 + 0.01 * (double)(j % 7); }

__global__ void k_power_fill(double *v, int64_t n) {
    GRID_LOOP(j, n) { v[j] = power_start(j); }
}

// ‖start‖², reduced by one block in a fixed order (the terms are formed, not loaded;
// j mod 7 steps by NT mod 7 from one term of a thread to its next).
__global__ void k_power_init(int64_t n, double *part) {
    __shared__ double sh[NT / 32];
    double s[1] = {0.0};
    int r = threadIdx.x % 7;
    for (int64_t j = threadIdx.x; j < n; j += NT) {
        const double x = 1.0 + 0.01 * (double)r;
        s[0] += x * x;
        r += NT % 7;
        if (r >= 7) r -= 7;
    }
    block_sum<1>(s, sh);
    if (threadIdx.x == 0) part[0] = s[0];
}

__global__ void k_power_start(const double *part, DevState *st) {
    if (threadIdx.x) return;
    st->pi_scale = 1.0 / sqrt(part[0]);  // solver.rs:223
    st->pi_lambda = 0.0;
    st->pi_done = 0;
    st->pi_iters = 0;
    st->error = ERR_NONE;
}

__global__ void __launch_bounds__(NT) k_power_fin(const double *part, int tiles, unsigned long long max_iters,
                                                  DevState *st) {
    __shared__ double sh[NT / 32];
    if (st->pi_done) return;
    double s[1];
    sum_slots<1>(part, tiles, s, sh);
    if (threadIdx.x) return;
    const double norm = sqrt(s[0]);  // solver.rs:229-238
    if (isnan(norm) || norm <= 0.0 || isinf(norm)) {
        st->error = ERR_NUMERICAL_POWER;
        st->pi_done = 1;
        return;
    }
    st->pi_scale = 1.0 / norm;
    const bool done = fabs(norm - st->pi_lambda) <= 1e-6 * norm;
    st->pi_lambda = norm;
    st->pi_iters += 1;
    if (done || (unsigned long long)st->pi_iters >= max_iters) st->pi_done = 1;
}

// ============================================================ scaling passes (scaling.rs:53-103)

__device__ __forceinline__ double inv_sqrt_d(double v) {  // scaling.rs:139-141
    return (v > 0.0 && isfinite(v)) ? 1.0 / sqrt(v) : 1.0;
}

// Per-row geometric-mean factor 1/sqrt(min·max) of |a| (scaling.rs:62-63, min_max :159-178).
// The row passes of the scaling below take each row with a group of G lanes (G = 4 … 32,
// from the matrix's mean row length): min and max do not depend on the order, so the group
// size changes no bit, and short rows no longer leave most of a warp idle. The row loop
// steps a whole warp (32 / G rows) at a time so that every lane reaches each shuffle.
template <int G>
__global__ void k_row_geo(const int *rp, const double *v, int64_t rows, double *f) {
    const int lane = threadIdx.x & 31, sub = lane % G;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = warp * (32 / G); base < rows; base += nw * (32 / G)) {
        const int64_t r = base + lane / G;
        double lo = INFINITY, hi = 0.0;
        if (r < rows)
            for (int k = rp[r] + sub; k < rp[r + 1]; k += G) {
                const double a = fabs(v[k]);
                lo = fmin(lo, a);
                hi = fmax(hi, a);
            }
        for (int o = G / 2; o; o >>= 1) {
            lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        if (sub == 0 && r < rows) {
            if (hi == 0.0) lo = 0.0;
            f[r] = inv_sqrt_d(lo * hi);
        }
    }
}
template <int G>
__global__ void k_row_ruiz(const int *rp, const double *v, int64_t rows, double *f) {
    const int lane = threadIdx.x & 31, sub = lane % G;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = warp * (32 / G); base < rows; base += nw * (32 / G)) {
        const int64_t r = base + lane / G;
        double hi = 0.0;
        if (r < rows)
            for (int k = rp[r] + sub; k < rp[r + 1]; k += G) hi = fmax(hi, fabs(v[k]));
        for (int o = G / 2; o; o >>= 1) hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        if (sub == 0 && r < rows) f[r] = inv_sqrt_d(hi);
    }
}
__global__ void k_row_pc(const int *rp, const double *v, int64_t rows, double alpha, double *f) {
    GRID_LOOP(r, rows) {
        double s = 0.0;
        for (int k = rp[r]; k < rp[r + 1]; ++k) {
            const double a = fabs(v[k]);
            s = s + (alpha == 1.0 ? a : pow(a, alpha));
        }
        f[r] = inv_sqrt_d(s);
    }
}

// The scaling's sweeps. The reference scales A' in place with a.scale(r, c)
// (values[k] *= r[i] * c[j], problem.rs:118-125) and forms each next factor from the
// scaled values (scaling.rs:53-79); it builds A'ᵀ only at the end. Here A'ᵀ exists
// from the start, so every step updates both layouts with the same operations (an
// entry gets the same roundings in both) and forms the statistic of the next step from
// the values it has just written, in the same sweep: one read and one write of each
// layout per step, instead of a statistics sweep plus an apply sweep of both layouts
// per half-step, and no multiplications by the all-ones vector (r·1 = r exactly).
enum NextStat : int { NEXT_NONE = 0, NEXT_GEO = 1, NEXT_MAX = 2 };

template <int G>
__device__ __forceinline__ void group_min_max(double &lo, double &hi) {
    for (int o = G / 2; o; o >>= 1) {
        lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
}

// The factor a NEXT statistic gives a row: 1/sqrt(min·max) of its magnitudes
// (min_max, scaling.rs:159-178: an empty or all-zero row counts min as 0), or
// 1/sqrt(max) (the Ruiz step, scaling.rs:68-70).
template <int NEXT>
__device__ __forceinline__ double next_factor(double lo, double hi) {
    return NEXT == NEXT_GEO ? inv_sqrt_d((hi == 0.0 ? 0.0 : lo) * hi) : inv_sqrt_d(hi);
}

// Short rows (at most SWEEP_TRIPS·G entries) go to a group of G lanes; a longer row is
// taken by the whole warp after the group pass (a ballot finds them), so one long row does
// not hold up the warp's other groups for many trips. Neither choice changes a bit: every
// entry is computed alone and min / max do not depend on the order. (Measured on the 40M
// LP's layouts: plain loads beat chunks of loads issued ahead and the streaming cache hints
// here, 0.31 against 0.42-0.69 ms on A', 0.37 against 0.52 ms on A'ᵀ.)
constexpr int SWEEP_TRIPS = 4;

// Entry k's new value: GEO2 (v·own)·gat, else v·(own·gat).
template <bool GEO2>
__device__ __forceinline__ double sweep_value(double v, double own, double g) {
    return GEO2 ? (v * own) * g : v * (own * g);
}

// Entries k, k + step, ... < k1 of one row (a long row: step 32, all lanes): new values
// written, min / max of their magnitudes into lo / hi.
template <bool GEO2, bool STATS>
__device__ __forceinline__ void sweep_span(const int *__restrict__ ci, double *__restrict__ v,
                                           const double *__restrict__ gat, int k, int k1, int step, double f,
                                           double &lo, double &hi) {
    for (; k < k1; k += step) {
        const double a = sweep_value<GEO2>(v[k], f, __ldg(gat + ci[k]));
        v[k] = a;
        if (STATS) {
            lo = fmin(lo, fabs(a));
            hi = fmax(hi, fabs(a));
        }
    }
}

// One sweep over a layout, G lanes per row: every entry of row `r` is multiplied by its
// row's factor own[r] and the factor gat[ci] of its other index, as
//   GEO2:  (v·own)·gat — the A' side of a geometric-mean pass, whose two applies each
//          had a factor of 1 on the other side (two roundings, as the reference);
//   else:  v·(own·gat) — Ruiz and Pock-Chambolle, one product as problem.rs:123 forms
//          it (on the A'ᵀ side the product is c_j·r_i, the same number: IEEE
//          multiplication commutes).
// scale[r] *= own[r] (apply, scaling.rs:181-183); next[r] = the NEXT statistic's
// factor of the row's new values.
template <int G, bool GEO2, int NEXT>
__global__ void __launch_bounds__(NT) k_scale_sweep(const int *__restrict__ rp, const int *__restrict__ ci,
                                                    double *__restrict__ v, int64_t rows,
                                                    const double *__restrict__ own, const double *__restrict__ gat,
                                                    double *__restrict__ scale, double *__restrict__ next) {
    constexpr bool STATS = NEXT != NEXT_NONE;
    const int lane = threadIdx.x & 31, sub = lane % G;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = warp * (32 / G); base < rows; base += nw * (32 / G)) {
        const int64_t r = base + lane / G;
        const bool live = r < rows;
        const int k0 = live ? rp[r] : 0, k1 = live ? rp[r + 1] : 0;
        const bool longrow = k1 - k0 > SWEEP_TRIPS * G;
        const double f = live ? own[r] : 1.0;
        double lo = INFINITY, hi = 0.0;
        if (!longrow) sweep_span<GEO2, STATS>(ci, v, gat, k0 + sub, k1, G, f, lo, hi);
        if (STATS) group_min_max<G>(lo, hi);
        if (sub == 0 && live && !longrow) {
            scale[r] *= f;
            if (STATS) next[r] = next_factor<NEXT>(lo, hi);
        }
        for (unsigned mask = __ballot_sync(0xffffffffu, sub == 0 && longrow); mask; mask &= mask - 1) {
            const int src = __ffs(mask) - 1;
            const int a = __shfl_sync(0xffffffffu, k0, src), b = __shfl_sync(0xffffffffu, k1, src);
            const double ff = __shfl_sync(0xffffffffu, f, src);
            double l2 = INFINITY, h2 = 0.0;
            sweep_span<GEO2, STATS>(ci, v, gat, a + lane, b, 32, ff, l2, h2);
            if (STATS) group_min_max<32>(l2, h2);
            if (lane == 0) {
                const int64_t rr = base + src / G;
                scale[rr] *= ff;
                if (STATS) next[rr] = next_factor<NEXT>(l2, h2);
            }
        }
    }
}

// The A'ᵀ side of a geometric-mean pass (row j of A'ᵀ is column j of A'): the row factor
// of A' (gathered) comes first; the column factor c_j = 1/sqrt(min·max) of the column
// after it (scaling.rs:64-65) needs the whole column, so a first walk forms it from the
// products v·r and a second writes (v·r)·c_j — from the products a short row's lanes
// kept in registers, a long row's formed again. fac[j] = c_j (the A' side gathers it),
// scale[j] *= c_j; NEXT_MAX also gives the first Ruiz factor of the column from the
// written values.
template <int G, int NEXT>
__global__ void __launch_bounds__(NT) k_scale_geo_cols(const int *__restrict__ rp, const int *__restrict__ ci,
                                                       double *__restrict__ v, int64_t rows,
                                                       const double *__restrict__ gat, double *__restrict__ fac,
                                                       double *__restrict__ scale, double *__restrict__ next) {
    constexpr bool STATS = NEXT != NEXT_NONE;
    const int lane = threadIdx.x & 31, sub = lane % G;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = warp * (32 / G); base < rows; base += nw * (32 / G)) {
        const int64_t r = base + lane / G;
        const bool live = r < rows;
        const int k0 = live ? rp[r] : 0, k1 = live ? rp[r + 1] : 0;
        const bool longrow = k1 - k0 > SWEEP_TRIPS * G;
        double pr[SWEEP_TRIPS];
        double lo = INFINITY, hi = 0.0;
        if (!longrow) {
            int c[SWEEP_TRIPS];
            double x[SWEEP_TRIPS];
#pragma unroll
            for (int t = 0; t < SWEEP_TRIPS; ++t) {
                const int k = k0 + sub + t * G;
                if (k < k1) {
                    c[t] = __ldcs(ci + k);
                    x[t] = __ldcs(v + k);
                }
            }
#pragma unroll
            for (int t = 0; t < SWEEP_TRIPS; ++t)
                if (k0 + sub + t * G < k1) {
                    pr[t] = x[t] * __ldg(gat + c[t]);
                    lo = fmin(lo, fabs(pr[t]));
                    hi = fmax(hi, fabs(pr[t]));
                }
        }
        group_min_max<G>(lo, hi);
        const double cf = next_factor<NEXT_GEO>(lo, hi);
        double lo2 = INFINITY, hi2 = 0.0;
        if (!longrow) {
#pragma unroll
            for (int t = 0; t < SWEEP_TRIPS; ++t) {
                const int k = k0 + sub + t * G;
                if (k < k1) {
                    const double a = pr[t] * cf;
                    __stcs(v + k, a);
                    if (STATS) hi2 = fmax(hi2, fabs(a));
                }
            }
        }
        if (STATS) group_min_max<G>(lo2, hi2);
        if (sub == 0 && live && !longrow) {
            fac[r] = cf;
            scale[r] *= cf;
            if (STATS) next[r] = next_factor<NEXT>(lo2, hi2);
        }
        for (unsigned mask = __ballot_sync(0xffffffffu, sub == 0 && longrow); mask; mask &= mask - 1) {
            const int src = __ffs(mask) - 1;
            const int a = __shfl_sync(0xffffffffu, k0, src), b = __shfl_sync(0xffffffffu, k1, src);
            double l3 = INFINITY, h3 = 0.0;
            for (int k = a + lane; k < b; k += 32) {
                const double p = fabs(v[k] * __ldg(gat + ci[k]));  // read again below: cached loads
                l3 = fmin(l3, p);
                h3 = fmax(h3, p);
            }
            group_min_max<32>(l3, h3);
            const double c3 = next_factor<NEXT_GEO>(l3, h3);
            double l4 = INFINITY, h4 = 0.0;
            for (int k = a + lane; k < b; k += 32) {
                const double x = (v[k] * __ldg(gat + ci[k])) * c3;
                v[k] = x;
                if (STATS) h4 = fmax(h4, fabs(x));
            }
            if (STATS) group_min_max<32>(l4, h4);
            if (lane == 0) {
                const int64_t rr = base + src / G;
                fac[rr] = c3;
                scale[rr] *= c3;
                if (STATS) next[rr] = next_factor<NEXT>(l4, h4);
            }
        }
    }
}

__global__ void k_fill(double *v, double x, int64_t n) {
    GRID_LOOP(i, n) { v[i] = x; }
}

// c' = c·C, lc' = lc·R, uc' = uc·R, lv' = lv/C, uv' = uv/C (scaling.rs:83-87).
__global__ void k_scale_vectors(const double *c, const double *lc, const double *uc, const double *lv, const double *uv,
                                const double *rs, const double *cs, double *c2, double *lc2, double *uc2, double *lv2,
                                double *uv2, int64_t m, int64_t n) {
    GRID_LOOP(j, n) {
        c2[j] = c[j] * cs[j];
        lv2[j] = lv[j] / cs[j];
        uv2[j] = uv[j] / cs[j];
    }
    GRID_LOOP(i, m) {
        lc2[i] = lc[i] * rs[i];
        uc2[i] = uc[i] * rs[i];
    }
}

// The four norms the solve needs, each a sequential sum from -0.0 in index order,
// as the reference computes them (scaling.rs:186-201): finite_bound_norm and norm2
// of the scaled bounds and objective, and of the original ones (solver.rs:317-318).
// Each norm is one sequential sum in index order, added by thread 0 of its block
// while the other threads stage the next chunk in shared memory (the add chain, not
// the loads, sets the pace). Block b computes norm b: the bound and cost norms of
// the original problem (norms[2], norms[3]) and of the scaled one (norms[0],
// norms[1]).
constexpr int SEQ_CHUNK = 2048;

__global__ void __launch_bounds__(NT) k_seq_norms(const double *olc, const double *ouc, const double *oc,
                                                  const double *lc, const double *uc, const double *c, int64_t m,
                                                  int64_t n, double *norms) {
    // The terms of the sum are independent of one another: threads 1..NT-1 form the next
    // chunk's terms (each with the reference's operations) while thread 0 adds this chunk's
    // in index order; the additions, the one dependent chain, are exactly the reference's.
    __shared__ double st[2][SEQ_CHUNK];
    const int which = blockIdx.x & 1;  // 0: bound norm over m rows, 1: cost norm over n columns
    const bool orig = blockIdx.x < 2;
    const double *a = which == 0 ? (orig ? olc : lc) : (orig ? oc : c);
    const double *b = orig ? ouc : uc;
    const int64_t len = which == 0 ? m : n;
    const int64_t nchunks = (len + SEQ_CHUNK - 1) / SEQ_CHUNK;
    auto stage = [&](int64_t k, int buf) {  // threads 1..NT-1
        const int64_t base = k * SEQ_CHUNK;
        for (int i = threadIdx.x - 1; i < SEQ_CHUNK; i += NT - 1) {
            const int64_t e = base + i;
            if (e >= len) break;
            if (which == 0) {  // finite_bound_norm's term (scaling.rs:191-201)
                const double l = isfinite(a[e]) ? a[e] : 0.0;
                const double u = isfinite(b[e]) ? b[e] : 0.0;
                st[buf][i] = (l == u) ? l * l : l * l + u * u;
            } else {
                st[buf][i] = a[e] * a[e];  // norm2's term (scaling.rs:186-188)
            }
        }
    };
    if (threadIdx.x > 0 && nchunks > 0) stage(0, 0);
    __syncthreads();
    double s = -0.0;
    for (int64_t k = 0; k < nchunks; ++k) {
        const int buf = (int)(k & 1);
        if (threadIdx.x == 0) {
            const int cnt = (int)min((int64_t)SEQ_CHUNK, len - k * SEQ_CHUNK);
            const double *t = st[buf];
            int i = 0;
            for (; i + 8 <= cnt; i += 8) {
                double v[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) v[u] = t[i + u];
#pragma unroll
                for (int u = 0; u < 8; ++u) s += v[u];
            }
            for (; i < cnt; ++i) s += t[i];
        } else if (k + 1 < nchunks) {
            stage(k + 1, buf ^ 1);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) norms[(orig ? 2 : 0) + which] = sqrt(s);
}

__global__ void k_rescale(double *lc, double *uc, double *lv, double *uv, double *c, const double *norms, int64_t m,
                          int64_t n, int enabled, double *scales) {
    const double bs = enabled ? 1.0 / (1.0 + norms[0]) : 1.0;  // scaling.rs:91-92
    const double os = enabled ? 1.0 / (1.0 + norms[1]) : 1.0;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        scales[0] = bs;
        scales[1] = os;
    }
    if (!enabled) return;
    GRID_LOOP(i, m) {
        lc[i] *= bs;
        uc[i] *= bs;
    }
    GRID_LOOP(j, n) {
        lv[j] *= bs;
        uv[j] *= bs;
        c[j] *= os;
    }
}

__global__ void k_factors(const double *rs, const double *cs, const double *scales, double *pf, double *df, int64_t m,
                          int64_t n) {
    const double bs = scales[0], os = scales[1];
    GRID_LOOP(i, m) { pf[i] = 1.0 / (rs[i] * bs); }  // scaling.rs:124-126
    GRID_LOOP(j, n) { df[j] = 1.0 / (cs[j] * os); }  // scaling.rs:129-131
}

__global__ void k_to_f32(const double *v, float *o, int64_t n) {
    GRID_LOOP(i, n) { o[i] = (float)v[i]; }
}

// Transpose helpers: the row of every nonzero, then A'ᵀ from a stable sort by column.
__global__ void k_row_ids(const int *rp, int64_t rows, int *row_of) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = warp; i < rows; i += nw)
        for (int k = rp[i] + lane; k < rp[i + 1]; k += 32) row_of[k] = (int)i;
}
__global__ void k_iota(int *v, int64_t n) {
    GRID_LOOP(i, n) { v[i] = (int)i; }
}
// A'ᵀ row pointers from the sorted column keys: rp_t[j] = first position with key >= j.
__global__ void k_rowptr_from_sorted(const int *keys, int64_t nnz, int64_t ncols, int *rp_t) {
    GRID_LOOP(j, ncols + 1) {
        int64_t lo = 0, hi = nnz;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (keys[mid] < j) lo = mid + 1;
            else hi = mid;
        }
        rp_t[j] = (int)lo;
    }
}
__global__ void k_gather_transpose(const int *perm, const int *row_of, const double *v, int *ci_t, double *v_t,
                                   int64_t nnz) {
    GRID_LOOP(k, nnz) {
        const int src = perm[k];
        ci_t[k] = row_of[src];
        v_t[k] = v[src];
    }
}

// x = x_t C / β, y = y_t R / γ (scaling.rs:113-121).
__global__ void k_unscale(const double *xt, const double *yt, const double *cs, const double *rs, const double *scales,
                          double *x, double *y, int64_t n, int64_t m) {
    const double bs = scales[0], os = scales[1];
    GRID_LOOP(j, n) { x[j] = xt[j] * cs[j] / bs; }
    GRID_LOOP(i, m) { y[i] = yt[i] * rs[i] / os; }
}

// A starting point given in the original space, mapped into the scaled one (the inverse of
// k_unscale: x' = x·β / col_scale, y' = y·γ / row_scale), as iterate and anchor; the mixed
// form's FP32 shadow of y too (the first primal pass gathers it).
__global__ void k_warm_start(const double *x0, const double *y0, const double *cs, const double *rs,
                             const double *scales, double *x, double *xa, double *y, double *ya, float *y32,
                             int64_t n, int64_t m) {
    const double bs = scales[0], os = scales[1];
    GRID_LOOP(j, n) {
        const double v = x0 ? x0[j] * bs / cs[j] : 0.0;
        x[j] = v;
        xa[j] = v;
    }
    GRID_LOOP(i, m) {
        const double v = y0 ? y0[i] * os / rs[i] : 0.0;
        y[i] = v;
        ya[i] = v;
        if (y32) y32[i] = (float)v;
    }
}

}  // namespace sp

// ============================================================ host side

using namespace sp;

namespace {

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

int grid_of(const sp_ctx *ctx, int64_t n, int per_thread_items = 1) {
    int64_t b = (n / per_thread_items + NT - 1) / NT;
    int64_t cap = (int64_t)ctx->sms * 16;
    return (int)std::max<int64_t>(1, std::min(b, cap));
}

// Device arrays carry CSR_PAD elements of slack: the bulk copies of the stream
// engine round their ranges out to 16-byte boundaries.
template <class T>
int dalloc(T **p, int64_t n) {
    return dmalloc((void **)p, sizeof(T) * (std::max<int64_t>(n, 1) + CSR_PAD));
}

}  // namespace

namespace sp {

size_t smem_P() { return std::max(tile_smem_bytes<1, double>(), (size_t)(NP_P * (NT / 32) * 8)); }
size_t smem_D() { return std::max(tile_smem_bytes<4, double>(), (size_t)(NP_D * (NT / 32) * 8)); }
size_t smem_T() { return tile_smem_bytes<2, double>(); }

// Everything a pass needs, by value.
SolverPtrs ptrs_of(sp_solver *s) {
    SolverPtrs p{};
    p.a_rp = s->A.rp;
    p.a_ci = s->A.ci;
    p.a_v = s->A.v;
    p.a_v32 = s->A.v32;
    p.a_tiles = s->A.tiles;
    p.a_sched = s->A.sched;
    p.t_sched = s->AT.sched;
    p.t_rp = s->AT.rp;
    p.t_ci = s->AT.ci;
    p.t_v = s->AT.v;
    p.t_v32 = s->AT.v32;
    p.t_tiles = s->AT.tiles;
    p.c = s->c;
    p.lc = s->lc;
    p.uc = s->uc;
    p.lv = s->lv;
    p.uv = s->uv;
    p.pf = s->pf;
    p.df = s->df;
    p.x = s->x;
    p.y = s->y;
    p.xt = s->xt;
    p.yt = s->yt;
    p.xbar = s->xbar;
    p.xa = s->xa;
    p.ya = s->ya;
    p.aty = s->aty;
    p.xbar32 = s->xbar32;
    p.y32 = s->y32;
    p.pk = s->pk;
    p.pky = s->pky;
    p.partP = s->partP;
    p.partD = s->partD;
    p.partT = s->partT;
    p.partP0 = s->partP0;
    p.partD0 = s->partD0;
    p.prm = s->d_prm;
    p.st = s->d_st;
    p.mixed = s->mixed;
    return p;
}

template <bool LO, int MODE>
PrimalPass<LO, MODE> mkP(const SolverPtrs &p, int i, int role) {
    PrimalPass<LO, MODE> o{};
    o.rp = p.t_rp;
    o.ci = p.t_ci;
    if constexpr (LO) o.vals = p.t_v32;
    else o.vals = p.t_v;
    o.tiles = p.t_tiles;
    o.sched = p.t_sched;
    o.s = p;
    o.i = i;
    o.role = role;
    return o;
}
template <bool LO, int MODE>
DualPass<LO, MODE> mkD(const SolverPtrs &p, int i, int role) {
    DualPass<LO, MODE> o{};
    o.rp = p.a_rp;
    o.ci = p.a_ci;
    if constexpr (LO && MODE == 0) o.vals = p.a_v32;
    else o.vals = p.a_v;
    o.tiles = p.a_tiles;
    o.sched = p.a_sched;
    o.s = p;
    o.i = i;
    o.role = role;
    return o;
}

// The stream engine kernels of one FUSED op: one CTA per SM. Variants differ in the
// gatherer warps (count, loads in flight per lane, register or cp.async gathers) and
// in the slot count; choose_engines() picks one per pass when a solver is created.
constexpr int ENGINE_SELL = 100;  // a pass on its SELL copy (sell.cuh)

enum StreamVariant : int {
    SV_LDG4 = 0,   // 4 register-gatherer warps, 8 loads in flight per lane
    SV_LDG4_DEEP,  // ... with as many slots as fit
    SV_LDG8B16,    // 8 warps, 16 loads in flight per lane
    SV_CP4,        // 4 cp.async gatherer warps
    SV_LDG8_DEEP,  // 8 warps, 8 loads in flight per lane, as many slots as fit
    SV_LDG6_DEEP,  // 6 warps, 8 loads, as many slots as fit
    SV_LDG4B16_DEEP,  // 4 warps, 16 loads, as many slots as fit
    SV_LDG4_PAIR,  // 4 warps, 8 loads, 2 slots, two CTAs per SM
    SV_LDG6_PAIR,  // 6 warps, 8 loads, 2 slots, two CTAs per SM
    SV_COUNT
};
constexpr const char *STREAM_VARIANT_NAMES[SV_COUNT] = {"ldg4", "ldg4deep", "ldg8b16", "cp4", "ldg8deep", "ldg6deep",
                                                        "ldg4b16deep", "ldg4pair", "ldg6pair"};

template <class Op>
struct StreamKernel {
    template <bool LDG, int DEEP>
    static constexpr size_t smem_of() { return StreamLayout<Op, !LDG, DEEP>::total; }
    static std::atomic<int> ready[64];
    template <int GW, bool LDG, int B, int DEEP>
    static int prepare_one() {
        constexpr size_t smem = smem_of<LDG, DEEP>();
        auto *f = k_stream<Op, GW, LDG, B, DEEP>;
        SP_CUDA_TRY(cudaFuncSetAttribute((const void *)f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int b = 0;
        SP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, f, stream_threads(GW), smem));
        if (b < 1) return fail(SP_ERR_CUDA, "stream engine kernel cannot be resident");
        return SP_OK;
    }
    // Runs before any graph capture: opts every variant in to its shared memory.
    static int prepare(int dev) {
        if (dev < 0 || dev >= 64) return fail(SP_ERR_INVALID, "device ordinal out of range");
        if (ready[dev].load()) return SP_OK;
        int rc;
        if ((rc = prepare_one<4, true, 8, SLOTS_FEW>()) || (rc = prepare_one<4, true, 8, SLOTS_DEEP>()) ||
            (rc = prepare_one<8, true, 16, SLOTS_FEW>()) || (rc = prepare_one<4, false, 1, SLOTS_FEW>()) ||
            (rc = prepare_one<8, true, 8, SLOTS_DEEP>()) || (rc = prepare_one<6, true, 8, SLOTS_DEEP>()) ||
            (rc = prepare_one<4, true, 16, SLOTS_DEEP>()) || (rc = prepare_one<4, true, 8, SLOTS_PAIR>()) ||
            (rc = prepare_one<6, true, 8, SLOTS_PAIR>()))
            return rc;
        ready[dev].store(1);
        return SP_OK;
    }
    template <int GW, bool LDG, int B, int DEEP>
    static void go(int grid, const DevCsr &M, cudaStream_t st, const Op &op, const StreamTrial &tr) {
        const int g = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)grid * stream_ctas_per_sm(DEEP), M.ntiles));
        k_stream<Op, GW, LDG, B, DEEP><<<g, stream_threads(GW), smem_of<LDG, DEEP>(), st>>>(M.ntiles, M.nlong, op, tr);
    }
    static void launch(const sp_solver *s, const DevCsr &M, cudaStream_t st, const Op &op, int variant) {
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(s->ctx->sms, M.ntiles));
        StreamTrial tr = s->trial;
        if (tr.withhold >= 0) tr.withhold += M.nlong;  // the knob counts the tiles after the long rows
        switch (variant) {
        case SV_LDG4: go<4, true, 8, SLOTS_FEW>(grid, M, st, op, tr); break;
        case SV_LDG4_DEEP: go<4, true, 8, SLOTS_DEEP>(grid, M, st, op, tr); break;
        case SV_LDG8B16: go<8, true, 16, SLOTS_FEW>(grid, M, st, op, tr); break;
        case SV_LDG8_DEEP: go<8, true, 8, SLOTS_DEEP>(grid, M, st, op, tr); break;
        case SV_LDG6_DEEP: go<6, true, 8, SLOTS_DEEP>(grid, M, st, op, tr); break;
        case SV_LDG4B16_DEEP: go<4, true, 16, SLOTS_DEEP>(grid, M, st, op, tr); break;
        case SV_LDG4_PAIR: go<4, true, 8, SLOTS_PAIR>(grid, M, st, op, tr); break;
        case SV_LDG6_PAIR: go<6, true, 8, SLOTS_PAIR>(grid, M, st, op, tr); break;
        default: go<4, false, 1, SLOTS_FEW>(grid, M, st, op, tr); break;
        }
    }
};
template <class Op>
std::atomic<int> StreamKernel<Op>::ready[64];

using StreamP64 = StreamKernel<PrimalPass<false, 0>>;
using StreamP32 = StreamKernel<PrimalPass<true, 0>>;
using StreamD64 = StreamKernel<DualPass<false, 0>>;
using StreamD32 = StreamKernel<DualPass<true, 0>>;

void free_sell(SellMat *S, cudaStream_t st);

// Passes over at least this many nonzeros run their SELL parts on two streams; smaller
// ones in one launch (on small LPs an iteration's time is mostly launch latency).
constexpr int64_t SELL_SPLIT_NNZ = 4 << 20;

// The SELL copy of one matrix (sell.cuh), built on the device from its CSR arrays after
// scaling: the rows' sort keys and a stable radix sort of them (each window's rows by
// decreasing length), the slice widths and slot offsets, the warp-row list and its chunk
// offsets, then the two copies. Left unbuilt (ok = false) for a matrix with a row longer
// than TILE_NNZ, or whose copy would hold more than SELL_MAX_SLOTS_PER_NNZ slots per nonzero.
int build_sell(sp_solver *s, const DevCsr &M, SellMat *S) {
    cudaStream_t st = s->ctx->stream;
    *S = SellMat{};
    if (M.nlong > 0 || M.nrows == 0) return SP_OK;
    const int64_t nrows = M.nrows, nwin = (nrows + SELL_WIN - 1) / SELL_WIN, npad = nwin * SELL_WIN;
    const int64_t nslices = npad / 32;
    S->nrows = nrows;
    S->nwin = nwin;
    S->nslices = nslices;
    int64_t *slots = nullptr, *cnt = nullptr;
    int *flag = nullptr, *nsel = nullptr;
    uint32_t *key = nullptr, *skey = nullptr;
    uint16_t *loc = nullptr;
    void *tmp = nullptr;
    auto release = [&] {
        for (void *p : {(void *)slots, (void *)cnt, (void *)flag, (void *)nsel, (void *)key, (void *)skey,
                        (void *)loc, tmp})
            dfree(p, st);
    };
    auto fail = [&](int rc) {
        release();
        free_sell(S, st);
        return rc;
    };
    int rc;
    if ((rc = dmalloc((void **)&S->len, npad)) || (rc = dmalloc((void **)&S->lsort, npad)) ||
        (rc = dmalloc((void **)&S->perm, sizeof(uint16_t) * npad)) ||
        (rc = dmalloc((void **)&S->slen, sizeof(int) * nslices)) ||
        (rc = dmalloc((void **)&S->off, sizeof(int64_t) * nslices)) ||
        (rc = dmalloc((void **)&slots, sizeof(int64_t) * nslices)) || (rc = dmalloc((void **)&flag, sizeof(int) * nrows)) ||
        (rc = dmalloc((void **)&key, sizeof(uint32_t) * npad)) || (rc = dmalloc((void **)&skey, sizeof(uint32_t) * npad)) ||
        (rc = dmalloc((void **)&loc, sizeof(uint16_t) * npad)) ||
        (rc = dmalloc((void **)&S->heavy, sizeof(int) * nrows)) || (rc = dmalloc((void **)&nsel, sizeof(int))))
        return fail(rc);
    const int g = grid_of(s->ctx, npad);
    k_sell_keys<<<g, NT, 0, st>>>(M.rp, nrows, npad, S->len, flag, key, loc);
    int end_bit = 6;  // the window number above the 6 bits of the length
    while (end_bit < 32 && ((uint64_t)(nwin - 1) >> (end_bit - 6))) ++end_bit;
    size_t b0 = 0, b1 = 0, b2 = 0;
    thrust::counting_iterator<int> rows(0);
    SP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, b0, key, skey, loc, S->perm, npad, 0, end_bit, st));
    SP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, b1, slots, S->off, nslices, st));
    SP_CUDA_TRY(cub::DeviceSelect::Flagged(nullptr, b2, rows, flag, S->heavy, nsel, (int)nrows, st));
    size_t btmp = std::max({b0, b1, b2});
    if ((rc = dmalloc(&tmp, btmp))) return fail(rc);
    SP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, b0, key, skey, loc, S->perm, npad, 0, end_bit, st));
    k_sell_slices<<<g, NT, 0, st>>>(skey, npad, S->lsort, S->slen, slots);
    SP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp, b1, slots, S->off, nslices, st));
    SP_CUDA_TRY(cub::DeviceSelect::Flagged(tmp, b2, rows, flag, S->heavy, nsel, (int)nrows, st));
    int64_t last[2];
    int nh = 0;
    SP_CUDA_TRY(cudaMemcpyAsync(&last[0], S->off + nslices - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    SP_CUDA_TRY(cudaMemcpyAsync(&last[1], slots + nslices - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    SP_CUDA_TRY(cudaMemcpyAsync(&nh, nsel, sizeof(int), cudaMemcpyDeviceToHost, st));
    SP_CUDA_TRY(cudaStreamSynchronize(st));
    S->slots = last[0] + last[1];
    S->nheavy = nh;
    // the warp rows' chunk offsets
    if ((rc = dmalloc((void **)&S->choff, sizeof(int64_t) * (nh + 1))) ||
        (rc = dmalloc((void **)&cnt, sizeof(int64_t) * (nh + 1))))
        return fail(rc);
    k_sell_chunk_counts<<<grid_of(s->ctx, (int64_t)nh + 1), NT, 0, st>>>(M.rp, S->heavy, nh, cnt);
    size_t b3 = 0;
    SP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, b3, cnt, S->choff, (int64_t)nh + 1, st));
    if (b3 > btmp) {
        dfree(tmp, st);
        tmp = nullptr;
        if ((rc = dmalloc(&tmp, b3))) return fail(rc);
    }
    SP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp, b3, cnt, S->choff, (int64_t)nh + 1, st));
    SP_CUDA_TRY(cudaMemcpyAsync(&S->chunks, S->choff + nh, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    SP_CUDA_TRY(cudaStreamSynchronize(st));
    S->nseg = (S->chunks + SELL_SEG_CHUNKS - 1) / SELL_SEG_CHUNKS;
    if ((rc = dmalloc((void **)&S->segrow, sizeof(int) * (S->nseg + 1)))) return fail(rc);
    k_sell_segments<<<grid_of(s->ctx, S->nseg + 1), NT, 0, st>>>(S->choff, nh, S->nseg, S->segrow);
    S->split = M.nnz >= SELL_SPLIT_NNZ;
    // rows too uneven for slices: more padding than the pass would save
    if (S->slots + 32 * S->chunks > SELL_MAX_SLOTS_PER_NNZ * std::max<int64_t>(M.nnz, 1024)) return fail(SP_OK);
    const int64_t hs = 32 * S->chunks;
    if ((rc = dmalloc((void **)&S->ci, sizeof(int) * std::max<int64_t>(S->slots, 1))) ||
        (rc = dmalloc((void **)&S->v, sizeof(double) * std::max<int64_t>(S->slots, 1))) ||
        (s->mixed && (rc = dmalloc((void **)&S->v32, sizeof(float) * std::max<int64_t>(S->slots, 1)))) ||
        (rc = dmalloc((void **)&S->hci, sizeof(int) * std::max<int64_t>(hs, 1))) ||
        (rc = dmalloc((void **)&S->hv, sizeof(double) * std::max<int64_t>(hs, 1))) ||
        (s->mixed && (rc = dmalloc((void **)&S->hv32, sizeof(float) * std::max<int64_t>(hs, 1)))))
        return fail(rc);
    k_sell_fill<<<g, NT, 0, st>>>(M.rp, M.ci, M.v, npad, S->lsort, S->perm, S->off, S->ci, S->v, S->v32);
    if (nh > 0)
        k_sell_chunk_fill<<<grid_of(s->ctx, 32 * (int64_t)nh), NT, 0, st>>>(M.rp, M.ci, M.v, S->heavy, nh, S->choff,
                                                                             S->hci, S->hv, S->hv32);
    SP_CUDA_TRY(cudaGetLastError());
    release();
    S->ok = true;
    return SP_OK;
}

void free_sell(SellMat *S, cudaStream_t st) {
    for (void *p : {(void *)S->ci, (void *)S->v, (void *)S->v32, (void *)S->off, (void *)S->slen, (void *)S->len,
                    (void *)S->lsort, (void *)S->perm, (void *)S->heavy, (void *)S->choff, (void *)S->segrow,
                    (void *)S->hci, (void *)S->hv, (void *)S->hv32})
        dfree(p, st);
    *S = SellMat{};
}

SellArgs sell_args(const SellMat &S) {
    return SellArgs{S.ci,     S.v,   S.v32, S.off,  S.slen,  S.len,  S.lsort,  S.perm, S.heavy,
                    S.choff,  S.segrow, S.hci, S.hv, S.hv32, S.nrows, S.nwin, S.nheavy, S.nseg};
}

// A check pass on the SELL copy: rows' contributions, then the tile partials from them
// (sell.cuh: k_sell_chk, k_sell_refold). The same bits as the tile engine's pass.
template <class Op>
void launch_sell_check(sp_solver *s, const SellMat &S, const DevCsr &M, cudaStream_t st, const Op &op) {
    const SellArgs a = sell_args(S);
    const unsigned g = (unsigned)((S.nseg + NT / 32 - 1) / (NT / 32) + S.nwin);
    k_sell_chk<Op, 2, 4><<<g, NT, 0, st>>>(op, a, s->contrib);
    k_sell_refold<Op><<<M.ntiles, NT, 0, st>>>(op, S.len, s->contrib, S.nrows);
}

// A SELL pass: on a large pass the warp rows on the solver's second stream, beside the
// windows on the pass's stream (they write disjoint rows), joined before the next pass; on a
// small one both in one launch. Kernel shapes from a sweep on the 40M LP (ms per pass, SELL
// path for both passes, 16-row segments): warp rows with 2 chunks per batch at 4 CTAs/SM in
// FP64 (primal pass 0.276; 4 chunks at 3 CTAs/SM 0.290, 4 or 8 at the registers' natural
// occupancy 0.288–0.293), 4 at 4 CTAs/SM in FP32 (0.255; 2 chunks 0.264); windows with 8
// slice entries in flight at 4 CTAs/SM in both (1,024-row windows: dual pass 0.193 FP64, 0.191 FP32; 4 entries
// 0.198, 8 at natural occupancy 0.207, 16 0.233). On the transport LP's 63-chunk rows, 4
// chunks per batch: dual pass 0.053 ms (2 chunks 0.060, 8 0.060).
template <class Op>
void launch_sell(sp_solver *s, const SellMat &S, cudaStream_t st, const Op &op) {
    const SellArgs a = sell_args(S);
    if (!S.split) {
        const unsigned g = (unsigned)((S.nseg + NT / 32 - 1) / (NT / 32) + S.nwin);
        if constexpr (sizeof(typename Op::VT) == 4) k_sell_both<Op, 4, 8, 1><<<g, NT, 0, st>>>(op, a);
        else k_sell_both<Op, 2, 8, 1><<<g, NT, 0, st>>>(op, a);
        return;
    }
    const bool rows = S.nseg > 0;
    if (rows) {
        cudaEventRecord(s->fork, st);
        cudaStreamWaitEvent(s->aux, s->fork, 0);
        const unsigned gr = (unsigned)((S.nseg + NT / 32 - 1) / (NT / 32));
        // rows of 16+ chunks on average (the transport LP's 63): 4 chunks per batch
        if (sizeof(typename Op::VT) == 4 || S.chunks >= 16 * S.nheavy) k_sell_rows<Op, 4, 4><<<gr, NT, 0, s->aux>>>(op, a);
        else k_sell_rows<Op, 2, 4><<<gr, NT, 0, s->aux>>>(op, a);
    }
    // FP32 values: 5 CTAs per SM (0.176 ms against 0.182 at 4, with 512-row windows)
    if constexpr (sizeof(typename Op::VT) == 4) k_sell_win<Op, 8, 5><<<(unsigned)S.nwin, NT, 0, st>>>(op, a);
    else k_sell_win<Op, 8, 4><<<(unsigned)S.nwin, NT, 0, st>>>(op, a);
    if (rows) {
        cudaEventRecord(s->join, s->aux);
        cudaStreamWaitEvent(st, s->join, 0);
    }
}

// Which engine runs each MID pass (-1: the tile engine, ENGINE_SELL the SELL path, else a
// stream-engine variant). The defaults are the fastest measured on the 40M power-law LP (ms
// per launch): the primal pass on the stream engine with 4 register-gatherer warps and 8
// loads in flight per lane, 4 slots in FP64 (0.255; 3 slots 0.265, 6 or 8 gatherer warps
// 0.266-0.285, 16 loads in flight 0.275-0.309, two CTAs per SM with 2 slots 0.269; tile
// engine 0.297, SELL 0.31) and two CTAs per SM with 2 slots in FP32 (0.242; one CTA with 4
// slots 0.246, deeper slots 0.32-0.39); the dual pass on its SELL copy in both precisions
// (0.185 FP64, 0.182 FP32 with 512-row windows; tile engine 0.238 and 0.249, stream engine
// 0.300 and 0.227).
// A problem under SMALL_NNZ nonzeros keeps both passes on the tile engine: there an
// iteration's time is launch latency and tile parallelism (32 LPs of the batch workload,
// one device solve each: 9.1 µs per iteration on tiles, 9.5 stream, 11.6 SELL).
// SP_PASS_ENGINE=tiles|stream|sell overrides all four (large: the assignment above for a
// problem of any size), SP_PRIMAL_ENGINE and SP_DUAL_ENGINE one pass; SP_STREAM_GATHER
// names the stream variant.
constexpr int64_t SMALL_NNZ = 1 << 20;

int choose_engines(sp_solver *s) {
    const char *eng = getenv("SP_PASS_ENGINE");
    // "large": the large-problem assignment whatever the size (tests of small LPs use it)
    const bool small = s->nnz < SMALL_NNZ && !(eng && !strcmp(eng, "large"));
    s->sv_p64 = small ? -1 : SV_LDG4_DEEP;
    s->sv_p32 = small ? -1 : SV_LDG4_PAIR;
    s->sv_d64 = small ? -1 : ENGINE_SELL;
    s->sv_d32 = small ? -1 : ENGINE_SELL;
    // test knob of the stream engine's stall path (stream.cuh: StreamTrial): the copies
    // of one tile are never issued and every wait gives up after 100 µs
    if (const char *w = getenv("SP_TEST_STREAM_WITHHOLD")) {
        s->trial.withhold = std::max(0, atoi(w));
        s->trial.wait_ns = 100000ull;
    }
    if (eng && !strcmp(eng, "tiles")) s->sv_p64 = s->sv_p32 = s->sv_d64 = s->sv_d32 = -1;
    if (eng && !strcmp(eng, "sell")) s->sv_p64 = s->sv_p32 = s->sv_d64 = s->sv_d32 = ENGINE_SELL;
    int sv = SV_LDG4;
    if (const char *gv = getenv("SP_STREAM_GATHER"))
        for (int k = 0; k < SV_COUNT; ++k)
            if (!strcmp(gv, STREAM_VARIANT_NAMES[k])) sv = k;
    if (eng && !strcmp(eng, "stream")) s->sv_p64 = s->sv_p32 = s->sv_d64 = s->sv_d32 = sv;
    // one pass's engine alone (measurements): SP_PRIMAL_ENGINE / SP_DUAL_ENGINE = tiles|stream|sell
    auto pick = [&](const char *name, int *v64, int *v32) {
        const char *e = getenv(name);
        if (!e) return;
        const int v = !strcmp(e, "tiles") ? -1 : !strcmp(e, "sell") ? ENGINE_SELL : !strcmp(e, "stream") ? sv : -2;
        if (v != -2) *v64 = *v32 = v;
    };
    pick("SP_PRIMAL_ENGINE", &s->sv_p64, &s->sv_p32);
    pick("SP_DUAL_ENGINE", &s->sv_d64, &s->sv_d32);
    const int dev = s->ctx->device;
    int rc;
    // the SELL copies, where a pass uses them (a matrix with a row longer than a tile
    // has none: its passes fall back to the tile engine)
    const bool sell_p = s->sv_p64 == ENGINE_SELL || (s->mixed && s->sv_p32 == ENGINE_SELL);
    const bool sell_d = s->sv_d64 == ENGINE_SELL || (s->mixed && s->sv_d32 == ENGINE_SELL);
    if (sell_p && (rc = build_sell(s, s->AT, &s->sellAT))) return rc;
    if (sell_d && (rc = build_sell(s, s->A, &s->sellA))) return rc;
    for (int *v : {&s->sv_p64, &s->sv_p32})
        if (*v == ENGINE_SELL && !s->sellAT.ok) *v = -1;
    for (int *v : {&s->sv_d64, &s->sv_d32})
        if (*v == ENGINE_SELL && !s->sellA.ok) *v = -1;
    // the check's dual pass on the SELL copy too, where the iteration's dual pass uses it
    if (s->sellA.ok && s->sv_d64 == ENGINE_SELL && !s->contrib &&
        (rc = dmalloc((void **)&s->contrib, sizeof(double) * NP_D * std::max<int64_t>(s->A.nrows, 1))))
        return rc;
    if (((s->sellA.ok && s->sellA.split) || (s->sellAT.ok && s->sellAT.split)) && !s->aux) {
        SP_CUDA_TRY(cudaStreamCreateWithFlags(&s->aux, cudaStreamNonBlocking));
        SP_CUDA_TRY(cudaEventCreateWithFlags(&s->fork, cudaEventDisableTiming));
        SP_CUDA_TRY(cudaEventCreateWithFlags(&s->join, cudaEventDisableTiming));
    }
    auto stream = [](int v) { return v >= 0 && v < SV_COUNT; };
    if (stream(s->sv_p64) && (rc = StreamP64::prepare(dev))) return rc;
    if (stream(s->sv_d64) && (rc = StreamD64::prepare(dev))) return rc;
    if (s->mixed && stream(s->sv_p32) && (rc = StreamP32::prepare(dev))) return rc;
    if (s->mixed && stream(s->sv_d32) && (rc = StreamD32::prepare(dev))) return rc;
    return SP_OK;
}

// Launches the primal pass of iteration i with the given role. MID iterations go
// through the stream engine when it is on (in the mixed form one launch per
// precision; the one that does not match the device state returns at once).
void launch_P(sp_solver *s, int i, int role, cudaStream_t st) {
    const SolverPtrs p = ptrs_of(s);
    const int g = s->AT.ntiles;
    if (g == 0) return;
    const size_t sm = smem_P();
    // MID passes, and the FUSED variant of an epoch's first pass (it returns at once when the
    // epoch opens at k = 0), on the pass's engine; the first pass's k = 0 variant on tiles
    if ((role == ROLE_MID || role == ROLE_FIRST) && (s->sv_p64 >= 0 || (s->mixed && s->sv_p32 >= 0))) {
        if (s->mixed) {
            if (s->sv_p32 == ENGINE_SELL) launch_sell(s, s->sellAT, st, mkP<true, 0>(p, i, role));
            else if (s->sv_p32 >= 0) StreamP32::launch(s, s->AT, st, mkP<true, 0>(p, i, role), s->sv_p32);
            else launch_tiles(s->ctx->sms, s->ctx->d_tiles, g, sm, st, mkP<true, 0>(p, i, role));
        }
        if (s->sv_p64 == ENGINE_SELL) launch_sell(s, s->sellAT, st, mkP<false, 0>(p, i, role));
        else if (s->sv_p64 >= 0) StreamP64::launch(s, s->AT, st, mkP<false, 0>(p, i, role), s->sv_p64);
        else launch_tiles(s->ctx->sms, s->ctx->d_tiles, g, sm, st, mkP<false, 0>(p, i, role));
        if (role == ROLE_FIRST) {
            if (s->mixed) launch_tiles(s->ctx->sms, s->ctx->d_tiles, g, sm, st, mkP<true, 1>(p, i, role), mkP<false, 1>(p, i, role));
            else launch_tiles(s->ctx->sms, s->ctx->d_tiles, g, sm, st, mkP<false, 1>(p, i, role));
        }
        return;
    }
    if (s->mixed) {
        if (role == ROLE_MID)
            launch_tiles(s->ctx->sms, s->ctx->d_tiles, g, sm, st, mkP<true, 0>(p, i, role), mkP<false, 0>(p, i, role));
        else if (role == ROLE_FIRST) {
            // FUSED and K0 as launches of their own (one of them returns at once), so
            // the FUSED one keeps its own register and shared-memory footprint
            launch_tiles(s->ctx->sms, s->ctx->d_tiles, g, sm, st, mkP<true, 0>(p, i, role), mkP<false, 0>(p, i, role));
            launch_tiles(s->ctx->sms, s->ctx->d_tiles, g, sm, st, mkP<true, 1>(p, i, role), mkP<false, 1>(p, i, role));
        }
        else
            launch_tiles(s->ctx->sms, s->ctx->d_tiles, g, sm, st, mkP<true, 2>(p, i, role), mkP<false, 2>(p, i, role));
    } else {
        if (role == ROLE_MID) launch_tiles(s->ctx->sms, s->ctx->d_tiles, g, sm, st, mkP<false, 0>(p, i, role));
        else if (role == ROLE_FIRST) {
            launch_tiles(s->ctx->sms, s->ctx->d_tiles, g, sm, st, mkP<false, 0>(p, i, role));
            launch_tiles(s->ctx->sms, s->ctx->d_tiles, g, sm, st, mkP<false, 1>(p, i, role));
        }
        else launch_tiles(s->ctx->sms, s->ctx->d_tiles, g, sm, st, mkP<false, 2>(p, i, role));
    }
}

void launch_D(sp_solver *s, int i, int role, cudaStream_t st) {
    const SolverPtrs p = ptrs_of(s);
    const int g = s->A.ntiles;
    if (g == 0) return;
    const size_t sm = smem_D();
    if (role == ROLE_CHECK && s->contrib) {
        if (s->mixed) launch_sell_check(s, s->sellA, s->A, st, mkD<true, 2>(p, i, role));
        launch_sell_check(s, s->sellA, s->A, st, mkD<false, 2>(p, i, role));
        return;
    }
    if ((role == ROLE_MID || role == ROLE_FIRST) && (s->sv_d64 >= 0 || (s->mixed && s->sv_d32 >= 0))) {
        const size_t s1 = tile_smem_bytes<1, double>();
        if (s->mixed) {
            if (s->sv_d32 == ENGINE_SELL) launch_sell(s, s->sellA, st, mkD<true, 0>(p, i, role));
            else if (s->sv_d32 >= 0) StreamD32::launch(s, s->A, st, mkD<true, 0>(p, i, role), s->sv_d32);
            else launch_tiles(s->ctx->sms, s->ctx->d_tiles, g, s1, st, mkD<true, 0>(p, i, role));
        }
        if (s->sv_d64 == ENGINE_SELL) launch_sell(s, s->sellA, st, mkD<false, 0>(p, i, role));
        else if (s->sv_d64 >= 0) StreamD64::launch(s, s->A, st, mkD<false, 0>(p, i, role), s->sv_d64);
        else launch_tiles(s->ctx->sms, s->ctx->d_tiles, g, s1, st, mkD<false, 0>(p, i, role));
        if (role == ROLE_FIRST) {
            // the k = 0 variant: two products and two partial sums per row
            if (s->contrib) {
                if (s->mixed) launch_sell_check(s, s->sellA, s->A, st, mkD<true, 1>(p, i, role));
                launch_sell_check(s, s->sellA, s->A, st, mkD<false, 1>(p, i, role));
            } else if (s->mixed) {
                launch_tiles(s->ctx->sms, s->ctx->d_tiles, g, tile_smem_bytes<2, double>(), st, mkD<true, 1>(p, i, role),
                             mkD<false, 1>(p, i, role));
            } else {
                launch_tiles(s->ctx->sms, s->ctx->d_tiles, g, tile_smem_bytes<2, double>(), st, mkD<false, 1>(p, i, role));
            }
        }
        return;
    }
    if (s->mixed) {
        if (role == ROLE_MID)
            launch_tiles(s->ctx->sms, s->ctx->d_tiles, g, tile_smem_bytes<1, double>(), st, mkD<true, 0>(p, i, role), mkD<false, 0>(p, i, role));
        else if (role == ROLE_FIRST) {
            launch_tiles(s->ctx->sms, s->ctx->d_tiles, g, tile_smem_bytes<1, double>(), st, mkD<true, 0>(p, i, role), mkD<false, 0>(p, i, role));
            launch_tiles(s->ctx->sms, s->ctx->d_tiles, g, tile_smem_bytes<2, double>(), st, mkD<true, 1>(p, i, role), mkD<false, 1>(p, i, role));
        }
        else
            launch_tiles(s->ctx->sms, s->ctx->d_tiles, g, sm, st, mkD<true, 2>(p, i, role), mkD<false, 2>(p, i, role));
    } else {
        if (role == ROLE_MID)
            launch_tiles(s->ctx->sms, s->ctx->d_tiles, g, tile_smem_bytes<1, double>(), st, mkD<false, 0>(p, i, role));
        else if (role == ROLE_FIRST) {
            launch_tiles(s->ctx->sms, s->ctx->d_tiles, g, tile_smem_bytes<1, double>(), st, mkD<false, 0>(p, i, role));
            launch_tiles(s->ctx->sms, s->ctx->d_tiles, g, tile_smem_bytes<2, double>(), st, mkD<false, 1>(p, i, role));
        }
        else launch_tiles(s->ctx->sms, s->ctx->d_tiles, g, sm, st, mkD<false, 2>(p, i, role));
    }
}

void launch_T(sp_solver *s, int i, cudaStream_t st) {
    const SolverPtrs p = ptrs_of(s);
    if (s->AT.ntiles == 0) return;
    CheckPassT o{};
    o.rp = p.t_rp;
    o.ci = p.t_ci;
    o.vals = p.t_v;
    o.tiles = p.t_tiles;
    o.sched = p.t_sched;
    o.s = p;
    o.i = i;
    launch_tiles(s->ctx->sms, s->ctx->d_tiles, s->AT.ntiles, smem_T(), st, o);
}

// One epoch of E iterations (the last is the check) on stream `st`. With timing
// on, CUDA events bracket the P and D launches of sampled MID iterations.
void enqueue_epoch(sp_solver *s, int E, cudaStream_t st, bool timed) {
    const SolverPtrs p = ptrs_of(s);
    const int gn = grid_of(s->ctx, std::max(s->n, s->m));
    for (int i = 0; i < E; ++i) {
        const bool last = i == E - 1;
        const int role = last ? ROLE_CHECK : (i == 0 ? ROLE_FIRST : ROLE_MID);
        bool sample = timed && role == ROLE_MID && s->timing_every > 0 && (s->timing_counter++ % s->timing_every == 0);
        cudaEvent_t e0 = nullptr, e1 = nullptr, e2 = nullptr;
        if (sample) {
            e0 = s->event();
            e1 = s->event();
            e2 = s->event();
            sample = e0 && e1 && e2;  // no sample where the pool could not grow
        }
        if (sample) cudaEventRecord(e0, st);
        launch_P(s, i, role, st);
        if (sample) cudaEventRecord(e1, st);
        launch_D(s, i, role, st);
        if (sample) {
            cudaEventRecord(e2, st);
            s->samples.push_back({e0, e1, e2});
        }
        if (role == ROLE_FIRST) k_halpern_x0<<<gn, NT, 0, st>>>(p, s->n);
        if (last) {
            launch_T(s, i, st);
            CtrlArgs a{s->partP, s->partD, s->partT, s->partP0, s->partD0, s->AT.ntiles, s->A.ntiles, E, s->d_trace,
                       (long long)s->trace_cap};
            k_controller<<<1, NT, 0, st>>>(a, s->d_prm, s->d_st);
            k_finish<<<gn, NT, 0, st>>>(p, s->n, s->m);
        }
    }
}

int set_smem_limits() {
    static bool done = false;
    if (done) return SP_OK;
    // Opt in to more than 48 KB of dynamic shared memory for the 4-product check pass.
    auto set = [](const void *f, size_t bytes) {
        return cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    };
    using DL0 = DualPass<true, 2>;
    using DH0 = DualPass<false, 2>;
    SP_CUDA_TRY(set((const void *)k_tiles_any<DL0, DH0>, smem_D()));
    SP_CUDA_TRY(set((const void *)k_tiles_any<DH0>, smem_D()));
    done = true;
    return SP_OK;
}

int build_graph(sp_solver *s, int E, cudaGraphExec_t *out) {
    cudaStream_t st = s->ctx->stream;
    cudaGraph_t g;
    SP_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    enqueue_epoch(s, E, st, false);
    SP_CUDA_TRY(cudaStreamEndCapture(st, &g));
    // the epoch's kernel launches, for the callers that count them
    size_t nodes = 0;
    int64_t kernels = 0;
    if (cudaGraphGetNodes(g, nullptr, &nodes) == cudaSuccess && nodes > 0) {
        std::vector<cudaGraphNode_t> all(nodes);
        if (cudaGraphGetNodes(g, all.data(), &nodes) == cudaSuccess)
            for (size_t k = 0; k < nodes; ++k) {
                cudaGraphNodeType t;
                if (cudaGraphNodeGetType(all[k], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++kernels;
            }
    }
    s->graph_kernels[E] = kernels;
    cudaError_t e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(SP_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    return SP_OK;
}

}  // namespace sp

// ------------------------------------------------------------------ creation

namespace sp {

void solver_release(sp_solver *s) {
    if (!s) return;
    cudaSetDevice(s->ctx->device);
    cudaStreamSynchronize(s->ctx->stream);
    for (auto &kv : s->graphs) cudaGraphExecDestroy(kv.second);
    for (cudaEvent_t e : s->event_pool) cudaEventDestroy(e);
    if (s->aux) {
        cudaStreamSynchronize(s->aux);
        cudaStreamDestroy(s->aux);
        cudaEventDestroy(s->fork);
        cudaEventDestroy(s->join);
    }
    cudaStream_t fst = s->ctx->stream;
    free_csr(&s->A, fst);
    free_csr(&s->AT, fst);
    free_sell(&s->sellA, fst);
    free_sell(&s->sellAT, fst);
    void *bufs[] = {s->c, s->lc, s->uc, s->lv, s->uv, s->pf, s->df, s->x, s->y, s->xt, s->yt, s->xbar, s->xa, s->ya,
                    s->aty, s->xbar32, s->y32, s->pk, s->pky, s->partP, s->partD, s->partT, s->partP0, s->partD0, s->pv, s->ptmp,
                    s->contrib,
                    s->ppart, s->row_scale, s->col_scale, s->scales, s->d_prm, s->d_st, s->d_trace, s->norms,
                    s->out_x, s->out_y};
    for (void *b : bufs) dfree(b, fst);
    cudaStreamSynchronize(fst);
    cudaFreeHost(s->h_st);
    delete s;
}

// Scaling passes on the device (ScaledProblem::new, scaling.rs:53-103). A' and
// A'ᵀ are kept in step: each pass multiplies both by the same r_i * c_j products.
// The norms of the bounds and costs (k_seq_norms, sequential sums: tens of ms on a
// large problem) and the rescaling that depends on them run on the context's second
// stream, beside the power iteration, which needs only the scaled matrix. SideNorms
// holds that work until join(): the host waits for the second stream, and the main
// stream then releases the original vectors the side work read.
struct SideNorms {
    sp_solver *s = nullptr;
    double *keep[3] = {};
    void arm(sp_solver *solver, double *a, double *b, double *c) {
        s = solver;
        keep[0] = a;
        keep[1] = b;
        keep[2] = c;
    }
    cudaError_t join() {
        if (!s) return cudaSuccess;
        const cudaError_t e = cudaStreamSynchronize(s->ctx->aux);
        for (double *&b : keep) {
            dfree(b, s->ctx->stream);
            b = nullptr;
        }
        s = nullptr;
        return e;
    }
    ~SideNorms() { join(); }
};

// Calls f(std::integral_constant<int, G>) for the group size g (2, 4, 8, 16 or 32).
template <class F>
void with_group(int g, F &&f) {
    switch (g) {
    case 2: f(std::integral_constant<int, 2>{}); break;
    case 4: f(std::integral_constant<int, 4>{}); break;
    case 8: f(std::integral_constant<int, 8>{}); break;
    case 16: f(std::integral_constant<int, 16>{}); break;
    default: f(std::integral_constant<int, 32>{}); break;
    }
}

template <int G>
void launch_sweep(const DevCsr &M, bool geo2, int next, int grid, cudaStream_t st, const double *own,
                  const double *gat, double *scale, double *nxt) {
#define SP_SWEEP(GEO, NX) k_scale_sweep<G, GEO, NX><<<grid, NT, 0, st>>>(M.rp, M.ci, M.v, M.nrows, own, gat, scale, nxt)
    if (geo2) {
        if (next == NEXT_GEO) SP_SWEEP(true, NEXT_GEO);
        else if (next == NEXT_MAX) SP_SWEEP(true, NEXT_MAX);
        else SP_SWEEP(true, NEXT_NONE);
    } else {
        if (next == NEXT_MAX) SP_SWEEP(false, NEXT_MAX);
        else SP_SWEEP(false, NEXT_NONE);
    }
#undef SP_SWEEP
}

int scale_on_device(sp_solver *s, const sp_lp *lp, const std::vector<int> &rp_t, SideNorms *side) {
    sp_ctx *ctx = s->ctx;
    cudaStream_t st = ctx->stream;
    const int64_t m = s->m, n = s->n, nnz = s->nnz;
    const sp_solver_params &P = s->prm;
    double *rb[2] = {}, *cb[2] = {};  // factors of the rows of A' and of its columns (two of each)
    int rc;
    // The original bounds and objective come in through the output slots of the scaled
    // ones. They are copied first: a copy from pageable memory waits for the work queued
    // before it on the stream, and the sweeps below are meant to run while the host
    // goes on (plan_transpose).
    double *oc = nullptr, *olc = nullptr, *ouc = nullptr, *olv = nullptr, *ouv = nullptr;
    if ((rc = upload_vec(ctx, &oc, lp->c, n)) || (rc = upload_vec(ctx, &olc, lp->lc, m)) ||
        (rc = upload_vec(ctx, &ouc, lp->uc, m)) || (rc = upload_vec(ctx, &olv, lp->lv, n)) ||
        (rc = upload_vec(ctx, &ouv, lp->uv, n))) {
        for (double *b : {oc, olc, ouc, olv, ouv}) dfree(b, st);
        return rc;
    }
    auto release = [&]() {
        for (double *b : {rb[0], rb[1], cb[0], cb[1]}) dfree(b, st);
    };
    if ((rc = dalloc(&rb[0], m)) || (rc = dalloc(&rb[1], m)) || (rc = dalloc(&cb[0], n)) || (rc = dalloc(&cb[1], n))) {
        release();
        for (double *b : {oc, olc, ouc, olv, ouv}) dfree(b, st);
        return rc;
    }
    const int gm = grid_of(ctx, m), gn = grid_of(ctx, n);
    // lanes per row of the row sweeps: the smallest power of two g >= 2 with 2.5·g at
    // least the median row length (of 4096 rows spread over the layout), at most 32; the
    // rows longer than SWEEP_TRIPS·g go to whole warps (on the 40M LP: g = 8 for A', whose
    // rows hold 20 entries on average, and 2 for A'ᵀ, whose median row holds 3)
    auto group_of = [](auto row_len, int64_t rows) {
        if (rows <= 0) return 2;
        const int64_t samples = std::min<int64_t>(rows, 4096);
        std::vector<int64_t> len(samples);
        for (int64_t q = 0; q < samples; ++q) len[q] = row_len(q * rows / samples);
        std::nth_element(len.begin(), len.begin() + samples / 2, len.end());
        const int64_t med = len[samples / 2];
        int g = 2;
        while (g < 32 && 5 * g < 2 * med) g *= 2;
        return g;
    };
    const int64_t *arp = lp->a.row_ptr;
    const int Gm = group_of([&](int64_t i) { return arp[i + 1] - arp[i]; }, m);
    const int Gn = group_of([&](int64_t j) { return (int64_t)rp_t[j + 1] - rp_t[j]; }, n);
    const int wm = grid_of(ctx, m * Gm), wn = grid_of(ctx, n * Gn);
    k_fill<<<gm, NT, 0, st>>>(s->row_scale, 1.0, m);
    k_fill<<<gn, NT, 0, st>>>(s->col_scale, 1.0, n);
    // sweep over A' (rows i) or A'ᵀ (rows j): own = the layout's row factors, gat = the others
    auto sweep = [&](bool a_side, bool geo2, int next, const double *own, const double *gat, double *nxt) {
        const DevCsr &M = a_side ? s->A : s->AT;
        double *scale = a_side ? s->row_scale : s->col_scale;
        with_group(a_side ? Gm : Gn, [&](auto G) {
            launch_sweep<decltype(G)::value>(M, geo2, next, a_side ? wm : wn, st, own, gat, scale, nxt);
        });
    };
    const uint64_t GP = P.geometric_mean_passes, RZ = P.ruiz_iterations;
    if (nnz > 0) {  // with no entries every factor is 1 (inv_sqrt of 0) and the scales stay 1
        int ri = 0, cc = 0;  // which of rb / cb holds the current factors
        if (GP > 0) {
            // geometric-mean passes (scaling.rs:60-66): the first row factors from A' as
            // given, each later one from the sweep that finished the pass before
            with_group(Gm, [&](auto G) {
                k_row_geo<decltype(G)::value><<<wm, NT, 0, st>>>(s->A.rp, s->A.v, m, rb[0]);
            });
            for (uint64_t p = 0; p < GP; ++p) {
                const bool last = p + 1 == GP;
                const int next_t = last && RZ > 0 ? NEXT_MAX : NEXT_NONE;
                with_group(Gn, [&](auto G) {
                    constexpr int g = decltype(G)::value;
                    if (next_t == NEXT_MAX)
                        k_scale_geo_cols<g, NEXT_MAX><<<wn, NT, 0, st>>>(s->AT.rp, s->AT.ci, s->AT.v, n, rb[ri], cb[0],
                                                                         s->col_scale, cb[1]);
                    else
                        k_scale_geo_cols<g, NEXT_NONE><<<wn, NT, 0, st>>>(s->AT.rp, s->AT.ci, s->AT.v, n, rb[ri], cb[0],
                                                                          s->col_scale, nullptr);
                });
                sweep(true, true, !last ? NEXT_GEO : (RZ > 0 ? NEXT_MAX : NEXT_NONE), rb[ri], cb[0], rb[ri ^ 1]);
                ri ^= 1;
            }
            cc = 1;  // the first Ruiz column factors (written by the last pass's A'ᵀ sweep)
        } else if (RZ > 0) {
            with_group(Gm, [&](auto G) {
                k_row_ruiz<decltype(G)::value><<<wm, NT, 0, st>>>(s->A.rp, s->A.v, m, rb[0]);
            });
            with_group(Gn, [&](auto G) {
                k_row_ruiz<decltype(G)::value><<<wn, NT, 0, st>>>(s->AT.rp, s->AT.v, n, cb[0]);
            });
        }
        // Ruiz iterations (scaling.rs:67-72): both factors from the same matrix, so each
        // sweep reads the current pair and writes the next into the other buffer
        for (uint64_t q = 0; q < RZ; ++q) {
            const int next = q + 1 < RZ ? NEXT_MAX : NEXT_NONE;
            sweep(true, false, next, rb[ri], cb[cc], rb[ri ^ 1]);
            sweep(false, false, next, cb[cc], rb[ri], cb[cc ^ 1]);
            ri ^= 1;
            cc ^= 1;
        }
        if (P.pock_chambolle_enabled) {  // scaling.rs:73-79: sums in index order, one row per thread
            k_row_pc<<<gm, NT, 0, st>>>(s->A.rp, s->A.v, m, P.pock_chambolle_alpha, rb[0]);
            k_row_pc<<<gn, NT, 0, st>>>(s->AT.rp, s->AT.v, n, 2.0 - P.pock_chambolle_alpha, cb[0]);
            sweep(true, false, NEXT_NONE, rb[0], cb[0], nullptr);
            sweep(false, false, NEXT_NONE, cb[0], rb[0], nullptr);
        }
    }
    release();
    k_scale_vectors<<<std::max(gm, gn), NT, 0, st>>>(oc, olc, ouc, olv, ouv, s->row_scale, s->col_scale, s->c, s->lc,
                                                     s->uc, s->lv, s->uv, m, n);
    dfree(olv, st);
    dfree(ouv, st);
    SP_CUDA_TRY(cudaGetLastError());
    // the norms (of the original problem too, solver.rs:317-318), the rescaling and the
    // residual factors, on the second stream
    SP_CUDA_TRY(cudaEventRecord(ctx->aux_ev, st));
    SP_CUDA_TRY(cudaStreamWaitEvent(ctx->aux, ctx->aux_ev, 0));
    side->arm(s, oc, olc, ouc);
    cudaStream_t ax = ctx->aux;
    // Each norm's block asks for all the shared memory a CTA may have, so that no other
    // CTA shares its SM: beside the power iteration's CTAs the chain of additions ran 2-3
    // times slower (4M terms: 22 ms alone, 45-60 ms beside a gather-bound kernel).
    int optin = 0;
    SP_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device));
    cudaFuncAttributes fa{};
    SP_CUDA_TRY(cudaFuncGetAttributes(&fa, (const void *)k_seq_norms));
    const int pad = std::max(0, optin - (int)fa.sharedSizeBytes);
    SP_CUDA_TRY(cudaFuncSetAttribute((const void *)k_seq_norms, cudaFuncAttributeMaxDynamicSharedMemorySize, pad));
    k_seq_norms<<<4, NT, pad, ax>>>(olc, ouc, oc, s->lc, s->uc, s->c, m, n, s->norms);
    k_rescale<<<std::max(gm, gn), NT, 0, ax>>>(s->lc, s->uc, s->lv, s->uv, s->c, s->norms, m, n,
                                               P.bound_objective_rescaling, s->scales);
    k_factors<<<std::max(gm, gn), NT, 0, ax>>>(s->row_scale, s->col_scale, s->scales, s->pf, s->df, m, n);
    SP_CUDA_TRY(cudaGetLastError());
    return SP_OK;
}

// A'ᵀ on the device: a stable radix sort of the column indices (cub) gives, per
// column, its entries in increasing row order: CsrMatrix::transpose's order
// (problem.rs:88-109), bit for bit.
int transpose_on_device(sp_solver *s, std::vector<int> &rp32) {
    sp_ctx *ctx = s->ctx;
    cudaStream_t st = ctx->stream;
    const int64_t m = s->m, n = s->n, nnz = s->nnz;
    DevCsr &T = s->AT;
    T.nrows = n;
    T.ncols = m;
    T.nnz = nnz;
    int rc;
    if ((rc = dalloc(&T.rp, n + 1)) || (rc = dalloc(&T.ci, nnz)) || (rc = dalloc(&T.v, nnz))) return rc;
    int *row_of, *keys_out, *perm_in, *perm_out;
    if ((rc = dalloc(&row_of, nnz)) || (rc = dalloc(&keys_out, nnz)) || (rc = dalloc(&perm_in, nnz)) ||
        (rc = dalloc(&perm_out, nnz)))
        return rc;
    k_row_ids<<<grid_of(ctx, m * 32), NT, 0, st>>>(s->A.rp, m, row_of);
    k_iota<<<grid_of(ctx, nnz), NT, 0, st>>>(perm_in, nnz);
    int bits = 1;
    while ((int64_t(1) << bits) < n) ++bits;
    size_t temp = 0;
    SP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, temp, s->A.ci, keys_out, perm_in, perm_out, (int)nnz, 0, bits,
                                                st));
    void *tmp = nullptr;
    if ((rc = dmalloc(&tmp, std::max<size_t>(temp, 1)))) return rc;
    SP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, temp, s->A.ci, keys_out, perm_in, perm_out, (int)nnz, 0, bits, st));
    k_rowptr_from_sorted<<<grid_of(ctx, n + 1), NT, 0, st>>>(keys_out, nnz, n, T.rp);
    k_gather_transpose<<<grid_of(ctx, nnz), NT, 0, st>>>(perm_out, row_of, s->A.v, T.ci, T.v, nnz);
    SP_CUDA_TRY(cudaGetLastError());
    SP_CUDA_TRY(cudaStreamSynchronize(st));
    for (void *b : {(void *)row_of, (void *)keys_out, (void *)perm_in, (void *)perm_out, tmp}) dfree(b, st);
    // the row pointers for the host's tile plan (plan_transpose), which the scaling
    // sweeps do not need: the host builds it while they run
    rp32.resize(n + 1);
    SP_CUDA_TRY(cudaMemcpyAsync(rp32.data(), T.rp, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost, st));
    SP_CUDA_TRY(cudaStreamSynchronize(st));
    return SP_OK;
}

// The tile plan and row schedule of A'ᵀ, from its row pointers, built on the host and
// uploaded (the SpMV engines and the power iteration need them). Both are built before
// the first copy: a copy from pageable memory waits for the work queued before it on
// the stream (the scaling sweeps), and the host work is meant to run beside that.
int plan_transpose(sp_solver *s, const std::vector<int> &rp32) {
    cudaStream_t st = s->ctx->stream;
    const int64_t n = s->n;
    DevCsr &T = s->AT;
    std::vector<int64_t> rp64(rp32.begin(), rp32.end());
    std::vector<Tile> tiles = build_tiles(rp64.data(), n);
    T.ntiles = (int)tiles.size();
    T.nlong = count_long_tiles(tiles);
    const std::vector<uint16_t> sched = build_schedule(rp64.data(), n, tiles);
    int rc;
    // Memory from the stream-ordered pool is ours only in the order of `st` (the pool may hand
    // out memory whose previous owner, on another stream, is still running, with a wait
    // for it inserted into `st`): every copy into it goes through `st`, never through the
    // legacy stream of a synchronous cudaMemcpy.
    if ((rc = dmalloc((void **)&T.tiles, sizeof(Tile) * std::max<size_t>(tiles.size(), 1)))) return rc;
    if ((rc = dalloc(&T.sched, n))) return rc;
    if (!tiles.empty())
        SP_CUDA_TRY(cudaMemcpyAsync(T.tiles, tiles.data(), sizeof(Tile) * tiles.size(), cudaMemcpyHostToDevice, st));
    if (n) SP_CUDA_TRY(cudaMemcpyAsync(T.sched, sched.data(), sizeof(uint16_t) * n, cudaMemcpyHostToDevice, st));
    SP_CUDA_TRY(cudaStreamSynchronize(st));  // the host vectors end here
    return SP_OK;
}

// The first index in [0, len) at which bad(i) returns a nonzero code, with that code (-1, 0
// when there is none): up to 16 host threads scan contiguous ranges, and the lowest range
// with a failure holds the first one, so the answer is the sequential scan's.
template <class F>
std::pair<int64_t, int> first_bad(int64_t len, const F &bad) {
    const int workers = (int)std::max<int64_t>(1, std::min<int64_t>(16, len >> 18));
    std::vector<std::pair<int64_t, int>> found(workers, {-1, 0});
    auto scan = [&](int w) {
        for (int64_t k = len * w / workers, k1 = len * (w + 1) / workers; k < k1; ++k)
            if (const int c = bad(k)) {
                found[w] = {k, c};
                return;
            }
    };
    if (workers == 1) {
        scan(0);
    } else {
        std::vector<std::thread> th;
        for (int w = 0; w < workers; ++w) th.emplace_back(scan, w);
        for (auto &t : th) t.join();
    }
    for (const auto &f : found)
        if (f.first >= 0) return f;
    return {-1, 0};
}

// A double as Rust's `{}` prints it: the shortest digits that read back to the same value,
// written out without an exponent ("2", "0.1", "1500", "-0", "inf", "NaN").
std::string rust_display(double v) {
    if (std::isnan(v)) return "NaN";
    if (std::isinf(v)) return v > 0 ? "inf" : "-inf";
    if (v == 0.0) return std::signbit(v) ? "-0" : "0";
    char buf[64];
    for (int p = 0; p <= 17; ++p) {
        snprintf(buf, sizeof buf, "%.*e", p, v);
        if (strtod(buf, nullptr) == v) break;
    }
    // buf = [-]d[.ddd]e±XX
    std::string m(buf), digits;
    const bool neg = m[0] == '-';
    const size_t e = m.find('e');
    for (size_t k = neg ? 1 : 0; k < e; ++k)
        if (m[k] != '.') digits += m[k];
    const int exp10 = atoi(m.c_str() + e + 1);
    std::string out = neg ? "-" : "";
    if (exp10 >= 0) {
        if ((int)digits.size() <= exp10 + 1) {
            out += digits + std::string(exp10 + 1 - digits.size(), '0');
        } else {
            out += digits.substr(0, exp10 + 1) + "." + digits.substr(exp10 + 1);
        }
    } else {
        out += "0." + std::string(-exp10 - 1, '0') + digits;
    }
    return out;
}

// Calls body(w, k0, k1) for up to 16 contiguous ranges [k0, k1) of [0, len), each on a host
// thread of its own when there is more than one.
template <class F>
void split_ranges(int64_t len, const F &body) {
    const int workers = (int)std::max<int64_t>(1, std::min<int64_t>(16, len >> 18));
    if (workers == 1) {
        body(0, 0, len);
        return;
    }
    std::vector<std::thread> th;
    for (int w = 0; w < workers; ++w) th.emplace_back(body, w, len * w / workers, len * (w + 1) / workers);
    for (auto &t : th) t.join();
}

// LpProblem::validate (problem.rs:166-194), its checks in its order and with its messages
// (SP_ERR_PROBLEM): the variables' bounds (NaN, then crossed) over all columns, then the
// constraints', then NaN among the coefficients c and then A's values (numbered after c).
// Then the matrix's structure, which a C caller can break although the reference's
// CsrMatrix keeps it by construction (SP_ERR_INVALID): row pointers from 0 to nnz, never
// decreasing, and column indices in [0, ncols) — an index out of range would make a pass
// read outside its vector on the GPU. A's values and column indices are read in one pass.
int lp_check(const sp_lp *lp, std::string *msg) {
    const int64_t m = lp->a.nrows, n = lp->a.ncols, nnz = lp->a.nnz;
    auto bounds = [&](const char *what, const double *lo, const double *hi, int64_t len) -> std::string {
        const auto f = first_bad(len, [&](int64_t i) {
            if (std::isnan(lo[i]) || std::isnan(hi[i])) return 1;
            return lo[i] > hi[i] ? 2 : 0;
        });
        const std::string at = std::string(what) + " " + std::to_string(f.first);
        if (f.second == 1) return at + " is NaN";
        if (f.second == 2)
            return at + " has lower bound " + rust_display(lo[f.first]) + " above upper bound " +
                   rust_display(hi[f.first]);
        return "";
    };
    *msg = bounds("variable", lp->lv, lp->uv, n);
    if (msg->empty()) *msg = bounds("constraint", lp->lc, lp->uc, m);
    if (!msg->empty()) return SP_ERR_PROBLEM;
    const int64_t kc = first_bad(n, [&](int64_t j) { return std::isnan(lp->c[j]) ? 1 : 0; }).first;
    if (kc >= 0) {
        *msg = "coefficient " + std::to_string(kc) + " is NaN";
        return SP_ERR_PROBLEM;
    }
    const int64_t *rp = lp->a.row_ptr;
    const int32_t *ci = lp->a.col_idx;
    const double *v = lp->a.values;
    if (!rp || (nnz > 0 && (!ci || !v))) {
        *msg = "A lacks an array";
        return SP_ERR_INVALID;
    }
    // per range: the first NaN value, and the first column out of range before it
    std::vector<std::pair<int64_t, int64_t>> found(16, {-1, -1});
    split_ranges(nnz, [&](int w, int64_t k0, int64_t k1) {
        int64_t fc = -1;
        for (int64_t k = k0; k < k1; ++k) {
            if (std::isnan(v[k])) {
                found[w] = {k, fc};
                return;
            }
            if (fc < 0 && (ci[k] < 0 || ci[k] >= n)) fc = k;
        }
        found[w] = {-1, fc};
    });
    int64_t nan_at = -1, col_at = -1;
    for (const auto &f : found) {
        if (nan_at < 0 && f.first >= 0) nan_at = f.first;
        if (col_at < 0 && f.second >= 0) col_at = f.second;
    }
    if (nan_at >= 0) {
        *msg = "coefficient " + std::to_string(n + nan_at) + " is NaN";
        return SP_ERR_PROBLEM;
    }
    if (rp[0] != 0 || rp[m] != nnz) {
        *msg = "A's row pointers run from " + std::to_string(rp[0]) + " to " + std::to_string(rp[m]) +
               ", not from 0 to " + std::to_string(nnz);
        return SP_ERR_INVALID;
    }
    const int64_t row = first_bad(m, [&](int64_t i) { return rp[i + 1] < rp[i] ? 1 : 0; }).first;
    if (row >= 0) {
        *msg = "A's row pointers decrease after row " + std::to_string(row);
        return SP_ERR_INVALID;
    }
    if (col_at >= 0) {
        *msg = "A's column index " + std::to_string(ci[col_at]) + " at entry " + std::to_string(col_at) +
               " is out of range for " + std::to_string(n) + " columns";
        return SP_ERR_INVALID;
    }
    msg->clear();
    return SP_OK;
}

int validate_lp(const sp_lp *lp) {
    std::string msg;
    const int rc = lp_check(lp, &msg);
    return rc ? fail(rc, msg) : SP_OK;
}

int power_iteration(sp_solver *s) {  // Solver::estimate_norm (solver.rs:215-242)
    cudaStream_t st = s->ctx->stream;
    if (s->n == 0 || s->nnz == 0) {
        s->norm_est = 1.0;
        return SP_OK;
    }
    k_power_fill<<<grid_of(s->ctx, s->n), NT, 0, st>>>(s->pv, s->n);
    k_power_init<<<1, NT, 0, st>>>(s->n, s->ppart);
    k_power_start<<<1, 32, 0, st>>>(s->ppart, s->d_st);
    const uint64_t maxit = s->prm.power_iterations;
    PowerA a{s->A.rp, s->A.ci, s->A.v, s->A.tiles, s->pv, s->ptmp, s->d_st, 0.0};
    PowerT t{s->AT.rp, s->AT.ci, s->AT.v, s->AT.tiles, s->ptmp, s->pv, s->ppart, s->d_st};
    const uint64_t chunk = 8;
    DevState h{};  // with no iterations, λ stays 0 as in the reference
    for (uint64_t done_it = 0; done_it < maxit;) {
        const uint64_t c = std::min(chunk, maxit - done_it);
        for (uint64_t q = 0; q < c; ++q) {
            // A'·v on the SELL copy where the dual passes have one (the same bits; 0.21 ms on
            // the tile engine for the 40M LP), else on the tile engine
            if (s->sellA.ok) launch_sell(s, s->sellA, st, a);
            else k_tiles<<<s->A.ntiles, NT, tile_smem_bytes<1, double>(), st>>>(a);
            k_tiles<<<s->AT.ntiles, NT, tile_smem_bytes<1, double>(), st>>>(t);
            k_power_fin<<<1, NT, 0, st>>>(s->ppart, s->AT.ntiles, maxit, s->d_st);
        }
        done_it += c;
        SP_CUDA_TRY(cudaMemcpyAsync(&h, s->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, st));
        SP_CUDA_TRY(cudaStreamSynchronize(st));
        if (h.pi_done) break;
    }
    if (h.error == ERR_NUMERICAL_POWER) return fail(SP_ERR_NUMERICAL, "numerical breakdown: power iteration collapsed");
    s->norm_est = sqrt(h.pi_lambda) * 1.01;  // solver.rs:241
    s->pi_iters = h.pi_iters;
    return SP_OK;
}

}  // namespace sp

extern "C" void sp_solver_params_default(sp_solver_params *p) {
    if (!p) return;
    memset(p, 0, sizeof *p);
    p->tolerance = 1e-6;  // solver.rs:70-93
    p->infeasibility_tolerance = 1e-8;
    p->max_iterations = 1000000;
    p->time_limit_s = 0.0;
    p->check_every = 64;
    p->step_size_factor = 0.998;
    p->reflection = 1.0;
    p->restart_sufficient = 0.2;
    p->restart_necessary = 0.5;
    p->restart_artificial = 0.36;
    p->pid_kp = 0.99;
    p->pid_ki = 0.01;
    p->pid_kd = 0.0;
    p->pid_discount = 0.3;
    p->power_iterations = 200;
    p->geometric_mean_passes = 12;  // scaling.rs:25-34
    p->ruiz_iterations = 10;
    p->pock_chambolle_enabled = 1;
    p->pock_chambolle_alpha = 1.0;
    p->bound_objective_rescaling = 1;
    p->log_every_checks = 0;
    p->termination = SP_TERMINATION_PROJECTED;
    p->precision = SP_PRECISION_FP64;
    p->mixed_switch_tolerance = 1e-5;
}

extern "C" int sp_solver_reset(sp_solver *s) {
    if (!s) return SP_ERR_INVALID;
    int rc = enter(s->ctx);
    if (rc) return rc;
    cudaStream_t st = s->ctx->stream;
    const int64_t m = s->m, n = s->n;
    for (double *v : {s->x, s->xt, s->xbar, s->xa, s->aty}) SP_CUDA_TRY(cudaMemsetAsync(v, 0, sizeof(double) * n, st));
    for (double *v : {s->y, s->yt, s->ya}) SP_CUDA_TRY(cudaMemsetAsync(v, 0, sizeof(double) * m, st));
    if (s->mixed) {
        SP_CUDA_TRY(cudaMemsetAsync(s->xbar32, 0, sizeof(float) * n, st));
        SP_CUDA_TRY(cudaMemsetAsync(s->y32, 0, sizeof(float) * m, st));
    }
    DevState h{};
    h.total = 0;
    h.k = 0;
    // Initial primal weight (solver.rs:322).
    h.omega = s->prm.bound_objective_rescaling ? 1.0 : (1.0 + s->c_norm) / (1.0 + s->b_norm);
    h.status = -1;
    h.fp64 = s->mixed ? 0 : 1;
    h.anchor_residual = INFINITY;
    h.prev_residual = INFINITY;
    h.pid_best_weight = h.omega;  // PidState::new (solver.rs:453-455)
    h.pid_best_balance = INFINITY;
    h.pi_done = 1;
    h.mx_best = INFINITY;
    *s->h_st = h;
    SP_CUDA_TRY(cudaMemcpyAsync(s->d_st, s->h_st, sizeof(DevState), cudaMemcpyHostToDevice, st));
    SP_CUDA_TRY(cudaStreamSynchronize(st));
    s->launched = 0;
    s->time_limited = false;
    return SP_OK;
}

extern "C" int sp_solver_warm_start(sp_solver *s, const double *x, const double *y) {
    if (!s) return SP_ERR_INVALID;
    int rc = sp_solver_reset(s);
    if (rc) return rc;
    if (!x && !y) return SP_OK;
    cudaStream_t st = s->ctx->stream;
    double *dx = nullptr, *dy = nullptr;
    if (x && (rc = dalloc(&dx, s->n))) return rc;
    if (y && (rc = dalloc(&dy, s->m))) {
        dfree(dx, st);
        return rc;
    }
    if (x && s->n) SP_CUDA_TRY(cudaMemcpyAsync(dx, x, sizeof(double) * s->n, cudaMemcpyHostToDevice, st));
    if (y && s->m) SP_CUDA_TRY(cudaMemcpyAsync(dy, y, sizeof(double) * s->m, cudaMemcpyHostToDevice, st));
    k_warm_start<<<grid_of(s->ctx, std::max(s->n, s->m)), NT, 0, st>>>(dx, dy, s->col_scale, s->row_scale, s->scales,
                                                                        s->x, s->xa, s->y, s->ya, s->mixed ? s->y32 : nullptr,
                                                                        s->n, s->m);
    SP_CUDA_TRY(cudaGetLastError());
    SP_CUDA_TRY(cudaStreamSynchronize(st));
    dfree(dx, st);
    dfree(dy, st);
    return SP_OK;
}

extern "C" int sp_solver_create(sp_ctx *ctx, const sp_lp *lp, const sp_solver_params *params, sp_solver **out) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!lp || !out || !lp->c || !lp->lc || !lp->uc || !lp->lv || !lp->uv)
        return fail(SP_ERR_INVALID, "sp_solver_create: null argument");
    if ((rc = validate_lp(lp))) return rc;
    double t0 = now_s();
    // SP_SETUP_TRACE=1: each set-up stage's wall time on stderr (the stages synchronise)
    const bool trace = getenv("SP_SETUP_TRACE") != nullptr;
    double tl = t0;
    auto stage = [&](const char *what) {
        if (!trace) return;
        cudaStreamSynchronize(ctx->stream);
        const double t = now_s();
        fprintf(stderr, "setup %-12s %8.2f ms\n", what, (t - tl) * 1e3);
        tl = t;
    };
    auto *s = new sp_solver();
    s->ctx = ctx;
    sp_solver_params_default(&s->prm);
    if (params) s->prm = *params;
    s->mixed = s->prm.precision == SP_PRECISION_MIXED;
    s->m = lp->a.nrows;
    s->n = lp->a.ncols;
    s->nnz = lp->a.nnz;
    s->c0 = lp->c0;
    s->maximize = lp->maximize;
    if (s->prm.check_every == 0) s->prm.check_every = 1ull << 62;  // never a multiple: only the iteration limit checks
    const int64_t m = s->m, n = s->n;
    // the set-up work on the second stream (scale_on_device); an early return joins it
    // before the solver's buffers are released
    SideNorms side;
    auto cleanup = [&](int code) {
        side.join();
        solver_release(s);
        return code;
    };
    if ((rc = upload_csr(ctx, &lp->a, &s->A, false))) return cleanup(rc);
    stage("upload");
    std::vector<int> rp_t;
    if ((rc = transpose_on_device(s, rp_t))) return cleanup(rc);
    stage("transpose");
    if ((rc = dalloc(&s->c, n)) || (rc = dalloc(&s->lc, m)) || (rc = dalloc(&s->uc, m)) || (rc = dalloc(&s->lv, n)) ||
        (rc = dalloc(&s->uv, n)) || (rc = dalloc(&s->pf, m)) || (rc = dalloc(&s->df, n)) ||
        (rc = dalloc(&s->row_scale, m)) || (rc = dalloc(&s->col_scale, n)) || (rc = dalloc(&s->scales, 2)) ||
        (rc = dalloc(&s->norms, 4)))
        return cleanup(rc);
    if ((rc = scale_on_device(s, lp, rp_t, &side))) return cleanup(rc);
    // the host's tile plan of A'ᵀ while the GPU runs the scaling sweeps
    if ((rc = plan_transpose(s, rp_t))) return cleanup(rc);
    rp_t = std::vector<int>();
    stage("scaling");
    if (s->mixed) {
        if ((rc = dalloc(&s->A.v32, s->nnz)) || (rc = dalloc(&s->AT.v32, s->nnz))) return cleanup(rc);
        k_to_f32<<<grid_of(ctx, s->nnz), NT, 0, ctx->stream>>>(s->A.v, s->A.v32, s->nnz);
        k_to_f32<<<grid_of(ctx, s->nnz), NT, 0, ctx->stream>>>(s->AT.v, s->AT.v32, s->nnz);
    }
    if ((rc = dalloc(&s->x, n)) || (rc = dalloc(&s->y, m)) || (rc = dalloc(&s->xt, n)) || (rc = dalloc(&s->yt, m)) ||
        (rc = dalloc(&s->xbar, n)) || (rc = dalloc(&s->xa, n)) || (rc = dalloc(&s->ya, m)) ||
        (rc = dalloc(&s->aty, n)) || (rc = dalloc(&s->xbar32, n)) || (rc = dalloc(&s->y32, m)) ||
        (rc = dalloc(&s->pk, n)) || (rc = dalloc(&s->pky, m)) ||
        (rc = dalloc(&s->partP, (int64_t)s->AT.ntiles * NP_P)) || (rc = dalloc(&s->partT, (int64_t)s->AT.ntiles * NP_T)) ||
        (rc = dalloc(&s->partP0, (int64_t)s->AT.ntiles * NP_P0)) ||
        (rc = dalloc(&s->partD, (int64_t)s->A.ntiles * NP_D)) || (rc = dalloc(&s->partD0, (int64_t)s->A.ntiles * NP_D0)) ||
        (rc = dalloc(&s->pv, n)) || (rc = dalloc(&s->ptmp, m)) ||
        (rc = dalloc(&s->ppart, std::max<int64_t>(s->AT.ntiles, 1))) || (rc = dalloc(&s->d_st, 1)) ||
        (rc = dalloc(&s->d_prm, 1)))
        return cleanup(rc);
    s->trace_cap = (int64_t)std::min<uint64_t>(s->prm.max_iterations / std::max<uint64_t>(s->prm.check_every, 1) + 2,
                                               1 << 20);
    if ((rc = dalloc(&s->d_trace, s->trace_cap))) return cleanup(rc);
    SP_CUDA_TRY(cudaMallocHost(&s->h_st, sizeof(DevState) * (SolverLookahead + 2)));
    if ((rc = set_smem_limits())) return cleanup(rc);
    if ((rc = choose_engines(s))) return cleanup(rc);
    stage("engines");
    // ‖A'‖₂ and η (solver.rs:316), while the second stream forms the norms
    if ((rc = power_iteration(s))) return cleanup(rc);
    stage("power");
    if (side.join() != cudaSuccess) return cleanup(fail(SP_ERR_CUDA, "set-up: norms on the second stream failed"));
    double hn[4], hs[2];
    SP_CUDA_TRY(cudaMemcpyAsync(hn, s->norms, sizeof hn, cudaMemcpyDeviceToHost, ctx->stream));
    SP_CUDA_TRY(cudaMemcpyAsync(hs, s->scales, sizeof hs, cudaMemcpyDeviceToHost, ctx->stream));
    SP_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    s->b_norm = hn[2];
    s->c_norm = hn[3];
    s->bound_scale = hs[0];
    s->obj_scale = hs[1];
    if ((rc = sp_solver_reset(s))) return cleanup(rc);
    stage("norms");
    DevParams dp{};
    const sp_solver_params &P = s->prm;
    dp.tolerance = P.tolerance;
    dp.infeasibility_tolerance = P.infeasibility_tolerance;
    dp.max_iterations = P.max_iterations;
    dp.check_every = P.check_every;
    dp.reflection = P.reflection;
    dp.restart_sufficient = P.restart_sufficient;
    dp.restart_necessary = P.restart_necessary;
    dp.restart_artificial = P.restart_artificial;
    dp.pid_kp = P.pid_kp;
    dp.pid_ki = P.pid_ki;
    dp.pid_kd = P.pid_kd;
    dp.pid_discount = P.pid_discount;
    dp.termination = P.termination;
    dp.mixed = s->mixed;
    dp.mixed_switch_tolerance = P.mixed_switch_tolerance;
    dp.mixed_stall_checks = MIXED_STALL_CHECKS;
    if (const char *e = getenv("SP_MIXED_STALL_CHECKS")) dp.mixed_stall_checks = std::max(1, atoi(e));
    dp.b_norm = s->b_norm;
    dp.c_norm = s->c_norm;
    dp.c0 = s->c0;
    dp.obj_factor = 1.0 / (s->bound_scale * s->obj_scale);  // scaling.rs:134-136
    dp.eta = P.step_size_factor / s->norm_est;
    dp.bound_objective_rescaling = P.bound_objective_rescaling;
    SP_CUDA_TRY(cudaMemcpyAsync(s->d_prm, &dp, sizeof dp, cudaMemcpyHostToDevice, ctx->stream));
    SP_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if ((rc = sp_solver_reset(s))) return cleanup(rc);
    s->setup_s = now_s() - t0;
    *out = s;
    return SP_OK;
}

namespace sp {

int epoch_graph(sp_solver *s, int E, cudaGraphExec_t *g) {
    auto it = s->graphs.find(E);
    if (it != s->graphs.end()) {
        *g = it->second;
        return SP_OK;
    }
    const double t0 = now_s();
    int rc = build_graph(s, E, g);
    if (rc) return rc;
    if (getenv("SP_SETUP_TRACE")) fprintf(stderr, "solve graph(%d)    %8.2f ms\n", E, (now_s() - t0) * 1e3);
    s->graphs[E] = *g;
    return SP_OK;
}

// Enqueues one epoch (graph, or direct launches when timing samples are due).
int launch_epoch(sp_solver *s, int E) {
    cudaStream_t st = s->ctx->stream;
    if (s->timing_every > 0) {
        enqueue_epoch(s, E, st, true);
    } else {
        cudaGraphExec_t g;
        int rc = epoch_graph(s, E, &g);
        if (rc) return rc;
        SP_CUDA_TRY(cudaGraphLaunch(g, st));
    }
    SP_CUDA_TRY(cudaGetLastError());
    s->launched += (uint64_t)E;
    return SP_OK;
}

void fill_info(sp_solver *s, const DevState &h, sp_solution_info *info) {
    if (!info) return;
    const double sign = s->maximize ? -1.0 : 1.0;
    info->status = h.done ? h.status : (s->time_limited ? SP_STATUS_TIME_LIMIT : -1);
    info->objective = sign * h.primal_obj;
    info->dual_objective = sign * h.dual_obj;
    info->primal_residual = h.primal_res;
    info->dual_residual = h.dual_res;
    info->gap = fabs(h.primal_obj - h.dual_obj);
    info->iterations = h.total;
    info->restarts = h.restarts;
    info->solve_time_s = s->solve_s;
    info->setup_time_s = s->setup_s;
    info->norm_estimate = s->norm_est;
    info->fp64_from_iteration = s->mixed ? h.fp64_from : 0;
}

}  // namespace sp

extern "C" int sp_solver_run_epochs(sp_solver *s, uint64_t epochs) {
    if (!s) return SP_ERR_INVALID;
    int rc = enter(s->ctx);
    if (rc) return rc;
    for (uint64_t e = 0; e < epochs; ++e) {
        const uint64_t E = std::min<uint64_t>(s->prm.check_every, s->prm.max_iterations - std::min(s->launched, s->prm.max_iterations));
        if (E == 0) break;
        if ((rc = launch_epoch(s, (int)E))) return rc;
    }
    return SP_OK;
}

extern "C" int sp_solver_sync(sp_solver *s) {
    if (!s) return SP_ERR_INVALID;
    int rc = enter(s->ctx);
    if (rc) return rc;
    SP_CUDA_TRY(cudaStreamSynchronize(s->ctx->stream));
    return SP_OK;
}

extern "C" int sp_solver_solve(sp_solver *s, sp_solution_info *info) {
    if (!s) return SP_ERR_INVALID;
    int rc = enter(s->ctx);
    if (rc) return rc;
    cudaStream_t st = s->ctx->stream;
    const double t0 = now_s();
    const double limit = s->prm.time_limit_s;
    // Epochs are queued SolverLookahead ahead of the state the host has seen;
    // each queued epoch is followed by a copy of the state into its own slot.
    // the epochs' completion events, destroyed on every way out
    struct Events {
        std::vector<cudaEvent_t> e;
        ~Events() {
            for (cudaEvent_t x : e) cudaEventDestroy(x);
        }
    } events;
    for (int k = 0; k < SolverLookahead + 1; ++k) {
        cudaEvent_t e = nullptr;
        SP_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        events.e.push_back(e);
    }
    std::vector<cudaEvent_t> &ev = events.e;
    uint64_t queued = 0, seen = 0;
    bool stop = false;
    DevState last{};
    uint64_t logged_checks = 0;
    while (!stop) {
        while (!stop && queued - seen < (uint64_t)SolverLookahead + 1) {
            const uint64_t E = std::min<uint64_t>(s->prm.check_every,
                                                  s->prm.max_iterations - std::min(s->launched, s->prm.max_iterations));
            if (E == 0) {
                stop = queued == seen;
                break;
            }
            if ((rc = launch_epoch(s, (int)E))) return rc;
            const int slot = (int)(queued % ev.size());
            SP_CUDA_TRY(cudaMemcpyAsync(&s->h_st[slot], s->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, st));
            SP_CUDA_TRY(cudaEventRecord(ev[slot], st));
            ++queued;
        }
        if (seen == queued) break;
        const int slot = (int)(seen % ev.size());
        SP_CUDA_TRY(cudaEventSynchronize(ev[slot]));
        last = s->h_st[slot];
        ++seen;
        if (s->prm.log_every_checks > 0 && last.checks > logged_checks && last.checks % s->prm.log_every_checks == 0) {
            logged_checks = last.checks;
            fprintf(stderr, "%9llu %14.6e %14.6e %9.2e %9.2e %9.2e %9.2e %5llu %8.2fs %7llu %9.2e\n",
                    (unsigned long long)last.total, last.primal_obj, last.dual_obj, last.primal_res, last.dual_res,
                    fabs(last.primal_obj - last.dual_obj), last.omega, (unsigned long long)last.restarts,
                    now_s() - t0, (unsigned long long)last.k, last.last_residual / last.anchor_residual);
        }
        if (last.done) stop = true;
        if (!stop && limit > 0 && now_s() - t0 >= limit) {  // solver.rs:392-394, observed per epoch
            s->time_limited = true;
            stop = true;
        }
    }
    SP_CUDA_TRY(cudaStreamSynchronize(st));
    SP_CUDA_TRY(cudaMemcpy(s->h_st, s->d_st, sizeof(DevState), cudaMemcpyDeviceToHost));
    last = s->h_st[0];
    s->solve_s = now_s() - t0;
    if (last.error == ERR_NUMERICAL_ITERATES) return fail(SP_ERR_NUMERICAL, "numerical breakdown: iterates are not finite");
    if (last.error == ERR_PIPELINE_STALL)
        return fail(SP_ERR_CUDA, "a bulk copy of the pass pipeline did not complete within its wait limit");
    if (!last.done && !s->time_limited) s->time_limited = true;  // only reachable with an exhausted limit
    fill_info(s, last, info);
    return SP_OK;
}

extern "C" int sp_solver_info(sp_solver *s, sp_solution_info *info) {
    if (!s || !info) return SP_ERR_INVALID;
    int rc = enter(s->ctx);
    if (rc) return rc;
    SP_CUDA_TRY(cudaStreamSynchronize(s->ctx->stream));
    DevState h;
    SP_CUDA_TRY(cudaMemcpy(&h, s->d_st, sizeof h, cudaMemcpyDeviceToHost));
    fill_info(s, h, info);
    return SP_OK;
}

extern "C" int sp_solver_download(sp_solver *s, double *x, double *y) {
    if (!s) return SP_ERR_INVALID;
    int rc = enter(s->ctx);
    if (rc) return rc;
    cudaStream_t st = s->ctx->stream;
    if (!s->out_x) {
        if ((rc = dalloc(&s->out_x, s->n)) || (rc = dalloc(&s->out_y, s->m))) return rc;
    }
    k_unscale<<<grid_of(s->ctx, std::max(s->n, s->m)), NT, 0, st>>>(s->xt, s->yt, s->col_scale, s->row_scale, s->scales,
                                                                    s->out_x, s->out_y, s->n, s->m);
    if (x && s->n) SP_CUDA_TRY(cudaMemcpyAsync(x, s->out_x, sizeof(double) * s->n, cudaMemcpyDeviceToHost, st));
    if (y && s->m) SP_CUDA_TRY(cudaMemcpyAsync(y, s->out_y, sizeof(double) * s->m, cudaMemcpyDeviceToHost, st));
    SP_CUDA_TRY(cudaStreamSynchronize(st));
    return SP_OK;
}

extern "C" int sp_solver_trace(sp_solver *s, sp_check_record *out, int64_t cap, int64_t *len) {
    if (!s || !len) return SP_ERR_INVALID;
    int rc = enter(s->ctx);
    if (rc) return rc;
    SP_CUDA_TRY(cudaStreamSynchronize(s->ctx->stream));
    DevState h;
    SP_CUDA_TRY(cudaMemcpy(&h, s->d_st, sizeof h, cudaMemcpyDeviceToHost));
    const int64_t avail = std::min<int64_t>((int64_t)h.trace_len, s->trace_cap);
    *len = avail;
    const int64_t k = std::min(avail, cap);
    if (k > 0 && out) SP_CUDA_TRY(cudaMemcpy(out, s->d_trace, sizeof(sp_check_record) * k, cudaMemcpyDeviceToHost));
    return SP_OK;
}

extern "C" int sp_solver_set_timing(sp_solver *s, int every) {
    if (!s) return SP_ERR_INVALID;
    s->timing_every = every > 0 ? every : 0;
    s->timing_counter = 0;
    s->samples.clear();
    s->event_next = 0;
    return SP_OK;
}

extern "C" int sp_solver_kernel_timing(sp_solver *s, int id, int64_t *launches, double *total_ms,
                                       double *bytes_per_launch) {
    if (!s || id < 0 || id > 1) return SP_ERR_INVALID;
    int rc = enter(s->ctx);
    if (rc) return rc;
    SP_CUDA_TRY(cudaStreamSynchronize(s->ctx->stream));
    double tot = 0.0;
    int64_t cnt = 0;
    for (auto &smp : s->samples) {
        float ms = 0.f;
        cudaEvent_t a = id == 0 ? smp.e0 : smp.e1, b = id == 0 ? smp.e1 : smp.e2;
        if (cudaEventElapsedTime(&ms, a, b) == cudaSuccess) {
            tot += ms;
            ++cnt;
        }
    }
    if (launches) *launches = cnt;
    if (total_ms) *total_ms = tot;
    if (bytes_per_launch) *bytes_per_launch = s->pass_bytes(id);
    return SP_OK;
}

extern "C" double sp_solver_bytes_per_iteration(sp_solver *s) { return s ? s->pass_bytes(0) + s->pass_bytes(1) : 0.0; }

namespace sp {

// The gathers of a pass and nothing else: every nonzero's entry of the gathered vector,
// addressed through the pass's own column-index stream (coalesced, 8 loads in flight per
// thread), summed per warp into `out` so nothing is optimised away. Its time is the floor
// the pass's random gathers set on this GPU (no values, no epilogue, no staging).
template <class GT>
__global__ void __launch_bounds__(NT) k_gather_floor(const int *__restrict__ ci, int64_t nnz,
                                                     const GT *__restrict__ gv, double *__restrict__ out) {
    const int64_t stride = (int64_t)gridDim.x * NT;
    int64_t k = blockIdx.x * (int64_t)NT + threadIdx.x;
    double acc = 0.0;
    for (; k + 7 * stride < nnz; k += 8 * stride) {
        int c[8];
        GT g[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) c[u] = ld_stream(ci + k + u * stride);
#pragma unroll
        for (int u = 0; u < 8; ++u) g[u] = __ldg(gv + c[u]);
#pragma unroll
        for (int u = 0; u < 8; ++u) acc += double(g[u]);
    }
    for (; k < nnz; k += stride) acc += double(__ldg(gv + ld_stream(ci + k)));
    acc = warp_sum_down(acc);
    if ((threadIdx.x & 31) == 0) out[blockIdx.x * (NT / 32) + (threadIdx.x >> 5)] = acc;
}

}  // namespace sp

extern "C" int sp_solver_gather_floor(sp_solver *s, int pass, int fp32, int reps, double *ms_per_launch) {
    if (!s || pass < 0 || pass > 1 || reps < 1 || !ms_per_launch) return SP_ERR_INVALID;
    if (fp32 && !s->mixed) return fail(SP_ERR_INVALID, "FP32 gathers exist in the mixed form only");
    int rc = enter(s->ctx);
    if (rc) return rc;
    cudaStream_t st = s->ctx->stream;
    const DevCsr &M = pass == 0 ? s->AT : s->A;
    if (M.nnz == 0) {
        *ms_per_launch = 0.0;
        return SP_OK;
    }
    int per_sm = 0;
    const void *f = fp32 ? (const void *)k_gather_floor<float> : (const void *)k_gather_floor<double>;
    SP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f, NT, 0));
    const int grid = std::max(1, per_sm) * s->ctx->sms;
    double *out = nullptr;
    if ((rc = dalloc(&out, (int64_t)grid * (NT / 32)))) return rc;
    EventPair ep;
    if ((rc = ep.init())) return rc;
    auto launch = [&] {
        if (fp32) k_gather_floor<float><<<grid, NT, 0, st>>>(M.ci, M.nnz, pass == 0 ? s->y32 : s->xbar32, out);
        else k_gather_floor<double><<<grid, NT, 0, st>>>(M.ci, M.nnz, pass == 0 ? s->y : s->xbar, out);
    };
    launch();
    SP_CUDA_TRY(cudaEventRecord(ep.e0, st));
    for (int r = 0; r < reps; ++r) launch();
    SP_CUDA_TRY(cudaEventRecord(ep.e1, st));
    SP_CUDA_TRY(cudaEventSynchronize(ep.e1));
    float ms = 0.f;
    SP_CUDA_TRY(cudaEventElapsedTime(&ms, ep.e0, ep.e1));
    dfree(out, st);
    SP_CUDA_TRY(cudaGetLastError());
    *ms_per_launch = (double)ms / reps;
    return SP_OK;
}

extern "C" int sp_solver_engines(sp_solver *s, int32_t out[4]) {
    if (!s || !out) return SP_ERR_INVALID;
    const int v[4] = {s->sv_p64, s->sv_p32, s->sv_d64, s->sv_d32};
    for (int k = 0; k < 4; ++k) out[k] = v[k] < 0 ? SP_ENGINE_TILES : (v[k] == ENGINE_SELL ? SP_ENGINE_SELL : SP_ENGINE_STREAM);
    return SP_OK;
}

extern "C" int sp_solver_epoch_kernels(sp_solver *s, int64_t *count) {
    if (!s || !count) return SP_ERR_INVALID;
    int rc = enter(s->ctx);
    if (rc) return rc;
    const int E = (int)std::max<uint64_t>(1, s->prm.check_every);
    cudaGraphExec_t g;
    if ((rc = epoch_graph(s, E, &g))) return rc;
    *count = s->graph_kernels[E];
    return SP_OK;
}

extern "C" void sp_solver_free(sp_solver *s) { solver_release(s); }

// The whole solve in one call (Part 2).
extern "C" int sp_solve(sp_ctx *ctx, const sp_lp *lp, const sp_solver_params *params, double *x, double *y,
                        sp_solution_info *info) {
    sp_solver *s = nullptr;
    const bool trace = getenv("SP_SETUP_TRACE") != nullptr;  // the stages' wall times on stderr
    double t = now_s();
    auto mark = [&](const char *what) {
        if (!trace) return;
        const double u = now_s();
        fprintf(stderr, "solve %-12s %8.2f ms\n", what, (u - t) * 1e3);
        t = u;
    };
    int rc = sp_solver_create(ctx, lp, params, &s);
    if (rc) return rc;
    mark("create");
    rc = sp_solver_solve(s, info);
    mark("iterations");
    if (!rc) rc = sp_solver_download(s, x, y);
    mark("download");
    if (!rc && info) {
        info->setup_time_s = s->setup_s;
        info->solve_time_s = s->solve_s;
    }
    sp_solver_free(s);
    mark("free");
    return rc;
}

extern "C" int sp_problem_validate(const sp_lp *lp, char *message, size_t cap) {
    if (!lp || !lp->c || !lp->lc || !lp->uc || !lp->lv || !lp->uv || lp->a.nrows < 0 || lp->a.ncols < 0 ||
        lp->a.nnz < 0)
        return SP_ERR_INVALID;
    std::string e;
    const int rc = sp::lp_check(lp, &e);
    if (message && cap > 0) snprintf(message, cap, "%s", e.c_str());
    return rc;
}

extern "C" int sp_solver_scaled(sp_solver *s, int64_t *a_row_ptr, int32_t *a_col_idx, double *a_values,
                                int64_t *at_row_ptr, int32_t *at_col_idx, double *at_values, double *c, double *lc,
                                double *uc, double *lv, double *uv, double *row_scale, double *col_scale,
                                double *bound_scale, double *obj_scale) {
    if (!s) return SP_ERR_INVALID;
    int rc = enter(s->ctx);
    if (rc) return rc;
    SP_CUDA_TRY(cudaStreamSynchronize(s->ctx->stream));
    const int64_t m = s->m, n = s->n, nnz = s->nnz;
    auto rowptr = [&](const int *d, int64_t rows, int64_t *out) -> int {
        if (!out) return SP_OK;
        std::vector<int> tmp(rows + 1);
        SP_CUDA_TRY(cudaMemcpy(tmp.data(), d, sizeof(int) * (rows + 1), cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i <= rows; ++i) out[i] = tmp[i];
        return SP_OK;
    };
    auto copy = [&](void *dst, const void *src, size_t bytes) -> int {
        if (dst && bytes) SP_CUDA_TRY(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost));
        return SP_OK;
    };
    if ((rc = rowptr(s->A.rp, m, a_row_ptr)) || (rc = rowptr(s->AT.rp, n, at_row_ptr)) ||
        (rc = copy(a_col_idx, s->A.ci, sizeof(int) * nnz)) || (rc = copy(a_values, s->A.v, sizeof(double) * nnz)) ||
        (rc = copy(at_col_idx, s->AT.ci, sizeof(int) * nnz)) || (rc = copy(at_values, s->AT.v, sizeof(double) * nnz)) ||
        (rc = copy(c, s->c, sizeof(double) * n)) || (rc = copy(lc, s->lc, sizeof(double) * m)) ||
        (rc = copy(uc, s->uc, sizeof(double) * m)) || (rc = copy(lv, s->lv, sizeof(double) * n)) ||
        (rc = copy(uv, s->uv, sizeof(double) * n)) || (rc = copy(row_scale, s->row_scale, sizeof(double) * m)) ||
        (rc = copy(col_scale, s->col_scale, sizeof(double) * n)))
        return rc;
    if (bound_scale) *bound_scale = s->bound_scale;
    if (obj_scale) *obj_scale = s->obj_scale;
    return SP_OK;
}
