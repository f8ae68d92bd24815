// solver_state.h — the device-resident solver handle (sp_solver).
#pragma once

#include <map>
#include <vector>

#include "internal.cuh"
#include "sell.cuh"
#include "stream.cuh"

namespace sp {
constexpr int SolverLookahead = 2;  // epochs queued ahead of the state the host has read
struct TimingSample {
    cudaEvent_t e0, e1, e2;  // before P, between P and D, after D
};
}  // namespace sp

struct sp_solver {
    sp_ctx *ctx = nullptr;
    sp_solver_params prm{};
    int mixed = 0;
    // engine of each MID pass: -1 the tile engine, ENGINE_SELL the SELL path (sell.cuh),
    // else a stream-engine variant (stream.cuh)
    int sv_p64 = -1, sv_p32 = -1, sv_d64 = -1, sv_d32 = -1;
    sp::StreamTrial trial;      // wait limits of the stream engine (and its test knob)
    sp::SellMat sellA, sellAT;  // SELL copies of A' (dual pass) and A'ᵀ (primal pass), when used
    cudaStream_t aux = nullptr;  // second stream of a SELL pass: its warp rows beside its windows
    cudaEvent_t fork = nullptr, join = nullptr;
    double *contrib = nullptr;   // [NP_D][m] row contributions of the check's dual pass on the SELL copy
    int64_t m = 0, n = 0, nnz = 0;
    double c0 = 0.0;
    int maximize = 0;
    // scaled problem
    sp::DevCsr A, AT;
    double *c = nullptr, *lc = nullptr, *uc = nullptr, *lv = nullptr, *uv = nullptr, *pf = nullptr, *df = nullptr;
    double *row_scale = nullptr, *col_scale = nullptr;
    double *scales = nullptr;  // [bound_scale, obj_scale] on the device
    double *norms = nullptr;   // [‖b'‖, ‖c'‖, ‖b‖, ‖c‖]
    double b_norm = 0, c_norm = 0, bound_scale = 1, obj_scale = 1;
    // iterates
    double *x = nullptr, *y = nullptr, *xt = nullptr, *yt = nullptr, *xbar = nullptr, *xa = nullptr, *ya = nullptr,
           *aty = nullptr;
    float *xbar32 = nullptr, *y32 = nullptr;
    sp::CheckQuad *pk = nullptr;  // the check's packed column records
    double2 *pky = nullptr;       // ... and row records
    // partial sums per tile
    double *partP = nullptr, *partD = nullptr, *partT = nullptr, *partP0 = nullptr, *partD0 = nullptr;
    // power iteration
    double *pv = nullptr, *ptmp = nullptr, *ppart = nullptr;
    double norm_est = 1.0;
    int pi_iters = 0;
    // state
    sp::DevParams *d_prm = nullptr;
    sp::DevState *d_st = nullptr;
    sp::DevState *h_st = nullptr;  // pinned, one slot per queued epoch
    sp_check_record *d_trace = nullptr;
    int64_t trace_cap = 0;
    std::map<int, cudaGraphExec_t> graphs;  // epoch length -> instantiated graph
    std::map<int, int64_t> graph_kernels;    // epoch length -> kernel nodes of its graph
    uint64_t launched = 0;
    bool time_limited = false;
    double setup_s = 0, solve_s = 0;
    double *out_x = nullptr, *out_y = nullptr;
    // timing
    int timing_every = 0;
    uint64_t timing_counter = 0;
    std::vector<sp::TimingSample> samples;
    std::vector<cudaEvent_t> event_pool;
    size_t event_next = 0;

    // A timing event from the pool (null when none can be created).
    cudaEvent_t event() {
        if (event_next == event_pool.size()) {
            cudaEvent_t e = nullptr;
            if (cudaEventCreate(&e) != cudaSuccess) {
                cudaGetLastError();
                return nullptr;
            }
            event_pool.push_back(e);
        }
        return event_pool[event_next++];
    }

    // Algorithmic bytes of one launch of the primal pass (id 0) or the dual pass
    // (id 1) in the current precision: every array counted once per launch, a
    // gathered vector once (ideal reuse), int32 indices.
    //   P (A'ᵀ rows): nnz·(v + 4) + 4(n+1) + gather y + x, c, lv, uv, x_anchor read + x̄, x written
    //   D (A' rows):  nnz·(v + 4) + 4(m+1) + gather x̄ + y, lc, uc, y_anchor read + y (+ FP32 y) written
    // FP64 total: 24·nnz + 68n + 52m; mixed: 16·nnz + 60n + 52m (plus the 8 bytes of two row-pointer ends).
    double pass_bytes(int id) const {
        const bool lo = mixed != 0;
        const double vb = lo ? 4.0 : 8.0, gb = lo ? 4.0 : 8.0;
        const double M = (double)m, N = (double)n, Z = (double)nnz;
        if (id == 0) return Z * (vb + 4.0) + 4.0 * (N + 1) + gb * M + 40.0 * N + (lo ? 12.0 : 16.0) * N;
        return Z * (vb + 4.0) + 4.0 * (M + 1) + gb * N + 32.0 * M + (lo ? 12.0 : 8.0) * M;
    }
};

namespace sp {
void solver_release(sp_solver *s);
}
