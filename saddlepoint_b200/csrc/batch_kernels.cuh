// batch_kernels.cuh — the batched form: one persistent kernel solves many LPs.
//
// Each CTA takes the next instance from a device counter and runs its whole
// solve: the scaling passes (scaling.rs:53-103), power iteration (solver.rs:215-242)
// and the PDHG loop with checks, restarts, PID and termination (solver.rs:311-438),
// synchronising with __syncthreads only — an instance never waits on another CTA,
// so nothing in the kernel spins. All of an instance's work is done by one CTA in
// a fixed order, so its result is the same bits whether it is solved alone or in
// a mix of thousands.
//
// SpMV inside a CTA: rows are dealt to groups of L lanes (L = 1, 2, ..., 32, the
// "lanes per row" the tuner picks per instance and per matrix). A lane sums a
// strided slice of its row from -0.0, the group adds the slices with a fixed
// shuffle tree; with L = 1 a row is summed in column order by one thread, the
// reference CPU backend's order.
#pragma once

#include "control.cuh"
#include "solver_kernels.cuh"

namespace sp {

struct BatchInst {
    int m, n, nnz;
    int lanes_a, lanes_t;  // lanes per row for A' and for A'ᵀ (lane-group variant)
    int variant;           // VARIANT_LANES or VARIANT_TILES, picked by the tuner
    long long rpa, rpt;    // offsets of the row pointers (m + 1 and n + 1 entries, instance-local values)
    long long nz;          // offset of the nonzeros
    long long mo, no;      // offsets of the m- and n-vectors
    long long ta, tt;      // offsets of the tile plans of A' and A'ᵀ (instance-local rows)
    long long pa, pt;      // offsets of the per-tile partial sums (10 per A' tile, 15 per A'ᵀ tile)
    int nta, ntt;          // tiles of A' and A'ᵀ
    double c0;
    int maximize, pad2;
};

enum : int { VARIANT_LANES = 0, VARIANT_TILES = 1 };

struct BatchArgs {
    const BatchInst *inst;
    const int *order;  // processing order (largest first)
    int count;
    int *counter;
    // The tail hand-off: once every instance has been claimed (drain_ns: when, 0 before),
    // an instance still running handoff_ns later stops at its next check and is
    // finished by the single-LP solver on the host's side (0: never).
    unsigned long long *drain_ns;
    unsigned long long handoff_ns;
    const int *a_rp, *a_ci, *t_rp, *t_ci;
    double *a_v, *t_v;
    float *a_v32, *t_v32;
    const double *oc, *olc, *ouc, *olv, *ouv;  // original vectors
    double *c, *lc, *uc, *lv, *uv, *pf, *df, *rs, *cs;
    double *x, *y, *xt, *yt, *xbar, *xa, *ya, *aty, *pv, *pt, *ox, *oy;
    float *xbar32, *y32;
    CheckQuad *pk;  // the tile variant's packed column records (n per instance)
    double2 *pky;   // ... and row records (m per instance)
    const Tile *a_tiles, *t_tiles;
    double *part;  // per-tile partial sums of every instance
    sp_batch_result *res;
    DevParams base;
    unsigned long long power_iterations, geo_passes, ruiz_iterations;
    int pc_enabled, rescale;
    double pc_alpha, step_size_factor;
    int mixed;
};

// Thread 0, after a check that did not end the solve: stop for the hand-off when the
// queue drained more than handoff_ns ago (the instance is a straggler of the tail).
__device__ __forceinline__ void tail_handoff(const BatchArgs &A, DevState &st) {
    if (st.done || A.handoff_ns == 0) return;
    const unsigned long long drained = *reinterpret_cast<volatile unsigned long long *>(A.drain_ns);
    if (drained && global_ns() - drained > A.handoff_ns) {
        st.done = 1;
        st.status = SP_STATUS_ITERATION_LIMIT;
        st.handoff = 1;
    }
}

template <int BT, int K>
__device__ __forceinline__ void bsum(double (&v)[K], double *sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int W = BT / 32;
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

// Runs `body(r, gl)` for the rows of a matrix dealt to groups of L lanes, with a
// uniform trip count per warp so the group shuffles are safe. body returns the
// group's slot sums through `acc` reduced onto lane gl == 0 by reduce().
template <int BT>
struct Rows {
    int L, lane, warp, gl, gid, rpw;
    __device__ Rows(int L_) : L(L_) {
        lane = threadIdx.x & 31;
        warp = threadIdx.x >> 5;
        gl = lane % L;
        gid = lane / L;
        rpw = 32 / L;
    }
    template <class T>
    __device__ __forceinline__ T reduce(T v) const {
        for (int o = L >> 1; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o, L);
        return v;
    }
};

// Runs a tile pass over one instance's tiles if its setup() accepts (uniform over the CTA).
template <class Op>
__device__ __forceinline__ void cta_tiles(Op op, int ntiles, unsigned char *dsm) {
    if (!op.setup()) return;
    for (int t = 0; t < ntiles; ++t) {
        tile_body(op, dsm, t);
        __syncthreads();
    }
}

template <bool LO>
__device__ __forceinline__ void cta_primal(const SolverPtrs &S, int role, int nt, unsigned char *dsm) {
    auto mk = [&](auto tag) {
        constexpr int MODE = decltype(tag)::value;
        PrimalPass<LO, MODE> o{};
        o.rp = S.t_rp;
        o.ci = S.t_ci;
        if constexpr (LO) o.vals = S.t_v32;
        else o.vals = S.t_v;
        o.tiles = S.t_tiles;
        o.s = S;
        o.i = 0;
        o.role = role;
        return o;
    };
    cta_tiles(mk(std::integral_constant<int, 0>{}), nt, dsm);
    cta_tiles(mk(std::integral_constant<int, 1>{}), nt, dsm);
    cta_tiles(mk(std::integral_constant<int, 2>{}), nt, dsm);
}

template <bool LO>
__device__ __forceinline__ void cta_dual(const SolverPtrs &S, int role, int nt, unsigned char *dsm) {
    auto mk = [&](auto tag) {
        constexpr int MODE = decltype(tag)::value;
        DualPass<LO, MODE> o{};
        o.rp = S.a_rp;
        o.ci = S.a_ci;
        if constexpr (LO && MODE == 0) o.vals = S.a_v32;
        else o.vals = S.a_v;
        o.tiles = S.a_tiles;
        o.s = S;
        o.i = 0;
        o.role = role;
        return o;
    };
    cta_tiles(mk(std::integral_constant<int, 0>{}), nt, dsm);
    cta_tiles(mk(std::integral_constant<int, 1>{}), nt, dsm);
    cta_tiles(mk(std::integral_constant<int, 2>{}), nt, dsm);
}

// An instance solved by the tile passes of the single-LP solve, driven by this CTA
// instead of by kernel launches: the same tiles, the same partial sums reduced in
// the same order, the same controller — so the same bits as sp_solve.
template <int BT>
__device__ void batch_tiles_solve(const BatchArgs &A, const BatchInst &I, const SolverPtrs &S, double *ppart,
                                  double *pv, double *ptmp, double *sh, unsigned char *dsm, DevState &st,
                                  DevParams &prm) {
    static_assert(BT == NT, "the tile passes are written for NT threads");
    const int tid = threadIdx.x, m = I.m, n = I.n;
    const bool mixed = A.mixed != 0;
    // power iteration (solver.rs:215-242), as k_power_init / PowerA / PowerT / k_power_fin
    double lambda = 0.0;
    bool numerical = false;
    if (n > 0 && I.nnz > 0) {
        double s1[1] = {0.0};
        for (int j = tid; j < n; j += BT) {
            const double v0 = 1.0 + 0.01 * (double)(j % 7);
            pv[j] = v0;
            s1[0] += v0 * v0;
        }
        block_sum<1>(s1, sh);
        if (tid == 0) {
            st.pi_scale = 1.0 / sqrt(s1[0]);
            st.pi_lambda = 0.0;
            st.pi_done = 0;
            st.pi_iters = 0;
            st.error = ERR_NONE;
        }
        __syncthreads();
        for (unsigned long long it = 0; it < A.power_iterations && !st.pi_done; ++it) {
            PowerA pa{S.a_rp, S.a_ci, S.a_v, S.a_tiles, pv, ptmp, &st, 0.0};
            cta_tiles(pa, I.nta, dsm);
            PowerT ptr{S.t_rp, S.t_ci, S.t_v, S.t_tiles, ptmp, pv, ppart, &st};
            cta_tiles(ptr, I.ntt, dsm);
            double s[1];
            sum_slots<1>(ppart, I.ntt, s, sh);
            if (tid == 0) {
                const double norm = sqrt(s[0]);
                if (isnan(norm) || norm <= 0.0 || isinf(norm)) {
                    st.error = ERR_NUMERICAL_POWER;
                    st.pi_done = 1;
                } else {
                    st.pi_scale = 1.0 / norm;
                    const bool done = fabs(norm - st.pi_lambda) <= 1e-6 * norm;
                    st.pi_lambda = norm;
                    st.pi_iters += 1;
                    if (done || (unsigned long long)st.pi_iters >= A.power_iterations) st.pi_done = 1;
                }
            }
            __syncthreads();
        }
        lambda = st.pi_lambda;
        numerical = st.error == ERR_NUMERICAL_POWER;
    }
    const double norm_est = (n > 0 && I.nnz > 0) ? sqrt(lambda) * 1.01 : 1.0;
    __syncthreads();
    if (tid == 0) {
        prm.eta = A.step_size_factor / norm_est;
        st = DevState{};
        st.omega = A.rescale ? 1.0 : (1.0 + prm.c_norm) / (1.0 + prm.b_norm);
        st.status = -1;
        st.fp64 = mixed ? 0 : 1;
        st.anchor_residual = INFINITY;
        st.prev_residual = INFINITY;
        st.pid_best_weight = st.omega;
        st.pid_best_balance = INFINITY;
        st.mx_best = INFINITY;
        st.pi_done = 1;
        if (numerical) {
            st.done = 1;
            st.error = ERR_NUMERICAL_POWER;
        }
    }
    for (int j = tid; j < n; j += BT) S.x[j] = S.xa[j] = 0.0;
    for (int i = tid; i < m; i += BT) {
        S.y[i] = S.ya[i] = 0.0;
        if (mixed) S.y32[i] = 0.0f;
    }
    __syncthreads();
    // the PDHG loop (solver.rs:332-420), one iteration at a time
    while (!st.done) {
        const bool check = (prm.check_every != 0 && (st.total + 1) % prm.check_every == 0) ||
                           st.total + 1 >= prm.max_iterations;
        const bool k0 = st.k == 0;
        const bool lo = mixed && !st.fp64;
        const int role = check ? ROLE_CHECK : ROLE_FIRST;  // FIRST: K0 at k == 0, else fused
        if (lo) cta_primal<true>(S, role, I.ntt, dsm);
        else cta_primal<false>(S, role, I.ntt, dsm);
        if (lo) cta_dual<true>(S, role, I.nta, dsm);
        else cta_dual<false>(S, role, I.nta, dsm);
        if (!check) {
            if (k0) {
                const double rho = prm.reflection;
                for (int j = tid; j < n; j += BT) S.x[j] = halpern(S.x[j], S.xt[j], S.xa[j], 0.5, rho);
                double P0[1], D0[2];
                sum_slots<1>(S.partP0, I.ntt, P0, sh);
                sum_slots<2>(S.partD0, I.nta, D0, sh);
                if (tid == 0) {
                    bool bad = false;
                    st.anchor_residual = fixed_point_residual(prm.eta, st.omega, P0[0], D0[0], D0[1], &bad);
                    if (bad) {
                        st.error = ERR_NUMERICAL_ITERATES;
                        st.done = 1;
                    }
                }
            }
            if (tid == 0) {
                st.k += 1;
                st.total += 1;
            }
            __syncthreads();
            continue;
        }
        CheckPassT tp{};
        tp.rp = S.t_rp;
        tp.ci = S.t_ci;
        tp.vals = S.t_v;
        tp.tiles = S.t_tiles;
        tp.s = S;
        tp.i = 0;
        cta_tiles(tp, I.ntt, dsm);
        double P[NP_P], D[NP_D], T[NP_T];
        sum_slots<NP_P>(S.partP, I.ntt, P, sh);
        sum_slots<NP_D>(S.partD, I.nta, D, sh);
        sum_slots<NP_T>(S.partT, I.ntt, T, sh);
        if (tid == 0) {
            bool bad = false;
            sp_check_record rec;
            check_decide(&st, &prm, P, D, T, st.k, st.total + 1, &bad, &rec);
            tail_handoff(A, st);
        }
        __syncthreads();
        if (st.done) break;
        // k_finish: the Halpern step, or the restart's copies
        const double w = st.w_last, rho = prm.reflection;
        const bool rs = st.restart_flag != 0, y32 = mixed && !st.fp64;
        for (int j = tid; j < n; j += BT) {
            if (rs) S.x[j] = S.xa[j] = S.xt[j];
            else S.x[j] = halpern(S.x[j], S.xt[j], S.xa[j], w, rho);
        }
        for (int i = tid; i < m; i += BT) {
            double v;
            if (rs) v = S.ya[i] = S.yt[i];
            else v = halpern(S.y[i], S.yt[i], S.ya[i], w, rho);
            S.y[i] = v;
            if (y32) S.y32[i] = (float)v;
        }
        __syncthreads();
    }
}

template <int BT>
__device__ void batch_solve_one(const BatchArgs &A, int id, double *sh, DevState &st, DevParams &prm, double *bc,
                                unsigned char *dsm) {
    const BatchInst I = A.inst[id];
    const int m = I.m, n = I.n;
    const int *arp = A.a_rp + I.rpa, *aci = A.a_ci + I.nz, *trp = A.t_rp + I.rpt, *tci = A.t_ci + I.nz;
    double *av = A.a_v + I.nz, *tv = A.t_v + I.nz;
    float *av32 = A.a_v32 ? A.a_v32 + I.nz : nullptr, *tv32 = A.t_v32 ? A.t_v32 + I.nz : nullptr;
    const double *oc = A.oc + I.no, *olv = A.olv + I.no, *ouv = A.ouv + I.no, *olc = A.olc + I.mo,
                 *ouc = A.ouc + I.mo;
    double *c = A.c + I.no, *lv = A.lv + I.no, *uv = A.uv + I.no, *df = A.df + I.no, *cs = A.cs + I.no;
    double *lc = A.lc + I.mo, *uc = A.uc + I.mo, *pf = A.pf + I.mo, *rs = A.rs + I.mo;
    double *x = A.x + I.no, *xt = A.xt + I.no, *xbar = A.xbar + I.no, *xa = A.xa + I.no, *aty = A.aty + I.no,
           *pv = A.pv + I.no, *ox = A.ox + I.no;
    double *y = A.y + I.mo, *yt = A.yt + I.mo, *ya = A.ya + I.mo, *pt = A.pt + I.mo, *oy = A.oy + I.mo;
    float *xbar32 = A.xbar32 ? A.xbar32 + I.no : nullptr, *y32 = A.y32 ? A.y32 + I.mo : nullptr;
    const int tid = threadIdx.x;
    const bool mixed = A.mixed != 0;

    // ---------------- scaling passes (ScaledProblem::new)
    for (int i = tid; i < m; i += BT) rs[i] = 1.0;
    for (int j = tid; j < n; j += BT) cs[j] = 1.0;
    __syncthreads();
    auto apply = [&](const double *r, const double *cc, bool rows_only, bool cols_only) {
        // values[k] *= r[i] * c[j] in A' and A'ᵀ (problem.rs:120-126); a missing side is 1.0
        for (int i = tid; i < m; i += BT)
            for (int k = arp[i]; k < arp[i + 1]; ++k) {
                const double ri = cols_only ? 1.0 : r[i], cj = rows_only ? 1.0 : cc[aci[k]];
                av[k] *= ri * cj;
            }
        for (int j = tid; j < n; j += BT)
            for (int k = trp[j]; k < trp[j + 1]; ++k) {
                const double ri = cols_only ? 1.0 : r[tci[k]], cj = rows_only ? 1.0 : cc[j];
                tv[k] *= ri * cj;
            }
        if (!cols_only)
            for (int i = tid; i < m; i += BT) rs[i] *= r[i];
        if (!rows_only)
            for (int j = tid; j < n; j += BT) cs[j] *= cc[j];
        __syncthreads();
    };
    auto inv_sqrt = [](double v) { return (v > 0.0 && isfinite(v)) ? 1.0 / sqrt(v) : 1.0; };
    auto geo = [&](const int *rp, const double *v, int rows, double *f) {
        for (int r = tid; r < rows; r += BT) {
            double lo = INFINITY, hi = 0.0;
            for (int k = rp[r]; k < rp[r + 1]; ++k) {
                const double a = fabs(v[k]);
                lo = fmin(lo, a);
                hi = fmax(hi, a);
            }
            if (hi == 0.0) lo = 0.0;
            f[r] = inv_sqrt(lo * hi);
        }
        __syncthreads();
    };
    for (unsigned long long ps = 0; ps < A.geo_passes; ++ps) {
        geo(arp, av, m, pt);
        apply(pt, nullptr, true, false);
        geo(trp, tv, n, pv);
        apply(nullptr, pv, false, true);
    }
    for (unsigned long long it = 0; it < A.ruiz_iterations; ++it) {
        for (int r = tid; r < m; r += BT) {
            double hi = 0.0;
            for (int k = arp[r]; k < arp[r + 1]; ++k) hi = fmax(hi, fabs(av[k]));
            pt[r] = inv_sqrt(hi);
        }
        for (int r = tid; r < n; r += BT) {
            double hi = 0.0;
            for (int k = trp[r]; k < trp[r + 1]; ++k) hi = fmax(hi, fabs(tv[k]));
            pv[r] = inv_sqrt(hi);
        }
        __syncthreads();
        apply(pt, pv, false, false);
    }
    if (A.pc_enabled) {  // sums in the reference's order (one thread per row)
        const double a1 = A.pc_alpha, a2 = 2.0 - A.pc_alpha;
        for (int r = tid; r < m; r += BT) {
            double s = 0.0;
            for (int k = arp[r]; k < arp[r + 1]; ++k) {
                const double a = fabs(av[k]);
                s = s + (a1 == 1.0 ? a : pow(a, a1));
            }
            pt[r] = inv_sqrt(s);
        }
        for (int r = tid; r < n; r += BT) {
            double s = 0.0;
            for (int k = trp[r]; k < trp[r + 1]; ++k) {
                const double a = fabs(tv[k]);
                s = s + (a2 == 1.0 ? a : pow(a, a2));
            }
            pv[r] = inv_sqrt(s);
        }
        __syncthreads();
        apply(pt, pv, false, false);
    }
    for (int j = tid; j < n; j += BT) {
        c[j] = oc[j] * cs[j];
        lv[j] = olv[j] / cs[j];
        uv[j] = ouv[j] / cs[j];
    }
    for (int i = tid; i < m; i += BT) {
        lc[i] = olc[i] * rs[i];
        uc[i] = ouc[i] * rs[i];
    }
    __syncthreads();
    if (tid == 0) {  // the four sequential norms (scaling.rs:186-201, solver.rs:317-318)
        auto fbn = [&](const double *lo, const double *hi) {
            double s = -0.0;
            for (int i = 0; i < m; ++i) {
                const double l = isfinite(lo[i]) ? lo[i] : 0.0, u = isfinite(hi[i]) ? hi[i] : 0.0;
                s += (l == u) ? l * l : l * l + u * u;
            }
            return sqrt(s);
        };
        auto n2 = [&](const double *v) {
            double s = -0.0;
            for (int j = 0; j < n; ++j) s += v[j] * v[j];
            return sqrt(s);
        };
        const double bs = A.rescale ? 1.0 / (1.0 + fbn(lc, uc)) : 1.0;
        const double os = A.rescale ? 1.0 / (1.0 + n2(c)) : 1.0;
        bc[0] = bs;
        bc[1] = os;
        prm = A.base;
        prm.b_norm = fbn(olc, ouc);
        prm.c_norm = n2(oc);
        prm.c0 = I.c0;
        prm.obj_factor = 1.0 / (bs * os);
    }
    __syncthreads();
    const double bs = bc[0], os = bc[1];
    if (A.rescale) {
        for (int i = tid; i < m; i += BT) {
            lc[i] *= bs;
            uc[i] *= bs;
        }
        for (int j = tid; j < n; j += BT) {
            lv[j] *= bs;
            uv[j] *= bs;
            c[j] *= os;
        }
    }
    for (int i = tid; i < m; i += BT) pf[i] = 1.0 / (rs[i] * bs);
    for (int j = tid; j < n; j += BT) df[j] = 1.0 / (cs[j] * os);
    if (mixed) {
        for (int k = tid; k < I.nnz; k += BT) {
            av32[k] = (float)av[k];
            tv32[k] = (float)tv[k];
        }
    }
    __syncthreads();

    if (I.variant == VARIANT_TILES) {
        SolverPtrs S{};
        S.a_rp = arp;
        S.a_ci = aci;
        S.a_v = av;
        S.a_v32 = av32;
        S.a_tiles = A.a_tiles + I.ta;
        S.t_rp = trp;
        S.t_ci = tci;
        S.t_v = tv;
        S.t_v32 = tv32;
        S.t_tiles = A.t_tiles + I.tt;
        S.c = c;
        S.lc = lc;
        S.uc = uc;
        S.lv = lv;
        S.uv = uv;
        S.pf = pf;
        S.df = df;
        S.x = x;
        S.y = y;
        S.xt = xt;
        S.yt = A.yt + I.mo;
        S.xbar = xbar;
        S.xa = xa;
        S.ya = ya;
        S.aty = aty;
        S.xbar32 = xbar32;
        S.y32 = y32;
        S.pk = A.pk + I.no;
        S.pky = A.pky + I.mo;
        double *pt_base = A.part + I.pt, *pa_base = A.part + I.pa;
        S.partP = pt_base;
        S.partT = pt_base + (long long)I.ntt * NP_P;
        S.partP0 = pt_base + (long long)I.ntt * (NP_P + NP_T);
        S.partD = pa_base;
        S.partD0 = pa_base + (long long)I.nta * NP_D;
        S.prm = &prm;
        S.st = &st;
        S.mixed = mixed;
        batch_tiles_solve<BT>(A, I, S, pt_base + (long long)I.ntt * (NP_P + NP_T + NP_P0), pv, pt, sh, dsm, st,
                              prm);
    } else {
    const Rows<BT> RA(I.lanes_a), RT(I.lanes_t);

    // ---------------- power iteration (solver.rs:215-242)
    double lambda = 0.0;
    bool numerical = false;
    if (n > 0 && I.nnz > 0) {
        double s1[1] = {0.0};
        for (int j = tid; j < n; j += BT) {
            const double v0 = 1.0 + 0.01 * (double)(j % 7);
            pv[j] = v0;
            s1[0] += v0 * v0;
        }
        bsum<BT, 1>(s1, sh);
        if (tid == 0) bc[2] = 1.0 / sqrt(s1[0]);
        __syncthreads();
        for (unsigned long long it = 0; it < A.power_iterations; ++it) {
            const double sc = bc[2];
            for (int base = RA.warp * RA.rpw; base < m; base += (BT / 32) * RA.rpw) {
                const int r = base + RA.gid;
                double a = -0.0;
                if (r < m)
                    for (int k = arp[r] + RA.gl; k < arp[r + 1]; k += RA.L) a += av[k] * (pv[aci[k]] * sc);
                a = RA.reduce(a);
                if (r < m && RA.gl == 0) pt[r] = a;
            }
            __syncthreads();
            double s2[1] = {0.0};
            for (int base = RT.warp * RT.rpw; base < n; base += (BT / 32) * RT.rpw) {
                const int r = base + RT.gid;
                double a = -0.0;
                if (r < n)
                    for (int k = trp[r] + RT.gl; k < trp[r + 1]; k += RT.L) a += tv[k] * pt[tci[k]];
                a = RT.reduce(a);
                if (r < n && RT.gl == 0) {
                    pv[r] = a;
                    s2[0] += a * a;
                }
            }
            bsum<BT, 1>(s2, sh);
            if (tid == 0) {
                const double norm = sqrt(s2[0]);
                if (isnan(norm) || norm <= 0.0 || isinf(norm)) {
                    bc[3] = -1.0;
                } else {
                    bc[2] = 1.0 / norm;
                    const bool done = fabs(norm - lambda) <= 1e-6 * norm;
                    lambda = norm;
                    bc[3] = done ? 1.0 : 0.0;
                }
                bc[4] = lambda;
            }
            __syncthreads();
            lambda = bc[4];
            if (bc[3] != 0.0) {
                numerical = bc[3] < 0.0;
                break;
            }
        }
    }
    const double norm_est = (n > 0 && I.nnz > 0) ? sqrt(lambda) * 1.01 : 1.0;
    if (tid == 0) {
        prm.eta = A.step_size_factor / norm_est;
        st = DevState{};
        st.omega = A.rescale ? 1.0 : (1.0 + prm.c_norm) / (1.0 + prm.b_norm);
        st.status = -1;
        st.fp64 = mixed ? 0 : 1;
        st.anchor_residual = INFINITY;
        st.prev_residual = INFINITY;
        st.pid_best_weight = st.omega;
        st.pid_best_balance = INFINITY;
        st.mx_best = INFINITY;
        if (numerical) {
            st.done = 1;
            st.error = ERR_NUMERICAL_POWER;
        }
    }
    for (int j = tid; j < n; j += BT) x[j] = xa[j] = 0.0;
    for (int i = tid; i < m; i += BT) {
        y[i] = ya[i] = 0.0;
        if (mixed) y32[i] = 0.0f;
    }
    __syncthreads();

    // ---------------- the PDHG loop (solver.rs:332-420)
    unsigned long long total = 0;
    const double rho = prm.reflection;
    while (!st.done) {
        const double omega = st.omega, eta = prm.eta;
        const double tau = eta / omega, sigma = eta * omega;
        const unsigned long long k = st.k;
        const double w = (double)(k + 1) / (double)(k + 2);
        const bool check = (prm.check_every != 0 && (total + 1) % prm.check_every == 0) || total + 1 >= prm.max_iterations;
        const bool k0 = k == 0;
        const bool lo = mixed && !st.fp64;
        double P[NP_P] = {0}, D[NP_D] = {0}, T[NP_T] = {0};
        // P: A'ᵀ rows
        for (int base = RT.warp * RT.rpw; base < n; base += (BT / 32) * RT.rpw) {
            const int j = base + RT.gid;
            double a;
            if (lo) {
                float af = -0.0f;
                if (j < n)
                    for (int q = trp[j] + RT.gl; q < trp[j + 1]; q += RT.L) af += tv32[q] * y32[tci[q]];
                a = (double)RT.reduce(af);
            } else {
                a = -0.0;
                if (j < n)
                    for (int q = trp[j] + RT.gl; q < trp[j + 1]; q += RT.L) a += tv[q] * y[tci[q]];
                a = RT.reduce(a);
            }
            if (j < n && RT.gl == 0) {
                const double xj = x[j];
                const double t = clampd(xj - tau * (c[j] - a), lv[j], uv[j]);
                const double xb = 2.0 * t - xj;
                if (lo) xbar32[j] = (float)xb;
                else xbar[j] = xb;
                if (!check && !k0) {
                    x[j] = halpern(xj, t, xa[j], w, rho);
                } else {
                    xt[j] = t;
                    const double dx = t - xj;
                    P[0] += dx * dx;
                    if (check) {
                        aty[j] = a;
                        const double cj = c[j], dxa = t - xa[j];
                        const double rv = recession_violation(dxa, lv[j], uv[j]);
                        P[1] += cj * t;
                        P[2] += a * t;
                        P[3] += t * t;
                        P[4] += xj * t;
                        P[5] += rv * rv;
                        P[6] += dxa * dxa;
                        P[7] += cj * dxa;
                    }
                }
            }
        }
        __syncthreads();
        // D: A' rows
        for (int base = RA.warp * RA.rpw; base < m; base += (BT / 32) * RA.rpw) {
            const int i = base + RA.gid;
            double s0, s1 = -0.0, s2 = -0.0, s3 = -0.0;
            if (lo) {
                float af = -0.0f;
                if (i < m)
                    for (int q = arp[i] + RA.gl; q < arp[i + 1]; q += RA.L) af += av32[q] * xbar32[aci[q]];
                s0 = (double)RA.reduce(af);
            } else {
                double a = -0.0;
                if (i < m)
                    for (int q = arp[i] + RA.gl; q < arp[i + 1]; q += RA.L) a += av[q] * xbar[aci[q]];
                s0 = RA.reduce(a);
            }
            if (check || k0) {
                if (i < m)
                    for (int q = arp[i] + RA.gl; q < arp[i + 1]; q += RA.L) {
                        const int cc = aci[q];
                        const double v = av[q], xtc = xt[cc];
                        s1 += v * (xtc - x[cc]);
                        if (check) {
                            s2 += v * xtc;
                            s3 += v * (xtc - xa[cc]);
                        }
                    }
                s1 = RA.reduce(s1);
                if (check) {
                    s2 = RA.reduce(s2);
                    s3 = RA.reduce(s3);
                }
            }
            if (i < m && RA.gl == 0) {
                const double yi = y[i];
                const double v = s0 - yi / sigma;
                const double ytv = yi - sigma * (s0 - clampd(v, lc[i], uc[i]));
                if (!check) {
                    const double yn = halpern(yi, ytv, ya[i], w, rho);
                    y[i] = yn;
                    if (lo) y32[i] = (float)yn;
                    if (k0) {
                        const double dy = ytv - yi;
                        D[0] += dy * dy;
                        D[1] += dy * s1;
                    }
                } else {
                    yt[i] = ytv;
                    const double dy = ytv - yi, dya = ytv - ya[i];
                    const double e = excess(s2, lc[i], uc[i]) * pf[i];
                    const double rv = recession_violation(s3, lc[i], uc[i]);
                    const double fb = forbidden(dya, lc[i], uc[i]);
                    D[0] += dy * dy;
                    D[1] += dy * s1;
                    D[2] += e * e;
                    D[3] += bound_term(ytv, lc[i], uc[i]);
                    D[4] += rv * rv;
                    D[5] += fb * fb;
                    D[6] += bound_term(dya, lc[i], uc[i]);
                    D[7] += dya * dya;
                }
            }
        }
        __syncthreads();
        total += 1;
        if (!check) {
            if (k0) {  // the anchor's residual (solver.rs:341-346), then x's Halpern step
                for (int j = tid; j < n; j += BT) x[j] = halpern(x[j], xt[j], xa[j], w, rho);
                double r3[3] = {P[0], D[0], D[1]};
                bsum<BT, 3>(r3, sh);
                if (tid == 0) {
                    bool bad = false;
                    st.anchor_residual = fixed_point_residual(eta, omega, r3[0], r3[1], r3[2], &bad);
                    if (bad) {
                        st.error = ERR_NUMERICAL_ITERATES;
                        st.done = 1;
                    }
                    st.k = k + 1;
                }
            } else if (tid == 0) {
                st.k = k + 1;
            }
            __syncthreads();
            continue;
        }
        // T: the A'ᵀ check pass
        const double inv_tau = 1.0 / tau;
        for (int base = RT.warp * RT.rpw; base < n; base += (BT / 32) * RT.rpw) {
            const int j = base + RT.gid;
            double a0 = -0.0, a1 = -0.0;
            if (j < n)
                for (int q = trp[j] + RT.gl; q < trp[j + 1]; q += RT.L) {
                    const int rr = tci[q];
                    const double v = tv[q], ytc = yt[rr];
                    a0 += v * ytc;
                    a1 += v * (ytc - ya[rr]);
                }
            a0 = RT.reduce(a0);
            a1 = RT.reduce(a1);
            if (j < n && RT.gl == 0) {
                const double r = c[j] - a0;
                const double f = forbidden(r, lv[j], uv[j]) * df[j];
                const double sd = (aty[j] - a0 - (xt[j] - x[j]) * inv_tau) * df[j];
                const double ra = -a1, fa = forbidden(ra, lv[j], uv[j]);
                T[0] += f * f;
                T[1] += bound_term(r, lv[j], uv[j]);
                T[2] += sd * sd;
                T[3] += fa * fa;
                T[4] += bound_term(ra, lv[j], uv[j]);
            }
        }
        bsum<BT, NP_P>(P, sh);
        bsum<BT, NP_D>(D, sh);
        bsum<BT, NP_T>(T, sh);
        if (tid == 0) {
            bool bad = false;
            sp_check_record rec;
            check_decide(&st, &prm, P, D, T, k, total, &bad, &rec);
            tail_handoff(A, st);
        }
        __syncthreads();
        if (st.done) break;
        const bool rs_flag = st.restart_flag != 0;
        const double wl = st.w_last;
        const bool lo2 = mixed && !st.fp64;
        for (int j = tid; j < n; j += BT) {
            if (rs_flag) x[j] = xa[j] = xt[j];
            else x[j] = halpern(x[j], xt[j], xa[j], wl, rho);
        }
        for (int i = tid; i < m; i += BT) {
            double v;
            if (rs_flag) v = ya[i] = yt[i];
            else v = halpern(y[i], yt[i], ya[i], wl, rho);
            y[i] = v;
            if (lo2) y32[i] = (float)v;
        }
        __syncthreads();
    }
    }  // lane-group variant
    // Solution in the original space (solver.rs:422-437)
    for (int j = tid; j < n; j += BT) ox[j] = xt[j] * cs[j] / bs;
    for (int i = tid; i < m; i += BT) oy[i] = yt[i] * rs[i] / os;
    if (tid == 0) {
        sp_batch_result r;
        const double sign = I.maximize ? -1.0 : 1.0;
        r.status = st.error ? -1 - st.error : st.status;
        r.objective = sign * st.primal_obj;
        r.dual_objective = sign * st.dual_obj;
        r.primal_residual = st.primal_res;
        r.dual_residual = st.dual_res;
        r.gap = fabs(st.primal_obj - st.dual_obj);
        r.iterations = st.total;
        r.restarts = st.restarts;
        r.lanes_per_row = I.variant == VARIANT_TILES ? 0 : I.lanes_a * 100 + I.lanes_t;
        r.handed_off = st.handoff ? 2 : 0;  // 2: the host finishes it
        A.res[id] = r;
    }
    __syncthreads();
}

template <int BT>
__global__ void __launch_bounds__(BT) k_batch(BatchArgs A) {
    extern __shared__ __align__(16) unsigned char dsm[];  // tile staging of the tile variant
    __shared__ double sh[NP_P * (BT / 32)];
    __shared__ DevState st;
    __shared__ DevParams prm;
    __shared__ double bc[8];
    __shared__ int next;
    for (;;) {
        if (threadIdx.x == 0) next = atomicAdd(A.counter, 1);
        __syncthreads();
        const int slot = next;
        __syncthreads();
        if (slot >= A.count) {
            if (threadIdx.x == 0) atomicCAS(A.drain_ns, 0ull, global_ns());
            return;
        }
        batch_solve_one<BT>(A, A.order[slot], sh, st, prm, bc, dsm);
    }
}

// Dynamic shared memory of k_batch: the largest tile pass (four products per nonzero).
constexpr size_t batch_smem_bytes() { return tile_smem_bytes<4, double>(); }

}  // namespace sp
