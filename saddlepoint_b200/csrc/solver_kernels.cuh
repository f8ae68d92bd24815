// solver_kernels.cuh — the fused passes of one PDHG iteration and of its checks.
//
// Per iteration the reference runs spmv_t, primal_step, spmv, dual_step and two
// halpern_steps (crates/saddlepoint-core/src/solver.rs:334-362), six launches and
// six sweeps over the vectors. Here an iteration is two tile passes:
//   P (over A'ᵀ rows = columns j): aty_j = (A'ᵀy)_j, then in the epilogue
//      x_t = clamp(x - τ(c - aty)), x̄ = 2x_t - x, and the Halpern update of x;
//   D (over A' rows i): (A'x̄)_i, then y_t = y - σ(ax̄ - clamp(ax̄ - y/σ)) and
//      the Halpern update of y.
// x_t, y_t and aty are stored only where a check or a restart reads them. Every
// element is computed with the reference's operations in the reference's order.
//
// Iteration roles inside an epoch of E = check_every iterations:
//   FIRST (i = 0): FUSED, or K0 when the epoch starts at k = 0 (the fixed-point
//          residual of the anchor is measured, solver.rs:341-346);
//   MID:   FUSED;
//   CHECK (i = E-1): writes x_t, y_t, aty and the partial sums of the residual,
//          KKT and ray statistics; the controller kernel then decides.
#pragma once

#include "control.cuh"
#include "stream.cuh"
#include "tiles.cuh"

namespace sp {

enum Role : int { ROLE_FIRST = 0, ROLE_MID = 1, ROLE_CHECK = 2 };

// What the dual pass of a check (and of the first iteration at k = 0) gathers per
// column, packed into one 32-byte sector: x̄ (in the iteration precision), x_t - x,
// x_t and x_t - x_anchor, each rounded exactly as the vector the reference forms
// before its SpMV. Written by the primal pass of the same iteration.
struct __align__(32) CheckQuad {
    double xbar, dx, xt, dxa;
};

// Pointers of the device-resident solve.
struct SolverPtrs {
    // A' (rows i) and A'ᵀ (rows j)
    const int *a_rp, *a_ci, *t_rp, *t_ci;
    const double *a_v, *t_v;
    const float *a_v32, *t_v32;
    const Tile *a_tiles, *t_tiles;
    const uint16_t *a_sched, *t_sched;
    // problem vectors
    const double *c, *lc, *uc, *lv, *uv, *pf, *df;
    // iterates
    double *x, *y, *xt, *yt, *xbar, *xa, *ya, *aty;
    float *xbar32, *y32;
    CheckQuad *pk;
    double2 *pky;  // the check's dual records for T: y_t, y_t - y_anchor (16 bytes per row)
    // partial sums per tile
    double *partP, *partD, *partT, *partP0, *partD0;
    const DevParams *prm;
    DevState *st;
    int mixed;
};

struct IterScalars {
    double tau, sigma, w, rho;
};

__device__ __forceinline__ IterScalars iter_scalars(const SolverPtrs &s, int i) {
    IterScalars r;
    const double omega = s.st->omega, eta = s.prm->eta;
    r.tau = eta / omega;  // solver.rs:333
    r.sigma = eta * omega;
    const unsigned long long k = s.st->k + (unsigned long long)i;
    r.w = (double)(k + 1) / (double)(k + 2);  // solver.rs:360
    r.rho = s.prm->reflection;
    return r;
}

// Whether a pass of precision LO (FP32 SpMV) should run now.
__device__ __forceinline__ bool precision_matches(const SolverPtrs &s, bool lo) {
    return lo ? (s.mixed && !s.st->fp64) : (!s.mixed || s.st->fp64);
}

// ----------------------------------------------------------------------------------
// P: the primal pass over A'ᵀ. MODE 0 = FUSED, 1 = K0, 2 = CHECK.
template <bool LO, int MODE>
struct PrimalPass {
    using VT = typename std::conditional<LO, float, double>::type;
    using ST = VT;
    static constexpr int G = 1;
    static constexpr int NP = MODE == 2 ? NP_P : (MODE == 1 ? NP_P0 : 0);
    static constexpr unsigned F32 = LO ? 1u : 0u;
    const int *rp, *ci;
    const VT *vals;
    const Tile *tiles;
    const uint16_t *sched;  // null: rows in order
    SolverPtrs s;
    int i, role;
    IterScalars sc;

    __device__ bool setup() {
        if (s.st->done || !precision_matches(s, LO)) return false;
        int mode = role == ROLE_MID ? 0 : (role == ROLE_CHECK ? 2 : (s.st->k == 0 ? 1 : 0));
        if (mode != MODE) return false;
        sc = iter_scalars(s, i);
        return true;
    }
    __device__ __forceinline__ void prod(int c, VT v, ST (&p)[1]) const {
        if constexpr (LO) p[0] = v * __ldg(s.y32 + c);
        else p[0] = v * __ldg(s.y + c);
    }
    // The row's inputs, loaded at the start of the tile.
    struct Pre {
        double x, c, lv, uv, xa;
    };
    __device__ __forceinline__ Pre pre(int j) const {
        Pre p;
        p.x = __ldcs(s.x + j);
        p.c = __ldcs(s.c + j);
        p.lv = __ldcs(s.lv + j);
        p.uv = __ldcs(s.uv + j);
        p.xa = MODE == 1 ? 0.0 : __ldcs(s.xa + j);
        return p;
    }
    // The stream engine's view of the pass (FUSED only): the gathered vector, the
    // product, the row inputs as arrays it stages (x, c, lv, uv, x_anchor) and the
    // Pre read back from shared memory (p: row q of array 0).
    using GT = VT;
    __device__ __forceinline__ const GT *gvec() const {
        if constexpr (LO) return s.y32;
        else return s.y;
    }
    __device__ __forceinline__ ST mul(VT v, GT g) const { return v * g; }
    static constexpr int NPRE = 5;
    __device__ __forceinline__ const double *pre_array(int q) const {
        return q == 0 ? s.x : q == 1 ? s.c : q == 2 ? s.lv : q == 3 ? s.uv : s.xa;
    }
    __device__ __forceinline__ Pre pre_smem(const double *p, int stride) const {
        return Pre{p[0], p[stride], p[2 * stride], p[3 * stride], MODE == 1 ? 0.0 : p[4 * stride]};
    }
    __device__ void fault() const {
        s.st->error = ERR_PIPELINE_STALL;
        s.st->done = 1;
    }
    __device__ __forceinline__ void row(int j, const double (&sum)[1], double *part, const Pre &in) const {
        const double aty = sum[0];
        const double xj = in.x;
        const double t = clampd(xj - sc.tau * (in.c - aty), in.lv, in.uv);  // cpu lib.rs:156
        const double xb = 2.0 * t - xj;                                     // cpu lib.rs:158
        if constexpr (LO) s.xbar32[j] = (float)xb;
        else s.xbar[j] = xb;
        if constexpr (MODE == 0) {
            s.x[j] = halpern(xj, t, in.xa, sc.w, sc.rho);  // solver.rs:361
        } else {
            s.xt[j] = t;
            const double dx = t - xj;  // fixed_point_residual: x_t - x (solver.rs:277)
            part[0] += dx * dx;
            const double xbq = LO ? (double)(float)xb : xb;  // x̄ as the dual pass gathers it
            if constexpr (MODE == 1) s.pk[j] = CheckQuad{xbq, dx, t, 0.0};
            if constexpr (MODE == 2) {
                s.aty[j] = aty;
                const double cj = in.c;
                const double dxa = t - in.xa;  // infeasibility: x_t - x_anchor (solver.rs:302)
                s.pk[j] = CheckQuad{xbq, dx, t, dxa};
                const double rv = recession_violation(dxa, in.lv, in.uv);
                part[1] += cj * t;       // primal objective c'ᵀx_t
                part[2] += aty * t;      // step-implied dual objective terms (solver.rs:268-269)
                part[3] += t * t;
                part[4] += xj * t;
                part[5] += rv * rv;      // primal ray: column violations
                part[6] += dxa * dxa;    // primal ray norm = distance_sq(x_t, x_anchor)
                part[7] += cj * dxa;     // primal ray objective
            }
        }
    }
    __device__ void store(int tile, const double *t) const {
        double *out = MODE == 2 ? s.partP : s.partP0;
#pragma unroll
        for (int q = 0; q < NP; ++q) out[tile * NP + q] = t[q];
    }
};

// ----------------------------------------------------------------------------------
// D: the dual pass over A'. MODE 0 = FUSED, 1 = K0, 2 = CHECK.
// FUSED reads the iteration precision's values; K0 and CHECK read FP64 values and
// form the iteration's own product in the iteration precision from them.
template <bool LO, int MODE>
struct DualPass {
    using VT = typename std::conditional<LO && MODE == 0, float, double>::type;
    using ST = typename std::conditional<LO && MODE == 0, float, double>::type;
    static constexpr int G = MODE == 2 ? 4 : (MODE == 1 ? 2 : 1);
    static constexpr int NP = MODE == 2 ? NP_D : (MODE == 1 ? NP_D0 : 0);
    static constexpr unsigned F32 = LO ? 1u : 0u;  // slot 0 is the iteration's product
    const int *rp, *ci;
    const VT *vals;
    const Tile *tiles;
    const uint16_t *sched;  // null: rows in order
    SolverPtrs s;
    int i, role;
    IterScalars sc;

    __device__ bool setup() {
        if (s.st->done || !precision_matches(s, LO)) return false;
        int mode = role == ROLE_MID ? 0 : (role == ROLE_CHECK ? 2 : (s.st->k == 0 ? 1 : 0));
        if (mode != MODE) return false;
        sc = iter_scalars(s, i);
        return true;
    }
    __device__ __forceinline__ void prod(int c, VT v, ST (&p)[G]) const {
        if constexpr (MODE == 0) {
            if constexpr (LO) p[0] = ST((float)v * __ldg(s.xbar32 + c));
            else p[0] = v * __ldg(s.xbar + c);
        } else {
            // one sector per nonzero: the packed column record of the primal pass
            const double2 *q = reinterpret_cast<const double2 *>(s.pk + c);
            const double2 q0 = __ldg(q);
            if constexpr (LO) p[0] = ST((float)v * (float)q0.x);
            else p[0] = v * q0.x;
            p[1] = v * q0.y;  // A'(x_t - x)
            if constexpr (MODE == 2) {
                const double2 q1 = __ldg(q + 1);
                p[2] = v * q1.x;  // A' x_t
                p[3] = v * q1.y;  // A'(x_t - x_anchor)
            }
        }
    }
    // The row's inputs, loaded at the start of the tile.
    struct Pre {
        double y, lc, uc, ya, pf;
    };
    __device__ __forceinline__ Pre pre(int r) const {
        Pre p;
        p.y = __ldcs(s.y + r);
        p.lc = __ldcs(s.lc + r);
        p.uc = __ldcs(s.uc + r);
        p.ya = __ldcs(s.ya + r);
        p.pf = MODE == 2 ? __ldcs(s.pf + r) : 0.0;
        return p;
    }
    // The stream engine's view of the pass (FUSED only): the gathered vector, the
    // product and the row inputs it stages (y, lc, uc, y_anchor).
    using GT = typename std::conditional<LO && MODE == 0, float, double>::type;
    __device__ __forceinline__ const GT *gvec() const {
        if constexpr (LO && MODE == 0) return s.xbar32;
        else return s.xbar;
    }
    __device__ __forceinline__ ST mul(VT v, GT g) const { return ST(v * g); }
    static constexpr int NPRE = 4;
    __device__ __forceinline__ const double *pre_array(int q) const {
        return q == 0 ? s.y : q == 1 ? s.lc : q == 2 ? s.uc : s.ya;
    }
    __device__ __forceinline__ Pre pre_smem(const double *p, int stride) const {
        return Pre{p[0], p[stride], p[2 * stride], p[3 * stride], 0.0};
    }
    __device__ void fault() const {
        s.st->error = ERR_PIPELINE_STALL;
        s.st->done = 1;
    }
    __device__ __forceinline__ void row(int r, const double (&sum)[G], double *part, const Pre &in) const {
        const double a = sum[0], yi = in.y;
        const double v = a - yi / sc.sigma;                              // cpu lib.rs:171
        const double yt = yi - sc.sigma * (a - clampd(v, in.lc, in.uc)); // cpu lib.rs:172
        if constexpr (MODE == 0) {
            const double yn = halpern(yi, yt, in.ya, sc.w, sc.rho);
            s.y[r] = yn;
            if constexpr (LO) s.y32[r] = (float)yn;  // the FP32 shadow the next P pass gathers
        } else {
            const double dy = yt - yi;  // fixed_point_residual: y_t - y (solver.rs:278)
            part[0] += dy * dy;
            part[1] += dy * sum[1];     // cross term dyᵀ A'(x_t - x)
            if constexpr (MODE == 1) {
                const double yn = halpern(yi, yt, in.ya, sc.w, sc.rho);
                s.y[r] = yn;
                if constexpr (LO) s.y32[r] = (float)yn;
            } else {
                s.yt[r] = yt;
                const double lc = in.lc, uc = in.uc;
                const double e = excess(sum[2], lc, uc) * in.pf;
                const double dya = yt - in.ya;
                s.pky[r] = make_double2(yt, dya);
                const double rv = recession_violation(sum[3], lc, uc);
                const double fb = forbidden(dya, lc, uc);
                part[2] += e * e;                       // primal residual
                part[3] += bound_term(yt, lc, uc);      // dual objective: row terms
                part[4] += rv * rv;                     // primal ray: row violations
                part[5] += fb * fb;                     // dual ray: row violations
                part[6] += bound_term(dya, lc, uc);     // dual ray objective: row terms
                part[7] += dya * dya;                   // dual ray norm = distance_sq(y_t, y_anchor)
            }
        }
    }
    __device__ void store(int tile, const double *t) const {
        double *out = MODE == 2 ? s.partD : s.partD0;
#pragma unroll
        for (int q = 0; q < NP; ++q) out[tile * NP + q] = t[q];
    }
};

// ----------------------------------------------------------------------------------
// T: the check pass over A'ᵀ with y_t and y_t - y_anchor (always FP64).
struct CheckPassT {
    using VT = double;
    using ST = double;
    static constexpr int G = 2, NP = NP_T;
    static constexpr unsigned F32 = 0;
    const int *rp, *ci;
    const double *vals;
    const Tile *tiles;
    const uint16_t *sched;  // null: rows in order
    SolverPtrs s;
    int i;
    double inv_tau;

    __device__ bool setup() {
        if (s.st->done) return false;
        inv_tau = 1.0 / iter_scalars(s, i).tau;  // cpu lib.rs:235
        return true;
    }
    __device__ __forceinline__ void prod(int c, double v, double (&p)[2]) const {
        const double2 q = __ldg(s.pky + c);  // y_t and y_t - y_anchor, one sector
        p[0] = v * q.x;
        p[1] = v * q.y;
    }
    struct Pre {
        double lv, uv, df, c, aty, xt, x;
    };
    __device__ __forceinline__ Pre pre(int j) const {
        return Pre{__ldcs(s.lv + j), __ldcs(s.uv + j), __ldcs(s.df + j), __ldcs(s.c + j),
                   __ldcs(s.aty + j), __ldcs(s.xt + j), __ldcs(s.x + j)};
    }
    __device__ __forceinline__ void row(int j, const double (&sum)[2], double *part, const Pre &in) const {
        const double lv = in.lv, uv = in.uv, df = in.df;
        const double aty_t = sum[0];
        const double r = in.c - aty_t;
        const double f = forbidden(r, lv, uv) * df;
        const double sd = (in.aty - aty_t - (in.xt - in.x) * inv_tau) * df;
        const double ra = -sum[1];
        const double fa = forbidden(ra, lv, uv);
        part[0] += f * f;                   // dual residual
        part[1] += bound_term(r, lv, uv);   // dual objective: column terms
        part[2] += sd * sd;                 // step-implied dual residual
        part[3] += fa * fa;                 // dual ray: column violations
        part[4] += bound_term(ra, lv, uv);  // dual ray objective: column terms
    }
    __device__ void store(int tile, const double *t) const {
#pragma unroll
        for (int q = 0; q < NP; ++q) s.partT[tile * NP + q] = t[q];
    }
};

// ----------------------------------------------------------------------------------
// Power iteration on A'ᵀA' (solver.rs:215-242), device-resident.
struct PowerA {  // tmp = A' (v * s)
    using VT = double;
    using ST = double;
    static constexpr int G = 1, NP = 0;
    static constexpr unsigned F32 = 0;
    const int *rp, *ci;
    const double *vals;
    const Tile *tiles;
    const double *v;
    double *tmp;
    DevState *st;
    double scale;
    __device__ bool setup() {
        if (st->pi_done) return false;
        scale = st->pi_scale;
        return true;
    }
    struct Pre {};
    __device__ __forceinline__ Pre pre(int) const { return {}; }
    __device__ __forceinline__ void prod(int c, double val, double (&p)[1]) const {
        p[0] = val * (__ldg(v + c) * scale);  // the gather sees v after `scale(v, s)`
    }
    // the SELL path's view (sell.cuh): the gathered vector and the same product
    using GT = double;
    __device__ __forceinline__ const double *gvec() const { return v; }
    __device__ __forceinline__ double mul(double val, double g) const { return val * (g * scale); }
    __device__ __forceinline__ void row(int r, const double (&s)[1], double *, const Pre &) const { tmp[r] = s[0]; }
    __device__ void store(int, const double *) const {}
};

struct PowerT {  // v = A'ᵀ tmp, partial ‖v‖²
    using VT = double;
    using ST = double;
    static constexpr int G = 1, NP = 1;
    static constexpr unsigned F32 = 0;
    const int *rp, *ci;
    const double *vals;
    const Tile *tiles;
    const double *tmp;
    double *v;
    double *part;
    DevState *st;
    struct Pre {};
    __device__ bool setup() { return !st->pi_done; }
    __device__ __forceinline__ Pre pre(int) const { return {}; }
    __device__ __forceinline__ void prod(int c, double val, double (&p)[1]) const { p[0] = val * __ldg(tmp + c); }
    __device__ __forceinline__ void row(int r, const double (&s)[1], double *pp, const Pre &) const {
        v[r] = s[0];
        pp[0] += s[0] * s[0];
    }
    __device__ void store(int tile, const double *t) const { part[tile] = t[0]; }
};

template <bool PERSIST, class Op>
__device__ __forceinline__ bool try_run(Op &op, unsigned char *smem, int ntiles, int *ctr) {
    if (!op.setup()) return false;
    if constexpr (PERSIST) run_tiles(op, smem, ntiles, ctr);
    else tile_body(op, smem, blockIdx.x);
    return true;
}

// Whether a tile launch runs persistent CTAs (run_tiles) instead of one CTA per tile:
// measured on the 40M LP, the 4-product check pass (64 KB of staged products per tile)
// takes 0.65 ms with persistent CTAs against 1.22 ms with one CTA per tile, while the
// passes with one or two products run 5–17 % slower persistent (the loop costs them
// registers and occupancy).
template <class... Ops>
__host__ __device__ constexpr bool tiles_persistent() {
    return ((Ops::G >= 3) || ...);
}

// Runs the first of the passes whose setup() accepts this launch (the choice is
// uniform over the grid: it depends only on the device state).
template <class... Ops>
__global__ void __launch_bounds__(NT) k_tiles_any(int ntiles, int *ctr, Ops... ops) {
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr bool P = tiles_persistent<Ops...>();
    (void)(try_run<P>(ops, smem, ntiles, ctr) || ...);
    if constexpr (P) tiles_exit(ctr);
}

// Launches k_tiles_any over ntiles tiles: persistent CTAs on the grid of tile_grid, with
// ctr (two zeroed ints that only launches on stream st use), or one CTA per tile.
template <class... Ops>
void launch_tiles(int sms, int *ctr, int ntiles, size_t smem, cudaStream_t st, const Ops &...ops) {
    if constexpr (tiles_persistent<Ops...>()) {
        const unsigned g = tile_grid((const void *)&k_tiles_any<Ops...>, sms, ntiles, smem);
        k_tiles_any<Ops...><<<g, NT, smem, st>>>(ntiles, ctr, ops...);
    } else {
        k_tiles_any<Ops...><<<(unsigned)ntiles, NT, smem, st>>>(ntiles, nullptr, ops...);
    }
}

}  // namespace sp
