// polish.cpp — feasibility polishing after a solve (Part 6 of the C ABI).
//
// A PDHG answer at tolerance ε has primal and dual residuals of order ε. cuPDLPx, which
// the reference's benchmark compares against (bench/README.md:1-6), polishes such an answer
// into one that is feasible to a much tighter tolerance. This is the same idea built on
// this library's device-resident solve with a warm start:
//   * primal: the feasibility problem (the LP's constraints and bounds, zero cost) started
//     from (x, 0) — its optimal set is the LP's feasible set, so the solve moves x to a
//     nearby point that is feasible to the tolerance;
//   * dual: the LP with every finite bound set to zero (infinite ones kept) started from
//     (0, y) — a bound's finiteness alone decides which signs the duals and reduced costs
//     may take, so this problem has the LP's dual feasible set and a zero dual objective,
//     and the solve moves y to a nearby dual-feasible point.
// Both solves run in FP64 with the caller's parameters otherwise. The residuals of the
// polished pair fall to the polishing tolerance; its objective gap moves by the size of the
// steps, which is of the order of the original residuals (measured on Netlib from 1e-4
// answers: 1.1 to 70 times the original relative gap). Solving without restarts, so that
// the Halpern anchor stays at the start and the step is the shortest in the PDHG metric,
// kept the gap lower on some LPs but took up to 1M iterations (seconds instead of
// milliseconds), so the solves keep the restart rules.
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/saddlepoint_b200.h"

namespace {

// One warm-started device solve of `lp` from (x0, y0); the answer into (x, y).
int solve_from(sp_ctx *ctx, const sp_lp *lp, const sp_solver_params &p, const double *x0, const double *y0,
               double *x, double *y, uint64_t *iterations) {
    sp_solver *s = nullptr;
    int rc = sp_solver_create(ctx, lp, &p, &s);
    if (rc) return rc;
    sp_solution_info info{};
    if (!(rc = sp_solver_warm_start(s, x0, y0)) && !(rc = sp_solver_solve(s, &info)))
        rc = sp_solver_download(s, x, y);
    if (!rc && iterations) *iterations = info.iterations;
    sp_solver_free(s);
    return rc;
}

}  // namespace

extern "C" int sp_polish(sp_ctx *ctx, const sp_lp *lp, const sp_solver_params *params, double tolerance, double *x,
                         double *y, uint64_t iterations[2]) {
    if (!ctx || !lp || !x || !y || !(tolerance > 0.0)) return SP_ERR_INVALID;
    const int64_t m = lp->a.nrows, n = lp->a.ncols;
    sp_solver_params p;
    sp_solver_params_default(&p);
    if (params) p = *params;
    p.tolerance = tolerance;
    p.precision = SP_PRECISION_FP64;
    // primal: zero cost, the same constraints and bounds, from (x, 0)
    std::vector<double> zero_c(std::max<int64_t>(n, 1), 0.0);
    sp_lp primal = *lp;
    primal.c = zero_c.data();
    primal.c0 = 0.0;
    std::vector<double> xp(std::max<int64_t>(n, 1)), yp(std::max<int64_t>(m, 1));
    uint64_t it[2] = {0, 0};
    int rc = solve_from(ctx, &primal, p, x, nullptr, xp.data(), yp.data(), &it[0]);
    if (rc) return rc;
    // dual: every finite bound at zero, from (0, y)
    auto zeroed = [](const double *v, int64_t k) {
        std::vector<double> out(std::max<int64_t>(k, 1));
        for (int64_t i = 0; i < k; ++i) out[i] = std::isfinite(v[i]) ? 0.0 : v[i];
        return out;
    };
    std::vector<double> lc = zeroed(lp->lc, m), uc = zeroed(lp->uc, m), lv = zeroed(lp->lv, n), uv = zeroed(lp->uv, n);
    sp_lp dual = *lp;
    dual.lc = lc.data();
    dual.uc = uc.data();
    dual.lv = lv.data();
    dual.uv = uv.data();
    std::vector<double> xd(std::max<int64_t>(n, 1)), yd(std::max<int64_t>(m, 1));
    if ((rc = solve_from(ctx, &dual, p, nullptr, y, xd.data(), yd.data(), &it[1]))) return rc;
    if (n) memcpy(x, xp.data(), sizeof(double) * n);
    if (m) memcpy(y, yd.data(), sizeof(double) * m);
    if (iterations) {
        iterations[0] = it[0];
        iterations[1] = it[1];
    }
    return SP_OK;
}
