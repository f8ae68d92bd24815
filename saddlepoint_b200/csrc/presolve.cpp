// presolve.cpp — reductions of an LP before the PDHG solve, and the postsolve that maps
// the reduced problem's (x, y) back to the original problem.
//
// The reference has no presolve (cuPDLPx, which its benchmark compares against, has one:
// bench/README.md:1-6). These are the classic exact reductions, applied until none
// applies (at most 64 rounds):
//   * an empty row is dropped (its bounds must hold 0, else the LP is primal infeasible);
//   * a singleton row lc <= a·x_j <= uc becomes bounds on x_j and is dropped;
//   * a fixed column (lv = uv) is substituted: its contribution a·x_j moves into the row
//     bounds and c_j·x_j into the objective constant;
//   * an empty column is set to the bound its cost points at (the LP is dual infeasible if
//     that bound is infinite) and dropped.
// The problem is in the reference's minimisation form (LpProblem, problem.rs:129-145: c and
// c0 already negated for a maximisation, `maximize` only flips the reported objective), and
// the duals follow the solver's convention (y_i > 0 when lc_i is active, reduced costs
// r = c - Aᵀy, saddlepoint-check's lib.rs:59-61). Postsolve gives removed columns their
// values, empty rows y = 0, and a singleton row the part of its column's reduced cost that
// the bound it implied carries (rows undone in reverse order of removal, each row's dual
// entering the reduced costs of all its columns before the rows removed earlier), so the answer
// satisfies the original problem's KKT conditions as well as the reduced one did.
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/saddlepoint_b200.h"

namespace {

struct Singleton {
    int64_t row, col;
    double a;
    bool lower, upper;  // which bounds of the column this row tightened
};

}  // namespace

struct sp_presolve {
    int64_t m = 0, n = 0;
    std::vector<double> c;             // original costs (for the reduced costs of postsolve)
    std::vector<int64_t> row_ptr;      // original A in CSR
    std::vector<int32_t> col_idx;
    std::vector<double> values;
    std::vector<int64_t> row_new, col_new;  // original -> reduced index, -1 when removed
    std::vector<double> col_value;          // value of each removed column
    std::vector<Singleton> singles;         // in order of removal
    int64_t empty_rows = 0, singleton_rows = 0, fixed_cols = 0, empty_cols = 0;
    int status = -1;  // -1: solve the reduced LP; else the status presolve found
    // the reduced LP's arrays (sp_lp points into them)
    std::vector<int64_t> r_rp;
    std::vector<int32_t> r_ci;
    std::vector<double> r_v, r_c, r_lc, r_uc, r_lv, r_uv;
};

namespace {

// Whether lo <= v <= hi, with a rounding allowance relative to the bounds.
bool holds(double v, double lo, double hi) {
    const double tol = 1e-9 * (1.0 + std::fabs(v) + (std::isfinite(lo) ? std::fabs(lo) : 0.0) +
                               (std::isfinite(hi) ? std::fabs(hi) : 0.0));
    return v >= lo - tol && v <= hi + tol;
}

}  // namespace

extern "C" int sp_presolve_create(const sp_lp *lp, sp_lp *reduced, sp_presolve **out, int *status) {
    if (!lp || !reduced || !out || !status || !lp->a.row_ptr) return SP_ERR_INVALID;
    const int64_t m = lp->a.nrows, n = lp->a.ncols, nnz = lp->a.nnz;
    if (m < 0 || n < 0 || nnz < 0 || lp->a.row_ptr[m] != nnz) return SP_ERR_INVALID;
    auto *p = new sp_presolve();
    p->m = m;
    p->n = n;
    p->c.assign(lp->c, lp->c + n);
    p->row_ptr.assign(lp->a.row_ptr, lp->a.row_ptr + m + 1);
    p->col_idx.assign(lp->a.col_idx, lp->a.col_idx + nnz);
    p->values.assign(lp->a.values, lp->a.values + nnz);
    for (int64_t k = 0; k < nnz; ++k)
        if (p->col_idx[k] < 0 || p->col_idx[k] >= n) {
            delete p;
            return SP_ERR_INVALID;
        }
    std::vector<double> lc(lp->lc, lp->lc + m), uc(lp->uc, lp->uc + m), lv(lp->lv, lp->lv + n), uv(lp->uv, lp->uv + n);
    double c0 = lp->c0;
    // column-wise view for the column reductions
    std::vector<int64_t> cp(n + 1, 0);
    for (int64_t k = 0; k < nnz; ++k) cp[p->col_idx[k] + 1] += 1;
    for (int64_t j = 0; j < n; ++j) cp[j + 1] += cp[j];
    std::vector<int64_t> crow(nnz), cpos(nnz);
    {
        std::vector<int64_t> next(cp.begin(), cp.end() - 1);
        for (int64_t i = 0; i < m; ++i)
            for (int64_t k = p->row_ptr[i]; k < p->row_ptr[i + 1]; ++k) {
                const int64_t t = next[p->col_idx[k]]++;
                crow[t] = i;
                cpos[t] = k;
            }
    }
    std::vector<char> row_live(m, 1), col_live(n, 1);
    std::vector<int64_t> row_cnt(m), col_cnt(n);
    for (int64_t i = 0; i < m; ++i) row_cnt[i] = p->row_ptr[i + 1] - p->row_ptr[i];
    for (int64_t j = 0; j < n; ++j) col_cnt[j] = cp[j + 1] - cp[j];
    // explicit zeros do not count as entries
    for (int64_t i = 0; i < m; ++i)
        for (int64_t k = p->row_ptr[i]; k < p->row_ptr[i + 1]; ++k)
            if (p->values[k] == 0.0) {
                row_cnt[i] -= 1;
                col_cnt[p->col_idx[k]] -= 1;
            }
    p->col_value.assign(n, 0.0);
    int st = -1;
    auto drop_col = [&](int64_t j, double x) {
        col_live[j] = 0;
        p->col_value[j] = x;
        c0 += p->c[j] * x;
        for (int64_t t = cp[j]; t < cp[j + 1]; ++t) {
            const int64_t i = crow[t];
            const double a = p->values[cpos[t]];
            if (!row_live[i] || a == 0.0) continue;
            if (std::isfinite(lc[i])) lc[i] -= a * x;
            if (std::isfinite(uc[i])) uc[i] -= a * x;
            row_cnt[i] -= 1;
        }
    };
    for (int round = 0; round < 64 && st < 0; ++round) {
        bool changed = false;
        for (int64_t i = 0; i < m && st < 0; ++i) {
            if (!row_live[i]) continue;
            if (row_cnt[i] == 0) {  // empty row
                if (!holds(0.0, lc[i], uc[i])) st = SP_STATUS_PRIMAL_INFEASIBLE;
                row_live[i] = 0;
                p->empty_rows += 1;
                changed = true;
            } else if (row_cnt[i] == 1) {  // singleton row: bounds on its column
                int64_t j = -1;
                double a = 0.0;
                for (int64_t k = p->row_ptr[i]; k < p->row_ptr[i + 1]; ++k)
                    if (col_live[p->col_idx[k]] && p->values[k] != 0.0) {
                        j = p->col_idx[k];
                        a = p->values[k];
                    }
                double lo = a > 0 ? lc[i] / a : uc[i] / a, hi = a > 0 ? uc[i] / a : lc[i] / a;
                if (!std::isfinite(lo)) lo = -INFINITY;
                if (!std::isfinite(hi)) hi = INFINITY;
                Singleton s{i, j, a, lo > lv[j], hi < uv[j]};
                if (s.lower) lv[j] = lo;
                if (s.upper) uv[j] = hi;
                if (lv[j] > uv[j]) {
                    if (holds(lv[j], uv[j], uv[j])) lv[j] = uv[j];  // equal up to rounding
                    else st = SP_STATUS_PRIMAL_INFEASIBLE;
                }
                p->singles.push_back(s);
                row_live[i] = 0;
                col_cnt[j] -= 1;
                p->singleton_rows += 1;
                changed = true;
            }
        }
        for (int64_t j = 0; j < n && st < 0; ++j) {
            if (!col_live[j]) continue;
            if (lv[j] == uv[j] && std::isfinite(lv[j])) {  // fixed column
                drop_col(j, lv[j]);
                p->fixed_cols += 1;
                changed = true;
            } else if (col_cnt[j] == 0) {  // empty column: its cost picks the bound
                const double cj = p->c[j];
                double x;
                if (cj > 0.0) x = lv[j];
                else if (cj < 0.0) x = uv[j];
                else x = std::fmin(std::fmax(0.0, lv[j]), uv[j]);
                if (!std::isfinite(x)) {
                    st = SP_STATUS_DUAL_INFEASIBLE;
                    break;
                }
                drop_col(j, x);
                p->empty_cols += 1;
                changed = true;
            }
        }
        if (!changed) break;
    }
    // the reduced LP: live rows and columns, entries in the original order
    p->row_new.assign(m, -1);
    p->col_new.assign(n, -1);
    int64_t mr = 0, nr = 0;
    for (int64_t i = 0; i < m; ++i)
        if (row_live[i]) p->row_new[i] = mr++;
    for (int64_t j = 0; j < n; ++j)
        if (col_live[j]) p->col_new[j] = nr++;
    p->r_rp.assign(1, 0);
    for (int64_t i = 0; i < m; ++i) {
        if (!row_live[i]) continue;
        for (int64_t k = p->row_ptr[i]; k < p->row_ptr[i + 1]; ++k) {
            const int64_t j = p->col_idx[k];
            if (!col_live[j] || p->values[k] == 0.0) continue;
            p->r_ci.push_back((int32_t)p->col_new[j]);
            p->r_v.push_back(p->values[k]);
        }
        p->r_rp.push_back((int64_t)p->r_v.size());
        p->r_lc.push_back(lc[i]);
        p->r_uc.push_back(uc[i]);
    }
    for (int64_t j = 0; j < n; ++j) {
        if (!col_live[j]) continue;
        p->r_c.push_back(p->c[j]);
        p->r_lv.push_back(lv[j]);
        p->r_uv.push_back(uv[j]);
    }
    if (st < 0 && nr == 0) st = SP_STATUS_OPTIMAL;  // every column fixed: nothing left to solve
    p->status = st;
    for (auto *v : {&p->r_v, &p->r_c, &p->r_lc, &p->r_uc, &p->r_lv, &p->r_uv}) v->reserve(1);
    p->r_ci.reserve(1);
    memset(reduced, 0, sizeof *reduced);
    reduced->a.nrows = mr;
    reduced->a.ncols = nr;
    reduced->a.nnz = (int64_t)p->r_v.size();
    reduced->a.row_ptr = p->r_rp.data();
    reduced->a.col_idx = p->r_ci.data();
    reduced->a.values = p->r_v.data();
    reduced->c = p->r_c.data();
    reduced->lc = p->r_lc.data();
    reduced->uc = p->r_uc.data();
    reduced->lv = p->r_lv.data();
    reduced->uv = p->r_uv.data();
    reduced->c0 = c0;
    reduced->maximize = lp->maximize;
    *status = st;
    *out = p;
    return SP_OK;
}

extern "C" int sp_presolve_postsolve(const sp_presolve *p, const double *x_red, const double *y_red, double *x,
                                     double *y) {
    if (!p || !x || !y) return SP_ERR_INVALID;
    const int64_t m = p->m, n = p->n;
    int64_t nr = 0, mr = 0;
    for (int64_t j = 0; j < n; ++j) nr += p->col_new[j] >= 0;
    for (int64_t i = 0; i < m; ++i) mr += p->row_new[i] >= 0;
    if ((nr > 0 && !x_red) || (mr > 0 && !y_red)) return SP_ERR_INVALID;
    for (int64_t j = 0; j < n; ++j) x[j] = p->col_new[j] >= 0 ? x_red[p->col_new[j]] : p->col_value[j];
    for (int64_t i = 0; i < m; ++i) y[i] = p->row_new[i] >= 0 ? y_red[p->row_new[i]] : 0.0;
    if (p->singles.empty()) return SP_OK;
    // reduced costs r = c - Aᵀy over the rows kept so far, then the singleton rows undone
    // in reverse order of removal, each taking the part of r_j its implied bound carries
    std::vector<double> r(p->c);
    for (int64_t i = 0; i < m; ++i) {
        if (p->row_new[i] < 0 || y[i] == 0.0) continue;
        for (int64_t k = p->row_ptr[i]; k < p->row_ptr[i + 1]; ++k) r[p->col_idx[k]] -= p->values[k] * y[i];
    }
    // (a row's dual enters the reduced cost of every column of the row, the columns
    // removed before it became a singleton included)
    for (auto it = p->singles.rbegin(); it != p->singles.rend(); ++it) {
        const int64_t j = it->col, i = it->row;
        double yi = 0.0;
        if ((r[j] > 0.0 && it->lower) || (r[j] < 0.0 && it->upper)) yi = r[j] / it->a;
        y[i] = yi;
        if (yi != 0.0)
            for (int64_t k = p->row_ptr[i]; k < p->row_ptr[i + 1]; ++k) r[p->col_idx[k]] -= p->values[k] * yi;
    }
    return SP_OK;
}

extern "C" int sp_presolve_counts(const sp_presolve *p, int64_t counts[4]) {
    if (!p || !counts) return SP_ERR_INVALID;
    counts[0] = p->empty_rows;
    counts[1] = p->singleton_rows;
    counts[2] = p->fixed_cols;
    counts[3] = p->empty_cols;
    return SP_OK;
}

extern "C" void sp_presolve_free(sp_presolve *p) { delete p; }
