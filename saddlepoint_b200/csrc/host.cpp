// host.cpp — host-side parts of the library:
//   * sp_solve_stepwise: the reference's solver loop (crates/saddlepoint-core/src/solver.rs:311-438)
//     driven over the Part 1 entry points only, as a Rust host drives a Backend;
//   * the seeded synthetic LP generators.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/saddlepoint_b200.h"

namespace {

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// ===================================================================== stepwise solve

struct Vecs {
    sp_ctx *ctx;
    std::vector<sp_vec *> all;
    ~Vecs() {
        for (sp_vec *v : all) sp_vec_free(v);
    }
    int make(const std::vector<double> &h, sp_vec **out) {
        int rc = sp_vec_upload(ctx, h.data(), (int64_t)h.size(), out);
        if (!rc) all.push_back(*out);
        return rc;
    }
};

#define TRY(x)              \
    do {                    \
        int _rc = (x);      \
        if (_rc) return _rc; \
    } while (0)

double seq_norm2(const double *v, int64_t n) {  // scaling.rs:186-188
    double s = -0.0;
    for (int64_t i = 0; i < n; ++i) s += v[i] * v[i];
    return std::sqrt(s);
}
double seq_finite_bound_norm(const double *lo, const double *hi, int64_t n) {  // scaling.rs:191-201
    double s = -0.0;
    for (int64_t i = 0; i < n; ++i) {
        const double l = std::isfinite(lo[i]) ? lo[i] : 0.0, u = std::isfinite(hi[i]) ? hi[i] : 0.0;
        s += (l == u) ? l * l : l * l + u * u;
    }
    return std::sqrt(s);
}

struct Pid {  // PidState (solver.rs:445-480)
    double integral = 0, prev_error = 0, best_weight, best_balance = INFINITY;
    bool has_prev = false;
    explicit Pid(double omega) : best_weight(omega) {}
    double update(const sp_solver_params &p, double omega, double dx, double dy, double rel_primal, double rel_dual) {
        auto sane = [](double v) { return v >= 1e-16 && v <= 1e12; };
        const double ratio = rel_dual / rel_primal;
        if (!sane(dx) || !sane(dy) || !(ratio >= 1e-8 && ratio <= 1e8)) {
            integral = 0.0;
            has_prev = false;
            return best_weight;
        }
        const double e = std::log(omega * dx / dy);
        integral = p.pid_discount * integral + e;
        const double derivative = has_prev ? e - prev_error : 0.0;
        prev_error = e;
        has_prev = true;
        const double next = std::exp(std::log(omega) - (p.pid_kp * e + p.pid_ki * integral + p.pid_kd * derivative));
        const double balance = std::fabs(std::log10(ratio));
        if (balance < best_balance) {
            best_balance = balance;
            best_weight = next;
        }
        return next;
    }
};

struct Kkt {
    double primal_obj = 0, dual_obj = 0, primal_res = 0, dual_res = 0;
    double gap() const { return std::fabs(primal_obj - dual_obj); }
    bool converged(double eps, double b, double c) const {  // solver.rs:147-151
        return primal_res <= eps * (1.0 + b) && dual_res <= eps * (1.0 + c) &&
               gap() <= eps * (1.0 + std::fabs(primal_obj) + std::fabs(dual_obj));
    }
};

int stepwise(sp_ctx *ctx, const sp_lp *lp, const sp_solver_params &p, double *x_out, double *y_out,
             sp_solution_info *info) {
    const int64_t m = lp->a.nrows, n = lp->a.ncols, nnz = lp->a.nnz;
    const double t_setup = now_s();
    // ScaledProblem::new: the scaling passes run on the device and the scaled
    // problem is downloaded, which is what a Rust host hands to Backend::load.
    sp_solver_params sp = p;
    sp.precision = SP_PRECISION_FP64;
    sp.power_iterations = 0;
    sp_solver *s = nullptr;
    TRY(sp_solver_create(ctx, lp, &sp, &s));
    std::vector<int64_t> arp(m + 1), trp(n + 1);
    std::vector<int32_t> aci(nnz), tci(nnz);
    std::vector<double> av(nnz), tv(nnz), c(n), lc(m), uc(m), lv(n), uv(n), rs(m), cs(n);
    double bs = 1, os = 1;
    int rc = sp_solver_scaled(s, arp.data(), aci.data(), av.data(), trp.data(), tci.data(), tv.data(), c.data(),
                              lc.data(), uc.data(), lv.data(), uv.data(), rs.data(), cs.data(), &bs, &os);
    sp_solver_free(s);
    if (rc) return rc;
    std::vector<double> pf(m), df(n);
    for (int64_t i = 0; i < m; ++i) pf[i] = 1.0 / (rs[i] * bs);  // scaling.rs:124-126
    for (int64_t j = 0; j < n; ++j) df[j] = 1.0 / (cs[j] * os);  // scaling.rs:129-131
    const double obj_factor = 1.0 / (bs * os);
    sp_csr A{m, n, nnz, arp.data(), aci.data(), av.data()};
    sp_csr AT{n, m, nnz, trp.data(), tci.data(), tv.data()};
    sp_problem *dev = nullptr;
    TRY(sp_problem_load(ctx, &A, &AT, c.data(), lc.data(), uc.data(), lv.data(), uv.data(), pf.data(), df.data(), &dev));
    struct Free {
        sp_problem *p;
        ~Free() { sp_problem_free(p); }
    } free_dev{dev};

    // Solver::new (solver.rs:185-212)
    Vecs V{ctx, {}};
    const std::vector<double> zn(n, 0.0), zm(m, 0.0);
    sp_vec *x, *y, *x_t, *y_t, *x_bar, *x_anchor, *y_anchor, *ax, *aty, *tmp_n, *tmp_m, *tmp_m2, *cv;
    TRY(V.make(zn, &x));
    TRY(V.make(zm, &y));
    TRY(V.make(zn, &x_t));
    TRY(V.make(zm, &y_t));
    TRY(V.make(zn, &x_bar));
    TRY(V.make(zn, &x_anchor));
    TRY(V.make(zm, &y_anchor));
    TRY(V.make(zm, &ax));
    TRY(V.make(zn, &aty));
    TRY(V.make(zn, &tmp_n));
    TRY(V.make(zm, &tmp_m));
    TRY(V.make(zm, &tmp_m2));
    TRY(V.make(c, &cv));
    const double setup_s = now_s() - t_setup;

    const double start = now_s();
    // estimate_norm (solver.rs:215-242)
    double norm_est = 1.0;
    if (n > 0 && nnz > 0) {
        std::vector<double> st(n);
        for (int64_t j = 0; j < n; ++j) st[j] = 1.0 + 0.01 * (double)(j % 7);
        sp_vec *v;
        TRY(V.make(st, &v));
        double ns;
        TRY(sp_norm_sq(ctx, v, &ns));
        TRY(sp_scale(ctx, v, 1.0 / std::sqrt(ns)));
        double lambda = 0.0;
        for (uint64_t it = 0; it < p.power_iterations; ++it) {
            TRY(sp_spmv(ctx, dev, v, tmp_m));
            TRY(sp_spmv_t(ctx, dev, tmp_m, v));
            TRY(sp_norm_sq(ctx, v, &ns));
            const double norm = std::sqrt(ns);
            if (std::isnan(norm) || norm <= 0.0 || std::isinf(norm)) return SP_ERR_NUMERICAL;
            TRY(sp_scale(ctx, v, 1.0 / norm));
            const bool done = std::fabs(norm - lambda) <= 1e-6 * norm;
            lambda = norm;
            if (done) break;
        }
        norm_est = std::sqrt(lambda) * 1.01;
    }
    // run (solver.rs:311-438)
    const double eta = p.step_size_factor / norm_est;
    const double b_norm = seq_finite_bound_norm(lp->lc, lp->uc, m);
    const double c_norm = seq_norm2(lp->c, n);
    double omega = p.bound_objective_rescaling ? 1.0 : (1.0 + c_norm) / (1.0 + b_norm);
    Pid pid(omega);
    uint64_t total = 0, k = 0, restarts = 0;
    double anchor_residual = INFINITY, prev_residual = INFINITY;
    int status = -1;
    Kkt kkt;
    for (;;) {
        const double tau = eta / omega, sigma = eta * omega;
        TRY(sp_spmv_t(ctx, dev, y, aty));
        TRY(sp_primal_step(ctx, dev, x, aty, tau, x_t, x_bar));
        TRY(sp_spmv(ctx, dev, x_bar, ax));
        TRY(sp_dual_step(ctx, dev, y, ax, sigma, y_t));
        total += 1;
        const bool check = (p.check_every != 0 && total % p.check_every == 0) || total >= p.max_iterations;
        double residual = 0.0;
        if (check || k == 0) {  // fixed_point_residual (solver.rs:275-288)
            TRY(sp_sub(ctx, x_t, x, tmp_n));
            TRY(sp_sub(ctx, y_t, y, tmp_m2));
            TRY(sp_spmv(ctx, dev, tmp_n, tmp_m));
            double dx2, dy2, cross;
            TRY(sp_norm_sq(ctx, tmp_n, &dx2));
            TRY(sp_norm_sq(ctx, tmp_m2, &dy2));
            TRY(sp_dot(ctx, tmp_m2, tmp_m, &cross));
            const double r2 = omega / eta * dx2 + dy2 / (eta * omega) + 2.0 * cross;
            if (!std::isfinite(r2)) return SP_ERR_NUMERICAL;
            residual = std::sqrt(std::max(r2, 0.0));
        }
        if (k == 0) anchor_residual = residual;
        double step_dual = 0.0, step_obj = 0.0;
        if (check) {  // kkt (solver.rs:245-258)
            sp_primal_stats_t ps;
            sp_dual_stats_t ds;
            TRY(sp_spmv(ctx, dev, x_t, tmp_m));
            TRY(sp_primal_stats(ctx, dev, x_t, tmp_m, &ps));
            TRY(sp_spmv_t(ctx, dev, y_t, tmp_n));
            TRY(sp_dual_stats(ctx, dev, y_t, tmp_n, &ds));
            kkt.primal_obj = ps.objective * obj_factor + lp->c0;
            kkt.dual_obj = ds.objective * obj_factor + lp->c0;
            kkt.primal_res = std::sqrt(ps.residual_sq);
            kkt.dual_res = std::sqrt(ds.residual_sq);
            double sd;
            TRY(sp_step_dual_residual_sq(ctx, dev, x, x_t, aty, tmp_n, tau, &sd));
            step_dual = std::sqrt(sd);
            if (p.termination == SP_TERMINATION_STEP_IMPLIED) {  // step_dual_objective (solver.rs:263-271)
                sp_dual_stats_t rows;
                TRY(sp_dual_stats(ctx, dev, y_t, cv, &rows));
                double d1, d2, d3, d4;
                TRY(sp_dot(ctx, cv, x_t, &d1));
                TRY(sp_dot(ctx, aty, x_t, &d2));
                TRY(sp_dot(ctx, x_t, x_t, &d3));
                TRY(sp_dot(ctx, x, x_t, &d4));
                step_obj = (rows.objective + (d1 - d2 + (d3 - d4) / tau)) * obj_factor + lp->c0;
            }
        }
        const double w = (double)(k + 1) / (double)(k + 2);
        TRY(sp_halpern_step(ctx, x, x_t, x_anchor, w, p.reflection));
        TRY(sp_halpern_step(ctx, y, y_t, y_anchor, w, p.reflection));
        k += 1;
        if (!check) continue;
        Kkt test = kkt;
        if (p.termination == SP_TERMINATION_STEP_IMPLIED) {
            test.dual_obj = step_obj;
            test.dual_res = step_dual;
        }
        if (test.converged(p.tolerance, b_norm, c_norm)) {
            status = SP_STATUS_OPTIMAL;
            break;
        }
        // infeasibility (solver.rs:291-309)
        const double eps = p.infeasibility_tolerance;
        sp_ray_stats_t d, pr;
        TRY(sp_sub(ctx, y_t, y_anchor, tmp_m));
        TRY(sp_spmv_t(ctx, dev, tmp_m, tmp_n));
        TRY(sp_dual_ray_stats(ctx, dev, tmp_m, tmp_n, &d));
        if (d.objective > 0.0 && std::sqrt(d.violation_sq) <= eps * d.objective &&
            d.objective > eps * std::sqrt(d.norm_sq)) {
            status = SP_STATUS_PRIMAL_INFEASIBLE;
            break;
        }
        TRY(sp_sub(ctx, x_t, x_anchor, tmp_n));
        TRY(sp_spmv(ctx, dev, tmp_n, tmp_m));
        TRY(sp_primal_ray_stats(ctx, dev, tmp_n, tmp_m, &pr));
        if (pr.objective < 0.0 && std::sqrt(pr.violation_sq) <= -eps * pr.objective &&
            -pr.objective > eps * std::sqrt(pr.norm_sq)) {
            status = SP_STATUS_DUAL_INFEASIBLE;
            break;
        }
        if (total >= p.max_iterations) {
            status = SP_STATUS_ITERATION_LIMIT;
            break;
        }
        if (p.time_limit_s > 0 && now_s() - start >= p.time_limit_s) {
            status = SP_STATUS_TIME_LIMIT;
            break;
        }
        const double r0 = anchor_residual;
        const bool restart = residual <= p.restart_sufficient * r0 ||
                             (residual <= p.restart_necessary * r0 && residual > prev_residual) ||
                             (double)k >= p.restart_artificial * (double)total;
        prev_residual = residual;
        if (restart) {
            double dx, dy;
            TRY(sp_distance_sq(ctx, x_t, x_anchor, &dx));
            TRY(sp_distance_sq(ctx, y_t, y_anchor, &dy));
            omega = pid.update(p, omega, std::sqrt(dx), std::sqrt(dy), kkt.primal_res / (1.0 + b_norm),
                               step_dual / (1.0 + c_norm));
            TRY(sp_vec_copy(ctx, x_t, x_anchor));
            TRY(sp_vec_copy(ctx, y_t, y_anchor));
            TRY(sp_vec_copy(ctx, x_t, x));
            TRY(sp_vec_copy(ctx, y_t, y));
            k = 0;
            restarts += 1;
            prev_residual = INFINITY;
        }
    }
    // Solution (solver.rs:422-437)
    std::vector<double> hx(n), hy(m);
    TRY(sp_vec_download(ctx, x_t, hx.data(), n));
    TRY(sp_vec_download(ctx, y_t, hy.data(), m));
    if (x_out)
        for (int64_t j = 0; j < n; ++j) x_out[j] = hx[j] * cs[j] / bs;
    if (y_out)
        for (int64_t i = 0; i < m; ++i) y_out[i] = hy[i] * rs[i] / os;
    if (info) {
        const double sign = lp->maximize ? -1.0 : 1.0;
        info->status = status;
        info->objective = sign * kkt.primal_obj;
        info->dual_objective = sign * kkt.dual_obj;
        info->primal_residual = kkt.primal_res;
        info->dual_residual = kkt.dual_res;
        info->gap = kkt.gap();
        info->iterations = total;
        info->restarts = restarts;
        info->solve_time_s = now_s() - start;
        info->setup_time_s = setup_s;
        info->norm_estimate = norm_est;
        info->fp64_from_iteration = 0;
    }
    return SP_OK;
}

// ===================================================================== generators

// xorshift64 (crates/saddlepoint-cuda/examples/speedup.rs:22-34), one stream per
// column (and per row), each seeded by splitmix64 so columns generate in parallel.
struct Rng {
    uint64_t s;
    explicit Rng(uint64_t seed) : s(seed ? seed : 0x2545F4914F6CDD1Dull) {}
    uint64_t next() {
        s ^= s << 13;
        s ^= s >> 7;
        s ^= s << 17;
        return s;
    }
    double unit() { return (double)(next() >> 11) / (double)(1ull << 53); }
    double normal() {  // Box-Muller, first of the pair
        const double u1 = 1.0 - unit(), u2 = unit();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
    uint64_t below(uint64_t n) { return next() % n; }
};

uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
enum : uint64_t { FAMILY_COL = 1, FAMILY_ROW = 2, FAMILY_GLOBAL = 3 };
Rng stream(uint64_t seed, uint64_t family, uint64_t index) {
    return Rng(splitmix64(seed ^ splitmix64(family * 0x100000001B3ull + index)));
}

struct Owned {  // host arrays behind a generated sp_lp
    std::vector<int64_t> rp;
    std::vector<int32_t> ci;
    std::vector<double> v, c, lc, uc, lv, uv;
};

void parallel_for(int64_t n, const std::function<void(int64_t, int64_t)> &f);

// Column-major entries -> CSR with columns ascending in each row.
void csc_to_csr(int64_t m, int64_t n, const std::vector<int64_t> &cp, const std::vector<int32_t> &ri,
                const std::vector<double> &vals, Owned &o) {
    const int64_t nnz = cp[n];
    o.rp.assign(m + 1, 0);
    for (int64_t k = 0; k < nnz; ++k) o.rp[ri[k] + 1] += 1;
    for (int64_t i = 0; i < m; ++i) o.rp[i + 1] += o.rp[i];
    std::vector<int64_t> next(o.rp.begin(), o.rp.end() - 1);
    o.ci.resize(nnz);
    o.v.resize(nnz);
    for (int64_t j = 0; j < n; ++j)
        for (int64_t k = cp[j]; k < cp[j + 1]; ++k) {
            const int64_t t = next[ri[k]]++;
            o.ci[t] = (int32_t)j;
            o.v[t] = vals[k];
        }
}

// Draws `d` distinct rows in [0, m) from `r` (rejection; d is small against m).
void distinct_rows(Rng &r, int64_t d, int64_t m, int32_t *out) {
    for (int64_t q = 0; q < d; ++q) {
        for (;;) {
            const int32_t cand = (int32_t)r.below((uint64_t)m);
            bool dup = false;
            for (int64_t t = 0; t < q; ++t)
                if (out[t] == cand) {
                    dup = true;
                    break;
                }
            if (!dup) {
                out[q] = cand;
                break;
            }
        }
    }
}

// Rows, bounds and cost as the random LP recipe: x0 ~ U[0,1]^n, the first m/2 rows
// equalities A x0, the rest A x0 + U[0,1] upper bounds; 0 <= x <= 10; c ~ U[-1,1].
void finish_random_lp(uint64_t seed, int64_t m, int64_t n, const std::vector<double> &x0, Owned &o) {
    std::vector<double> b(m);
    parallel_for(m, [&](int64_t lo, int64_t hi) {
        for (int64_t i = lo; i < hi; ++i) {
            double s = -0.0;
            for (int64_t k = o.rp[i]; k < o.rp[i + 1]; ++k) s += o.v[k] * x0[o.ci[k]];
            b[i] = s;
        }
    });
    o.lc.resize(m);
    o.uc.resize(m);
    for (int64_t i = 0; i < m; ++i) {
        if (i < m / 2) {
            o.lc[i] = o.uc[i] = b[i];
        } else {
            Rng r = stream(seed, FAMILY_ROW, (uint64_t)i);
            o.lc[i] = -INFINITY;
            o.uc[i] = b[i] + r.unit();
        }
    }
    o.lv.assign(n, 0.0);
    o.uv.assign(n, 10.0);
}

int gen_random(const sp_gen_params &g, Owned &o) {
    const int64_t m = g.nrows, n = g.ncols;
    const int64_t dmin = std::max<int64_t>(1, g.nnz_per_col_min), dmax = std::max(dmin, g.nnz_per_col_max);
    if (m <= 0 || n <= 0 || dmax > m) return SP_ERR_INVALID;
    std::vector<int64_t> deg(n);
    std::vector<Rng> rngs;
    rngs.reserve(n);
    for (int64_t j = 0; j < n; ++j) {
        rngs.push_back(stream(g.seed, FAMILY_COL, (uint64_t)j));
        deg[j] = dmin + (int64_t)rngs[j].below((uint64_t)(dmax - dmin + 1));
    }
    std::vector<int64_t> cp(n + 1, 0);
    for (int64_t j = 0; j < n; ++j) cp[j + 1] = cp[j] + deg[j];
    std::vector<int32_t> ri(cp[n]);
    std::vector<double> vals(cp[n]), x0(n);
    o.c.resize(n);
    parallel_for(n, [&](int64_t lo, int64_t hi) {
        for (int64_t j = lo; j < hi; ++j) {
            Rng &r = rngs[j];
            distinct_rows(r, deg[j], m, &ri[cp[j]]);
            for (int64_t k = cp[j]; k < cp[j + 1]; ++k) vals[k] = r.normal();
            x0[j] = r.unit();
            o.c[j] = 2.0 * r.unit() - 1.0;
        }
    });
    csc_to_csr(m, n, cp, ri, vals, o);
    finish_random_lp(g.seed, m, n, x0, o);
    return SP_OK;
}

// Power-law column degrees: d_j drawn from a Zipf(s) law truncated to
// [degree_min, degree_max], then rescaled by one factor f so that the total is
// target_nnz: d_j <- max(degree_min, floor(d_j f)), the remainder added one by one
// to the first columns (in index order) that stay within the bounds.
int gen_powerlaw(const sp_gen_params &g, Owned &o) {
    const int64_t m = g.nrows, n = g.ncols, dmin = g.degree_min, dmax = std::min<int64_t>(g.degree_max, m);
    if (m <= 0 || n <= 0 || dmin < 1 || dmax < dmin || g.target_nnz < n * dmin || g.target_nnz > n * dmax)
        return SP_ERR_INVALID;
    std::vector<double> cdf(dmax - dmin + 1);
    double acc = 0.0;
    for (int64_t d = dmin; d <= dmax; ++d) {
        acc += std::pow((double)d, -g.zipf_s);
        cdf[d - dmin] = acc;
    }
    for (double &v : cdf) v /= acc;
    std::vector<Rng> rngs;
    rngs.reserve(n);
    std::vector<int64_t> raw(n);
    for (int64_t j = 0; j < n; ++j) {
        rngs.push_back(stream(g.seed, FAMILY_COL, (uint64_t)j));
        const double u = rngs[j].unit();
        raw[j] = dmin + (int64_t)(std::lower_bound(cdf.begin(), cdf.end(), u) - cdf.begin());
        if (raw[j] > dmax) raw[j] = dmax;
    }
    auto total_for = [&](double f) {
        int64_t t = 0;
        for (int64_t j = 0; j < n; ++j) t += std::min(dmax, std::max(dmin, (int64_t)std::floor((double)raw[j] * f)));
        return t;
    };
    double lo = 0.0, hi = 1.0;
    while (total_for(hi) < g.target_nnz && hi < 1e9) hi *= 2.0;
    for (int it = 0; it < 100; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (total_for(mid) <= g.target_nnz) lo = mid;
        else hi = mid;
    }
    std::vector<int64_t> deg(n);
    int64_t sum = 0;
    for (int64_t j = 0; j < n; ++j) {
        deg[j] = std::min(dmax, std::max(dmin, (int64_t)std::floor((double)raw[j] * lo)));
        sum += deg[j];
    }
    for (int64_t pass = 0; sum < g.target_nnz && pass < dmax; ++pass)
        for (int64_t j = 0; j < n && sum < g.target_nnz; ++j)
            if (deg[j] < dmax) {
                deg[j] += 1;
                sum += 1;
            }
    std::vector<int64_t> cp(n + 1, 0);
    for (int64_t j = 0; j < n; ++j) cp[j + 1] = cp[j] + deg[j];
    std::vector<int32_t> ri(cp[n]);
    std::vector<double> vals(cp[n]), x0(n);
    o.c.resize(n);
    parallel_for(n, [&](int64_t a, int64_t b) {
        std::vector<int32_t> seen;
        for (int64_t j = a; j < b; ++j) {
            Rng &r = rngs[j];
            const int64_t d = deg[j];
            if (d <= 32) {
                distinct_rows(r, d, m, &ri[cp[j]]);
            } else {  // draw, then redraw duplicates found by sorting a copy
                int32_t *out = &ri[cp[j]];
                for (int64_t q = 0; q < d; ++q) out[q] = (int32_t)r.below((uint64_t)m);
                for (;;) {
                    seen.assign(out, out + d);
                    std::sort(seen.begin(), seen.end());
                    bool dup = false;
                    for (int64_t q = 1; q < d; ++q)
                        if (seen[q] == seen[q - 1]) {
                            dup = true;
                            break;
                        }
                    if (!dup) break;
                    // redraw every later duplicate of an earlier entry, in index order
                    for (int64_t q = 0; q < d; ++q)
                        for (int64_t t = 0; t < q; ++t)
                            if (out[t] == out[q]) {
                                out[q] = (int32_t)r.below((uint64_t)m);
                                break;
                            }
                }
            }
            for (int64_t k = cp[j]; k < cp[j + 1]; ++k) vals[k] = r.normal();
            x0[j] = r.unit();
            o.c[j] = 2.0 * r.unit() - 1.0;
        }
    });
    csc_to_csr(m, n, cp, ri, vals, o);
    finish_random_lp(g.seed, m, n, x0, o);
    return SP_OK;
}

// Transportation LP: supplies s_i ~ U{1..1000}; demands split the same total by
// seeded weights; one column per arc (i, j) with +1 in row i and +1 in row S + j;
// all rows equalities; costs U{1..100}; 0 <= x < inf.
int gen_transport(const sp_gen_params &g, Owned &o) {
    const int64_t S = g.supplies, D = g.demands;
    if (S <= 0 || D <= 0 || S * D > INT32_MAX) return SP_ERR_INVALID;
    const int64_t m = S + D, n = S * D;
    Rng gr = stream(g.seed, FAMILY_GLOBAL, 0);
    std::vector<double> sup(S), dem(D), w(D);
    double total = 0.0;
    for (int64_t i = 0; i < S; ++i) {
        sup[i] = (double)(1 + gr.below(1000));
        total += sup[i];
    }
    double wsum = 0.0;
    for (int64_t j = 0; j < D; ++j) {
        w[j] = 1.0 - gr.unit();
        wsum += w[j];
    }
    double dsum = 0.0;
    for (int64_t j = 0; j < D; ++j) {
        dem[j] = std::floor(total * w[j] / wsum);
        dsum += dem[j];
    }
    for (int64_t j = 0; dsum < total; j = (j + 1) % D) {
        dem[j] += 1.0;
        dsum += 1.0;
    }
    o.rp.resize(m + 1);
    o.ci.resize(2 * n);
    o.v.assign(2 * n, 1.0);
    int64_t k = 0;
    o.rp[0] = 0;
    for (int64_t i = 0; i < S; ++i) {  // supply rows: arcs i*D .. i*D + D-1
        for (int64_t j = 0; j < D; ++j) o.ci[k++] = (int32_t)(i * D + j);
        o.rp[i + 1] = k;
    }
    for (int64_t j = 0; j < D; ++j) {  // demand rows: arcs i*D + j
        for (int64_t i = 0; i < S; ++i) o.ci[k++] = (int32_t)(i * D + j);
        o.rp[S + j + 1] = k;
    }
    o.c.resize(n);
    parallel_for(S, [&](int64_t a, int64_t b) {
        for (int64_t i = a; i < b; ++i) {
            Rng r = stream(g.seed, FAMILY_COL, (uint64_t)i);
            for (int64_t j = 0; j < D; ++j) o.c[i * D + j] = (double)(1 + r.below(100));
        }
    });
    o.lc.resize(m);
    o.uc.resize(m);
    for (int64_t i = 0; i < S; ++i) o.lc[i] = o.uc[i] = sup[i];
    for (int64_t j = 0; j < D; ++j) o.lc[S + j] = o.uc[S + j] = dem[j];
    o.lv.assign(n, 0.0);
    o.uv.assign(n, INFINITY);
    return SP_OK;
}

void parallel_for(int64_t n, const std::function<void(int64_t, int64_t)> &f) {
    int nt = (int)std::thread::hardware_concurrency();
    if (nt < 1) nt = 1;
    if (nt > 64) nt = 64;
    if (n < 4096 || nt == 1) {
        f(0, n);
        return;
    }
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t) {
        const int64_t lo = n * t / nt, hi = n * (t + 1) / nt;
        th.emplace_back([=, &f] { f(lo, hi); });
    }
    for (auto &t : th) t.join();
}

}  // namespace

// Generated LPs: the arrays belong to the library until sp_lp_release.
std::map<const void *, Owned *> g_owned;
std::mutex g_owned_mu;

namespace sp {  // backend.cu: the calling thread's context and its last error
int enter(sp_ctx *ctx);
int fail(int code, const std::string &msg);
}  // namespace sp

extern "C" int sp_solve_stepwise(sp_ctx *ctx, const sp_lp *lp, const sp_solver_params *params, double *x, double *y,
                                 sp_solution_info *info) {
    if (!ctx || !lp) return SP_ERR_INVALID;
    // problem.validate()? before anything else (solver.rs:155)
    char msg[256] = "";
    const int v = sp_problem_validate(lp, msg, sizeof msg);
    if (v != SP_OK) {
        if (sp::enter(ctx) == SP_OK) sp::fail(v, msg);
        return v;
    }
    sp_solver_params p;
    sp_solver_params_default(&p);
    if (params) p = *params;
    return stepwise(ctx, lp, p, x, y, info);
}

extern "C" int sp_generate(const sp_gen_params *g, sp_lp *out) {
    if (!g || !out) return SP_ERR_INVALID;
    auto *o = new Owned();
    int rc;
    switch (g->kind) {
    case SP_GEN_RANDOM: rc = gen_random(*g, *o); break;
    case SP_GEN_POWERLAW: rc = gen_powerlaw(*g, *o); break;
    case SP_GEN_TRANSPORT: rc = gen_transport(*g, *o); break;
    default: rc = SP_ERR_INVALID;
    }
    if (rc) {
        delete o;
        return rc;
    }
    memset(out, 0, sizeof *out);
    out->a.nrows = (int64_t)o->rp.size() - 1;
    out->a.ncols = (int64_t)o->c.size();
    out->a.nnz = (int64_t)o->v.size();
    out->a.row_ptr = o->rp.data();
    out->a.col_idx = o->ci.data();
    out->a.values = o->v.data();
    out->c = o->c.data();
    out->lc = o->lc.data();
    out->uc = o->uc.data();
    out->lv = o->lv.data();
    out->uv = o->uv.data();
    out->c0 = 0.0;
    out->maximize = 0;
    std::lock_guard<std::mutex> lock(g_owned_mu);
    g_owned[out->a.row_ptr] = o;
    return SP_OK;
}

namespace sp {
// Hands arrays built elsewhere in the library (the MPS reader) to `out`, owned by the
// library until sp_lp_release.
void register_owned_lp(sp_lp *out, std::vector<int64_t> &&rp, std::vector<int32_t> &&ci, std::vector<double> &&v,
                       std::vector<double> &&c, std::vector<double> &&lc, std::vector<double> &&uc,
                       std::vector<double> &&lv, std::vector<double> &&uv) {
    auto *o = new Owned();
    o->rp = std::move(rp);
    o->ci = std::move(ci);
    o->v = std::move(v);
    o->c = std::move(c);
    o->lc = std::move(lc);
    o->uc = std::move(uc);
    o->lv = std::move(lv);
    o->uv = std::move(uv);
    // keep every pointer valid for empty problems
    for (auto *vec : {&o->v, &o->c, &o->lc, &o->uc, &o->lv, &o->uv}) vec->reserve(1);
    o->ci.reserve(1);
    memset(out, 0, sizeof *out);
    out->a.nrows = (int64_t)o->rp.size() - 1;
    out->a.ncols = (int64_t)o->c.size();
    out->a.nnz = (int64_t)o->v.size();
    out->a.row_ptr = o->rp.data();
    out->a.col_idx = o->ci.data();
    out->a.values = o->v.data();
    out->c = o->c.data();
    out->lc = o->lc.data();
    out->uc = o->uc.data();
    out->lv = o->lv.data();
    out->uv = o->uv.data();
    std::lock_guard<std::mutex> lock(g_owned_mu);
    g_owned[out->a.row_ptr] = o;
}
}  // namespace sp

extern "C" void sp_lp_release(sp_lp *lp) {
    if (!lp || !lp->a.row_ptr) return;
    Owned *o = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_owned_mu);
        auto it = g_owned.find(lp->a.row_ptr);
        if (it == g_owned.end()) return;  // not a generated LP
        o = it->second;
        g_owned.erase(it);
    }
    delete o;
    memset(lp, 0, sizeof *lp);
}
