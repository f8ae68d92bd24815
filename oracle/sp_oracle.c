/*
 * sp_oracle.c — CPU oracle (TEST INFRASTRUCTURE ONLY; see sp_oracle.h).
 *
 * Restates, in operation order, the reference's
 *   crates/saddlepoint-core/src/problem.rs   (CSR build, transpose, scale, validate)
 *   crates/saddlepoint-core/src/scaling.rs   (ScaledProblem::new and helpers)
 *   crates/saddlepoint-cpu/src/lib.rs        (CpuBackend)
 *   crates/saddlepoint-core/src/solver.rs    (Solver::run, PidState)
 *   crates/saddlepoint-check/src/lib.rs      (independent KKT checker)
 * Compile with -ffp-contract=off so that no multiply-add is fused.
 */
#define _GNU_SOURCE
#include "sp_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#define PAR_THRESHOLD 32768 /* crates/saddlepoint-cpu/src/lib.rs:12 */
#define MAX_THREADS 256

/* ===================================================================== */
/* Thread pool: fixed contiguous chunking, partials combined in order.    */
/* ===================================================================== */

typedef void (*or_chunk_fn)(void *ctx, int chunk, int64_t lo, int64_t hi);

static struct {
    int nthreads;
    int started;
    pthread_t th[MAX_THREADS];
    pthread_mutex_t mu;
    pthread_cond_t cv_work, cv_done;
    uint64_t gen;
    int pending;
    or_chunk_fn fn;
    void *ctx;
    int64_t n;
} g_pool = {0, 0, {0}, PTHREAD_MUTEX_INITIALIZER, PTHREAD_COND_INITIALIZER, PTHREAD_COND_INITIALIZER, 0, 0, 0, 0, 0};

static int g_requested_threads = 0;

static void chunk_range(int64_t n, int nchunks, int c, int64_t *lo, int64_t *hi) {
    int64_t base = n / nchunks, rem = n % nchunks;
    *lo = c * base + (c < rem ? c : rem);
    *hi = *lo + base + (c < rem ? 1 : 0);
}

static void *pool_worker(void *arg) {
    int id = (int)(intptr_t)arg;
    uint64_t seen = 0;
    for (;;) {
        pthread_mutex_lock(&g_pool.mu);
        while (g_pool.gen == seen) pthread_cond_wait(&g_pool.cv_work, &g_pool.mu);
        seen = g_pool.gen;
        or_chunk_fn fn = g_pool.fn;
        void *ctx = g_pool.ctx;
        int64_t n = g_pool.n;
        int nt = g_pool.nthreads;
        pthread_mutex_unlock(&g_pool.mu);
        int64_t lo, hi;
        chunk_range(n, nt, id, &lo, &hi);
        fn(ctx, id, lo, hi);
        pthread_mutex_lock(&g_pool.mu);
        if (--g_pool.pending == 0) pthread_cond_signal(&g_pool.cv_done);
        pthread_mutex_unlock(&g_pool.mu);
    }
    return NULL;
}

int or_get_threads(void) {
    if (g_pool.started) return g_pool.nthreads;
    int n = g_requested_threads;
    if (n <= 0) {
        const char *e = getenv("SP_ORACLE_THREADS");
        n = e ? atoi(e) : 0;
    }
    if (n <= 0) n = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (n < 1) n = 1;
    if (n > MAX_THREADS) n = MAX_THREADS;
    return n;
}

void or_set_threads(int n) {
    if (!g_pool.started) g_requested_threads = n;
}

static void pool_start(void) {
    if (g_pool.started) return;
    g_pool.nthreads = or_get_threads();
    for (int i = 1; i < g_pool.nthreads; ++i)
        pthread_create(&g_pool.th[i], NULL, pool_worker, (void *)(intptr_t)i);
    g_pool.started = 1;
}

/* Runs fn over nthreads contiguous chunks of [0, n); chunk 0 on the caller. */
static int or_parallel(int64_t n, or_chunk_fn fn, void *ctx) {
    pool_start();
    int nt = g_pool.nthreads;
    if (nt == 1) {
        fn(ctx, 0, 0, n);
        return 1;
    }
    pthread_mutex_lock(&g_pool.mu);
    g_pool.fn = fn;
    g_pool.ctx = ctx;
    g_pool.n = n;
    g_pool.pending = nt - 1;
    g_pool.gen++;
    pthread_cond_broadcast(&g_pool.cv_work);
    pthread_mutex_unlock(&g_pool.mu);
    int64_t lo, hi;
    chunk_range(n, nt, 0, &lo, &hi);
    fn(ctx, 0, lo, hi);
    pthread_mutex_lock(&g_pool.mu);
    while (g_pool.pending > 0) pthread_cond_wait(&g_pool.cv_done, &g_pool.mu);
    pthread_mutex_unlock(&g_pool.mu);
    return nt;
}

/* ===================================================================== */
/* CSR (crates/saddlepoint-core/src/problem.rs)                           */
/* ===================================================================== */

void or_csr_free(or_csr *a) {
    free(a->row_ptr);
    free(a->col_idx);
    free(a->values);
    memset(a, 0, sizeof *a);
}

int or_csr_copy(const or_csr *s, or_csr *d) {
    d->nrows = s->nrows;
    d->ncols = s->ncols;
    d->nnz = s->nnz;
    d->row_ptr = malloc(sizeof(int64_t) * (s->nrows + 1));
    d->col_idx = malloc(sizeof(int64_t) * (s->nnz ? s->nnz : 1));
    d->values = malloc(sizeof(double) * (s->nnz ? s->nnz : 1));
    if (!d->row_ptr || !d->col_idx || !d->values) return OR_ERR_ALLOC;
    memcpy(d->row_ptr, s->row_ptr, sizeof(int64_t) * (s->nrows + 1));
    memcpy(d->col_idx, s->col_idx, sizeof(int64_t) * s->nnz);
    memcpy(d->values, s->values, sizeof(double) * s->nnz);
    return OR_OK;
}

/* Stable insertion/merge sort of (col, val) pairs by col. The reference uses
 * sort_unstable_by_key (problem.rs:60), whose order of equal keys is unspecified;
 * this oracle sums duplicates in triplet order, the stable choice. */
typedef struct { int64_t c; double v; } cv_pair;

static void merge_sort_pairs(cv_pair *a, cv_pair *tmp, int64_t n) {
    if (n <= 16) {
        for (int64_t i = 1; i < n; ++i) {
            cv_pair x = a[i];
            int64_t j = i;
            while (j > 0 && a[j - 1].c > x.c) { a[j] = a[j - 1]; --j; }
            a[j] = x;
        }
        return;
    }
    int64_t h = n / 2;
    merge_sort_pairs(a, tmp, h);
    merge_sort_pairs(a + h, tmp, n - h);
    int64_t i = 0, j = h, k = 0;
    while (i < h && j < n) tmp[k++] = (a[j].c < a[i].c) ? a[j++] : a[i++];
    while (i < h) tmp[k++] = a[i++];
    while (j < n) tmp[k++] = a[j++];
    memcpy(a, tmp, sizeof(cv_pair) * n);
}

/* CsrMatrix::from_triplets (problem.rs:33-77). */
int or_csr_from_triplets(int64_t nrows, int64_t ncols, int64_t ntrip, const int64_t *rows, const int64_t *cols,
                         const double *vals, or_csr *out) {
    memset(out, 0, sizeof *out);
    int64_t *counts = calloc(nrows + 1, sizeof(int64_t));
    if (!counts) return OR_ERR_ALLOC;
    for (int64_t t = 0; t < ntrip; ++t) {
        if (rows[t] < 0 || rows[t] >= nrows || cols[t] < 0 || cols[t] >= ncols) {
            free(counts);
            return OR_ERR_PROBLEM; /* the reference asserts (problem.rs:36) */
        }
        counts[rows[t] + 1] += 1;
    }
    for (int64_t i = 0; i < nrows; ++i) counts[i + 1] += counts[i];
    int64_t *next = malloc(sizeof(int64_t) * (nrows + 1));
    cv_pair *bucket = malloc(sizeof(cv_pair) * (ntrip ? ntrip : 1));
    memcpy(next, counts, sizeof(int64_t) * (nrows + 1));
    for (int64_t t = 0; t < ntrip; ++t) {
        int64_t k = next[rows[t]]++;
        bucket[k].c = cols[t];
        bucket[k].v = vals[t];
    }
    out->nrows = nrows;
    out->ncols = ncols;
    out->row_ptr = malloc(sizeof(int64_t) * (nrows + 1));
    out->col_idx = malloc(sizeof(int64_t) * (ntrip ? ntrip : 1));
    out->values = malloc(sizeof(double) * (ntrip ? ntrip : 1));
    cv_pair *tmp = malloc(sizeof(cv_pair) * (ntrip ? ntrip : 1));
    int64_t nnz = 0;
    out->row_ptr[0] = 0;
    for (int64_t i = 0; i < nrows; ++i) {
        cv_pair *s = bucket + counts[i];
        int64_t len = counts[i + 1] - counts[i];
        merge_sort_pairs(s, tmp, len);
        int64_t k = 0;
        while (k < len) {
            int64_t c = s[k].c;
            double v = s[k].v;
            ++k;
            while (k < len && s[k].c == c) { v += s[k].v; ++k; }
            if (v != 0.0) {
                out->col_idx[nnz] = c;
                out->values[nnz] = v;
                ++nnz;
            }
        }
        out->row_ptr[i + 1] = nnz;
    }
    out->nnz = nnz;
    free(tmp);
    free(bucket);
    free(next);
    free(counts);
    return OR_OK;
}

/* CsrMatrix::transpose (problem.rs:88-109): stable counting sort by column. */
int or_csr_transpose(const or_csr *a, or_csr *out) {
    memset(out, 0, sizeof *out);
    int64_t *counts = calloc(a->ncols + 1, sizeof(int64_t));
    if (!counts) return OR_ERR_ALLOC;
    for (int64_t k = 0; k < a->nnz; ++k) counts[a->col_idx[k] + 1] += 1;
    for (int64_t j = 0; j < a->ncols; ++j) counts[j + 1] += counts[j];
    int64_t *next = malloc(sizeof(int64_t) * (a->ncols + 1));
    memcpy(next, counts, sizeof(int64_t) * (a->ncols + 1));
    out->col_idx = malloc(sizeof(int64_t) * (a->nnz ? a->nnz : 1));
    out->values = malloc(sizeof(double) * (a->nnz ? a->nnz : 1));
    for (int64_t i = 0; i < a->nrows; ++i) {
        for (int64_t k = a->row_ptr[i]; k < a->row_ptr[i + 1]; ++k) {
            int64_t c = a->col_idx[k];
            int64_t t = next[c]++;
            out->col_idx[t] = i;
            out->values[t] = a->values[k];
        }
    }
    free(next);
    out->nrows = a->ncols;
    out->ncols = a->nrows;
    out->nnz = a->nnz;
    out->row_ptr = counts;
    return OR_OK;
}

/* CsrMatrix::mul_vec (problem.rs:112-117): serial, each row summed from -0.0. */
void or_csr_mul_vec(const or_csr *a, const double *x, double *out) {
    for (int64_t i = 0; i < a->nrows; ++i) {
        double s = -0.0;
        for (int64_t k = a->row_ptr[i]; k < a->row_ptr[i + 1]; ++k) s += a->values[k] * x[a->col_idx[k]];
        out[i] = s;
    }
}

/* CsrMatrix::scale (problem.rs:120-126): values[k] *= row[i] * col[j]. */
void or_csr_scale(or_csr *a, const double *row, const double *col) {
    for (int64_t i = 0; i < a->nrows; ++i) {
        double ri = row[i];
        for (int64_t k = a->row_ptr[i]; k < a->row_ptr[i + 1]; ++k) a->values[k] *= ri * col[a->col_idx[k]];
    }
}

/* LpProblem::validate (problem.rs:166-194). */
/* LpProblem::validate (problem.rs:166-194) with the first failure it reports: *what 0 for a
 * variable, 1 a constraint, 2 a coefficient; *kind 1 NaN (ProblemError::NaN), 2 crossed
 * bounds (ProblemError::CrossedBounds); *index within that family, the coefficients
 * numbered c first, then A's values (the reference chains c with a.values). */
int or_lp_validate_at(const or_lp *p, int *what, int *kind, int64_t *index) {
    int64_t m = p->a.nrows, n = p->a.ncols;
    const double *lo[2] = {p->lv, p->lc}, *hi[2] = {p->uv, p->uc};
    int64_t len[2] = {n, m};
    *what = *kind = 0;
    *index = -1;
    for (int s = 0; s < 2; ++s)
        for (int64_t i = 0; i < len[s]; ++i) {
            if (isnan(lo[s][i]) || isnan(hi[s][i]) || lo[s][i] > hi[s][i]) {
                *what = s;
                *kind = (isnan(lo[s][i]) || isnan(hi[s][i])) ? 1 : 2;
                *index = i;
                return OR_ERR_PROBLEM;
            }
        }
    for (int64_t j = 0; j < n + p->a.nnz; ++j)
        if (isnan(j < n ? p->c[j] : p->a.values[j - n])) {
            *what = 2;
            *kind = 1;
            *index = j;
            return OR_ERR_PROBLEM;
        }
    return OR_OK;
}

int or_lp_validate(const or_lp *p) {
    int what, kind;
    int64_t index;
    return or_lp_validate_at(p, &what, &kind, &index);
}

/* LpProblem::objective (problem.rs:198-201). */
double or_lp_objective(const or_lp *p, const double *x) {
    double v = -0.0;
    for (int64_t j = 0; j < p->a.ncols; ++j) v += p->c[j] * x[j];
    v = v + p->c0;
    return p->maximize ? -v : v;
}

void or_lp_free(or_lp *p) {
    or_csr_free(&p->a);
    free(p->c);
    free(p->lc);
    free(p->uc);
    free(p->lv);
    free(p->uv);
    memset(p, 0, sizeof *p);
}

/* ===================================================================== */
/* Scaling (crates/saddlepoint-core/src/scaling.rs)                       */
/* ===================================================================== */

void or_scaling_params_default(or_scaling_params *p) { /* scaling.rs:25-34 */
    p->geometric_mean_passes = 12;
    p->ruiz_iterations = 10;
    p->pock_chambolle_enabled = 1;
    p->pock_chambolle_alpha = 1.0;
    p->bound_objective_rescaling = 1;
}

/* inv_sqrt (scaling.rs:139-141). */
static double inv_sqrt(double v) { return (v > 0.0 && isfinite(v)) ? 1.0 / sqrt(v) : 1.0; }

/* norm2 (scaling.rs:186-188): sequential, from -0.0. */
double or_norm2(const double *v, int64_t n) {
    double s = -0.0;
    for (int64_t i = 0; i < n; ++i) s += v[i] * v[i];
    return sqrt(s);
}

/* finite_bound_norm (scaling.rs:191-201). */
double or_finite_bound_norm(const double *lo, const double *hi, int64_t n) {
    double s = -0.0;
    for (int64_t i = 0; i < n; ++i) {
        double l = isfinite(lo[i]) ? lo[i] : 0.0;
        double u = isfinite(hi[i]) ? hi[i] : 0.0;
        s += (l == u) ? l * l : l * l + u * u;
    }
    return sqrt(s);
}

/* min_max (scaling.rs:159-178). */
static void min_max(const or_csr *a, double *rmin, double *rmax, double *cmin, double *cmax) {
    for (int64_t i = 0; i < a->nrows; ++i) { rmin[i] = INFINITY; rmax[i] = 0.0; }
    for (int64_t j = 0; j < a->ncols; ++j) { cmin[j] = INFINITY; cmax[j] = 0.0; }
    for (int64_t i = 0; i < a->nrows; ++i)
        for (int64_t k = a->row_ptr[i]; k < a->row_ptr[i + 1]; ++k) {
            int64_t j = a->col_idx[k];
            double v = fabs(a->values[k]);
            rmin[i] = fmin(rmin[i], v);
            rmax[i] = fmax(rmax[i], v);
            cmin[j] = fmin(cmin[j], v);
            cmax[j] = fmax(cmax[j], v);
        }
    for (int64_t i = 0; i < a->nrows; ++i)
        if (rmax[i] == 0.0) rmin[i] = 0.0;
    for (int64_t j = 0; j < a->ncols; ++j)
        if (cmax[j] == 0.0) cmin[j] = 0.0;
}

/* abs_stats (scaling.rs:144-155) for the two folds the reference uses. */
enum { FOLD_MAX = 0, FOLD_POW_SUM = 1 };
static double fold_pow(double v, double alpha) { return alpha == 1.0 ? v : pow(v, alpha); }
static void abs_stats(const or_csr *a, int fold, double alpha, double *rows, double *cols) {
    for (int64_t i = 0; i < a->nrows; ++i) rows[i] = 0.0;
    for (int64_t j = 0; j < a->ncols; ++j) cols[j] = 0.0;
    for (int64_t i = 0; i < a->nrows; ++i)
        for (int64_t k = a->row_ptr[i]; k < a->row_ptr[i + 1]; ++k) {
            int64_t j = a->col_idx[k];
            double v = fabs(a->values[k]);
            if (fold == FOLD_MAX) {
                rows[i] = fmax(rows[i], v);
                cols[j] = fmax(cols[j], v);
            } else {
                double f = fold_pow(v, alpha);
                rows[i] = rows[i] + f;
                cols[j] = cols[j] + f;
            }
        }
}

/* apply (scaling.rs:180-184). */
static void apply_scale(or_csr *a, double *row_scale, double *col_scale, const double *r, const double *c) {
    or_csr_scale(a, r, c);
    for (int64_t i = 0; i < a->nrows; ++i) row_scale[i] *= r[i];
    for (int64_t j = 0; j < a->ncols; ++j) col_scale[j] *= c[j];
}

static double *dalloc(int64_t n) { return malloc(sizeof(double) * (n > 0 ? n : 1)); }
static double *dfill(int64_t n, double v) {
    double *p = dalloc(n);
    for (int64_t i = 0; i < n; ++i) p[i] = v;
    return p;
}

/* ScaledProblem::new (scaling.rs:53-103). */
int or_scaled_new(const or_lp *p, const or_scaling_params *params, or_scaled *out) {
    memset(out, 0, sizeof *out);
    int64_t m = p->a.nrows, n = p->a.ncols;
    or_csr a;
    if (or_csr_copy(&p->a, &a) != OR_OK) return OR_ERR_ALLOC;
    double *row_scale = dfill(m, 1.0), *col_scale = dfill(n, 1.0);
    double *ones_m = dfill(m, 1.0), *ones_n = dfill(n, 1.0);
    double *rmin = dalloc(m), *rmax = dalloc(m), *cmin = dalloc(n), *cmax = dalloc(n);
    double *r = dalloc(m), *c = dalloc(n);
    for (int64_t pass = 0; pass < params->geometric_mean_passes; ++pass) {
        min_max(&a, rmin, rmax, cmin, cmax);
        for (int64_t i = 0; i < m; ++i) r[i] = inv_sqrt(rmin[i] * rmax[i]);
        apply_scale(&a, row_scale, col_scale, r, ones_n);
        min_max(&a, rmin, rmax, cmin, cmax);
        for (int64_t j = 0; j < n; ++j) c[j] = inv_sqrt(cmin[j] * cmax[j]);
        apply_scale(&a, row_scale, col_scale, ones_m, c);
    }
    for (int64_t it = 0; it < params->ruiz_iterations; ++it) {
        abs_stats(&a, FOLD_MAX, 0.0, rmax, cmax);
        for (int64_t i = 0; i < m; ++i) r[i] = inv_sqrt(rmax[i]);
        for (int64_t j = 0; j < n; ++j) c[j] = inv_sqrt(cmax[j]);
        apply_scale(&a, row_scale, col_scale, r, c);
    }
    if (params->pock_chambolle_enabled) {
        double alpha = params->pock_chambolle_alpha;
        abs_stats(&a, FOLD_POW_SUM, alpha, rmax, cmin); /* row sums of |v|^alpha */
        abs_stats(&a, FOLD_POW_SUM, 2.0 - alpha, rmin, cmax); /* column sums of |v|^(2-alpha) */
        for (int64_t i = 0; i < m; ++i) r[i] = inv_sqrt(rmax[i]);
        for (int64_t j = 0; j < n; ++j) c[j] = inv_sqrt(cmax[j]);
        apply_scale(&a, row_scale, col_scale, r, c);
    }
    out->c = dalloc(n);
    out->lv = dalloc(n);
    out->uv = dalloc(n);
    out->lc = dalloc(m);
    out->uc = dalloc(m);
    for (int64_t j = 0; j < n; ++j) {
        out->c[j] = p->c[j] * col_scale[j];
        out->lv[j] = p->lv[j] / col_scale[j];
        out->uv[j] = p->uv[j] / col_scale[j];
    }
    for (int64_t i = 0; i < m; ++i) {
        out->lc[i] = p->lc[i] * row_scale[i];
        out->uc[i] = p->uc[i] * row_scale[i];
    }
    double bound_scale = 1.0, obj_scale = 1.0;
    if (params->bound_objective_rescaling) {
        bound_scale = 1.0 / (1.0 + or_finite_bound_norm(out->lc, out->uc, m));
        obj_scale = 1.0 / (1.0 + or_norm2(out->c, n));
        for (int64_t i = 0; i < m; ++i) out->lc[i] *= bound_scale;
        for (int64_t i = 0; i < m; ++i) out->uc[i] *= bound_scale;
        for (int64_t j = 0; j < n; ++j) out->lv[j] *= bound_scale;
        for (int64_t j = 0; j < n; ++j) out->uv[j] *= bound_scale;
        for (int64_t j = 0; j < n; ++j) out->c[j] *= obj_scale;
    }
    out->a = a;
    or_csr_transpose(&out->a, &out->at);
    out->row_scale = row_scale;
    out->col_scale = col_scale;
    out->bound_scale = bound_scale;
    out->obj_scale = obj_scale;
    free(ones_m);
    free(ones_n);
    free(rmin);
    free(rmax);
    free(cmin);
    free(cmax);
    free(r);
    free(c);
    return OR_OK;
}

void or_scaled_free(or_scaled *s) {
    or_csr_free(&s->a);
    or_csr_free(&s->at);
    free(s->c);
    free(s->lc);
    free(s->uc);
    free(s->lv);
    free(s->uv);
    free(s->row_scale);
    free(s->col_scale);
    memset(s, 0, sizeof *s);
}

/* scaling.rs:113-136 */
void or_scaled_unscale_primal(const or_scaled *s, const double *xs, double *out) {
    for (int64_t j = 0; j < s->a.ncols; ++j) out[j] = xs[j] * s->col_scale[j] / s->bound_scale;
}
void or_scaled_unscale_dual(const or_scaled *s, const double *ys, double *out) {
    for (int64_t i = 0; i < s->a.nrows; ++i) out[i] = ys[i] * s->row_scale[i] / s->obj_scale;
}
void or_scaled_primal_factors(const or_scaled *s, double *out) {
    for (int64_t i = 0; i < s->a.nrows; ++i) out[i] = 1.0 / (s->row_scale[i] * s->bound_scale);
}
void or_scaled_dual_factors(const or_scaled *s, double *out) {
    for (int64_t j = 0; j < s->a.ncols; ++j) out[j] = 1.0 / (s->col_scale[j] * s->obj_scale);
}
double or_scaled_objective_factor(const or_scaled *s) { return 1.0 / (s->bound_scale * s->obj_scale); }

/* ===================================================================== */
/* CPU backend (crates/saddlepoint-cpu/src/lib.rs)                         */
/* ===================================================================== */

/* excess (lib.rs:70-80) */
static inline double excess(double v, double lo, double hi) {
    if (v < lo) return v - lo;
    if (v > hi) return v - hi;
    return 0.0;
}
/* bound_term (lib.rs:82-92) */
static inline double bound_term(double v, double lo, double hi) {
    if (v > 0.0 && isfinite(lo)) return v * lo;
    if (v < 0.0 && isfinite(hi)) return v * hi;
    return 0.0;
}
/* forbidden (lib.rs:94-99) */
static inline double forbidden(double v, double lo, double hi) {
    return ((v > 0.0 && lo == -INFINITY) || (v < 0.0 && hi == INFINITY)) ? v : 0.0;
}
/* recession_violation (lib.rs:262-269) */
static inline double recession_violation(double v, double lo, double hi) {
    double l = isfinite(lo) ? 0.0 : -INFINITY;
    double h = isfinite(hi) ? 0.0 : INFINITY;
    return excess(v, l, h);
}
/* f64::clamp: `if v < lo { lo } else if v > hi { hi } else { v }`, NaN passes through. */
static inline double clampd(double v, double lo, double hi) {
    if (v < lo) v = lo;
    if (v > hi) v = hi;
    return v;
}

int or_cpu_load(const or_scaled *s, or_cpu_problem *out) { /* lib.rs:110-122 */
    out->a = &s->a;
    out->at = &s->at;
    out->c = s->c;
    out->lc = s->lc;
    out->uc = s->uc;
    out->lv = s->lv;
    out->uv = s->uv;
    out->primal_factor = dalloc(s->a.nrows);
    out->dual_factor = dalloc(s->a.ncols);
    or_scaled_primal_factors(s, out->primal_factor);
    or_scaled_dual_factors(s, out->dual_factor);
    return OR_OK;
}
void or_cpu_free(or_cpu_problem *p) {
    free(p->primal_factor);
    free(p->dual_factor);
    memset(p, 0, sizeof *p);
}

/* ---- generic op dispatch: serial below PAR_THRESHOLD, else chunks ---- */

typedef struct {
    int op;
    const or_csr *csr;
    const or_cpu_problem *p;
    const double *a, *b, *c, *d;
    double *o1, *o2;
    double s1, s2;
    double part[MAX_THREADS][5];
} op_ctx;

enum {
    OP_CSR_MUL, OP_PRIMAL_XT, OP_PRIMAL_XBAR, OP_DUAL, OP_HALPERN, OP_SUB, OP_SCALE,
    OP_DIST, OP_DOT, OP_PRIM_RES, OP_DUAL_ROWS, OP_DUAL_COLS, OP_STEP_DUAL,
    OP_PRAY_ROWS, OP_PRAY_COLS, OP_DRAY_ROWS, OP_DRAY_COLS
};

static void op_chunk(void *vctx, int chunk, int64_t lo, int64_t hi) {
    op_ctx *x = (op_ctx *)vctx;
    const or_cpu_problem *p = x->p;
    double *part = x->part[chunk];
    switch (x->op) {
    case OP_CSR_MUL: { /* csr_mul (lib.rs:58-68) */
        const or_csr *a = x->csr;
        for (int64_t i = lo; i < hi; ++i) {
            double s = -0.0;
            for (int64_t k = a->row_ptr[i]; k < a->row_ptr[i + 1]; ++k) s += a->values[k] * x->a[a->col_idx[k]];
            x->o1[i] = s;
        }
        break;
    }
    case OP_PRIMAL_XT: /* primal_step, first pass (lib.rs:156) */
        for (int64_t j = lo; j < hi; ++j)
            x->o1[j] = clampd(x->a[j] - x->s1 * (p->c[j] - x->b[j]), p->lv[j], p->uv[j]);
        break;
    case OP_PRIMAL_XBAR: /* primal_step, second pass (lib.rs:158) */
        for (int64_t j = lo; j < hi; ++j) x->o1[j] = 2.0 * x->b[j] - x->a[j];
        break;
    case OP_DUAL: /* dual_step (lib.rs:170-173) */
        for (int64_t i = lo; i < hi; ++i) {
            double v = x->b[i] - x->a[i] / x->s1;
            x->o1[i] = x->a[i] - x->s1 * (x->b[i] - clampd(v, p->lc[i], p->uc[i]));
        }
        break;
    case OP_HALPERN: /* halpern_step (lib.rs:185) */
        for (int64_t i = lo; i < hi; ++i)
            x->o1[i] = x->s1 * ((1.0 + x->s2) * x->a[i] - x->s2 * x->o1[i]) + (1.0 - x->s1) * x->b[i];
        break;
    case OP_SUB:
        for (int64_t i = lo; i < hi; ++i) x->o1[i] = x->a[i] - x->b[i];
        break;
    case OP_SCALE:
        for (int64_t i = lo; i < hi; ++i) x->o1[i] *= x->s1;
        break;
    case OP_DIST: { /* distance_sq (lib.rs:189-191) */
        double s = -0.0;
        for (int64_t i = lo; i < hi; ++i) { double d = x->a[i] - x->b[i]; s += d * d; }
        part[0] = s;
        break;
    }
    case OP_DOT: {
        double s = -0.0;
        for (int64_t i = lo; i < hi; ++i) s += x->a[i] * x->b[i];
        part[0] = s;
        break;
    }
    case OP_PRIM_RES: { /* primal_stats residual (lib.rs:212) */
        double s = -0.0;
        for (int64_t i = lo; i < hi; ++i) {
            double e = excess(x->a[i], p->lc[i], p->uc[i]) * p->primal_factor[i];
            s += e * e;
        }
        part[0] = s;
        break;
    }
    case OP_DUAL_ROWS: { /* dual_stats rows (lib.rs:218) */
        double s = -0.0;
        for (int64_t i = lo; i < hi; ++i) s += bound_term(x->a[i], p->lc[i], p->uc[i]);
        part[0] = s;
        break;
    }
    case OP_DUAL_COLS: { /* dual_stats cols (lib.rs:219-222), sum2 from (0, 0) */
        double s0 = 0.0, s1 = 0.0;
        for (int64_t j = lo; j < hi; ++j) {
            double r = p->c[j] - x->a[j];
            double f = forbidden(r, p->lv[j], p->uv[j]) * p->dual_factor[j];
            s0 = s0 + f * f;
            s1 = s1 + bound_term(r, p->lv[j], p->uv[j]);
        }
        part[0] = s0;
        part[1] = s1;
        break;
    }
    case OP_STEP_DUAL: { /* step_dual_residual_sq (lib.rs:235-236) */
        double s = -0.0, inv_tau = x->s1;
        for (int64_t j = lo; j < hi; ++j) {
            double r = (x->c[j] - x->d[j] - (x->b[j] - x->a[j]) * inv_tau) * p->dual_factor[j];
            s += r * r;
        }
        part[0] = s;
        break;
    }
    case OP_PRAY_ROWS: { /* primal_ray_stats rows (lib.rs:242) */
        double s = -0.0;
        for (int64_t i = lo; i < hi; ++i) {
            double v = recession_violation(x->a[i], p->lc[i], p->uc[i]);
            s += v * v;
        }
        part[0] = s;
        break;
    }
    case OP_PRAY_COLS: { /* primal_ray_stats cols (lib.rs:243-244), sum2 then sum1 */
        double s0 = 0.0, s1 = 0.0, s2 = -0.0;
        for (int64_t j = lo; j < hi; ++j) {
            double d = x->a[j];
            double v = recession_violation(d, p->lv[j], p->uv[j]);
            s0 = s0 + v * v;
            s1 = s1 + d * d;
            s2 += p->c[j] * d;
        }
        part[0] = s0;
        part[1] = s1;
        part[2] = s2;
        break;
    }
    case OP_DRAY_ROWS: { /* dual_ray_stats rows (lib.rs:251-252) and norm (lib.rs:257) */
        double s0 = 0.0, s1 = 0.0, s2 = -0.0;
        for (int64_t i = lo; i < hi; ++i) {
            double d = x->a[i];
            double f = forbidden(d, p->lc[i], p->uc[i]);
            s0 = s0 + f * f;
            s1 = s1 + bound_term(d, p->lc[i], p->uc[i]);
            s2 += d * d;
        }
        part[0] = s0;
        part[1] = s1;
        part[2] = s2;
        break;
    }
    case OP_DRAY_COLS: { /* dual_ray_stats cols (lib.rs:253-256) */
        double s0 = 0.0, s1 = 0.0;
        for (int64_t j = lo; j < hi; ++j) {
            double r = -x->a[j];
            double f = forbidden(r, p->lv[j], p->uv[j]);
            s0 = s0 + f * f;
            s1 = s1 + bound_term(r, p->lv[j], p->uv[j]);
        }
        part[0] = s0;
        part[1] = s1;
        break;
    }
    }
}

/* Runs op over n elements; returns the number of chunks whose partials are valid. */
static int run_op(op_ctx *x, int64_t n, int64_t work) {
    if (work < PAR_THRESHOLD) {
        op_chunk(x, 0, 0, n);
        return 1;
    }
    return or_parallel(n, op_chunk, x);
}

/* Combines partial k over chunks: sum1 folds from -0.0, sum2 from +0.0. */
static double combine(const op_ctx *x, int nch, int k, double start) {
    double s = start;
    for (int c = 0; c < nch; ++c) s += x->part[c][k];
    return s;
}
/* A serial pass already folded from the right start value; a parallel one combines. */
static double total(const op_ctx *x, int nch, int k, double start) {
    return nch == 1 ? x->part[0][k] : combine(x, nch, k, start);
}

static op_ctx *new_ctx(int op, const or_cpu_problem *p) {
    op_ctx *x = calloc(1, sizeof(op_ctx));
    x->op = op;
    x->p = p;
    return x;
}

static void csr_mul(const or_csr *a, const double *v, double *out) {
    op_ctx *x = new_ctx(OP_CSR_MUL, NULL);
    x->csr = a;
    x->a = v;
    x->o1 = out;
    run_op(x, a->nrows, a->nnz); /* threshold on nnz (lib.rs:63) */
    free(x);
}

void or_cpu_spmv(const or_cpu_problem *p, const double *x, double *out) { csr_mul(p->a, x, out); }
void or_cpu_spmv_t(const or_cpu_problem *p, const double *y, double *out) { csr_mul(p->at, y, out); }

void or_cpu_primal_step(const or_cpu_problem *p, const double *xv, const double *aty, double tau, double *x_t,
                        double *x_bar) {
    int64_t n = p->a->ncols;
    op_ctx *x = new_ctx(OP_PRIMAL_XT, p);
    x->a = xv;
    x->b = aty;
    x->s1 = tau;
    x->o1 = x_t;
    run_op(x, n, n);
    x->op = OP_PRIMAL_XBAR;
    x->b = x_t;
    x->o1 = x_bar;
    run_op(x, n, n);
    free(x);
}

void or_cpu_dual_step(const or_cpu_problem *p, const double *y, const double *ax_bar, double sigma, double *y_t) {
    int64_t m = p->a->nrows;
    op_ctx *x = new_ctx(OP_DUAL, p);
    x->a = y;
    x->b = ax_bar;
    x->s1 = sigma;
    x->o1 = y_t;
    run_op(x, m, m);
    free(x);
}

void or_cpu_halpern_step(double *z, const double *z_t, const double *anchor, double w, double rho, int64_t n) {
    op_ctx *x = new_ctx(OP_HALPERN, NULL);
    x->a = z_t;
    x->b = anchor;
    x->o1 = z;
    x->s1 = w;
    x->s2 = rho;
    run_op(x, n, n);
    free(x);
}

double or_cpu_distance_sq(const double *a, const double *b, int64_t n) {
    op_ctx *x = new_ctx(OP_DIST, NULL);
    x->a = a;
    x->b = b;
    int nch = run_op(x, n, n);
    double r = total(x, nch, 0, -0.0);
    free(x);
    return r;
}

void or_cpu_sub(const double *a, const double *b, double *out, int64_t n) {
    op_ctx *x = new_ctx(OP_SUB, NULL);
    x->a = a;
    x->b = b;
    x->o1 = out;
    run_op(x, n, n);
    free(x);
}

double or_cpu_dot(const double *a, const double *b, int64_t n) {
    op_ctx *x = new_ctx(OP_DOT, NULL);
    x->a = a;
    x->b = b;
    int nch = run_op(x, n, n);
    double r = total(x, nch, 0, -0.0);
    free(x);
    return r;
}

double or_cpu_norm_sq(const double *v, int64_t n) { return or_cpu_dot(v, v, n); }

void or_cpu_scale(double *v, double alpha, int64_t n) {
    op_ctx *x = new_ctx(OP_SCALE, NULL);
    x->o1 = v;
    x->s1 = alpha;
    run_op(x, n, n);
    free(x);
}

or_primal_stats or_cpu_primal_stats(const or_cpu_problem *p, const double *xv, const double *ax) {
    or_primal_stats st;
    op_ctx *x = new_ctx(OP_PRIM_RES, p);
    x->a = ax;
    int nch = run_op(x, p->a->nrows, p->a->nrows);
    st.residual_sq = total(x, nch, 0, -0.0);
    x->op = OP_DOT;
    x->a = p->c;
    x->b = xv;
    nch = run_op(x, p->a->ncols, p->a->ncols);
    st.objective = total(x, nch, 0, -0.0);
    free(x);
    return st;
}

or_dual_stats or_cpu_dual_stats(const or_cpu_problem *p, const double *y, const double *aty) {
    or_dual_stats st;
    op_ctx *x = new_ctx(OP_DUAL_ROWS, p);
    x->a = y;
    int nch = run_op(x, p->a->nrows, p->a->nrows);
    double rows = total(x, nch, 0, -0.0);
    x->op = OP_DUAL_COLS;
    x->a = aty;
    nch = run_op(x, p->a->ncols, p->a->ncols);
    double res = total(x, nch, 0, 0.0), cols = total(x, nch, 1, 0.0);
    free(x);
    st.residual_sq = res;
    st.objective = rows + cols;
    return st;
}

double or_cpu_step_dual_residual_sq(const or_cpu_problem *p, const double *xv, const double *x_t, const double *aty,
                                    const double *aty_t, double tau) {
    op_ctx *x = new_ctx(OP_STEP_DUAL, p);
    x->a = xv;
    x->b = x_t;
    x->c = aty;
    x->d = aty_t;
    x->s1 = 1.0 / tau;
    int nch = run_op(x, p->a->ncols, p->a->ncols);
    double r = total(x, nch, 0, -0.0);
    free(x);
    return r;
}

or_ray_stats or_cpu_primal_ray_stats(const or_cpu_problem *p, const double *dx, const double *adx) {
    or_ray_stats st;
    op_ctx *x = new_ctx(OP_PRAY_ROWS, p);
    x->a = adx;
    int nch = run_op(x, p->a->nrows, p->a->nrows);
    double rows = total(x, nch, 0, -0.0);
    x->op = OP_PRAY_COLS;
    x->a = dx;
    nch = run_op(x, p->a->ncols, p->a->ncols);
    double cols = total(x, nch, 0, 0.0), norm_sq = total(x, nch, 1, 0.0), obj = total(x, nch, 2, -0.0);
    free(x);
    st.objective = obj;
    st.violation_sq = rows + cols;
    st.norm_sq = norm_sq;
    return st;
}

or_ray_stats or_cpu_dual_ray_stats(const or_cpu_problem *p, const double *dy, const double *atdy) {
    or_ray_stats st;
    op_ctx *x = new_ctx(OP_DRAY_ROWS, p);
    x->a = dy;
    int nch = run_op(x, p->a->nrows, p->a->nrows);
    double row_viol = total(x, nch, 0, 0.0), row_obj = total(x, nch, 1, 0.0), norm_sq = total(x, nch, 2, -0.0);
    x->op = OP_DRAY_COLS;
    x->a = atdy;
    nch = run_op(x, p->a->ncols, p->a->ncols);
    double col_viol = total(x, nch, 0, 0.0), col_obj = total(x, nch, 1, 0.0);
    free(x);
    st.objective = row_obj + col_obj;
    st.violation_sq = row_viol + col_viol;
    st.norm_sq = norm_sq;
    return st;
}

/* ===================================================================== */
/* Solver (crates/saddlepoint-core/src/solver.rs)                          */
/* ===================================================================== */

void or_solver_params_default(or_solver_params *p) { /* solver.rs:70-93 */
    p->tolerance = 1e-6;
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
    or_scaling_params_default(&p->scaling);
    p->termination = 0;
}

/* PidState (solver.rs:445-480). */
void or_pid_init(or_pid *pid, double omega) {
    pid->integral = 0.0;
    pid->has_prev = 0;
    pid->prev_error = 0.0;
    pid->best_weight = omega;
    pid->best_balance = INFINITY;
}

static int sane(double v) { return v >= 1e-16 && v <= 1e12; }

double or_pid_update(or_pid *pid, const or_solver_params *p, double omega, double dx, double dy, double rel_primal,
                     double rel_dual) {
    double ratio = rel_dual / rel_primal;
    if (!sane(dx) || !sane(dy) || !(ratio >= 1e-8 && ratio <= 1e8)) {
        pid->integral = 0.0;
        pid->has_prev = 0;
        return pid->best_weight;
    }
    double e = log(omega * dx / dy);
    pid->integral = p->pid_discount * pid->integral + e;
    double derivative = pid->has_prev ? e - pid->prev_error : 0.0;
    pid->prev_error = e;
    pid->has_prev = 1;
    double next = exp(log(omega) - (p->pid_kp * e + p->pid_ki * pid->integral + p->pid_kd * derivative));
    double balance = fabs(log10(ratio));
    if (balance < pid->best_balance) {
        pid->best_balance = balance;
        pid->best_weight = next;
    }
    return next;
}

typedef struct {
    double primal_obj, dual_obj, primal_res, dual_res;
} kkt_t;
static double kkt_gap(const kkt_t *k) { return fabs(k->primal_obj - k->dual_obj); }
static int kkt_converged(const kkt_t *k, double eps, double b_norm, double c_norm) { /* solver.rs:147-151 */
    return k->primal_res <= eps * (1.0 + b_norm) && k->dual_res <= eps * (1.0 + c_norm) &&
           kkt_gap(k) <= eps * (1.0 + fabs(k->primal_obj) + fabs(k->dual_obj));
}

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

typedef struct {
    const or_lp *problem;
    const or_solver_params *params;
    or_scaled scaled;
    or_cpu_problem dev;
    int64_t m, n;
    double *x, *y, *x_t, *y_t, *x_bar, *x_anchor, *y_anchor, *ax, *aty, *tmp_n, *tmp_m, *tmp_m2, *c;
    int owns_scaled;
} solver_t;

/* Solver::estimate_norm (solver.rs:215-242). */
static int estimate_norm(solver_t *s, double *out) {
    int64_t n = s->n;
    if (n == 0 || s->scaled.a.nnz == 0) {
        *out = 1.0;
        return OR_OK;
    }
    double *v = dalloc(n);
    for (int64_t j = 0; j < n; ++j) v[j] = 1.0 + 0.01 * (double)(j % 7);
    double sc = 1.0 / sqrt(or_cpu_norm_sq(v, n));
    or_cpu_scale(v, sc, n);
    double lambda = 0.0;
    for (uint64_t it = 0; it < s->params->power_iterations; ++it) {
        or_cpu_spmv(&s->dev, v, s->tmp_m);
        or_cpu_spmv_t(&s->dev, s->tmp_m, v);
        double norm = sqrt(or_cpu_norm_sq(v, n));
        if (isnan(norm) || norm <= 0.0 || isinf(norm)) {
            free(v);
            return OR_ERR_NUMERICAL;
        }
        or_cpu_scale(v, 1.0 / norm, n);
        int done = fabs(norm - lambda) <= 1e-6 * norm;
        lambda = norm;
        if (done) break;
    }
    free(v);
    *out = sqrt(lambda) * 1.01;
    return OR_OK;
}

/* Solver::kkt (solver.rs:245-258). Leaves A'ᵀ y_t in tmp_n. */
static kkt_t kkt(solver_t *s) {
    double f = or_scaled_objective_factor(&s->scaled);
    or_cpu_spmv(&s->dev, s->x_t, s->tmp_m);
    or_primal_stats ps = or_cpu_primal_stats(&s->dev, s->x_t, s->tmp_m);
    or_cpu_spmv_t(&s->dev, s->y_t, s->tmp_n);
    or_dual_stats ds = or_cpu_dual_stats(&s->dev, s->y_t, s->tmp_n);
    kkt_t k;
    k.primal_obj = ps.objective * f + s->problem->c0;
    k.dual_obj = ds.objective * f + s->problem->c0;
    k.primal_res = sqrt(ps.residual_sq);
    k.dual_res = sqrt(ds.residual_sq);
    return k;
}

/* Solver::step_dual_objective (solver.rs:263-271). */
static double step_dual_objective(solver_t *s, double tau) {
    double rows = or_cpu_dual_stats(&s->dev, s->y_t, s->c).objective;
    int64_t n = s->n;
    double lx = or_cpu_dot(s->c, s->x_t, n) - or_cpu_dot(s->aty, s->x_t, n) +
                (or_cpu_dot(s->x_t, s->x_t, n) - or_cpu_dot(s->x, s->x_t, n)) / tau;
    return (rows + lx) * or_scaled_objective_factor(&s->scaled) + s->problem->c0;
}

/* Solver::fixed_point_residual (solver.rs:275-288). */
static int fixed_point_residual(solver_t *s, double eta, double omega, double *out) {
    or_cpu_sub(s->x_t, s->x, s->tmp_n, s->n);
    or_cpu_sub(s->y_t, s->y, s->tmp_m2, s->m);
    or_cpu_spmv(&s->dev, s->tmp_n, s->tmp_m);
    double dx2 = or_cpu_norm_sq(s->tmp_n, s->n);
    double dy2 = or_cpu_norm_sq(s->tmp_m2, s->m);
    double cross = or_cpu_dot(s->tmp_m2, s->tmp_m, s->m);
    double r2 = omega / eta * dx2 + dy2 / (eta * omega) + 2.0 * cross;
    if (!isfinite(r2)) return OR_ERR_NUMERICAL;
    *out = sqrt(fmax(r2, 0.0));
    return OR_OK;
}

/* Solver::infeasibility (solver.rs:291-309). Returns -1 for none. */
static int infeasibility(solver_t *s) {
    double eps = s->params->infeasibility_tolerance;
    or_cpu_sub(s->y_t, s->y_anchor, s->tmp_m, s->m);
    or_cpu_spmv_t(&s->dev, s->tmp_m, s->tmp_n);
    or_ray_stats d = or_cpu_dual_ray_stats(&s->dev, s->tmp_m, s->tmp_n);
    if (d.objective > 0.0 && sqrt(d.violation_sq) <= eps * d.objective && d.objective > eps * sqrt(d.norm_sq))
        return OR_PRIMAL_INFEASIBLE;
    or_cpu_sub(s->x_t, s->x_anchor, s->tmp_n, s->n);
    or_cpu_spmv(&s->dev, s->tmp_n, s->tmp_m);
    or_ray_stats p = or_cpu_primal_ray_stats(&s->dev, s->tmp_n, s->tmp_m);
    if (p.objective < 0.0 && sqrt(p.violation_sq) <= -eps * p.objective && -p.objective > eps * sqrt(p.norm_sq))
        return OR_DUAL_INFEASIBLE;
    return -1;
}

static void push_trace(or_solution *out, int64_t *cap, or_check_record rec) {
    if (out->trace_len == *cap) {
        *cap = *cap ? *cap * 2 : 64;
        out->trace = realloc(out->trace, sizeof(or_check_record) * (*cap));
    }
    out->trace[out->trace_len++] = rec;
}

static void solver_free(solver_t *s) {
    double *v[] = {s->x, s->y, s->x_t, s->y_t, s->x_bar, s->x_anchor, s->y_anchor,
                   s->ax, s->aty, s->tmp_n, s->tmp_m, s->tmp_m2, s->c};
    for (size_t i = 0; i < sizeof v / sizeof v[0]; ++i) free(v[i]);
    or_cpu_free(&s->dev);
    if (s->owns_scaled) or_scaled_free(&s->scaled);
}

static int solve_impl(const or_lp *problem, const or_scaled *given, const or_solver_params *p, double norm_override,
                      uint64_t stop_after, or_solution *out);

/* solve (solver.rs:154-157) = validate + Solver::new (:185-212) + Solver::run (:311-438). */
int or_solve(const or_lp *problem, const or_solver_params *p, or_solution *out) {
    return solve_impl(problem, NULL, p, 0.0, 0, out);
}

/* Solver::run on an already scaled problem (borrowed), for timing the loop alone;
 * norm_override > 0 replaces estimate_norm's result; stop_after > 0 ends the loop
 * after that many iterations without forcing a check (checks stay every
 * check_every iterations, the reference's cadence). */
int or_solve_scaled(const or_lp *problem, const or_scaled *scaled, const or_solver_params *p, double norm_override,
                    uint64_t stop_after, or_solution *out) {
    return solve_impl(problem, scaled, p, norm_override, stop_after, out);
}

static int solve_impl(const or_lp *problem, const or_scaled *given, const or_solver_params *p, double norm_override,
                      uint64_t stop_after, or_solution *out) {
    memset(out, 0, sizeof *out);
    if (or_lp_validate(problem) != OR_OK) return OR_ERR_PROBLEM;
    solver_t S;
    memset(&S, 0, sizeof S);
    solver_t *s = &S;
    s->problem = problem;
    s->params = p;
    s->m = problem->a.nrows;
    s->n = problem->a.ncols;
    if (given) {
        s->scaled = *given;
        s->owns_scaled = 0;
    } else {
        if (or_scaled_new(problem, &p->scaling, &s->scaled) != OR_OK) return OR_ERR_ALLOC;
        s->owns_scaled = 1;
    }
    or_cpu_load(&s->scaled, &s->dev);
    int64_t m = s->m, n = s->n;
    s->x = dfill(n, 0.0);
    s->y = dfill(m, 0.0);
    s->x_t = dfill(n, 0.0);
    s->y_t = dfill(m, 0.0);
    s->x_bar = dfill(n, 0.0);
    s->x_anchor = dfill(n, 0.0);
    s->y_anchor = dfill(m, 0.0);
    s->ax = dfill(m, 0.0);
    s->aty = dfill(n, 0.0);
    s->tmp_n = dfill(n, 0.0);
    s->tmp_m = dfill(m, 0.0);
    s->tmp_m2 = dfill(m, 0.0);
    s->c = dalloc(n);
    memcpy(s->c, s->scaled.c, sizeof(double) * n);

    double start = now_s();
    double norm_est = norm_override;
    int rc = norm_override > 0.0 ? OR_OK : estimate_norm(s, &norm_est);
    if (rc != OR_OK) {
        solver_free(s);
        return rc;
    }
    out->norm_estimate = norm_est;
    double eta = p->step_size_factor / norm_est;
    double b_norm = or_finite_bound_norm(problem->lc, problem->uc, m);
    double c_norm = or_norm2(problem->c, n);
    double omega = p->scaling.bound_objective_rescaling ? 1.0 : (1.0 + c_norm) / (1.0 + b_norm);
    or_pid pid;
    or_pid_init(&pid, omega);

    uint64_t total = 0, k = 0, restarts = 0;
    double anchor_residual = INFINITY, prev_residual = INFINITY;
    int64_t trace_cap = 0;
    int status;
    kkt_t kk = {0.0, 0.0, 0.0, 0.0};
    for (;;) {
        double tau = eta / omega, sigma = eta * omega;
        or_cpu_spmv_t(&s->dev, s->y, s->aty);
        or_cpu_primal_step(&s->dev, s->x, s->aty, tau, s->x_t, s->x_bar);
        or_cpu_spmv(&s->dev, s->x_bar, s->ax);
        or_cpu_dual_step(&s->dev, s->y, s->ax, sigma, s->y_t);

        total += 1;
        /* u64::is_multiple_of(0) is true only for 0, and total >= 1 here. */
        int check = (p->check_every != 0 && total % p->check_every == 0) || total >= p->max_iterations;
        double residual = 0.0;
        if (check || k == 0) {
            rc = fixed_point_residual(s, eta, omega, &residual);
            if (rc != OR_OK) {
                solver_free(s);
                return rc;
            }
        }
        if (k == 0) anchor_residual = residual;
        double step_dual = 0.0, step_obj = 0.0;
        if (check) {
            kk = kkt(s);
            step_dual = sqrt(or_cpu_step_dual_residual_sq(&s->dev, s->x, s->x_t, s->aty, s->tmp_n, tau));
            if (p->termination == 1) step_obj = step_dual_objective(s, tau);
        }
        double w = (double)(k + 1) / (double)(k + 2);
        or_cpu_halpern_step(s->x, s->x_t, s->x_anchor, w, p->reflection, n);
        or_cpu_halpern_step(s->y, s->y_t, s->y_anchor, w, p->reflection, m);
        k += 1;
        if (!check) {
            if (stop_after && total >= stop_after) {  /* a timing sample ends without a forced check */
                status = OR_ITERATION_LIMIT;
                break;
            }
            continue;
        }

        or_check_record rec;
        memset(&rec, 0, sizeof rec);
        rec.total = total;
        rec.residual = residual;
        rec.primal_obj = kk.primal_obj;
        rec.dual_obj = kk.dual_obj;
        rec.primal_res = kk.primal_res;
        rec.dual_res = kk.dual_res;

        kkt_t test = kk;
        if (p->termination == 1) {
            test.dual_obj = step_obj;
            test.dual_res = step_dual;
        }
        int stop = -1;
        if (kkt_converged(&test, p->tolerance, b_norm, c_norm)) stop = OR_OPTIMAL;
        if (stop < 0) {
            int inf = infeasibility(s);
            if (inf >= 0) stop = inf;
        }
        if (stop < 0 && total >= p->max_iterations) stop = OR_ITERATION_LIMIT;
        if (stop < 0 && p->time_limit_s > 0.0 && now_s() - start >= p->time_limit_s) stop = OR_TIME_LIMIT;
        if (stop >= 0) {
            rec.omega = omega;
            rec.k_after = k;
            push_trace(out, &trace_cap, rec);
            status = stop;
            break;
        }
        double r0 = anchor_residual;
        int restart = residual <= p->restart_sufficient * r0 ||
                      (residual <= p->restart_necessary * r0 && residual > prev_residual) ||
                      (double)k >= p->restart_artificial * (double)total;
        prev_residual = residual;
        if (restart) {
            double dx = sqrt(or_cpu_distance_sq(s->x_t, s->x_anchor, n));
            double dy = sqrt(or_cpu_distance_sq(s->y_t, s->y_anchor, m));
            double rel_primal = kk.primal_res / (1.0 + b_norm);
            double rel_dual = step_dual / (1.0 + c_norm);
            omega = or_pid_update(&pid, p, omega, dx, dy, rel_primal, rel_dual);
            memcpy(s->x_anchor, s->x_t, sizeof(double) * n);
            memcpy(s->y_anchor, s->y_t, sizeof(double) * m);
            memcpy(s->x, s->x_t, sizeof(double) * n);
            memcpy(s->y, s->y_t, sizeof(double) * m);
            k = 0;
            restarts += 1;
            prev_residual = INFINITY;
        }
        rec.restarted = restart;
        rec.omega = omega;
        rec.k_after = k;
        push_trace(out, &trace_cap, rec);
        if (stop_after && total >= stop_after) {
            status = OR_ITERATION_LIMIT;
            break;
        }
    }
    out->x = dalloc(n);
    out->y = dalloc(m);
    or_scaled_unscale_primal(&s->scaled, s->x_t, out->x);
    or_scaled_unscale_dual(&s->scaled, s->y_t, out->y);
    double sign = problem->maximize ? -1.0 : 1.0;
    out->status = status;
    out->objective = sign * kk.primal_obj;
    out->dual_objective = sign * kk.dual_obj;
    out->primal_residual = kk.primal_res;
    out->dual_residual = kk.dual_res;
    out->gap = kkt_gap(&kk);
    out->iterations = total;
    out->restarts = restarts;
    out->solve_time_s = now_s() - start;
    solver_free(s);
    return OR_OK;
}

void or_solution_free(or_solution *s) {
    free(s->x);
    free(s->y);
    free(s->trace);
    memset(s, 0, sizeof *s);
}

/* ===================================================================== */
/* Checker (crates/saddlepoint-check/src/lib.rs:45-118)                    */
/* ===================================================================== */

static double outside(double v, double lo, double hi) {
    if (v < lo) return lo - v;
    if (v > hi) return v - hi;
    return 0.0;
}

void or_check(const or_lp *p, const double *x, const double *y, or_kkt_report *out) {
    int64_t m = p->a.nrows, n = p->a.ncols;
    double *ax = dfill(m, 0.0), *aty = dfill(n, 0.0);
    for (int64_t i = 0; i < m; ++i)
        for (int64_t k = p->a.row_ptr[i]; k < p->a.row_ptr[i + 1]; ++k) {
            int64_t j = p->a.col_idx[k];
            double v = p->a.values[k];
            ax[i] += v * x[j];
            aty[j] += v * y[i];
        }
    double po = -0.0;
    for (int64_t j = 0; j < n; ++j) po += p->c[j] * x[j];
    po = po + p->c0;
    double cv = -0.0;
    for (int64_t i = 0; i < m; ++i) { double o = outside(ax[i], p->lc[i], p->uc[i]); cv += o * o; }
    cv = sqrt(cv);
    double bv = -0.0;
    for (int64_t j = 0; j < n; ++j) { double o = outside(x[j], p->lv[j], p->uv[j]); bv += o * o; }
    bv = sqrt(bv);

    /* term() closure (lib.rs:85-91): violations are squared-summed in push order. */
    double dual_obj = p->c0, dv = -0.0;
#define TERM(v, lo, hi)                                    \
    do {                                                   \
        double vv = (v);                                   \
        if (vv > 0.0) {                                    \
            if (isfinite(lo)) dual_obj += vv * (lo);       \
            else dv += vv * vv;                            \
        } else if (vv < 0.0) {                             \
            if (isfinite(hi)) dual_obj += vv * (hi);       \
            else dv += vv * vv;                            \
        }                                                  \
    } while (0)
    for (int64_t i = 0; i < m; ++i) TERM(y[i], p->lc[i], p->uc[i]);
    for (int64_t j = 0; j < n; ++j) TERM(p->c[j] - aty[j], p->lv[j], p->uv[j]);
#undef TERM
    double dual_violation = sqrt(dv);

    double bn = -0.0;
    for (int64_t i = 0; i < m; ++i) {
        double l = isfinite(p->lc[i]) ? p->lc[i] : 0.0;
        double u = (isfinite(p->uc[i]) && p->uc[i] != p->lc[i]) ? p->uc[i] : 0.0;
        bn += l * l;
        bn += u * u;
    }
    bn = sqrt(bn);
    double c_norm = -0.0;
    for (int64_t j = 0; j < n; ++j) c_norm += p->c[j] * p->c[j];
    c_norm = sqrt(c_norm);
    double primal = sqrt(cv * cv + bv * bv);
    out->primal_objective = po;
    out->dual_objective = dual_obj;
    out->constraint_violation = cv;
    out->bound_violation = bv;
    out->dual_violation = dual_violation;
    out->relative_primal = primal / (1.0 + bn);
    out->relative_dual = dual_violation / (1.0 + c_norm);
    out->relative_gap = fabs(po - dual_obj) / (1.0 + fabs(po) + fabs(dual_obj));
    free(ax);
    free(aty);
}

double or_kkt_max_relative(const or_kkt_report *r) { /* lib.rs:28-30 */
    return fmax(fmax(r->relative_primal, r->relative_dual), r->relative_gap);
}
