/*
 * sp_gen.c — the seeded synthetic LP generators, restated in plain C for the oracle.
 *
 * TEST INFRASTRUCTURE ONLY. The CUDA library ships the same generators
 * (saddlepoint_b200/csrc/host.cpp, sp_generate); this copy lets the CPU side (the
 * reference arm of the benchmark, fixture scripts) build the identical LP without
 * loading the product library. tests/test_oracle.py checks that both give the same
 * arrays bit for bit.
 *
 * The random stream is the reference's xorshift64 (crates/saddlepoint-cuda/examples/
 * speedup.rs:22-34: x ^= x << 13; x ^= x >> 7; x ^= x << 17; unit = (x >> 11) / 2^53),
 * one stream per column (and per row for the slack draws), each seeded by splitmix64;
 * N(0,1) by Box-Muller.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "sp_oracle.h"

typedef struct { uint64_t s; } g_rng;

static uint64_t g_next(g_rng *r) {
    r->s ^= r->s << 13;
    r->s ^= r->s >> 7;
    r->s ^= r->s << 17;
    return r->s;
}
static double g_unit(g_rng *r) { return (double)(g_next(r) >> 11) / (double)(1ull << 53); }
static double g_normal(g_rng *r) { /* Box-Muller, first of the pair */
    const double u1 = 1.0 - g_unit(r), u2 = g_unit(r);
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}
static uint64_t g_below(g_rng *r, uint64_t n) { return g_next(r) % n; }

static uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
enum { FAMILY_COL = 1, FAMILY_ROW = 2, FAMILY_GLOBAL = 3 };
static g_rng g_stream(uint64_t seed, uint64_t family, uint64_t index) {
    g_rng r;
    r.s = splitmix64(seed ^ splitmix64(family * 0x100000001B3ull + index));
    if (!r.s) r.s = 0x2545F4914F6CDD1Dull;
    return r;
}

/* Draws d distinct rows in [0, m) (rejection, in draw order). */
static void distinct_rows(g_rng *r, int64_t d, int64_t m, int64_t *out) {
    for (int64_t q = 0; q < d; ++q) {
        for (;;) {
            const int64_t cand = (int64_t)(int32_t)g_below(r, (uint64_t)m);
            int dup = 0;
            for (int64_t t = 0; t < q; ++t)
                if (out[t] == cand) { dup = 1; break; }
            if (!dup) { out[q] = cand; break; }
        }
    }
}

static int cmp_i64(const void *a, const void *b) {
    const int64_t x = *(const int64_t *)a, y = *(const int64_t *)b;
    return (x > y) - (x < y);
}

/* Draws d rows, then redraws every later duplicate of an earlier entry (in index order)
 * until a sorted copy shows none: the rule for columns of more than 32 entries. */
static int long_rows(g_rng *r, int64_t d, int64_t m, int64_t *out, int64_t *scratch) {
    for (int64_t q = 0; q < d; ++q) out[q] = (int64_t)(int32_t)g_below(r, (uint64_t)m);
    for (;;) {
        memcpy(scratch, out, sizeof(int64_t) * d);
        qsort(scratch, (size_t)d, sizeof(int64_t), cmp_i64);
        int dup = 0;
        for (int64_t q = 1; q < d; ++q)
            if (scratch[q] == scratch[q - 1]) { dup = 1; break; }
        if (!dup) return 0;
        for (int64_t q = 0; q < d; ++q)
            for (int64_t t = 0; t < q; ++t)
                if (out[t] == out[q]) { out[q] = (int64_t)(int32_t)g_below(r, (uint64_t)m); break; }
    }
}

static void *xmalloc(size_t n) { return malloc(n ? n : 1); }

/* Column-major entries to CSR, columns ascending in each row. */
static int csc_to_csr(int64_t m, int64_t n, const int64_t *cp, const int64_t *ri, const double *vals, or_lp *o) {
    const int64_t nnz = cp[n];
    o->a.nrows = m;
    o->a.ncols = n;
    o->a.nnz = nnz;
    o->a.row_ptr = calloc((size_t)m + 1, sizeof(int64_t));
    o->a.col_idx = xmalloc(sizeof(int64_t) * nnz);
    o->a.values = xmalloc(sizeof(double) * nnz);
    int64_t *next = xmalloc(sizeof(int64_t) * (m + 1));
    if (!o->a.row_ptr || !o->a.col_idx || !o->a.values || !next) { free(next); return OR_ERR_ALLOC; }
    for (int64_t k = 0; k < nnz; ++k) o->a.row_ptr[ri[k] + 1] += 1;
    for (int64_t i = 0; i < m; ++i) o->a.row_ptr[i + 1] += o->a.row_ptr[i];
    memcpy(next, o->a.row_ptr, sizeof(int64_t) * m);
    for (int64_t j = 0; j < n; ++j)
        for (int64_t k = cp[j]; k < cp[j + 1]; ++k) {
            const int64_t t = next[ri[k]]++;
            o->a.col_idx[t] = j;
            o->a.values[t] = vals[k];
        }
    free(next);
    return OR_OK;
}

/* x0 ~ U[0,1]^n; the first m/2 rows equalities A x0, the rest <= A x0 + U[0,1];
 * 0 <= x <= 10 (c is drawn with the columns). */
static int finish_random_lp(uint64_t seed, int64_t m, int64_t n, const double *x0, or_lp *o) {
    o->lc = xmalloc(sizeof(double) * m);
    o->uc = xmalloc(sizeof(double) * m);
    o->lv = xmalloc(sizeof(double) * n);
    o->uv = xmalloc(sizeof(double) * n);
    if (!o->lc || !o->uc || !o->lv || !o->uv) return OR_ERR_ALLOC;
    for (int64_t i = 0; i < m; ++i) {
        double s = -0.0;
        for (int64_t k = o->a.row_ptr[i]; k < o->a.row_ptr[i + 1]; ++k) s += o->a.values[k] * x0[o->a.col_idx[k]];
        if (i < m / 2) {
            o->lc[i] = o->uc[i] = s;
        } else {
            g_rng r = g_stream(seed, FAMILY_ROW, (uint64_t)i);
            o->lc[i] = -INFINITY;
            o->uc[i] = s + g_unit(&r);
        }
    }
    for (int64_t j = 0; j < n; ++j) {
        o->lv[j] = 0.0;
        o->uv[j] = 10.0;
    }
    return OR_OK;
}

/* Rows and values of the columns, x0 and c, given each column's degree and stream. The
 * random LP draws every column's rows by rejection; the power-law LP (long_rule) uses
 * the redraw rule for columns of more than 32 entries. */
static int fill_columns(int64_t m, int64_t n, const int64_t *deg, g_rng *rngs, uint64_t seed, int long_rule,
                        or_lp *o) {
    int64_t *cp = xmalloc(sizeof(int64_t) * (n + 1));
    if (!cp) return OR_ERR_ALLOC;
    cp[0] = 0;
    int64_t dmax = 0;
    for (int64_t j = 0; j < n; ++j) {
        cp[j + 1] = cp[j] + deg[j];
        if (deg[j] > dmax) dmax = deg[j];
    }
    int64_t *ri = xmalloc(sizeof(int64_t) * cp[n]);
    double *vals = xmalloc(sizeof(double) * cp[n]);
    double *x0 = xmalloc(sizeof(double) * n);
    int64_t *scratch = xmalloc(sizeof(int64_t) * (dmax + 1));
    o->c = xmalloc(sizeof(double) * n);
    int rc = OR_ERR_ALLOC;
    if (ri && vals && x0 && scratch && o->c) {
        for (int64_t j = 0; j < n; ++j) {
            g_rng *r = &rngs[j];
            if (!long_rule || deg[j] <= 32) distinct_rows(r, deg[j], m, &ri[cp[j]]);
            else long_rows(r, deg[j], m, &ri[cp[j]], scratch);
            for (int64_t k = cp[j]; k < cp[j + 1]; ++k) vals[k] = g_normal(r);
            x0[j] = g_unit(r);
            o->c[j] = 2.0 * g_unit(r) - 1.0;
        }
        rc = csc_to_csr(m, n, cp, ri, vals, o);
        if (!rc) rc = finish_random_lp(seed, m, n, x0, o);
    }
    free(cp);
    free(ri);
    free(vals);
    free(x0);
    free(scratch);
    return rc;
}

static int gen_random(const or_gen_params *g, or_lp *o) {
    const int64_t m = g->nrows, n = g->ncols;
    const int64_t dmin = g->nnz_per_col_min < 1 ? 1 : g->nnz_per_col_min;
    const int64_t dmax = g->nnz_per_col_max > dmin ? g->nnz_per_col_max : dmin;
    if (m <= 0 || n <= 0 || dmax > m) return OR_ERR_PROBLEM;
    int64_t *deg = xmalloc(sizeof(int64_t) * n);
    g_rng *rngs = xmalloc(sizeof(g_rng) * n);
    int rc = OR_ERR_ALLOC;
    if (deg && rngs) {
        for (int64_t j = 0; j < n; ++j) {
            rngs[j] = g_stream(g->seed, FAMILY_COL, (uint64_t)j);
            deg[j] = dmin + (int64_t)g_below(&rngs[j], (uint64_t)(dmax - dmin + 1));
        }
        rc = fill_columns(m, n, deg, rngs, g->seed, 0, o);
    }
    free(deg);
    free(rngs);
    return rc;
}

static int64_t clamped(int64_t raw, double f, int64_t dmin, int64_t dmax) {
    const int64_t d = (int64_t)floor((double)raw * f);
    return d < dmin ? dmin : (d > dmax ? dmax : d);
}

/* Zipf(s) column degrees truncated to [dmin, dmax], rescaled by one factor f found by
 * bisection so the total is <= target, d_j <- max(dmin, floor(d_j f)); the remainder is
 * added one by one to the first columns in index order that stay within the bounds. */
static int gen_powerlaw(const or_gen_params *g, or_lp *o) {
    const int64_t m = g->nrows, n = g->ncols, dmin = g->degree_min;
    const int64_t dmax = g->degree_max < m ? g->degree_max : m;
    if (m <= 0 || n <= 0 || dmin < 1 || dmax < dmin || g->target_nnz < n * dmin || g->target_nnz > n * dmax)
        return OR_ERR_PROBLEM;
    const int64_t nd = dmax - dmin + 1;
    double *cdf = xmalloc(sizeof(double) * nd);
    int64_t *raw = xmalloc(sizeof(int64_t) * n), *deg = xmalloc(sizeof(int64_t) * n);
    g_rng *rngs = xmalloc(sizeof(g_rng) * n);
    int rc = OR_ERR_ALLOC;
    if (cdf && raw && deg && rngs) {
        double acc = 0.0;
        for (int64_t d = dmin; d <= dmax; ++d) {
            acc += pow((double)d, -g->zipf_s);
            cdf[d - dmin] = acc;
        }
        for (int64_t q = 0; q < nd; ++q) cdf[q] /= acc;
        for (int64_t j = 0; j < n; ++j) {
            rngs[j] = g_stream(g->seed, FAMILY_COL, (uint64_t)j);
            const double u = g_unit(&rngs[j]);
            int64_t lo = 0, hi = nd; /* first q with cdf[q] >= u */
            while (lo < hi) {
                const int64_t mid = lo + (hi - lo) / 2;
                if (cdf[mid] < u) lo = mid + 1;
                else hi = mid;
            }
            raw[j] = dmin + lo;
            if (raw[j] > dmax) raw[j] = dmax;
        }
        double flo = 0.0, fhi = 1.0;
        for (;;) {
            int64_t t = 0;
            for (int64_t j = 0; j < n; ++j) t += clamped(raw[j], fhi, dmin, dmax);
            if (!(t < g->target_nnz && fhi < 1e9)) break;
            fhi *= 2.0;
        }
        for (int it = 0; it < 100; ++it) {
            const double mid = 0.5 * (flo + fhi);
            int64_t t = 0;
            for (int64_t j = 0; j < n; ++j) t += clamped(raw[j], mid, dmin, dmax);
            if (t <= g->target_nnz) flo = mid;
            else fhi = mid;
        }
        int64_t sum = 0;
        for (int64_t j = 0; j < n; ++j) {
            deg[j] = clamped(raw[j], flo, dmin, dmax);
            sum += deg[j];
        }
        for (int64_t pass = 0; sum < g->target_nnz && pass < dmax; ++pass)
            for (int64_t j = 0; j < n && sum < g->target_nnz; ++j)
                if (deg[j] < dmax) {
                    deg[j] += 1;
                    sum += 1;
                }
        rc = fill_columns(m, n, deg, rngs, g->seed, 1, o);
    }
    free(cdf);
    free(raw);
    free(deg);
    free(rngs);
    return rc;
}

/* Transportation LP: supplies U{1..1000}; demands split the same total by seeded
 * weights; arc (i, j) is column i*D + j with +1 in rows i and S + j; equalities;
 * costs U{1..100}; 0 <= x < inf. */
static int gen_transport(const or_gen_params *g, or_lp *o) {
    const int64_t S = g->supplies, D = g->demands;
    if (S <= 0 || D <= 0 || S * D > INT32_MAX) return OR_ERR_PROBLEM;
    const int64_t m = S + D, n = S * D;
    g_rng gr = g_stream(g->seed, FAMILY_GLOBAL, 0);
    double *sup = xmalloc(sizeof(double) * S), *dem = xmalloc(sizeof(double) * D), *w = xmalloc(sizeof(double) * D);
    o->a.nrows = m;
    o->a.ncols = n;
    o->a.nnz = 2 * n;
    o->a.row_ptr = xmalloc(sizeof(int64_t) * (m + 1));
    o->a.col_idx = xmalloc(sizeof(int64_t) * 2 * n);
    o->a.values = xmalloc(sizeof(double) * 2 * n);
    o->c = xmalloc(sizeof(double) * n);
    o->lc = xmalloc(sizeof(double) * m);
    o->uc = xmalloc(sizeof(double) * m);
    o->lv = xmalloc(sizeof(double) * n);
    o->uv = xmalloc(sizeof(double) * n);
    int rc = OR_ERR_ALLOC;
    if (sup && dem && w && o->a.row_ptr && o->a.col_idx && o->a.values && o->c && o->lc && o->uc && o->lv && o->uv) {
        double total = 0.0, wsum = 0.0, dsum = 0.0;
        for (int64_t i = 0; i < S; ++i) {
            sup[i] = (double)(1 + g_below(&gr, 1000));
            total += sup[i];
        }
        for (int64_t j = 0; j < D; ++j) {
            w[j] = 1.0 - g_unit(&gr);
            wsum += w[j];
        }
        for (int64_t j = 0; j < D; ++j) {
            dem[j] = floor(total * w[j] / wsum);
            dsum += dem[j];
        }
        for (int64_t j = 0; dsum < total; j = (j + 1) % D) {
            dem[j] += 1.0;
            dsum += 1.0;
        }
        int64_t k = 0;
        o->a.row_ptr[0] = 0;
        for (int64_t i = 0; i < S; ++i) {
            for (int64_t j = 0; j < D; ++j) o->a.col_idx[k++] = i * D + j;
            o->a.row_ptr[i + 1] = k;
        }
        for (int64_t j = 0; j < D; ++j) {
            for (int64_t i = 0; i < S; ++i) o->a.col_idx[k++] = i * D + j;
            o->a.row_ptr[S + j + 1] = k;
        }
        for (int64_t q = 0; q < 2 * n; ++q) o->a.values[q] = 1.0;
        for (int64_t i = 0; i < S; ++i) {
            g_rng r = g_stream(g->seed, FAMILY_COL, (uint64_t)i);
            for (int64_t j = 0; j < D; ++j) o->c[i * D + j] = (double)(1 + g_below(&r, 100));
        }
        for (int64_t i = 0; i < S; ++i) o->lc[i] = o->uc[i] = sup[i];
        for (int64_t j = 0; j < D; ++j) o->lc[S + j] = o->uc[S + j] = dem[j];
        for (int64_t j = 0; j < n; ++j) {
            o->lv[j] = 0.0;
            o->uv[j] = INFINITY;
        }
        rc = OR_OK;
    }
    free(sup);
    free(dem);
    free(w);
    return rc;
}

int or_generate(const or_gen_params *g, or_lp *out) {
    if (!g || !out) return OR_ERR_PROBLEM;
    memset(out, 0, sizeof *out);
    int rc;
    switch (g->kind) {
    case 0: rc = gen_random(g, out); break;
    case 1: rc = gen_powerlaw(g, out); break;
    case 2: rc = gen_transport(g, out); break;
    default: rc = OR_ERR_PROBLEM;
    }
    if (rc) or_lp_free(out);
    return rc;
}
