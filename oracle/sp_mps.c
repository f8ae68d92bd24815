/*
 * sp_mps.c — free-format MPS reader for the oracle (TEST INFRASTRUCTURE ONLY).
 *
 * Restates crates/saddlepoint-io/src/lib.rs:59-309 (read_mps) so that the
 * Netlib fixtures can be loaded without the Rust toolchain: the same sections,
 * the same error cases (reported with 1-based line numbers), the same RANGES
 * and BOUNDS rules, the same handling of the objective row and of maximisation.
 */
#define _GNU_SOURCE
#include <ctype.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "sp_oracle.h"

/* ---- a small string -> index map (open addressing) ---------------------- */
typedef struct {
    char **keys;
    int64_t *vals;
    int64_t cap, len;
} smap;

static uint64_t hash_str(const char *s) {
    uint64_t h = 1469598103934665603ull;
    while (*s) h = (h ^ (unsigned char)*s++) * 1099511628211ull;
    return h;
}
static void smap_free(smap *m) {
    for (int64_t i = 0; i < m->cap; ++i) free(m->keys[i]);
    free(m->keys);
    free(m->vals);
    memset(m, 0, sizeof *m);
}
static int64_t smap_get(const smap *m, const char *k) {
    if (!m->cap) return -1;
    uint64_t i = hash_str(k) & (m->cap - 1);
    while (m->keys[i]) {
        if (!strcmp(m->keys[i], k)) return m->vals[i];
        i = (i + 1) & (m->cap - 1);
    }
    return -1;
}
static void smap_put(smap *m, const char *k, int64_t v);
static void smap_grow(smap *m) {
    smap n = {0};
    n.cap = m->cap ? m->cap * 2 : 64;
    n.keys = calloc(n.cap, sizeof(char *));
    n.vals = calloc(n.cap, sizeof(int64_t));
    for (int64_t i = 0; i < m->cap; ++i)
        if (m->keys[i]) {
            smap_put(&n, m->keys[i], m->vals[i]);
        }
    smap_free(m);
    *m = n;
}
/* Inserts or overwrites. */
static void smap_put(smap *m, const char *k, int64_t v) {
    if ((m->len + 1) * 2 > m->cap) smap_grow(m);
    uint64_t i = hash_str(k) & (m->cap - 1);
    while (m->keys[i]) {
        if (!strcmp(m->keys[i], k)) {
            m->vals[i] = v;
            return;
        }
        i = (i + 1) & (m->cap - 1);
    }
    m->keys[i] = strdup(k);
    m->vals[i] = v;
    m->len++;
}

/* ---- growable arrays ---------------------------------------------------- */
#define VEC(T) struct { T *d; int64_t n, cap; }
#define VPUSH(v, x)                                                        \
    do {                                                                   \
        if ((v).n == (v).cap) {                                            \
            (v).cap = (v).cap ? (v).cap * 2 : 16;                          \
            (v).d = realloc((v).d, sizeof(*(v).d) * (size_t)(v).cap);      \
        }                                                                  \
        (v).d[(v).n++] = (x);                                              \
    } while (0)

enum { S_NONE, S_NAME, S_OBJSENSE, S_ROWS, S_COLUMNS, S_RHS, S_RANGES, S_BOUNDS, S_END };
enum { ROW_E, ROW_L, ROW_G };

static void upper(char *d, const char *s, size_t cap) {
    size_t i = 0;
    for (; s[i] && i + 1 < cap; ++i) d[i] = (char)toupper((unsigned char)s[i]);
    d[i] = 0;
}
static int ieq(const char *a, const char *b) {
    while (*a && *b)
        if (toupper((unsigned char)*a++) != toupper((unsigned char)*b++)) return 0;
    return *a == *b;
}
/* parse_sense (io/src/lib.rs:311-317): 1 max, 0 min, -1 unknown. */
static int parse_sense(const char *s) {
    if (ieq(s, "MAX") || ieq(s, "MAXIMIZE") || ieq(s, "MAXIMISE")) return 1;
    if (ieq(s, "MIN") || ieq(s, "MINIMIZE") || ieq(s, "MINIMISE")) return 0;
    return -1;
}
/* parse_num (io/src/lib.rs:319-322): Rust's f64 grammar, NaN rejected. */
static int parse_num(const char *s, double *out) {
    const char *p = s;
    if (*p == '+' || *p == '-') ++p;
    if (p[0] == '0' && (p[1] == 'x' || p[1] == 'X')) return 0; /* Rust has no hex floats */
    char *end;
    double v = strtod(s, &end);
    if (end == s || *end) return 0;
    if (isnan(v)) return 0;
    *out = v;
    return 1;
}
/* Strips quote characters at both ends, like str::trim_matches('\''). */
static void trim_quotes(char *d, const char *s, size_t cap) {
    size_t n = strlen(s), a = 0;
    while (a < n && s[a] == '\'') ++a;
    while (n > a && s[n - 1] == '\'') --n;
    size_t k = 0;
    for (size_t i = a; i < n && k + 1 < cap; ++i) d[k++] = s[i];
    d[k] = 0;
}

#define MAXF 64

int or_read_mps(const char *text, size_t len, or_lp *out, int64_t *err_line, char *err, size_t errlen) {
    memset(out, 0, sizeof *out);
    int maximize = 0;
    char *obj_row = NULL;
    smap row_index = {0}, col_index = {0}, ignored = {0};
    VEC(int) row_kind = {0};
    VEC(double) c = {0}, rhs = {0}, range = {0}, lv = {0}, uv = {0};
    VEC(char) has_range = {0};
    VEC(int64_t) tr = {0}, tc = {0};
    VEC(double) tv = {0};
    double c0 = 0.0;
    char *rhs_set = NULL, *ranges_set = NULL, *bounds_set = NULL;
    int section = S_NONE;
    int rc = OR_OK;
    int64_t lineno = 0;
    char *line = NULL;
    size_t line_cap = 0;
    size_t pos = 0;
    *err_line = 0;
    if (errlen) err[0] = 0;

#define FAIL(...)                                     \
    do {                                              \
        snprintf(err, errlen, __VA_ARGS__);           \
        *err_line = lineno;                           \
        rc = OR_ERR_PARSE;                            \
        goto done;                                    \
    } while (0)

    while (pos < len) {
        size_t e = pos;
        while (e < len && text[e] != '\n') ++e;
        size_t l = e - pos;
        if (l && text[pos + l - 1] == '\r') --l; /* BufRead::lines strips "\r\n" */
        if (l + 1 > line_cap) {
            line_cap = l + 1;
            line = realloc(line, line_cap);
        }
        memcpy(line, text + pos, l);
        line[l] = 0;
        pos = e + 1;
        ++lineno;
        /* skip comments and blank lines */
        int blank = 1;
        for (size_t i = 0; i < l; ++i)
            if (!isspace((unsigned char)line[i])) { blank = 0; break; }
        if (line[0] == '*' || blank) continue;
        char *f[MAXF];
        int nf = 0;
        char *save = NULL;
        int indented = (line[0] == ' ' || line[0] == '\t');
        for (char *t = strtok_r(line, " \t\r\f\v", &save); t && nf < MAXF; t = strtok_r(NULL, " \t\r\f\v", &save))
            f[nf++] = t;
        if (!indented) {
            char up[64];
            upper(up, f[0], sizeof up);
            int prev = section;
            if (!strcmp(up, "NAME")) section = S_NAME;
            else if (!strcmp(up, "OBJSENSE")) {
                if (nf > 1) {
                    int s = parse_sense(f[1]);
                    if (s < 0) FAIL("bad OBJSENSE %s", f[1]);
                    maximize = s;
                }
                section = S_OBJSENSE;
            } else if (!strcmp(up, "OBJSENCE")) section = S_OBJSENSE;
            else if (!strcmp(up, "ROWS")) section = S_ROWS;
            else if (!strcmp(up, "COLUMNS")) section = S_COLUMNS;
            else if (!strcmp(up, "RHS")) section = S_RHS;
            else if (!strcmp(up, "RANGES")) section = S_RANGES;
            else if (!strcmp(up, "BOUNDS")) section = S_BOUNDS;
            else if (!strcmp(up, "ENDATA")) section = S_END;
            else if ((!strcmp(up, "OBJSENSE_MAX") || !strcmp(up, "MAX") || !strcmp(up, "MAXIMIZE") ||
                      !strcmp(up, "MIN") || !strcmp(up, "MINIMIZE")) &&
                     prev == S_OBJSENSE) {
                int s = parse_sense(f[0]);
                maximize = s < 0 ? 0 : s;
                section = S_OBJSENSE;
            } else if (!strcmp(up, "QUADOBJ") || !strcmp(up, "QMATRIX") || !strcmp(up, "QSECTION") ||
                       !strcmp(up, "CSECTION") || !strcmp(up, "SOS") || !strcmp(up, "INDICATORS"))
                FAIL("section %s is not supported", f[0]);
            else FAIL("unknown section %s", f[0]);
            if (section == S_END) break;
            continue;
        }
        switch (section) {
        case S_OBJSENSE: {
            int s = parse_sense(f[0]);
            if (s < 0) FAIL("bad OBJSENSE %s", f[0]);
            maximize = s;
            break;
        }
        case S_ROWS: {
            if (nf < 2) FAIL("ROWS line needs a type and a name");
            char up[8];
            upper(up, f[0], sizeof up);
            int kind;
            if (!strcmp(up, "N")) {
                if (!obj_row) obj_row = strdup(f[1]);
                else smap_put(&ignored, f[1], 1);
                continue;
            } else if (!strcmp(up, "E")) kind = ROW_E;
            else if (!strcmp(up, "L")) kind = ROW_L;
            else if (!strcmp(up, "G")) kind = ROW_G;
            else FAIL("unknown row type %s", f[0]);
            if (smap_get(&row_index, f[1]) >= 0) FAIL("duplicate row %s", f[1]);
            smap_put(&row_index, f[1], row_kind.n);
            VPUSH(row_kind, kind);
            VPUSH(rhs, 0.0);
            VPUSH(range, 0.0);
            VPUSH(has_range, 0);
            break;
        }
        case S_COLUMNS: {
            if (nf >= 3) {
                char q[64];
                trim_quotes(q, f[1], sizeof q);
                if (ieq(q, "MARKER")) {
                    char m[64], um[64];
                    trim_quotes(m, f[2], sizeof m);
                    upper(um, m, sizeof um);
                    if (strcmp(um, "INTORG") && strcmp(um, "INTEND")) FAIL("unknown marker %s", um);
                    continue; /* integrality is dropped */
                }
            }
            if (nf < 3 || nf % 2 == 0) FAIL("COLUMNS line needs a column and row/value pairs");
            int64_t j = smap_get(&col_index, f[0]);
            if (j < 0) {
                j = c.n;
                smap_put(&col_index, f[0], j);
                VPUSH(c, 0.0);
                VPUSH(lv, 0.0);
                VPUSH(uv, INFINITY);
            }
            for (int t = 1; t + 1 < nf; t += 2) {
                double v;
                if (!parse_num(f[t + 1], &v)) FAIL("bad number %s", f[t + 1]);
                if (obj_row && !strcmp(obj_row, f[t])) c.d[j] += v;
                else {
                    int64_t i = smap_get(&row_index, f[t]);
                    if (i >= 0) {
                        VPUSH(tr, i);
                        VPUSH(tc, j);
                        VPUSH(tv, v);
                    } else if (smap_get(&ignored, f[t]) < 0) FAIL("unknown row %s", f[t]);
                }
            }
            break;
        }
        case S_RHS:
        case S_RANGES: {
            const char *set = "";
            int first = 0;
            if (nf % 2 == 1) {
                set = f[0];
                first = 1;
            }
            char **chosen = section == S_RHS ? &rhs_set : &ranges_set;
            if (!*chosen) *chosen = strdup(set);
            if (strcmp(*chosen, set)) continue;
            for (int t = first; t + 1 < nf; t += 2) {
                double v;
                if (!parse_num(f[t + 1], &v)) FAIL("bad number %s", f[t + 1]);
                if (obj_row && !strcmp(obj_row, f[t])) {
                    if (section == S_RHS) c0 = -v;
                } else {
                    int64_t i = smap_get(&row_index, f[t]);
                    if (i >= 0) {
                        if (section == S_RHS) rhs.d[i] = v;
                        else {
                            range.d[i] = v;
                            has_range.d[i] = 1;
                        }
                    } else if (smap_get(&ignored, f[t]) < 0) FAIL("unknown row %s", f[t]);
                }
            }
            break;
        }
        case S_BOUNDS: {
            char kind[16];
            upper(kind, f[0], sizeof kind);
            int needs_value = !(!strcmp(kind, "FR") || !strcmp(kind, "MI") || !strcmp(kind, "PL") || !strcmp(kind, "BV"));
            const char *set, *col, *val;
            if ((nf == 4 && needs_value) || (nf == 3 && !needs_value)) {
                set = f[1]; col = f[2]; val = nf > 3 ? f[3] : NULL;
            } else if ((nf == 3 && needs_value) || (nf == 2 && !needs_value)) {
                set = ""; col = f[1]; val = nf > 2 ? f[2] : NULL;
            } else if (nf == 4 && !needs_value) {
                set = f[1]; col = f[2]; val = NULL;
            } else FAIL("malformed BOUNDS line");
            if (!bounds_set) bounds_set = strdup(set);
            if (strcmp(bounds_set, set)) continue;
            int64_t j = smap_get(&col_index, col);
            if (j < 0) FAIL("unknown column %s", col);
            double v = 0.0;
            if (val && !parse_num(val, &v)) FAIL("bad number %s", val);
            if (!strcmp(kind, "UP") || !strcmp(kind, "UI")) {
                uv.d[j] = v;
                if (v < 0.0 && lv.d[j] == 0.0) lv.d[j] = -INFINITY;
            } else if (!strcmp(kind, "LO") || !strcmp(kind, "LI")) lv.d[j] = v;
            else if (!strcmp(kind, "FX")) { lv.d[j] = v; uv.d[j] = v; }
            else if (!strcmp(kind, "FR")) { lv.d[j] = -INFINITY; uv.d[j] = INFINITY; }
            else if (!strcmp(kind, "MI")) lv.d[j] = -INFINITY;
            else if (!strcmp(kind, "PL")) uv.d[j] = INFINITY;
            else if (!strcmp(kind, "BV")) { lv.d[j] = 0.0; uv.d[j] = 1.0; }
            else FAIL("unsupported bound type %s", f[0]);
            break;
        }
        case S_NAME:
            break;
        case S_NONE:
            FAIL("data before the first section");
        default:
            break;
        }
    }

    {
        int64_t m = row_kind.n, n = c.n;
        out->lc = malloc(sizeof(double) * (m ? m : 1));
        out->uc = malloc(sizeof(double) * (m ? m : 1));
        for (int64_t i = 0; i < m; ++i) { /* io/src/lib.rs:276-289 */
            double b = rhs.d[i], lo, hi;
            if (!has_range.d[i]) {
                if (row_kind.d[i] == ROW_E) { lo = b; hi = b; }
                else if (row_kind.d[i] == ROW_L) { lo = -INFINITY; hi = b; }
                else { lo = b; hi = INFINITY; }
            } else {
                double r = range.d[i];
                if (row_kind.d[i] == ROW_E) {
                    if (r >= 0.0) { lo = b; hi = b + r; }
                    else { lo = b + r; hi = b; }
                } else if (row_kind.d[i] == ROW_L) { lo = b - fabs(r); hi = b; }
                else { lo = b; hi = b + fabs(r); }
            }
            out->lc[i] = lo;
            out->uc[i] = hi;
        }
        if (maximize) {
            for (int64_t j = 0; j < n; ++j) c.d[j] = -c.d[j];
            c0 = -c0;
        }
        or_csr_from_triplets(m, n, tr.n, tr.d, tc.d, tv.d, &out->a);
        out->c = c.d ? c.d : malloc(sizeof(double));
        out->lv = lv.d ? lv.d : malloc(sizeof(double));
        out->uv = uv.d ? uv.d : malloc(sizeof(double));
        c.d = lv.d = uv.d = NULL;
        out->c0 = c0;
        out->maximize = maximize;
    }
done:
#undef FAIL
    if (rc != OR_OK) {
        free(out->lc);
        free(out->uc);
        memset(out, 0, sizeof *out);
    }
    free(line);
    free(obj_row);
    free(rhs_set);
    free(ranges_set);
    free(bounds_set);
    smap_free(&row_index);
    smap_free(&col_index);
    smap_free(&ignored);
    free(row_kind.d);
    free(c.d);
    free(rhs.d);
    free(range.d);
    free(has_range.d);
    free(lv.d);
    free(uv.d);
    free(tr.d);
    free(tc.d);
    free(tv.d);
    return rc;
}
