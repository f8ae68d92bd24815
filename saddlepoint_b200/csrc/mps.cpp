// mps.cpp — the MPS reader of the library (Part 5 of the C ABI): free-format MPS text
// to an sp_lp with library-owned arrays (release with sp_lp_release).
//
// It follows saddlepoint-io's read_mps (crates/saddlepoint-io/src/lib.rs:59-309) rule
// for rule: sections NAME, OBJSENSE (also OBJSENCE and a sense keyword on its own
// line), ROWS (the first N row is the objective, later N rows are ignored), COLUMNS
// (MARKER lines skipped — integrality is dropped), RHS / RANGES / BOUNDS with only
// the first set used, the classic negative-UP rule, ranges per row kind, the
// objective constant as minus the objective row's RHS, and maximisation by negating
// c and c0. Errors carry the 1-based line number and the reference's message. The
// matrix is built as CsrMatrix::from_triplets builds it (problem.rs:33-77): rows by a
// counting sort, each row's entries sorted by column (stably: duplicates are summed in
// file order), duplicates summed, exact zeros dropped.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "../../include/saddlepoint_b200.h"

namespace sp {
void register_owned_lp(sp_lp *out, std::vector<int64_t> &&rp, std::vector<int32_t> &&ci, std::vector<double> &&v,
                       std::vector<double> &&c, std::vector<double> &&lc, std::vector<double> &&uc,
                       std::vector<double> &&lv, std::vector<double> &&uv);
}

namespace {

constexpr double INF = std::numeric_limits<double>::infinity();

enum class Section { None, Name, ObjSense, Rows, Columns, Rhs, Ranges, Bounds, End };
enum class RowKind { E, L, G };

std::string upper(const std::string &s) {
    std::string u(s);
    for (char &ch : u) ch = (char)std::toupper((unsigned char)ch);
    return u;
}

bool is_space(char ch) { return ch == ' ' || ch == '\t' || ch == '\r' || ch == '\n' || ch == '\f' || ch == '\v'; }

// parse_sense (io/src/lib.rs:311-317): 1 max, 0 min, -1 neither.
int parse_sense(const std::string &s) {
    const std::string u = upper(s);
    if (u == "MAX" || u == "MAXIMIZE" || u == "MAXIMISE") return 1;
    if (u == "MIN" || u == "MINIMIZE" || u == "MINIMISE") return 0;
    return -1;
}

// parse_num (io/src/lib.rs:319-322): Rust's f64 grammar (decimal, exponent,
// inf/infinity), the whole field, NaN rejected. strtod also reads hexadecimal
// floats and "nan(...)", which Rust does not: those are rejected here too.
bool parse_num(const std::string &s, double *out) {
    const char *p = s.c_str();
    const char *q = (*p == '+' || *p == '-') ? p + 1 : p;
    if (q[0] == '0' && (q[1] == 'x' || q[1] == 'X')) return false;
    char *end = nullptr;
    const double v = std::strtod(p, &end);
    if (end == p || *end != '\0' || std::isnan(v)) return false;
    *out = v;
    return true;
}

std::string trim_quotes(const std::string &s) {
    size_t a = 0, b = s.size();
    while (a < b && s[a] == '\'') ++a;
    while (b > a && s[b - 1] == '\'') --b;
    return s.substr(a, b - a);
}

struct ParseError {
    int64_t line;
    std::string msg;
};

struct Triplet {
    int64_t row, col;
    double v;
};

void from_triplets(int64_t m, const std::vector<Triplet> &trip, std::vector<int64_t> &rp, std::vector<int32_t> &ci,
                   std::vector<double> &v) {
    std::vector<int64_t> start(m + 1, 0);
    for (const Triplet &t : trip) ++start[t.row + 1];
    for (int64_t i = 0; i < m; ++i) start[i + 1] += start[i];
    std::vector<int64_t> next(start.begin(), start.end() - 1);
    std::vector<std::pair<int64_t, double>> bucket(trip.size());
    for (const Triplet &t : trip) bucket[next[t.row]++] = {t.col, t.v};
    rp.assign(1, 0);
    rp.reserve(m + 1);
    ci.clear();
    v.clear();
    ci.reserve(trip.size());
    v.reserve(trip.size());
    for (int64_t i = 0; i < m; ++i) {
        auto b = bucket.begin() + start[i], e = bucket.begin() + start[i + 1];
        std::stable_sort(b, e, [](const auto &x, const auto &y) { return x.first < y.first; });
        for (auto k = b; k != e;) {
            const int64_t col = k->first;
            double sum = k->second;
            for (++k; k != e && k->first == col; ++k) sum += k->second;
            if (sum != 0.0) {
                ci.push_back((int32_t)col);
                v.push_back(sum);
            }
        }
        rp.push_back((int64_t)ci.size());
    }
}

// The reader proper; throws ParseError.
void read(const char *text, size_t len, sp_lp *out) {
    bool maximize = false;
    std::string obj_row;
    bool have_obj = false;
    std::unordered_map<std::string, int64_t> row_index, col_index;
    std::unordered_set<std::string> ignored_rows;
    std::vector<RowKind> row_kind;
    std::vector<double> c, rhs, range, lv, uv;
    std::vector<char> has_range;
    std::vector<Triplet> trip;
    double c0 = 0.0;
    std::string rhs_set, ranges_set, bounds_set;
    bool have_rhs_set = false, have_ranges_set = false, have_bounds_set = false;
    Section section = Section::None;
    int64_t lineno = 0;
    std::vector<std::string> f;
    size_t pos = 0;
    while (pos < len) {
        size_t e = pos;
        while (e < len && text[e] != '\n') ++e;
        size_t l = e - pos;
        if (l && text[pos + l - 1] == '\r') --l;  // lines() drops "\r\n" as well as "\n"
        const std::string line(text + pos, l);
        pos = e + 1;
        ++lineno;
        auto fail = [&](const std::string &msg) { throw ParseError{lineno, msg}; };
        if (!line.empty() && line[0] == '*') continue;
        f.clear();
        for (size_t i = 0; i < line.size();) {
            while (i < line.size() && is_space(line[i])) ++i;
            size_t j = i;
            while (j < line.size() && !is_space(line[j])) ++j;
            if (j > i) f.emplace_back(line.substr(i, j - i));
            i = j;
        }
        if (f.empty()) continue;  // blank line
        const bool data = line[0] == ' ' || line[0] == '\t';
        if (!data) {
            const std::string key = upper(f[0]);
            const Section prev = section;
            if (key == "NAME") section = Section::Name;
            else if (key == "OBJSENSE") {
                if (f.size() > 1) {
                    const int s = parse_sense(f[1]);
                    if (s < 0) fail("bad OBJSENSE " + f[1]);
                    maximize = s == 1;
                }
                section = Section::ObjSense;
            } else if (key == "OBJSENCE") section = Section::ObjSense;
            else if (key == "ROWS") section = Section::Rows;
            else if (key == "COLUMNS") section = Section::Columns;
            else if (key == "RHS") section = Section::Rhs;
            else if (key == "RANGES") section = Section::Ranges;
            else if (key == "BOUNDS") section = Section::Bounds;
            else if (key == "ENDATA") section = Section::End;
            else if ((key == "OBJSENSE_MAX" || key == "MAX" || key == "MAXIMIZE" || key == "MIN" || key == "MINIMIZE") &&
                     prev == Section::ObjSense) {
                maximize = parse_sense(f[0]) == 1;
                section = Section::ObjSense;
            } else if (key == "QUADOBJ" || key == "QMATRIX" || key == "QSECTION" || key == "CSECTION" || key == "SOS" ||
                       key == "INDICATORS")
                fail("section " + f[0] + " is not supported");
            else fail("unknown section " + f[0]);
            if (section == Section::End) break;
            continue;
        }
        switch (section) {
        case Section::ObjSense: {
            const int s = parse_sense(f[0]);
            if (s < 0) fail("bad OBJSENSE " + f[0]);
            maximize = s == 1;
            break;
        }
        case Section::Rows: {
            if (f.size() < 2) fail("ROWS line needs a type and a name");
            const std::string t = upper(f[0]);
            RowKind kind;
            if (t == "N") {
                if (!have_obj) {
                    obj_row = f[1];
                    have_obj = true;
                } else {
                    ignored_rows.insert(f[1]);
                }
                continue;
            } else if (t == "E") kind = RowKind::E;
            else if (t == "L") kind = RowKind::L;
            else if (t == "G") kind = RowKind::G;
            else fail("unknown row type " + t);
            if (!row_index.emplace(f[1], (int64_t)row_kind.size()).second) fail("duplicate row " + f[1]);
            row_kind.push_back(kind);
            rhs.push_back(0.0);
            range.push_back(0.0);
            has_range.push_back(0);
            break;
        }
        case Section::Columns: {
            if (f.size() >= 3 && upper(trim_quotes(f[1])) == "MARKER") {
                const std::string mk = upper(trim_quotes(f[2]));
                if (mk != "INTORG" && mk != "INTEND") fail("unknown marker " + mk);
                continue;
            }
            if (f.size() < 3 || f.size() % 2 == 0) fail("COLUMNS line needs a column and row/value pairs");
            auto it = col_index.find(f[0]);
            int64_t j;
            if (it != col_index.end()) {
                j = it->second;
            } else {
                j = (int64_t)c.size();
                col_index.emplace(f[0], j);
                c.push_back(0.0);
                lv.push_back(0.0);
                uv.push_back(INF);
            }
            for (size_t t = 1; t + 1 < f.size(); t += 2) {
                double v;
                if (!parse_num(f[t + 1], &v)) fail("bad number " + f[t + 1]);
                if (have_obj && f[t] == obj_row) {
                    c[j] += v;
                } else {
                    auto r = row_index.find(f[t]);
                    if (r != row_index.end()) trip.push_back({r->second, j, v});
                    else if (!ignored_rows.count(f[t])) fail("unknown row " + f[t]);
                }
            }
            break;
        }
        case Section::Rhs:
        case Section::Ranges: {
            // an odd field count means a set name comes first
            const bool named = f.size() % 2 == 1;
            const std::string set = named ? f[0] : std::string();
            const bool is_rhs = section == Section::Rhs;
            std::string &chosen = is_rhs ? rhs_set : ranges_set;
            bool &have = is_rhs ? have_rhs_set : have_ranges_set;
            if (!have) {
                chosen = set;
                have = true;
            }
            if (chosen != set) continue;
            for (size_t t = named ? 1 : 0; t + 1 < f.size(); t += 2) {
                double v;
                if (!parse_num(f[t + 1], &v)) fail("bad number " + f[t + 1]);
                if (have_obj && f[t] == obj_row) {
                    if (is_rhs) c0 = -v;
                } else {
                    auto r = row_index.find(f[t]);
                    if (r != row_index.end()) {
                        if (is_rhs) {
                            rhs[r->second] = v;
                        } else {
                            range[r->second] = v;
                            has_range[r->second] = 1;
                        }
                    } else if (!ignored_rows.count(f[t])) {
                        fail("unknown row " + f[t]);
                    }
                }
            }
            break;
        }
        case Section::Bounds: {
            const std::string kind = upper(f[0]);
            const bool needs_value = !(kind == "FR" || kind == "MI" || kind == "PL" || kind == "BV");
            const size_t nf = f.size();
            std::string set, col, val;
            bool has_val = false;
            if ((nf == 4 && needs_value) || (nf == 3 && !needs_value)) {
                set = f[1];
                col = f[2];
                if (nf > 3) val = f[3], has_val = true;
            } else if ((nf == 3 && needs_value) || (nf == 2 && !needs_value)) {
                col = f[1];
                if (nf > 2) val = f[2], has_val = true;
            } else if (nf == 4 && !needs_value) {
                set = f[1];
                col = f[2];
            } else {
                fail("malformed BOUNDS line");
            }
            if (!have_bounds_set) {
                bounds_set = set;
                have_bounds_set = true;
            }
            if (bounds_set != set) continue;
            auto it = col_index.find(col);
            if (it == col_index.end()) fail("unknown column " + col);
            const int64_t j = it->second;
            double v = 0.0;
            if (has_val && !parse_num(val, &v)) fail("bad number " + val);
            if (kind == "UP" || kind == "UI") {
                uv[j] = v;
                if (v < 0.0 && lv[j] == 0.0) lv[j] = -INF;  // the classic negative-UP rule
            } else if (kind == "LO" || kind == "LI") {
                lv[j] = v;
            } else if (kind == "FX") {
                lv[j] = v;
                uv[j] = v;
            } else if (kind == "FR") {
                lv[j] = -INF;
                uv[j] = INF;
            } else if (kind == "MI") {
                lv[j] = -INF;
            } else if (kind == "PL") {
                uv[j] = INF;
            } else if (kind == "BV") {
                lv[j] = 0.0;
                uv[j] = 1.0;
            } else {
                fail("unsupported bound type " + kind);
            }
            break;
        }
        case Section::Name:
            break;
        case Section::None:
            fail("data before the first section");
            break;
        case Section::End:
            break;
        }
    }
    // row bounds from the row kinds, right-hand sides and ranges (io/src/lib.rs:276-289)
    const int64_t m = (int64_t)row_kind.size(), n = (int64_t)c.size();
    std::vector<double> lc(m), uc(m);
    for (int64_t i = 0; i < m; ++i) {
        const double b = rhs[i];
        if (!has_range[i]) {
            lc[i] = row_kind[i] == RowKind::L ? -INF : b;
            uc[i] = row_kind[i] == RowKind::G ? INF : b;
        } else {
            const double r = range[i];
            if (row_kind[i] == RowKind::E) {
                lc[i] = r >= 0.0 ? b : b + r;
                uc[i] = r >= 0.0 ? b + r : b;
            } else if (row_kind[i] == RowKind::L) {
                lc[i] = b - std::fabs(r);
                uc[i] = b;
            } else {
                lc[i] = b;
                uc[i] = b + std::fabs(r);
            }
        }
    }
    if (maximize) {
        for (double &x : c) x = -x;
        c0 = -c0;
    }
    if (n > INT32_MAX || (int64_t)trip.size() > INT32_MAX) throw ParseError{lineno, "problem too large"};
    std::vector<int64_t> rp;
    std::vector<int32_t> ci;
    std::vector<double> v;
    from_triplets(m, trip, rp, ci, v);
    sp::register_owned_lp(out, std::move(rp), std::move(ci), std::move(v), std::move(c), std::move(lc), std::move(uc),
                          std::move(lv), std::move(uv));
    out->c0 = c0;
    out->maximize = maximize ? 1 : 0;
}

}  // namespace

extern "C" int sp_read_mps(const char *text, size_t len, sp_lp *out, int64_t *err_line, char *err, size_t errlen) {
    if (err_line) *err_line = 0;
    if (err && errlen) err[0] = '\0';
    if (!out || (!text && len)) return SP_ERR_INVALID;
    std::memset(out, 0, sizeof *out);
    try {
        read(text, len, out);
    } catch (const ParseError &e) {
        if (err_line) *err_line = e.line;
        if (err && errlen) std::snprintf(err, errlen, "%s", e.msg.c_str());
        return SP_ERR_PARSE;
    } catch (const std::bad_alloc &) {
        return SP_ERR_INVALID;
    }
    return SP_OK;
}
