// MPS -> device ingest: reads an MPS file into CSR in one pass on the host and
// uploads its standard form to the engine.
//
// Semantics follow the reference's MpsParser (src/mps_parser.cpp:140-531), so an
// LP read here is the LP the reference reads from the same file:
//   * lines split on whitespace (free format; fixed-format files whose names have no
//     blanks read the same); '*' comment lines; section keywords NAME, OBJSENSE,
//     ROWS, COLUMNS, RHS, RANGES, BOUNDS, ENDATA;
//   * the first N row is the objective; further N rows are dropped;
//   * 'MARKER' lines with INTORG / INTEND delimit integer columns;
//   * the first RHS / RANGES / BOUNDS vector name seen is the one used (a line whose
//     first token names a row carries no vector name); an RHS on the objective row is
//     the negated objective offset;
//   * RANGES R on row type L: [rhs - R, rhs] for R > 0, [rhs, rhs - R] otherwise;
//     on G and E: [rhs, rhs + R] for R > 0, [rhs + R, rhs] otherwise
//     (src/mps_parser.cpp:462-499); the row keeps rhs = lower end, range = upper end;
//   * bounds LO, UP, FX, FR, MI, PL, BV, LI, UI; defaults [0, +inf); a column whose
//     bounds are both infinite is free; BV makes the column binary, LI / UI integer.
// The standard form (min c.x, rows <= or =) negates G rows and, unlike the
// reference's first-order path (which keeps only the lower end of a ranged row,
// src/first_order_solver.cpp:83-99), writes a ranged row as the two rows
// a.x <= upper and -a.x <= -lower (one equality when they coincide).
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "b2p_internal.cuh"

struct b2p_mps {
    std::string name;
    int maximize = 0;
    double obj_offset = 0.0;
    // columns
    std::vector<std::string> col_names;
    std::vector<double> obj, lb, ub;
    std::vector<uint8_t> col_type;  // 0 continuous, 1 integer, 2 binary
    // rows (objective excluded), in file order
    std::vector<std::string> row_names;
    std::vector<char> row_type;     // 'L', 'G', 'E' as declared
    std::vector<uint8_t> ranged;
    std::vector<double> rhs, range_upper;
    // CSR of the rows (column indices ascending, duplicates: the last value read)
    std::vector<int32_t> rowptr, colidx;
    std::vector<double> vals;
};

namespace {

void split(const std::string& line, std::vector<std::string>& tok) {
    tok.clear();
    size_t i = 0, n = line.size();
    while (i < n) {
        while (i < n && (line[i] == ' ' || line[i] == '\t' || line[i] == '\r')) ++i;
        if (i >= n) break;
        size_t j = i;
        while (j < n && line[j] != ' ' && line[j] != '\t' && line[j] != '\r') ++j;
        tok.emplace_back(line, i, j - i);
        i = j;
    }
}

bool number(const std::string& s, double* v) {
    errno = 0;
    char* end = nullptr;
    *v = std::strtod(s.c_str(), &end);
    return end && *end == '\0' && end != s.c_str() && errno != ERANGE;
}

std::string upper(std::string s) {
    for (auto& ch : s) ch = (char)std::toupper((unsigned char)ch);
    return s;
}

struct Bound {
    double lb = 0.0, ub = INFINITY;
    bool free = false;
    int type = -1;  // -1 unchanged, 1 integer, 2 binary
};

int read(std::istream& in, b2p_mps* out, std::string* err) {
    enum Sec { NONE, NAMESEC, OBJSENSE, ROWS, COLUMNS, RHS, RANGES, BOUNDS };
    Sec sec = NONE;
    std::string line, obj_row, rhs_vec, rng_vec, bnd_vec;
    std::vector<std::string> tok;
    std::unordered_map<std::string, int> row_of;   // row name -> index (-1: objective, -2: other N rows)
    std::unordered_map<std::string, int> col_of;
    std::vector<std::vector<std::pair<int32_t, double>>> rows;  // per row: (column, value)
    std::vector<uint8_t> cost_set;  // the column's first objective entry has been read
    std::vector<uint8_t> row_sorted;  // the row's entries are in increasing column order
    std::unordered_map<std::string, double> rhs_map, rng_map;
    std::unordered_map<std::string, Bound> bnd;
    bool in_int = false, endata = false;
    size_t ln = 0;
    auto fail = [&](const std::string& m) {
        *err = m + " at line " + std::to_string(ln);
        return B2P_INVALID_ARGUMENT;
    };
    while (std::getline(in, line)) {
        ++ln;
        if (line.empty() || line[0] == '*') continue;
        split(line, tok);
        if (tok.empty()) continue;
        const std::string kw = upper(tok[0]);
        const bool header = (line[0] != ' ' && line[0] != '\t') || sec == NONE;
        if (header && (kw == "NAME" || kw == "OBJSENSE" || kw == "ROWS" || kw == "COLUMNS" || kw == "RHS" ||
                       kw == "RANGES" || kw == "BOUNDS" || kw == "ENDATA")) {
            if (kw == "NAME") {
                out->name = tok.size() > 1 ? tok[1] : "";
                sec = NAMESEC;
            } else if (kw == "OBJSENSE") {
                sec = OBJSENSE;
                if (tok.size() > 1) {  // "OBJSENSE MAX" on one line
                    const std::string s = upper(tok[1]);
                    if (s == "MAX" || s == "MAXIMIZE") out->maximize = 1;
                }
            } else if (kw == "ROWS") sec = ROWS;
            else if (kw == "COLUMNS") sec = COLUMNS;
            else if (kw == "RHS") sec = RHS;
            else if (kw == "RANGES") sec = RANGES;
            else if (kw == "BOUNDS") sec = BOUNDS;
            else {
                endata = true;
                break;
            }
            continue;
        }
        if (sec == OBJSENSE) {
            const std::string s = upper(tok[0]);
            if (s == "MAX" || s == "MAXIMIZE") out->maximize = 1;
            else if (s == "MIN" || s == "MINIMIZE") out->maximize = 0;
        } else if (sec == ROWS) {
            if (tok.size() < 2) return fail("malformed ROWS line");
            const char t = (char)std::toupper((unsigned char)tok[0][0]);
            if (t != 'N' && t != 'L' && t != 'G' && t != 'E') return fail("invalid row type");
            if (t == 'N') {
                if (obj_row.empty()) {
                    obj_row = tok[1];
                    row_of[tok[1]] = -1;
                } else {
                    row_of[tok[1]] = -2;
                }
                continue;
            }
            row_of[tok[1]] = (int)out->row_names.size();
            out->row_names.push_back(tok[1]);
            out->row_type.push_back(t);
            rows.emplace_back();
            row_sorted.push_back(1);
        } else if (sec == COLUMNS) {
            bool marker = false;
            for (const auto& t : tok)
                if (upper(t).find("MARKER") != std::string::npos) marker = true;
            if (marker) {
                for (const auto& t : tok) {
                    const std::string u = upper(t);
                    if (u.find("INTORG") != std::string::npos) in_int = true;
                    else if (u.find("INTEND") != std::string::npos) in_int = false;
                }
                continue;
            }
            if (tok.size() < 3) return fail("malformed COLUMNS line");
            auto it = col_of.find(tok[0]);
            int j;
            if (it == col_of.end()) {
                j = (int)out->col_names.size();
                col_of.emplace(tok[0], j);
                out->col_names.push_back(tok[0]);
                out->obj.push_back(0.0);
                cost_set.push_back(0);
                out->col_type.push_back(in_int ? 1 : 0);
            } else {
                j = it->second;
            }
            for (size_t k = 1; k + 1 < tok.size(); k += 2) {
                double v;
                if (!number(tok[k + 1], &v)) return fail("invalid coefficient '" + tok[k + 1] + "'");
                auto r = row_of.find(tok[k]);
                if (r == row_of.end()) continue;  // unknown rows are ignored, as the reference does
                if (r->second == -1) {
                    // the first entry of this column on the objective row is its cost
                    if (!cost_set[j]) {
                        out->obj[j] = v;
                        cost_set[j] = 1;
                    }
                } else if (r->second >= 0) {
                    // a repeated entry replaces the earlier value; an explicit zero is kept
                    // only as such a replacement (LPModel::set_coeff, src/lp_model.cpp:121-141)
                    // (a row's entries arrive in increasing column order unless a column
                    // is revisited out of order; only then is the row searched)
                    auto& e = rows[r->second];
                    if (!e.empty() && e.back().first == (int32_t)j) {
                        e.back().second = v;
                    } else if (e.empty() || (e.back().first < (int32_t)j && row_sorted[r->second])) {
                        if (v != 0.0) e.push_back({(int32_t)j, v});
                    } else {
                        bool found = false;
                        for (auto& q : e)
                            if (q.first == (int32_t)j) {
                                q.second = v;
                                found = true;
                            }
                        if (!found && v != 0.0) {
                            e.push_back({(int32_t)j, v});
                            row_sorted[r->second] = 0;
                        }
                    }
                }
            }
        } else if (sec == RHS || sec == RANGES) {
            std::string& vec = sec == RHS ? rhs_vec : rng_vec;
            auto& mp = sec == RHS ? rhs_map : rng_map;
            size_t k = 0;
            if (row_of.find(tok[0]) == row_of.end() && tok.size() > 1) {
                if (vec.empty()) vec = tok[0];
                if (tok[0] != vec) continue;
                k = 1;
            }
            for (; k + 1 < tok.size(); k += 2) {
                double v;
                if (!number(tok[k + 1], &v)) return fail(sec == RHS ? "invalid RHS value" : "invalid RANGES value");
                mp[tok[k]] = v;
            }
        } else if (sec == BOUNDS) {
            if (tok.size() < 3) return fail("malformed BOUNDS line");
            const std::string bt = upper(tok[0]);
            if (bnd_vec.empty()) bnd_vec = tok[1];
            if (tok[1] != bnd_vec) continue;
            Bound& b = bnd[tok[2]];
            double v = 0.0;
            if (tok.size() > 3 && !number(tok[3], &v)) v = 0.0;
            if (bt == "LO") b.lb = v;
            else if (bt == "UP") b.ub = v;
            else if (bt == "FX") b.lb = b.ub = v;
            else if (bt == "FR") {
                b.free = true;
                b.lb = -INFINITY;
                b.ub = INFINITY;
            } else if (bt == "MI") b.lb = -INFINITY;
            else if (bt == "PL") b.ub = INFINITY;
            else if (bt == "BV") {
                b.lb = 0.0;
                b.ub = 1.0;
                b.type = 2;
            } else if (bt == "LI") {
                b.lb = v;
                b.type = 1;
            } else if (bt == "UI") {
                b.ub = v;
                b.type = 1;
            } else {
                return fail("unknown bound type '" + bt + "'");
            }
        }
    }
    if (!endata) return fail("missing ENDATA");
    if (in_int) return fail("unclosed integer marker section");
    // columns: bounds and kinds
    const size_t n = out->col_names.size(), m = out->row_names.size();
    out->lb.assign(n, 0.0);
    out->ub.assign(n, INFINITY);
    for (size_t j = 0; j < n; ++j) {
        auto it = bnd.find(out->col_names[j]);
        if (it == bnd.end()) continue;
        const Bound& b = it->second;
        if (b.free || (std::isinf(b.lb) && b.lb < 0 && std::isinf(b.ub) && b.ub > 0)) {
            out->lb[j] = -INFINITY;
            out->ub[j] = INFINITY;
        } else {
            out->lb[j] = b.lb;
            out->ub[j] = b.ub;
        }
        if (b.type == 2) out->col_type[j] = 2;
        else if (b.type == 1 && out->col_type[j] != 2) out->col_type[j] = 1;
    }
    if (!obj_row.empty()) {
        auto it = rhs_map.find(obj_row);
        if (it != rhs_map.end()) out->obj_offset = -it->second;
    }
    // rows: rhs, ranges
    out->rhs.assign(m, 0.0);
    out->range_upper.assign(m, 0.0);
    out->ranged.assign(m, 0);
    for (size_t i = 0; i < m; ++i) {
        auto it = rhs_map.find(out->row_names[i]);
        double r = it == rhs_map.end() ? 0.0 : it->second;
        auto g = rng_map.find(out->row_names[i]);
        if (g != rng_map.end()) {
            const double R = g->second;
            double lo = r, hi = r;
            if (out->row_type[i] == 'L') {
                if (R > 0.0) lo = r - R;
                else hi = r - R;
            } else {  // G and E
                if (R > 0.0) hi = r + R;
                else lo = r + R;
            }
            out->ranged[i] = 1;
            r = lo;
            out->range_upper[i] = hi;
        }
        out->rhs[i] = r;
    }
    // CSR, column indices ascending within each row
    out->rowptr.assign(m + 1, 0);
    for (size_t i = 0; i < m; ++i) {
        auto& e = rows[i];
        std::sort(e.begin(), e.end(), [](const std::pair<int32_t, double>& a, const std::pair<int32_t, double>& b) {
            return a.first < b.first;
        });
        out->rowptr[i + 1] = out->rowptr[i] + (int32_t)e.size();
    }
    out->colidx.resize(out->rowptr[m]);
    out->vals.resize(out->rowptr[m]);
    for (size_t i = 0; i < m; ++i) {
        int32_t p = out->rowptr[i];
        for (const auto& e : rows[i]) {
            out->colidx[p] = e.first;
            out->vals[p++] = e.second;
        }
    }
    return B2P_OK;
}

// Standard form: min c.x with c = +-obj, rows <= (is_eq 0) or = (is_eq 1).  L rows as is,
// G rows negated, E rows as equalities; a ranged row [lo, hi] becomes an equality when
// lo == hi, else a.x <= hi and -a.x <= -lo (an infinite end drops its row).
struct Std {
    std::vector<int32_t> rowptr{0}, colidx;
    std::vector<double> vals, b;
    std::vector<uint8_t> is_eq;
};

void standard_form(const b2p_mps* M, Std* s) {
    auto add = [&](size_t i, double sign, double rhs, uint8_t eq) {
        for (int32_t p = M->rowptr[i]; p < M->rowptr[i + 1]; ++p) {
            s->colidx.push_back(M->colidx[p]);
            s->vals.push_back(sign * M->vals[p]);
        }
        s->rowptr.push_back((int32_t)s->colidx.size());
        s->b.push_back(sign * rhs);
        s->is_eq.push_back(eq);
    };
    for (size_t i = 0; i < M->row_names.size(); ++i) {
        if (M->ranged[i]) {
            const double lo = M->rhs[i], hi = M->range_upper[i];
            if (lo == hi) {
                add(i, 1.0, lo, 1);
                continue;
            }
            if (std::isfinite(hi)) add(i, 1.0, hi, 0);
            if (std::isfinite(lo)) add(i, -1.0, lo, 0);
        } else if (M->row_type[i] == 'E') {
            add(i, 1.0, M->rhs[i], 1);
        } else if (M->row_type[i] == 'G') {
            add(i, -1.0, M->rhs[i], 0);
        } else {
            add(i, 1.0, M->rhs[i], 0);
        }
    }
}

}  // namespace

using namespace b2p;

extern "C" {

int b2p_mps_read(const char* path, b2p_mps** out, char* err, size_t errlen) {
    if (!path || !out) return B2P_INVALID_ARGUMENT;
    *out = nullptr;
    std::ifstream f(path);
    std::string msg;
    if (!f) {
        msg = std::string("cannot open ") + path;
        if (err && errlen) std::snprintf(err, errlen, "%s", msg.c_str());
        return B2P_INVALID_ARGUMENT;
    }
    b2p_mps* M = new b2p_mps();
    int st = read(f, M, &msg);
    if (st != B2P_OK) {
        delete M;
        if (err && errlen) std::snprintf(err, errlen, "%s", msg.c_str());
        return st;
    }
    *out = M;
    return B2P_OK;
}

void b2p_mps_free(b2p_mps* M) { delete M; }

int b2p_mps_dims(const b2p_mps* M, int* m, int* n, int64_t* nnz, int* maximize, double* obj_offset, int* std_m,
                 int64_t* std_nnz) {
    if (!M) return B2P_INVALID_ARGUMENT;
    if (m) *m = (int)M->row_names.size();
    if (n) *n = (int)M->col_names.size();
    if (nnz) *nnz = (int64_t)M->vals.size();
    if (maximize) *maximize = M->maximize;
    if (obj_offset) *obj_offset = M->obj_offset;
    if (std_m || std_nnz) {
        Std s;
        standard_form(M, &s);
        if (std_m) *std_m = (int)s.b.size();
        if (std_nnz) *std_nnz = (int64_t)s.vals.size();
    }
    return B2P_OK;
}

int b2p_mps_model(const b2p_mps* M, int32_t* rowptr, int32_t* colidx, double* vals, char* row_type, uint8_t* ranged,
                  double* rhs, double* range_upper, double* obj, double* lb, double* ub, uint8_t* col_type) {
    if (!M) return B2P_INVALID_ARGUMENT;
    const size_t m = M->row_names.size(), n = M->col_names.size();
    if (rowptr) std::copy(M->rowptr.begin(), M->rowptr.end(), rowptr);
    if (colidx) std::copy(M->colidx.begin(), M->colidx.end(), colidx);
    if (vals) std::copy(M->vals.begin(), M->vals.end(), vals);
    for (size_t i = 0; i < m; ++i) {
        if (row_type) row_type[i] = M->row_type[i];
        if (ranged) ranged[i] = M->ranged[i];
        if (rhs) rhs[i] = M->rhs[i];
        if (range_upper) range_upper[i] = M->range_upper[i];
    }
    for (size_t j = 0; j < n; ++j) {
        if (obj) obj[j] = M->obj[j];
        if (lb) lb[j] = M->lb[j];
        if (ub) ub[j] = M->ub[j];
        if (col_type) col_type[j] = M->col_type[j];
    }
    return B2P_OK;
}

int b2p_mps_standard_form(const b2p_mps* M, int32_t* rowptr, int32_t* colidx, double* vals, double* b, double* c,
                          double* lb, double* ub, uint8_t* is_eq) {
    if (!M) return B2P_INVALID_ARGUMENT;
    Std s;
    standard_form(M, &s);
    const double sense = M->maximize ? -1.0 : 1.0;
    if (rowptr) std::copy(s.rowptr.begin(), s.rowptr.end(), rowptr);
    if (colidx) std::copy(s.colidx.begin(), s.colidx.end(), colidx);
    if (vals) std::copy(s.vals.begin(), s.vals.end(), vals);
    if (b) std::copy(s.b.begin(), s.b.end(), b);
    if (is_eq) std::copy(s.is_eq.begin(), s.is_eq.end(), is_eq);
    for (size_t j = 0; j < M->col_names.size(); ++j) {
        if (c) c[j] = sense * M->obj[j];
        if (lb) lb[j] = M->lb[j];
        if (ub) ub[j] = M->ub[j];
    }
    return B2P_OK;
}

int b2p_upload_mps(void* ctx, const b2p_mps* M) {
    if (!ctx) return B2P_GPU_UNINITIALIZED;
    if (!M) return B2P_INVALID_ARGUMENT;
    Std s;
    standard_form(M, &s);
    const size_t n = M->col_names.size();
    std::vector<double> c(n);
    const double sense = M->maximize ? -1.0 : 1.0;
    for (size_t j = 0; j < n; ++j) c[j] = sense * M->obj[j];
    return b2p_upload_lp(ctx, (int)s.b.size(), (int)n, (int64_t)s.vals.size(), s.rowptr.data(), s.colidx.data(),
                         s.vals.data(), s.b.data(), c.data(), M->lb.data(), M->ub.data(), s.is_eq.data());
}

}  // extern "C"
