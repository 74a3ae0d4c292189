// MPS reader (fixed and free format) for callers without Clp.  The reference
// reads MPS through ClpModel::readMps (CoinUtils' CoinMpsIO) and then derives
// its bound types (Problem::readMps, problem.tpp:332-409); this file parses the
// file itself and hands the same arrays to ds_load_csr, which derives the types
// the same way.  Conventions (those of CoinMpsIO where the format leaves a
// choice):
//   * the first N row is the objective; further N rows carry no constraint and
//     are dropped;
//   * L: (-inf, rhs], G: [rhs, inf), E: [rhs, rhs]; RANGES r: L -> [rhs-|r|, rhs],
//     G -> [rhs, rhs+|r|], E -> [rhs, rhs+r] for r > 0 and [rhs+r, rhs] for r < 0;
//   * an RHS entry on the objective row is the objective offset: reported
//     objectives are c^T x - offset (ClpModel::objectiveOffset, problem.tpp:256);
//   * columns default to [0, inf); BOUNDS UP/LO/FX/FR/MI/PL/BV/LI/UI (integrality
//     is ignored: the LP relaxation), UP < 0 on a column whose lower bound is 0
//     makes the lower bound -inf; SC bounds and OBJSENSE MAX are rejected;
//   * only the first RHS, RANGES and BOUNDS set is read; MARKER lines are skipped;
//   * any value of magnitude >= 1e30 is infinite (stored as +-1e300).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/ds_api.h"

namespace {

constexpr double MPS_INF = 1e300;

thread_local std::string g_mps_error;

struct MpsLp {
    int m = 0, n = 0;
    std::vector<int> row_ptr, col_idx;
    std::vector<double> val, c, col_lb, col_ub, row_lb, row_ub;
    double offset = 0.0;
};

std::vector<std::string> tokens(const std::string& line) {
    std::vector<std::string> t;
    size_t i = 0;
    while (i < line.size()) {
        while (i < line.size() && (line[i] == ' ' || line[i] == '\t')) ++i;
        if (i >= line.size()) break;
        size_t j = i;
        while (j < line.size() && line[j] != ' ' && line[j] != '\t') ++j;
        t.push_back(line.substr(i, j - i));
        i = j;
    }
    return t;
}

bool number(const std::string& s, double* v) {
    char* end = nullptr;
    const double x = std::strtod(s.c_str(), &end);
    if (end == s.c_str() || *end != '\0') return false;
    *v = (x >= 1e30) ? MPS_INF : (x <= -1e30) ? -MPS_INF : x;
    return true;
}

bool fail(int lineno, const std::string& what) {
    g_mps_error = "MPS line " + std::to_string(lineno) + ": " + what;
    return false;
}

bool parse_mps(const char* path, MpsLp& lp) {
    FILE* f = std::fopen(path, "r");
    if (!f) { g_mps_error = std::string("cannot open ") + path; return false; }
    enum Sec { NONE, NAME, ROWS, COLUMNS, RHS, RANGES, BOUNDS, OBJSENSE, END } sec = NONE;
    std::string obj;                                   // objective row name
    std::unordered_map<std::string, int> row_of;       // constraint row -> index
    std::unordered_map<std::string, int> dropped;      // further N rows
    std::vector<char> rtype;                           // 'L', 'G', 'E'
    std::vector<double> rhs, range;
    std::vector<char> has_range;
    std::unordered_map<std::string, int> col_of;
    std::vector<std::vector<std::pair<int, double>>> cols;
    std::string rhs_set, range_set, bound_set;
    bool rhs_set_seen = false, range_set_seen = false, bound_set_seen = false;
    std::vector<char> lb_set;
    std::vector<int> mark;   // row -> last column with an entry in it (duplicate check)
    std::string line;
    char buf[65536];
    int lineno = 0;
    bool ok = true;
    while (ok && std::fgets(buf, sizeof(buf), f)) {
        ++lineno;
        line.assign(buf);
        while (!line.empty() && (line.back() == '\n' || line.back() == '\r')) line.pop_back();
        if (line.empty() || line[0] == '*') continue;
        const std::vector<std::string> t = tokens(line);
        if (t.empty()) continue;
        const std::string& h = t[0];
        const bool header = line[0] != ' ' && line[0] != '\t' &&
                            (h == "NAME" || h == "ROWS" || h == "COLUMNS" || h == "RHS" || h == "RANGES" ||
                             h == "BOUNDS" || h == "OBJSENSE" || h == "OBJSENS" || h == "ENDATA");
        if (header) {   // section header (free-format data lines may start in column 1 too)
            if (h == "NAME") sec = NAME;
            else if (h == "ROWS") sec = ROWS;
            else if (h == "COLUMNS") sec = COLUMNS;
            else if (h == "RHS") sec = RHS;
            else if (h == "RANGES") sec = RANGES;
            else if (h == "BOUNDS") sec = BOUNDS;
            else if (h == "OBJSENSE" || h == "OBJSENS") {
                sec = OBJSENSE;
                if (t.size() > 1 && (t[1] == "MAX" || t[1] == "MAXIMIZE"))
                    ok = fail(lineno, "OBJSENSE MAX is not supported (the solver minimises)");
            } else { sec = END; break; }   // ENDATA
            continue;
        }
        switch (sec) {
            case OBJSENSE:
                if (t[0] == "MAX" || t[0] == "MAXIMIZE") ok = fail(lineno, "OBJSENSE MAX is not supported (the solver minimises)");
                break;
            case ROWS: {
                if (t.size() < 2) { ok = fail(lineno, "ROWS entry needs a type and a name"); break; }
                const std::string& ty = t[0];
                if (ty == "N") {
                    if (obj.empty()) obj = t[1];
                    else dropped[t[1]] = 1;
                } else if (ty == "L" || ty == "G" || ty == "E") {
                    if (row_of.count(t[1]) || t[1] == obj) { ok = fail(lineno, "duplicate row " + t[1]); break; }
                    row_of[t[1]] = (int)rtype.size();
                    rtype.push_back(ty[0]);
                    rhs.push_back(0.0);
                    range.push_back(0.0);
                    has_range.push_back(0);
                } else {
                    ok = fail(lineno, "unknown row type " + ty);
                }
                break;
            }
            case COLUMNS: {
                if (t.size() >= 3 && t[1] == "'MARKER'") break;
                if (t.size() != 3 && t.size() != 5) { ok = fail(lineno, "COLUMNS entry needs name row value [row value]"); break; }
                auto it = col_of.find(t[0]);
                int j;
                if (it == col_of.end()) {
                    j = (int)cols.size();
                    col_of[t[0]] = j;
                    cols.emplace_back();
                } else {
                    j = it->second;
                }
                for (size_t k = 1; k + 1 < t.size(); k += 2) {
                    double v;
                    if (!number(t[k + 1], &v)) { ok = fail(lineno, "bad number " + t[k + 1]); break; }
                    if (t[k] == obj) {
                        cols[j].push_back({-1, v});
                    } else if (dropped.count(t[k])) {
                        continue;
                    } else {
                        auto r = row_of.find(t[k]);
                        if (r == row_of.end()) { ok = fail(lineno, "unknown row " + t[k]); break; }
                        if (mark.size() < rtype.size()) mark.resize(rtype.size(), -1);
                        if (mark[r->second] == j) { ok = fail(lineno, "duplicate entry " + t[0] + " " + t[k]); break; }
                        mark[r->second] = j;
                        cols[j].push_back({r->second, v});
                    }
                }
                break;
            }
            case RHS:
            case RANGES: {
                // [set] row value [row value]: an odd token count carries the set name
                const size_t first = (t.size() % 2 == 1) ? 1 : 0;
                if (t.size() < first + 2) { ok = fail(lineno, "entry needs row and value"); break; }
                std::string& set = (sec == RHS) ? rhs_set : range_set;
                bool& seen = (sec == RHS) ? rhs_set_seen : range_set_seen;
                const std::string name = first ? t[0] : std::string();
                if (!seen) { set = name; seen = true; }
                else if (name != set) break;   // a later set
                for (size_t k = first; k + 1 < t.size(); k += 2) {
                    double v;
                    if (!number(t[k + 1], &v)) { ok = fail(lineno, "bad number " + t[k + 1]); break; }
                    if (t[k] == obj) {
                        if (sec == RHS) lp.offset = v;
                        continue;
                    }
                    if (dropped.count(t[k])) continue;
                    auto r = row_of.find(t[k]);
                    if (r == row_of.end()) { ok = fail(lineno, "unknown row " + t[k]); break; }
                    if (sec == RHS) rhs[r->second] = v;
                    else { range[r->second] = v; has_range[r->second] = 1; }
                }
                break;
            }
            case BOUNDS: {
                const std::string& ty = t[0];
                const bool valued = !(ty == "FR" || ty == "MI" || ty == "PL" || ty == "BV");
                size_t ncol;   // index of the column name
                if (valued) {
                    if (t.size() == 4) ncol = 2;
                    else if (t.size() == 3) ncol = 1;
                    else { ok = fail(lineno, "bound " + ty + " needs [set] column value"); break; }
                } else {
                    if (t.size() >= 3) ncol = 2;
                    else if (t.size() == 2) ncol = 1;
                    else { ok = fail(lineno, "bound " + ty + " needs [set] column"); break; }
                }
                const std::string name = (ncol == 2) ? t[1] : std::string();
                if (!bound_set_seen) { bound_set = name; bound_set_seen = true; }
                else if (name != bound_set) break;
                auto it = col_of.find(t[ncol]);
                if (it == col_of.end()) { ok = fail(lineno, "unknown column " + t[ncol]); break; }
                const int j = it->second;
                if ((int)lp.col_lb.size() < (int)cols.size()) {
                    lp.col_lb.resize(cols.size(), 0.0);
                    lp.col_ub.resize(cols.size(), MPS_INF);
                    lb_set.resize(cols.size(), 0);
                }
                double v = 0.0;
                if (valued && !number(t[ncol + 1], &v)) { ok = fail(lineno, "bad number " + t[ncol + 1]); break; }
                if (ty == "UP" || ty == "UI") {
                    lp.col_ub[j] = v;
                    if (v < 0.0 && lp.col_lb[j] == 0.0 && !lb_set[j]) lp.col_lb[j] = -MPS_INF;
                } else if (ty == "LO" || ty == "LI") {
                    lp.col_lb[j] = v; lb_set[j] = 1;
                } else if (ty == "FX") {
                    lp.col_lb[j] = v; lp.col_ub[j] = v; lb_set[j] = 1;
                } else if (ty == "FR") {
                    lp.col_lb[j] = -MPS_INF; lp.col_ub[j] = MPS_INF; lb_set[j] = 1;
                } else if (ty == "MI") {
                    lp.col_lb[j] = -MPS_INF; lb_set[j] = 1;
                } else if (ty == "PL") {
                    lp.col_ub[j] = MPS_INF;
                } else if (ty == "BV") {
                    lp.col_lb[j] = 0.0; lp.col_ub[j] = 1.0; lb_set[j] = 1;
                } else {
                    ok = fail(lineno, "unsupported bound type " + ty);
                }
                break;
            }
            case NAME: case NONE: case END:
                break;
        }
    }
    std::fclose(f);
    if (!ok) return false;
    if (sec != END) { g_mps_error = "MPS file ends without ENDATA"; return false; }
    if (obj.empty()) { g_mps_error = "MPS file has no objective (N) row"; return false; }
    const int m = (int)rtype.size(), n = (int)cols.size();
    lp.m = m; lp.n = n;
    lp.col_lb.resize(n, 0.0);
    lp.col_ub.resize(n, MPS_INF);
    lp.c.assign(n, 0.0);
    lp.row_lb.resize(m);
    lp.row_ub.resize(m);
    for (int i = 0; i < m; ++i) {
        const double b = rhs[i], r = range[i];
        double lo, hi;
        if (rtype[i] == 'L') { lo = -MPS_INF; hi = b; if (has_range[i]) lo = b - std::fabs(r); }
        else if (rtype[i] == 'G') { lo = b; hi = MPS_INF; if (has_range[i]) hi = b + std::fabs(r); }
        else { lo = b; hi = b; if (has_range[i]) { if (r > 0) hi = b + r; else lo = b + r; } }
        lp.row_lb[i] = lo;
        lp.row_ub[i] = hi;
    }
    // CSR with the columns of each row in ascending order
    std::vector<int> cnt(m + 1, 0);
    for (int j = 0; j < n; ++j)
        for (const auto& e : cols[j]) {
            if (e.first < 0) lp.c[j] = e.second;
            else ++cnt[e.first + 1];
        }
    lp.row_ptr.assign(m + 1, 0);
    for (int i = 0; i < m; ++i) lp.row_ptr[i + 1] = lp.row_ptr[i] + cnt[i + 1];
    const int nnz = lp.row_ptr[m];
    lp.col_idx.assign(nnz, 0);
    lp.val.assign(nnz, 0.0);
    std::vector<int> fill(lp.row_ptr.begin(), lp.row_ptr.end() - 1);
    for (int j = 0; j < n; ++j)
        for (const auto& e : cols[j])
            if (e.first >= 0) {
                const int p = fill[e.first]++;
                lp.col_idx[p] = j;
                lp.val[p] = e.second;
            }
    return true;
}

}  // namespace

extern "C" {

const char* ds_mps_last_error(void) { return g_mps_error.c_str(); }

int ds_mps_read(const char* path, int* m, int* n, long long* nnz, int* row_ptr, int* col_idx, double* val,
                double* c, double* col_lb, double* col_ub, double* row_lb, double* row_ub, double* obj_offset) {
    if (!path || !m || !n || !nnz) { g_mps_error = "null argument"; return DS_ERR_ARG; }
    MpsLp lp;
    if (!parse_mps(path, lp)) return DS_ERR_ARG;
    *m = lp.m;
    *n = lp.n;
    *nnz = (long long)lp.row_ptr[lp.m];
    if (obj_offset) *obj_offset = lp.offset;
    auto put = [](auto* dst, const auto& src) {
        if (dst && !src.empty()) std::memcpy(dst, src.data(), src.size() * sizeof(src[0]));
    };
    put(row_ptr, lp.row_ptr); put(col_idx, lp.col_idx); put(val, lp.val); put(c, lp.c);
    put(col_lb, lp.col_lb); put(col_ub, lp.col_ub); put(row_lb, lp.row_lb); put(row_ub, lp.row_ub);
    return DS_OK;
}

int ds_load_mps(ds_solver* s, const char* path, double* obj_offset) {
    if (!s || !path) { g_mps_error = "null argument"; return DS_ERR_ARG; }
    MpsLp lp;
    if (!parse_mps(path, lp)) return DS_ERR_ARG;
    if (obj_offset) *obj_offset = lp.offset;
    return ds_load_csr(s, lp.m, lp.n, lp.row_ptr.data(), lp.col_idx.data(), lp.val.data(), lp.c.data(),
                       lp.col_lb.data(), lp.col_ub.data(), lp.row_lb.data(), lp.row_ub.data());
}

}  // extern "C"
