// TEST INFRASTRUCTURE ONLY -- CPU restatement of veret-v/parallel_ds's
// sequential bounded dual simplex (parity checker for the CUDA engine).
//
// Every routine names the reference lines it restates.  Paths are relative to
// the reference project root.  Arithmetic is written in the reference's
// operation order and built with -ffp-contract=off so that single operations
// round exactly as the reference's unfused x86-64 code does.
//
// Departures from the reference, each guarded by or_options:
//   * PARDISO (src/cpu/matrix.cpp:530-583) is replaced by a dense LU with
//     partial pivoting of the basis's structural block K = A[R', S]; slack
//     columns of the basis are eliminated exactly (they are unit columns).
//   * std::random_device in perturbCosts (baseDualSimplex.tpp:244) becomes a
//     seeded std::mt19937 so runs are repeatable.
//   * strict_reference = 0 adds two guards: a restart-loop stop and a
//     post-perturbation cleanup (phase 1 + phase 2 on the original costs when
//     the perturbed optimum is dual infeasible; the reference's callPrimalSolver
//     is an empty stub, baseDualSimplex.tpp:677-680);
//   * strict_reference = 0 also crashes free structural columns into the start
//     basis (crash_free_columns), as the engine does.
#include "ds_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <unordered_set>
#include <vector>

namespace {

// Tolerances and constants: baseDualSimplex.hpp:23-46.
constexpr double EPS_BOUND = 1e-10;
constexpr double EPS_D = 1e-7;
constexpr double EPS_COSTS = 1e-8;
constexpr double EPS_A = 1e-5;
constexpr double EPS_Z = 1e-10;
constexpr double EPS_R = 1e-9;
constexpr double EPS_F = 1e-10;
constexpr double PERTURB_RATIO = 0.25;
constexpr double PSI = 1e-5;
constexpr int MAX_CYCLE = 5;
constexpr int NEED_RESTART = 40;
constexpr double INF = 1e25;
constexpr double BOUND_INF = 1e100;  // problem.hpp:31

enum { FIXED = 0, FREE = 1, BOXED = 2, UPPER = 3, LOWER = 4 };
enum { ST_UNSOLVED = 0, ST_OPTIMAL = 1, ST_PRIMAL_INF = 2, ST_DUAL_INF = 3, ST_ITER = 4, ST_ERROR = 5 };
enum Phase1Out { P1_SOLVED, P1_DUALINF, P1_RESTART };

struct Stop {};  // thrown to unwind on iteration limit / numeric failure

struct Oracle {
    or_options opt{};
    int m = 0, n = 0, N = 0;
    // [A | I] in CSC (rows ascending) and CSR (slack entry last in each row):
    // Matrix::genSparseReprs (matrix.cpp:99-146), stackColUnitMatrix (matrix.cpp:349-372).
    std::vector<int> cptr, crow, rptr, rcol;
    std::vector<double> cval, rval;
    std::vector<double> lb, ub, costs, original_costs, diff_bounds;
    std::vector<int> type;

    std::vector<double> x, d, beta;
    std::vector<int> basis, nonbasis;
    std::vector<char> is_basic;

    // factor of B0: K = A[rp_row, s_var], P K = L U
    int k = 0;
    double min_pivot = 1e300, min_pivot_rel = 1e300, max_step = 0.0;   // phase-2 pivot statistics
    std::vector<int> p2_block;   // experiments (col_rel_tol): iteration until which a position is not priced
    int refused_pivots = 0;
    std::vector<int> s_pos, s_var, rp_row, row_slackpos, piv;
    std::vector<double> LU;
    // PFI eta file (PFIfactor / linalg::PFIsolve)
    std::vector<std::vector<double>> eta;
    std::vector<int> eta_p;

    int iteration = 0, phase1_iters = 0, refactors = 0, restarts = 0, flips = 0;
    long long pivots = 0;  // basis changes in either phase
    bool perturbed = false;
    double obj = 0.0;
    int status = ST_UNSOLVED;
    std::mt19937 gen;
    bool in_phase1 = false;

    // trace
    int* tp = nullptr; int* tq = nullptr; double* tth = nullptr; double* tob = nullptr;
    int tcap = 0, tcount = 0;

    // ---------------------------------------------------------------- setup
    void load(int m_, int n_, const int* row_ptr, const int* col_idx, const double* val,
              const double* c, const int* col_type, const double* col_lb, const double* col_ub,
              const int* row_type, const double* row_lb, const double* row_ub) {
        m = m_; n = n_; N = n + m;
        // CSR of [A | I]
        rptr.assign(m + 1, 0);
        for (int i = 0; i < m; ++i) rptr[i + 1] = rptr[i] + (row_ptr[i + 1] - row_ptr[i]) + 1;
        rcol.resize(rptr[m]); rval.resize(rptr[m]);
        for (int i = 0; i < m; ++i) {
            int p = rptr[i];
            for (int e = row_ptr[i]; e < row_ptr[i + 1]; ++e) { rcol[p] = col_idx[e]; rval[p] = val[e]; ++p; }
            rcol[p] = n + i; rval[p] = 1.0;
        }
        // CSC by walking rows in order
        cptr.assign(N + 1, 0);
        for (int e = 0; e < rptr[m]; ++e) cptr[rcol[e] + 1]++;
        for (int j = 0; j < N; ++j) cptr[j + 1] += cptr[j];
        crow.resize(rptr[m]); cval.resize(rptr[m]);
        std::vector<int> cur(cptr.begin(), cptr.end() - 1);
        for (int i = 0; i < m; ++i)
            for (int e = rptr[i]; e < rptr[i + 1]; ++e) { int p = cur[rcol[e]]++; crow[p] = i; cval[p] = rval[e]; }
        // bounds / types: structurals as given, slacks per transformToComputeForm
        lb.resize(N); ub.resize(N); costs.resize(N); type.resize(N);
        for (int j = 0; j < n; ++j) { lb[j] = col_lb[j]; ub[j] = col_ub[j]; costs[j] = c[j]; type[j] = col_type[j]; }
        for (int i = 0; i < m; ++i) {
            ub[n + i] = -row_lb[i];
            lb[n + i] = -row_ub[i];
            costs[n + i] = 0;
            switch (row_type[i]) {
                case FIXED: type[n + i] = FIXED; break;
                case BOXED: type[n + i] = BOXED; break;
                case LOWER: type[n + i] = UPPER; break;
                case UPPER: type[n + i] = LOWER; break;
                default: type[n + i] = FREE; break;  // reference has no case (problem.tpp:201-218)
            }
        }
        diff_bounds.resize(N);
        for (int j = 0; j < N; ++j) diff_bounds[j] = ub[j] - lb[j];
        // BaseDualSimplex ctor (baseDualSimplex.tpp:184-204): slack basis
        basis.resize(m); nonbasis.resize(n); is_basic.assign(N, 0);
        for (int i = 0; i < n; ++i) nonbasis[i] = i;
        for (int i = 0; i < m; ++i) { basis[i] = i + n; is_basic[i + n] = 1; }
        if (!opt.strict_reference) crash_free_columns();
        beta.assign(m, 0.0);
        x.assign(N, 0.0); d.assign(N, 0.0);
        gen.seed((unsigned)(opt.seed & 0xffffffffu) ^ (unsigned)(opt.seed >> 32));
    }

    // Departure (strict_reference = 0): a nonbasic free structural with a nonzero
    // reduced cost is dual infeasible, and the reference's phase 1 can leave one
    // behind (then "optimal" at a dual infeasible basis).  Before the solve each
    // free structural column takes the place of a slack whose row has a finite
    // bound, chosen by partial pivoting on the columns eliminated so far
    // (largest |entry|, lowest row on ties, pivots below 1e-9 of the column's
    // largest entry refused), which keeps the structural block nonsingular.  At
    // most CRASH_MAX columns; a free basic variable never leaves the basis.
    static constexpr int CRASH_MAX = 512;
    void crash_free_columns() {
        std::vector<int> cols;
        for (int j = 0; j < n && (int)cols.size() < CRASH_MAX; ++j)
            if (type[j] == FREE && cptr[j + 1] > cptr[j]) cols.push_back(j);
        if (cols.empty()) return;
        // Sparse elimination: the work column w is zero outside `touched`, and the
        // eliminated columns keep only the rows they touched.  Every operation and
        // its order equal the dense restatement (zeros subtract nothing), so the
        // chosen rows do not change; the cost is the eliminated columns' nonzeros,
        // not k*m.
        std::vector<char> used(m, 0), mark(m, 0);
        std::vector<double> w(m, 0.0);
        std::vector<int> touched;
        std::vector<std::vector<int>> eidx;      // eliminated columns: rows ...
        std::vector<std::vector<double>> eval;   // ... and values
        std::vector<int> prow;
        std::vector<double> pval;
        for (int j : cols) {
            touched.clear();
            double vmax = 0.0;
            for (int e = cptr[j]; e < cptr[j + 1]; ++e) {
                const int i = crow[e];
                w[i] = cval[e];
                if (!mark[i]) { mark[i] = 1; touched.push_back(i); }
                vmax = std::max(vmax, std::fabs(cval[e]));
            }
            for (size_t t = 0; t < eidx.size(); ++t) {
                const double f = w[prow[t]] / pval[t];
                if (f != 0.0)
                    for (size_t u = 0; u < eidx[t].size(); ++u) {
                        const int i = eidx[t][u];
                        w[i] -= f * eval[t][u];
                        if (!mark[i]) { mark[i] = 1; touched.push_back(i); }
                    }
            }
            int r = -1;
            double best = 0.0;
            for (int i : touched) {
                if (used[i] || type[n + i] == FREE) continue;
                const double a = std::fabs(w[i]);
                if (a > best || (a == best && a > 0.0 && i < r)) { best = a; r = i; }
            }
            const bool take = r >= 0 && best > 1e-9 * vmax;
            if (take) {
                std::vector<int> ix(touched);
                std::vector<double> vx(touched.size());
                for (size_t u = 0; u < touched.size(); ++u) vx[u] = w[touched[u]];
                used[r] = 1;
                eidx.push_back(std::move(ix));
                eval.push_back(std::move(vx));
                prow.push_back(r);
                pval.push_back(w[r]);
                basis[r] = j; is_basic[j] = 1;
                nonbasis[j] = n + r; is_basic[n + r] = 0;
            }
            for (int i : touched) { w[i] = 0.0; mark[i] = 0; }
        }
    }

    void tick() {
        if (iteration > opt.max_iterations) { status = ST_ITER; throw Stop{}; }
    }

    // ---------------------------------------------------------------- factor
    // reFactorize (sequentialDualSimplex.cpp:155-160): clear eta file, B <- A[:,basis], LU.
    void refactor() {
        ++refactors;
        eta.clear(); eta_p.clear();
        s_pos.clear(); s_var.clear(); rp_row.clear();
        row_slackpos.assign(m, -1);
        for (int i = 0; i < m; ++i) {
            int v = basis[i];
            if (v < n) { s_pos.push_back(i); s_var.push_back(v); }
            else row_slackpos[v - n] = i;
        }
        for (int r = 0; r < m; ++r) if (row_slackpos[r] < 0) rp_row.push_back(r);
        k = (int)s_pos.size();
        if ((int)rp_row.size() != k) { status = ST_ERROR; throw Stop{}; }
        std::vector<int> rowk(m, -1);
        for (int t = 0; t < k; ++t) rowk[rp_row[t]] = t;
        if (opt.block_lu) { block_factor(rowk); return; }
        LU.assign((size_t)k * k, 0.0);  // row-major K[t][j]
        for (int j = 0; j < k; ++j)
            for (int e = cptr[s_var[j]]; e < cptr[s_var[j] + 1]; ++e) {
                int t = rowk[crow[e]];
                if (t >= 0) LU[(size_t)t * k + j] = cval[e];
            }
        if (!dense_lu(LU, k, piv)) { status = ST_ERROR; throw Stop{}; }
    }
    // Dense LU with partial pivoting, row-major A (kk x kk), in place: PA = LU.
    static bool dense_lu(std::vector<double>& A, int kk, std::vector<int>& pv) {
        pv.resize(kk);
        for (int c = 0; c < kk; ++c) {
            int pr = c; double best = std::fabs(A[(size_t)c * kk + c]);
            for (int r = c + 1; r < kk; ++r) { double v = std::fabs(A[(size_t)r * kk + c]); if (v > best) { best = v; pr = r; } }
            pv[c] = pr;
            if (!(best > 1e-14)) return false;
            if (pr != c) for (int j = 0; j < kk; ++j) std::swap(A[(size_t)c * kk + j], A[(size_t)pr * kk + j]);
            const double pvv = A[(size_t)c * kk + c];
            double* rowc = &A[(size_t)c * kk];

            for (int r = c + 1; r < kk; ++r) {
                double* rowr = &A[(size_t)r * kk];
                const double l = rowr[c] / pvv;
                rowr[c] = l;
                if (l != 0.0)
                    for (int j = c + 1; j < kk; ++j) rowr[j] -= l * rowc[j];
            }
        }
        return true;
    }
    // A z = b in place (PA = LU)
    static void dense_solve(const std::vector<double>& A, int kk, const std::vector<int>& pv, double* z) {
        for (int c = 0; c < kk; ++c) if (pv[c] != c) std::swap(z[c], z[pv[c]]);
        for (int r = 0; r < kk; ++r) { double s = z[r]; const double* row = &A[(size_t)r * kk]; for (int j = 0; j < r; ++j) s -= row[j] * z[j]; z[r] = s; }
        for (int r = kk - 1; r >= 0; --r) { double s = z[r]; const double* row = &A[(size_t)r * kk]; for (int j = r + 1; j < kk; ++j) s -= row[j] * z[j]; z[r] = s / row[r]; }
    }
    // A^T z = b in place: U^T w = b, L^T v = w (unit diagonal), z = P^T v
    static void dense_tsolve(const std::vector<double>& A, int kk, const std::vector<int>& pv, double* z) {
        for (int j = 0; j < kk; ++j) {
            const double* row = &A[(size_t)j * kk];
            const double wj = z[j] / row[j];
            z[j] = wj;
            if (wj != 0.0) for (int r = j + 1; r < kk; ++r) z[r] -= row[r] * wj;
        }
        for (int j = kk - 1; j >= 0; --j) {
            const double* row = &A[(size_t)j * kk];
            const double vj = z[j];
            if (vj != 0.0) for (int r = 0; r < j; ++r) z[r] -= row[r] * vj;
        }
        for (int c = kk - 1; c >= 0; --c) if (pv[c] != c) std::swap(z[c], z[pv[c]]);
    }
    // K z = b (b, z length k), PK = LU
    void k_solve(std::vector<double>& z) const {
        if (opt.block_lu) { block_solve(z); return; }
        dense_solve(LU, k, piv, z.data());
    }
    // K^T z = b
    void kt_solve(std::vector<double>& z) const {
        if (opt.block_lu) { block_tsolve(z); return; }
        dense_tsolve(LU, k, piv, z.data());
    }
    // ---- experiments (opt.block_lu): K put in block upper triangular form by its
    // column singletons (first) and row singletons (last), the kernel left in
    // between factorised by the dense LU above; values straight from A.
    std::vector<int> bk_cptr, bk_crow, bk_rptr, bk_rcol, bt_u1t, bt_u1j, bt_u3t, bt_u3j, bt_krow, bt_kcol, bt_piv;
    std::vector<double> bk_cval, bk_rval, bt_M;
    std::vector<char> bt_u3col, bt_u1row;
    int bt_km = 0;
    // block_lu == 2: the kernel by sequential Markowitz with threshold pivoting
    std::vector<int> sk_prow, sk_pcol, sk_uptr, sk_ucol, sk_lptr, sk_lrow;
    std::vector<double> sk_uval, sk_lval, sk_udiag;
    std::vector<std::vector<std::pair<int, double>>> sk_rows;
    bool sparse_kernel_lu() {
        const int km = bt_km;
        std::vector<std::vector<std::pair<int, double>>>& rows = sk_rows;
        std::vector<std::vector<int>> cols(km);
        for (int a = 0; a < km; ++a)
            for (const auto& e : rows[a]) cols[e.first].push_back(a);
        std::vector<char> rdone(km, 0), cdone(km, 0);
        sk_prow.clear(); sk_pcol.clear(); sk_uptr.assign(1, 0); sk_ucol.clear(); sk_uval.clear(); sk_udiag.clear();
        sk_lptr.assign(1, 0); sk_lrow.clear(); sk_lval.clear();
        auto value = [&](int r, int c) {
            for (const auto& e : rows[r]) if (e.first == c) return e.second;
            return 0.0;
        };
        for (int step = 0; step < km; ++step) {
            // the columns of fewest active entries (up to four), their admissible rows of least cost
            int cmin = INT32_MAX;
            std::vector<int> cnt(km, 0);
            for (int b = 0; b < km; ++b) {
                if (cdone[b]) continue;
                int c2 = 0;
                for (int r : cols[b]) if (!rdone[r] && value(r, b) != 0.0) ++c2;
                cnt[b] = c2;
                if (c2 < cmin) cmin = c2;
            }
            if (cmin == 0 || cmin == INT32_MAX) return false;
            long best = -1; int bi = -1, bj = -1, seen = 0;
            for (int b = 0; b < km && seen < 4; ++b) {
                if (cdone[b] || cnt[b] != cmin) continue;
                ++seen;
                double mx = 0.0;
                for (int r : cols[b]) if (!rdone[r]) mx = std::max(mx, std::fabs(value(r, b)));
                for (int r : cols[b]) {
                    if (rdone[r]) continue;
                    const double v = value(r, b);
                    if (v == 0.0 || std::fabs(v) < 0.1 * mx) continue;
                    const long cost = (long)((int)rows[r].size() - 1) * (cmin - 1);
                    if (best < 0 || cost < best || (cost == best && (r < bi || (r == bi && b < bj)))) { best = cost; bi = r; bj = b; }
                }
            }
            if (bi < 0) return false;
            const double pv = value(bi, bj);
            if (!(std::fabs(pv) > 1e-14)) return false;
            sk_prow.push_back(bi); sk_pcol.push_back(bj); sk_udiag.push_back(pv);
            for (const auto& e : rows[bi]) if (e.first != bj) { sk_ucol.push_back(e.first); sk_uval.push_back(e.second); }
            sk_uptr.push_back((int)sk_ucol.size());
            rdone[bi] = 1; cdone[bj] = 1;
            for (int r : cols[bj]) {
                if (rdone[r]) continue;
                const double arj = value(r, bj);
                if (arj == 0.0) continue;
                const double l = arj / pv;
                sk_lrow.push_back(r); sk_lval.push_back(l);
                // row r <- row r - l * row bi (the pivot column's entry dropped)
                std::vector<std::pair<int, double>> nr;
                size_t x = 0, y = 0;
                const auto& R = rows[r];
                const auto& P = rows[bi];
                while (x < R.size() || y < P.size()) {
                    if (y == P.size() || (x < R.size() && R[x].first < P[y].first)) { if (R[x].first != bj) nr.push_back(R[x]); ++x; }
                    else if (x == R.size() || P[y].first < R[x].first) {
                        if (P[y].first != bj) { nr.push_back({P[y].first, -l * P[y].second}); cols[P[y].first].push_back(r); }
                        ++y;
                    } else {
                        if (R[x].first != bj) nr.push_back({R[x].first, R[x].second - l * P[y].second});
                        ++x; ++y;
                    }
                }
                rows[r].swap(nr);
            }
            sk_lptr.push_back((int)sk_lrow.size());
        }
        return true;
    }
    // kernel M w = b (b by kernel row in, w by kernel column out)
    void sparse_kernel_solve(double* z) const {
        const int km = bt_km;
        std::vector<double> b(z, z + km), x(km, 0.0);
        for (int st = 0; st < km; ++st) {
            const double bp = b[sk_prow[st]];
            for (int e = sk_lptr[st]; e < sk_lptr[st + 1]; ++e) b[sk_lrow[e]] -= sk_lval[e] * bp;
        }
        for (int st = km - 1; st >= 0; --st) {
            double v = b[sk_prow[st]];
            for (int e = sk_uptr[st]; e < sk_uptr[st + 1]; ++e) v -= sk_uval[e] * x[sk_ucol[e]];
            x[sk_pcol[st]] = v / sk_udiag[st];
        }
        for (int i = 0; i < km; ++i) z[i] = x[i];
    }
    // kernel M^T y = c (c by kernel column in, y by kernel row out)
    void sparse_kernel_tsolve(double* z) const {
        const int km = bt_km;
        std::vector<double> c(z, z + km), w(km, 0.0), y(km, 0.0);
        for (int st = 0; st < km; ++st) {
            const double ws = c[sk_pcol[st]] / sk_udiag[st];
            w[st] = ws;
            for (int e = sk_uptr[st]; e < sk_uptr[st + 1]; ++e) c[sk_ucol[e]] -= sk_uval[e] * ws;
        }
        for (int st = km - 1; st >= 0; --st) {
            double v = w[st];
            for (int e = sk_lptr[st]; e < sk_lptr[st + 1]; ++e) v -= sk_lval[e] * y[sk_lrow[e]];
            y[sk_prow[st]] = v;
        }
        for (int i = 0; i < km; ++i) z[i] = y[i];
    }
    void block_factor(const std::vector<int>& rowk) {
        bk_cptr.assign(k + 1, 0); bk_crow.clear(); bk_cval.clear();
        for (int j = 0; j < k; ++j) {
            for (int e = cptr[s_var[j]]; e < cptr[s_var[j] + 1]; ++e) {
                const int t = rowk[crow[e]];
                if (t >= 0 && cval[e] != 0.0) { bk_crow.push_back(t); bk_cval.push_back(cval[e]); }
            }
            bk_cptr[j + 1] = (int)bk_crow.size();
        }
        const int nz = bk_cptr[k];
        bk_rptr.assign(k + 1, 0); bk_rcol.assign(nz, 0); bk_rval.assign(nz, 0.0);
        for (int x = 0; x < nz; ++x) bk_rptr[bk_crow[x] + 1]++;
        for (int t = 0; t < k; ++t) bk_rptr[t + 1] += bk_rptr[t];
        {
            std::vector<int> cur(bk_rptr.begin(), bk_rptr.end() - 1);
            for (int j = 0; j < k; ++j)
                for (int x = bk_cptr[j]; x < bk_cptr[j + 1]; ++x) { const int q = cur[bk_crow[x]]++; bk_rcol[q] = j; bk_rval[q] = bk_cval[x]; }
        }
        std::vector<int> ccnt(k), rcnt(k), qu;
        std::vector<char> rdone(k, 0), cdone(k, 0);
        bt_u1t.clear(); bt_u1j.clear(); bt_u3t.clear(); bt_u3j.clear();
        auto singular = [&]() { status = ST_ERROR; throw Stop{}; };
        for (int j = 0; j < k; ++j) { ccnt[j] = bk_cptr[j + 1] - bk_cptr[j]; if (!ccnt[j]) singular(); if (ccnt[j] == 1) qu.push_back(j); }
        for (int t = 0; t < k; ++t) { rcnt[t] = bk_rptr[t + 1] - bk_rptr[t]; if (!rcnt[t]) singular(); }
        for (size_t h = 0; h < qu.size(); ++h) {
            const int j = qu[h];
            if (cdone[j] || ccnt[j] != 1) continue;
            int t = -1;
            for (int x = bk_cptr[j]; x < bk_cptr[j + 1]; ++x) if (!rdone[bk_crow[x]]) { t = bk_crow[x]; break; }
            if (t < 0) singular();
            rdone[t] = 1; cdone[j] = 1; bt_u1t.push_back(t); bt_u1j.push_back(j);
            for (int y = bk_rptr[t]; y < bk_rptr[t + 1]; ++y) {
                const int c = bk_rcol[y];
                if (cdone[c]) continue;
                if (--ccnt[c] == 1) qu.push_back(c); else if (ccnt[c] == 0) singular();
            }
        }
        qu.clear();
        for (int t = 0; t < k; ++t) if (!rdone[t] && rcnt[t] == 1) qu.push_back(t);
        for (size_t h = 0; h < qu.size(); ++h) {
            const int t = qu[h];
            if (rdone[t] || rcnt[t] != 1) continue;
            int j = -1;
            for (int y = bk_rptr[t]; y < bk_rptr[t + 1]; ++y) if (!cdone[bk_rcol[y]]) { j = bk_rcol[y]; break; }
            if (j < 0) singular();
            rdone[t] = 1; cdone[j] = 1; bt_u3t.push_back(t); bt_u3j.push_back(j);
            for (int x = bk_cptr[j]; x < bk_cptr[j + 1]; ++x) {
                const int r = bk_crow[x];
                if (rdone[r]) continue;
                if (--rcnt[r] == 1) qu.push_back(r); else if (rcnt[r] == 0) singular();
            }
        }
        bt_krow.clear(); bt_kcol.clear();
        std::vector<int> kcl(k, -1);
        for (int t = 0; t < k; ++t) if (!rdone[t]) bt_krow.push_back(t);
        for (int j = 0; j < k; ++j) if (!cdone[j]) { kcl[j] = (int)bt_kcol.size(); bt_kcol.push_back(j); }
        bt_km = (int)bt_krow.size();
        if ((int)bt_kcol.size() != bt_km) singular();
        bt_u3col.assign(k, 0); bt_u1row.assign(k, 0);
        for (int j : bt_u3j) bt_u3col[j] = 1;
        for (int t : bt_u1t) bt_u1row[t] = 1;
        if (opt.block_lu == 2) {   // kernel rows kept sparse, sorted by kernel column
            sk_rows.assign(bt_km, {});
            for (int a = 0; a < bt_km; ++a)
                for (int y = bk_rptr[bt_krow[a]]; y < bk_rptr[bt_krow[a] + 1]; ++y)
                    if (kcl[bk_rcol[y]] >= 0) sk_rows[a].push_back({kcl[bk_rcol[y]], bk_rval[y]});
        } else {
            bt_M.assign((size_t)bt_km * bt_km, 0.0);
            for (int a = 0; a < bt_km; ++a)
                for (int y = bk_rptr[bt_krow[a]]; y < bk_rptr[bt_krow[a] + 1]; ++y)
                    if (kcl[bk_rcol[y]] >= 0) bt_M[(size_t)a * bt_km + kcl[bk_rcol[y]]] = bk_rval[y];
        }
        if (bt_km > 0 && !(opt.block_lu == 2 ? sparse_kernel_lu() : dense_lu(bt_M, bt_km, bt_piv))) singular();
    }
    // K x = b: b by K rows in, x by K columns out
    void block_solve(std::vector<double>& z) const {
        const std::vector<double> b = z;
        std::vector<double> x(k, 0.0);
        auto row_step = [&](int t, int j) {
            double s = b[t], pv = 0.0;
            for (int y = bk_rptr[t]; y < bk_rptr[t + 1]; ++y) {
                if (bk_rcol[y] == j) pv = bk_rval[y]; else s -= bk_rval[y] * x[bk_rcol[y]];
            }
            x[j] = s / pv;
        };
        for (size_t i = 0; i < bt_u3t.size(); ++i) row_step(bt_u3t[i], bt_u3j[i]);
        if (bt_km > 0) {
            std::vector<double> w(bt_km);
            for (int a = 0; a < bt_km; ++a) {
                const int t = bt_krow[a];
                double s = b[t];
                for (int y = bk_rptr[t]; y < bk_rptr[t + 1]; ++y) if (bt_u3col[bk_rcol[y]]) s -= bk_rval[y] * x[bk_rcol[y]];
                w[a] = s;
            }
            if (opt.block_lu == 2) sparse_kernel_solve(w.data()); else dense_solve(bt_M, bt_km, bt_piv, w.data());
            for (int c = 0; c < bt_km; ++c) x[bt_kcol[c]] = w[c];
        }
        for (int i = (int)bt_u1t.size() - 1; i >= 0; --i) row_step(bt_u1t[i], bt_u1j[i]);
        z = x;
    }
    // K^T y = c: c by K columns in, y by K rows out
    void block_tsolve(std::vector<double>& z) const {
        const std::vector<double> c = z;
        std::vector<double> y(k, 0.0);
        auto col_step = [&](int t, int j) {
            double s = c[j], pv = 0.0;
            for (int x = bk_cptr[j]; x < bk_cptr[j + 1]; ++x) {
                if (bk_crow[x] == t) pv = bk_cval[x]; else s -= bk_cval[x] * y[bk_crow[x]];
            }
            y[t] = s / pv;
        };
        for (size_t i = 0; i < bt_u1t.size(); ++i) col_step(bt_u1t[i], bt_u1j[i]);
        if (bt_km > 0) {
            std::vector<double> g(bt_km);
            for (int b2 = 0; b2 < bt_km; ++b2) {
                const int j = bt_kcol[b2];
                double s = c[j];
                for (int x = bk_cptr[j]; x < bk_cptr[j + 1]; ++x) if (bt_u1row[bk_crow[x]]) s -= bk_cval[x] * y[bk_crow[x]];
                g[b2] = s;
            }
            if (opt.block_lu == 2) sparse_kernel_tsolve(g.data()); else dense_tsolve(bt_M, bt_km, bt_piv, g.data());
            for (int a = 0; a < bt_km; ++a) y[bt_krow[a]] = g[a];
        }
        for (int i = (int)bt_u3t.size() - 1; i >= 0; --i) col_step(bt_u3t[i], bt_u3j[i]);
        z = y;
    }

    // B0 x = b (b by rows, x by positions): Matrix::solve non-transposed.
    void b0_solve(const std::vector<double>& b, std::vector<double>& out) const {
        std::vector<double> z(k);
        for (int t = 0; t < k; ++t) z[t] = b[rp_row[t]];
        k_solve(z);
        out.assign(m, 0.0);
        std::vector<double> xs_of_var;  // dense lookup of structural solution by column
        std::vector<int> kcol(n, -1);
        for (int j = 0; j < k; ++j) { out[s_pos[j]] = z[j]; kcol[s_var[j]] = j; }
        for (int r = 0; r < m; ++r) {
            int i = row_slackpos[r];
            if (i < 0) continue;
            double s = b[r];
            for (int e = rptr[r]; e < rptr[r + 1]; ++e) {
                int c = rcol[e];
                if (c < n && kcol[c] >= 0) s -= rval[e] * z[kcol[c]];
            }
            out[i] = s;
        }
    }
    // B0^T y = c (c by positions, y by rows): Matrix::solve transposed.
    void b0t_solve(const std::vector<double>& c, std::vector<double>& y) const {
        y.assign(m, 0.0);
        std::vector<char> inR(m, 0);
        for (int r = 0; r < m; ++r) if (row_slackpos[r] >= 0) { y[r] = c[row_slackpos[r]]; inR[r] = 1; }
        std::vector<double> z(k);
        for (int j = 0; j < k; ++j) {
            double s = c[s_pos[j]];
            for (int e = cptr[s_var[j]]; e < cptr[s_var[j] + 1]; ++e)
                if (inR[crow[e]]) s -= cval[e] * y[crow[e]];
            z[j] = s;
        }
        kt_solve(z);
        for (int t = 0; t < k; ++t) y[rp_row[t]] = z[t];
    }
    // linalg::PFIsolve (linalg.cpp:12-46)
    void pfi(std::vector<double>& sol, bool transpose) const {
        const int T = (int)eta.size();
        if (!transpose) {
            for (int t = 0; t < T; ++t) {
                const int kk = eta_p[t]; const double* ev = eta[t].data();
                const double sk = sol[kk];
                for (int i = 0; i < m; ++i) sol[i] = sol[i] + sk * ev[i];
                sol[kk] = sk * ev[kk];
            }
        } else {
            for (int t = T - 1; t >= 0; --t) {
                const int kk = eta_p[t]; const double* ev = eta[t].data();
                double s = 0.0;
                for (int i = 0; i < m; ++i) s += ev[i] * sol[i];
                sol[kk] = s;
            }
        }
    }
    // SequentialDualSimplex::solveLinSys (sequentialDualSimplex.cpp:28-70)
    void ftran(const std::vector<double>& rhs, std::vector<double>& sol) const { b0_solve(rhs, sol); pfi(sol, false); }
    void btran(const std::vector<double>& rhs, std::vector<double>& sol) const {
        std::vector<double> tmp = rhs; pfi(tmp, true); b0t_solve(tmp, sol);
    }

    // ---------------------------------------------------------------- helpers
    // checkVarIsInfeas (baseDualSimplex.tpp:443-466), switch fallthrough kept.
    std::pair<bool, double> var_infeas(int i) const {
        switch (type[i]) {
            case LOWER:
                if (x[i] < lb[i] - EPS_BOUND) return {true, x[i] - lb[i]};
                [[fallthrough]];
            case UPPER:
                if (x[i] > ub[i] + EPS_BOUND) return {true, x[i] - ub[i]};
                [[fallthrough]];
            case FIXED:
                if (std::fabs(x[i] - lb[i]) < EPS_BOUND) return {true, x[i] - lb[i]};
                [[fallthrough]];
            case BOXED:
                if (x[i] > ub[i] + EPS_BOUND) return {true, x[i] - ub[i]};
                else if (x[i] < lb[i] - EPS_BOUND) return {true, x[i] - lb[i]};
        }
        return {false, 0.0};
    }
    // checkPrimalFeasible (tpp:296-324), fallthrough kept.
    bool primal_feasible() const {
        for (int i : basis) {
            switch (type[i]) {
                case FIXED:
                    if (std::fabs(x[i] - lb[i]) > EPS_BOUND) return false;
                    [[fallthrough]];
                case FREE: break;
                case BOXED:
                    if (x[i] > ub[i] + EPS_R * std::fabs(ub[i]) + EPS_BOUND || x[i] < lb[i] - EPS_R * std::fabs(lb[i]) - EPS_BOUND) return false;
                    [[fallthrough]];
                case UPPER:
                    if (x[i] > ub[i] + EPS_R * std::fabs(ub[i]) + EPS_BOUND) return false;
                    [[fallthrough]];
                case LOWER:
                    if (x[i] < lb[i] - EPS_R * std::fabs(lb[i]) - EPS_BOUND) return false;
            }
        }
        return true;
    }
    // checkDualFeasible / counterDualInfeasible (tpp:362-440)
    int dual_infeasible_count() const {
        int num = 0;
        for (int i : nonbasis) {
            switch (type[i]) {
                case FREE: if (std::fabs(d[i]) < EPS_D || std::isnan(d[i])) num++; break;
                case UPPER: if (d[i] > EPS_D || std::isnan(d[i])) num++; break;
                case LOWER: if (d[i] < -EPS_D || std::isnan(d[i])) num++; break;
                default: break;
            }
        }
        return num;
    }
    bool dual_feasible() const { return dual_infeasible_count() == 0; }
    // experiments (shift_costs): make every wrong-signed nonbasic reduced cost a
    // small margin of the right sign by shifting its cost; false if a free
    // variable is dual infeasible (no shift fixes that)
    bool shift_dual_infeasible() {
        for (int j : nonbasis) {
            const double margin = 1e-7 + 1e-5 * std::fabs(original_costs.empty() ? costs[j] : original_costs[j]);
            if (type[j] == LOWER && d[j] < -EPS_D) { costs[j] += -d[j] + margin; d[j] = margin; }
            else if (type[j] == UPPER && d[j] > EPS_D) { costs[j] += -d[j] - margin; d[j] = -margin; }
            else if (type[j] == FREE && std::fabs(d[j]) < EPS_D) return false;
        }
        return dual_feasible();
    }

    // setPrimalVars (tpp:74-101)
    void set_primal_vars() {
        for (int i : nonbasis) {
            switch (type[i]) {
                case FIXED: x[i] = lb[i]; break;
                case FREE: x[i] = 0; break;
                case BOXED: x[i] = (d[i] > 0) ? lb[i] : ub[i]; break;
                case UPPER: x[i] = ub[i]; break;
                case LOWER: x[i] = lb[i]; break;
            }
        }
    }
    // initBetaWeights (tpp:34-70)
    void init_beta(bool ibasis) {
        if (ibasis) { for (int i = 0; i < m; ++i) beta[i] = 1; return; }
        std::vector<double> e(m, 0.0), buf;
        for (int i = 0; i < m; ++i) {
            e.assign(m, 0.0); e[i] = 1;
            btran(e, buf);
            double s = 0; for (double v : buf) s += v * v;  // ValuesVector::norm = sum of squares
            beta[i] = s;
        }
    }
    // initReducedCosts (sequentialDualSimplex.cpp:119-132) with dotUpdate UPDATE_T set=true.
    void init_reduced_costs() {
        std::vector<double> cb(m), y;
        for (int i = 0; i < m; ++i) cb[i] = costs[basis[i]];
        btran(cb, y);
        for (int j : nonbasis) {
            double acc = 0.0;
            for (int e = cptr[j]; e < cptr[j + 1]; ++e) acc += cval[e] * y[crow[e]] * -1.0;
            d[j] = acc + costs[j] * 1.0;
        }
    }
    // dualSimplexInit (sequentialDualSimplex.cpp:230-250)
    void dual_simplex_init() {
        set_primal_vars();
        std::vector<double> buff(N, 0.0), rhs(m), xb;
        for (int j : nonbasis) buff[j] = x[j];
        for (int i = 0; i < m; ++i) {
            double s = 0.0 * 1.0;
            for (int e = rptr[i]; e < rptr[i + 1]; ++e) s += rval[e] * buff[rcol[e]] * -1.0;
            rhs[i] = s;
        }
        ftran(rhs, xb);
        for (int i = 0; i < m; ++i) x[basis[i]] = xb[i];
        init_reduced_costs();
        double s = 0; for (int j = 0; j < N; ++j) s += costs[j] * x[j];
        obj = s;
    }
    // checkPerturbNeed (tpp:223-234), std::unique semantics kept
    bool perturb_needed() const {
        std::vector<double> c(costs);
        std::sort(c.begin(), c.end());
        int uniq = c.empty() ? 0 : 1;
        double last = c.empty() ? 0 : c[0];
        for (size_t i = 1; i < c.size(); ++i) if (!(std::fabs(last - c[i]) < EPS_COSTS)) { last = c[i]; ++uniq; }
        return uniq < PERTURB_RATIO * (double)N;
    }
    static double weight_for(int i) {  // getWeight (tpp:278-292)
        static const double w[10] = {0.01, 0.1, 1, 2, 5, 10, 20, 30, 40, 100};
        int kk = (i > 10) ? 9 : (i == 0 ? 0 : i - 1);
        return w[kk];
    }
    // perturbCosts (tpp:238-275); the sign assignment is overwritten as in the reference
    void perturb() {
        original_costs = costs;
        std::uniform_real_distribution<> dist(0.0, 1.0);
        double mean = 0; for (double v : costs) mean += v; mean /= (double)N;
        const double min_p = std::min(1e-2 * EPS_D, PSI);
        const double max_p = std::max(1e+3 * EPS_D, PSI * 10 * mean);
        for (int i = 0; i < N; ++i) {
            const double mag = 100 * EPS_D + PSI * costs[i];
            double pert;
            if (type[i] != LOWER && type[i] != FREE) pert = -0.5 * mag * (1 + dist(gen));
            pert = 0.5 * mag * (1 + dist(gen));
            pert = weight_for(cptr[i + 1] - cptr[i]) * pert;
            while (std::fabs(pert) > std::fabs(max_p) || std::fabs(pert) < std::fabs(min_p)) {
                if (std::fabs(pert) > std::fabs(max_p)) pert = 0.1 * pert;
                else if (std::fabs(pert) < std::fabs(min_p)) pert = 10 * pert;
            }
            costs[i] += pert;
        }
        perturbed = true;
    }

    // pivotRow: Matrix::dotUpdate UPDATE_T, alpha=1, beta=0 (matrix.cpp:273-286)
    void pivot_row(const std::vector<double>& rho, std::vector<double>& alpha) const {
        alpha.resize(n);
        for (int i = 0; i < n; ++i) {
            const int j = nonbasis[i];
            double acc = 0.0;
            for (int e = cptr[j]; e < cptr[j + 1]; ++e) acc += cval[e] * rho[crow[e]] * 1.0;
            alpha[i] = acc + costs[j] * 0.0;
        }
    }
    // simpleRatioTest (tpp:546-572); q = -1 when nothing is taken (reference: uninitialised)
    void ratio_test(const std::vector<int>& F, const std::vector<double>& alpha, int& q, int& q_idx) const {
        q = -1; q_idx = -1;
        if (opt.harris) {   // experiments: two-pass Harris (not the reference's rule)
            double tmax = INF;
            for (int i : F) {
                const double a = alpha[i];
                tmax = std::min(tmax, (d[nonbasis[i]] + std::copysign(EPS_D, a)) / a);
            }
            double best = -1.0;
            for (int i : F) {
                const int j = nonbasis[i];
                if (d[j] / alpha[i] <= tmax && std::fabs(alpha[i]) > best) { best = std::fabs(alpha[i]); q = j; q_idx = i; }
            }
            return;
        }
        double theta = INF;
        for (int i : F) {
            const int j = nonbasis[i];
            const double tt = d[j] / alpha[i];
            if (tt < theta) { theta = tt; q = j; q_idx = i; }
            else if (q_idx >= 0 && std::fabs(tt - theta) < EPS_Z) {
                if (std::fabs(alpha[i]) > std::fabs(alpha[q_idx])) { theta = tt; q = j; q_idx = i; }
            }
        }
    }
    void record(int p, int q, double theta) {
        if (tp && tcount < tcap) { tp[tcount] = p; tq[tcount] = q; tth[tcount] = theta; tob[tcount] = obj; }
        ++tcount;
    }

    // ------------------------------------------------------------- phase 1
    // minimizeDualInfeasibilityInit + initPhase1PricingVector (tpp:776-795,
    // sequentialDualSimplex.cpp:135-152)
    void phase1_init(std::vector<double>& f) {
        init_reduced_costs();
        std::vector<int> inf_u, inf_l;
        for (int i = 0; i < n; ++i) {
            const int j = nonbasis[i];
            if ((type[j] == UPPER || type[j] == FREE) && d[j] > EPS_D) inf_u.push_back(j);
            else if ((type[j] == LOWER || type[j] == FREE) && d[j] < -EPS_D) inf_l.push_back(j);
        }
        std::vector<double> cc(m, 0.0);
        double Z = 0;
        for (int j : inf_l) { Z += d[j]; for (int e = cptr[j]; e < cptr[j + 1]; ++e) cc[crow[e]] += cval[e]; }
        for (int j : inf_u) { Z -= d[j]; for (int e = cptr[j]; e < cptr[j + 1]; ++e) cc[crow[e]] -= cval[e]; }
        obj = Z;
        ftran(cc, f);
    }
    // minimizeDualInfeasibility (tpp:799-934)
    Phase1Out phase1() {
        in_phase1 = true;
        Phase1Out st = P1_SOLVED;
        std::vector<double> rho, f, alpha, alpha_q, tau;
        phase1_init(f);
        int cycle = 0;
        std::unordered_set<int> blocked;
        long long pivots_at_nop = -1;   // guard: repeated "no row" restart without a pivot
        while (true) {
            ++iteration; ++phase1_iters; tick();
            if (!perturbed && cycle > MAX_CYCLE) { perturb(); phase1_init(f); }
            if (cycle > NEED_RESTART || obj > INF || std::isnan(obj)) phase1_init(f);
            if (iteration % opt.refactor_interval == 0) refactor();
            // phase1Pricing (tpp:746-772)
            double maxw = 0; int p = -1, p_idx = -1; bool found = false;
            for (int i = 0; i < m; ++i) {
                const int j = basis[i];
                if ((type[j] == LOWER && f[i] > EPS_F) || (type[j] == UPPER && f[i] < -EPS_F) || type[j] == BOXED || type[j] == FIXED) {
                    const double w = f[i] * f[i] / beta[i];
                    if (w > maxw && !blocked.count(j)) { p = j; p_idx = i; maxw = w; found = true; }
                }
            }
            const int ndinf = dual_infeasible_count();
            if (!found || !ndinf) {
                if (std::fabs(obj) < EPS_A || !ndinf) { st = P1_SOLVED; break; }
                else if (obj > 0) { st = P1_DUALINF; break; }
            }
            if (p < 0 || p_idx < 0) {
                // The reference's only dual-infeasible exit is obj > 0 (tpp:848), but the
                // phase-1 objective is a sum of infeasibilities and never positive; with
                // no leaving row and infeasibilities left the auxiliary problem is at its
                // optimum, so the LP is dual infeasible (the reference restarts forever).
                if (!opt.strict_reference && ndinf > 0 && obj < -EPS_A && pivots_at_nop == pivots) { st = P1_DUALINF; break; }
                pivots_at_nop = pivots;
                refactor(); phase1_init(f); init_beta(false); blocked.clear(); ++restarts; continue;
            }
            if (obj > EPS_BOUND) { refactor(); phase1_init(f); init_beta(false); blocked.clear(); ++restarts; continue; }
            std::vector<double> e(m, 0.0); e[p_idx] = 1;
            btran(e, rho);
            pivot_row(rho, alpha);
            const bool neg = f[p_idx] > 0;
            if (neg) for (double& a : alpha) a = -a;
            std::vector<int> F;  // phase1SetRatioTestCandidates (tpp:530-542)
            for (int i = 0; i < n; ++i) {
                const int j = nonbasis[i];
                if ((d[j] >= 0 && alpha[i] > EPS_A) || (d[j] <= 0 && alpha[i] < -EPS_A)) F.push_back(i);
            }
            if (F.empty()) { blocked.insert(p); refactor(); phase1_init(f); ++restarts; continue; }
            blocked.clear();
            int q, q_idx;
            ratio_test(F, alpha, q, q_idx);
            if (q < 0) { status = ST_ERROR; throw Stop{}; }
            if (neg) for (double& a : alpha) a = -a;
            const double theta = d[q] / alpha[q_idx];
            std::vector<double> aq(m, 0.0);
            for (int e2 = cptr[q]; e2 < cptr[q + 1]; ++e2) aq[crow[e2]] = cval[e2];
            ftran(aq, alpha_q);
            if (std::fabs(alpha_q[p_idx] - alpha[q_idx]) > EPS_R * (1 + std::fabs(alpha_q[p_idx]))) refactor();
            // infisibilityCorr (tpp:614-625)
            double corr = 0;
            if ((type[q] == UPPER || type[q] == FREE) && d[q] > EPS_D) corr = 1;
            else if ((type[q] == LOWER || type[q] == FREE) && d[q] < -EPS_D) corr = -1;
            obj = obj - theta * f[p_idx];
            // simpleReducedCostsUpate (sequentialDualSimplex.cpp:163-172)
            for (int i = 0; i < n; ++i) { const int j = nonbasis[i]; d[j] -= theta * alpha[i]; }
            d[p] = -theta; d[q] = 0;
            const double theta_P = f[p_idx] / alpha_q[p_idx];
            // phase1UpdateAndChangeBasis (sequentialDualSimplex.cpp:174-197)
            ftran(rho, tau);
            std::vector<double> ev(m);
            const double ap = alpha_q[p_idx], bp = beta[p_idx];
            for (int i = 0; i < m; ++i) {
                f[i] = (i != p_idx) ? f[i] - alpha_q[i] * theta_P : f[p_idx];
                ev[i] = (i != p_idx) ? -alpha_q[i] / ap : 1 / ap;
                if (i != p_idx) { const double r = alpha_q[i] / ap; beta[i] = beta[i] - 2 * alpha_q[i] / ap * tau[i] + (r * r) * bp; }
            }
            beta[p_idx] = beta[p_idx] / (ap * ap);
            basis[p_idx] = q; nonbasis[q_idx] = p; is_basic[q] = 1; is_basic[p] = 0;
            eta.push_back(std::move(ev)); eta_p.push_back(p_idx);
            f[p_idx] = f[p_idx] / alpha_q[p_idx] + corr;
            ++pivots;
            cycle = (std::fabs(theta) < EPS_A) ? cycle + 1 : 0;
        }
        in_phase1 = false;
        return st;
    }

    // ------------------------------------------------------------- phase 2
    // presolve (tpp:5-30)
    Phase1Out presolve() {
        if (perturb_needed()) perturb();
        init_beta(true);
        Phase1Out st = phase1();
        if (st == P1_DUALINF) return st;
        set_primal_vars();
        return st;
    }
    // callDualSolver (sequentialDualSimplex.cpp:253-515; GPU variant cudaDualSimplex.cpp:396-655)
    bool phase2() {
        std::vector<double> rho, alpha, alpha_q, tau, dxb;
        if (opt.gpu_control_flow) refactor();
        dual_simplex_init();
        int cycle = 0;
        bool unbound_checked = false;
        long long pivots_at_nop = -1;  // restart-loop guard
        while (true) {
            ++iteration; tick();
            if (iteration % opt.refactor_interval == 0) refactor();
            if (iteration % NEED_RESTART == 0 && !dual_feasible()) {
                if (!(opt.shift_costs && perturbed && shift_dual_infeasible())) {
                    refactor(); phase1(); dual_simplex_init(); ++restarts;
                }
            }
            if (!perturbed && cycle > MAX_CYCLE) {
                perturb(); refactor(); dual_simplex_init();
                // guard: the perturbed reduced costs may be dual infeasible
                if (!opt.strict_reference && !dual_feasible() && !(opt.shift_costs && shift_dual_infeasible())) {
                    refactor(); phase1(); dual_simplex_init(); ++restarts;
                }
            }
            if (primal_feasible()) { status = ST_OPTIMAL; break; }
            // DSEPricing (tpp:470-501); blocked set is always empty in phase 2
            double maxw = 0, delta = 0; int p = -1, p_idx = -1; bool is_lower = false;
            for (int i = 0; i < m; ++i) {
                if (!p2_block.empty() && p2_block[i] > iteration) continue;   // experiments (col_rel_tol)
                auto [inf, dt] = var_infeas(basis[i]);
                if (inf && std::fabs(dt) > 1e-8) {
                    double w = (dt * dt) / beta[i];
                    if (opt.var_weight) w *= opt.var_weight[basis[i]];
                    if (w > maxw) { p = basis[i]; p_idx = i; delta = dt; maxw = w; is_lower = dt < 0; }
                }
            }
            if ((p < 0 || p_idx < 0) && !p2_block.empty()) {   // experiments: blocked rows come back first
                bool any = false;
                for (int& b : p2_block) { any |= b > iteration; b = 0; }
                if (any) continue;
            }
            if (p < 0 || p_idx < 0) {
                if (!opt.strict_reference && pivots_at_nop == pivots) {
                    status = ST_OPTIMAL; break;  // a second restart cannot change anything: infeasibilities <= 1e-8
                }
                pivots_at_nop = pivots;
                refactor(); init_beta(false);
                if (opt.gpu_control_flow) phase1();
                dual_simplex_init(); ++restarts;
                continue;
            }
            std::vector<double> e(m, 0.0); e[p_idx] = 1;
            btran(e, rho);
            pivot_row(rho, alpha);
            delta = std::fabs(delta);
            const int sgn = is_lower ? -1 : 1;
            if (is_lower) for (double& a : alpha) a = -a;
            std::vector<int> F; F.reserve(n);
            const double eps_a = opt.pivot_abs_tol > 0 ? opt.pivot_abs_tol : EPS_A;   // experiments
            for (int i = 0; i < n; ++i) {
                bool cond = false;
                const double a = alpha[i];
                const int j = nonbasis[i];
                if (a > eps_a) cond = std::fabs(x[j] - lb[j]) < EPS_Z && (type[j] == LOWER || type[j] == BOXED);
                else if (a < -eps_a) cond = std::fabs(x[j] - ub[j]) < EPS_Z && (type[j] == UPPER || type[j] == BOXED);
                else cond = type[j] == FREE;
                if (cond) F.push_back(i);
            }
            if (opt.rt_rel_tol > 0 && !F.empty()) {   // experiments: drop relatively tiny pivots
                double amax = 0.0;
                for (int i : F) amax = std::max(amax, std::fabs(alpha[i]));
                std::vector<int> F2;
                for (int i : F) if (std::fabs(alpha[i]) >= opt.rt_rel_tol * amax) F2.push_back(i);
                F.swap(F2);
            }
            if (F.empty()) {
                if (unbound_checked) { status = ST_PRIMAL_INF; break; }
                unbound_checked = true;
                refactor(); init_beta(false); phase1(); dual_simplex_init(); ++restarts;
                continue;
            }
            unbound_checked = false;
            int q = -1, q_idx = -1;
            while (!F.empty()) {
                ratio_test(F, alpha, q, q_idx);
                if (q < 0) break;
                if (type[q] == BOXED) {
                    if (delta - (ub[q] - lb[q]) * std::fabs(alpha[q_idx]) <= 0) break;
                    delta -= (ub[q] - lb[q]) * std::fabs(alpha[q_idx]);
                    F.erase(std::remove(F.begin(), F.end(), q_idx), F.end());
                } else break;
            }
            if (q < 0) { status = ST_ERROR; throw Stop{}; }
            if (is_lower) for (double& a : alpha) a = -a;
            double theta = d[q] / alpha[q_idx];
            if (opt.harris && theta * sgn < 0) theta = 0.0;   // experiments: a wrong-signed step within the tolerance
            delta = sgn * delta;
            std::vector<double> aq(m, 0.0);
            for (int e2 = cptr[q]; e2 < cptr[q + 1]; ++e2) aq[crow[e2]] = cval[e2];
            ftran(aq, alpha_q);
            if (opt.col_rel_tol > 0) {   // experiments: refuse a pivot tiny against its column
                double amax = 0.0;
                for (double v : alpha_q) amax = std::max(amax, std::fabs(v));
                if (std::fabs(alpha_q[p_idx]) < opt.col_rel_tol * amax) {
                    if (p2_block.empty()) p2_block.assign(m, 0);
                    p2_block[p_idx] = iteration + 100;
                    ++refused_pivots;
                    refactor();
                    continue;
                }
            }
            if (std::fabs(alpha_q[p_idx] - alpha[q_idx]) > EPS_R * (1 + std::fabs(alpha_q[p_idx]))) refactor();
            // dual update + BFRT sets (sequentialDualSimplex.cpp:438-467)
            std::vector<int> low, up;
            std::vector<double> cc(m, 0.0);
            double dz = 0;
            for (int i = 0; i < n; ++i) {
                const int j = nonbasis[i];
                d[j] = d[j] - theta * alpha[i];
                if (type[j] == BOXED) {
                    if (std::fabs(x[j] - lb[j]) < EPS_Z && d[j] < -EPS_D) { low.push_back(j); dz += costs[j] * (ub[j] - lb[j]); }
                    else if (std::fabs(x[j] - ub[j]) < EPS_Z && d[j] > EPS_D) { up.push_back(j); dz -= costs[j] * (ub[j] - lb[j]); }
                }
            }
            for (int j : low) for (int e2 = cptr[j]; e2 < cptr[j + 1]; ++e2) cc[crow[e2]] += cval[e2] * diff_bounds[j] * 1.0;
            for (int j : up) for (int e2 = cptr[j]; e2 < cptr[j + 1]; ++e2) cc[crow[e2]] += cval[e2] * diff_bounds[j] * -1.0;
            d[p] = -theta; d[q] = 0;
            if (!up.empty() || !low.empty()) {
                ftran(cc, dxb);
                for (int i = 0; i < m; ++i) x[basis[i]] = x[basis[i]] - dxb[i];
                for (int i = 0; i < m; ++i) dz -= costs[basis[i]] * dxb[i];
                flips += (int)(low.size() + up.size());
            }
            obj += dz;
            const double theta_P = delta / alpha_q[p_idx];
            {
                double amax = 0.0;
                for (int i = 0; i < m; ++i) amax = std::max(amax, std::fabs(alpha_q[i]));
                min_pivot = std::min(min_pivot, std::fabs(alpha_q[p_idx]));
                if (amax > 0) min_pivot_rel = std::min(min_pivot_rel, std::fabs(alpha_q[p_idx]) / amax);
                max_step = std::max(max_step, std::fabs(theta_P));
            }
            // updateAndChangeBasis (sequentialDualSimplex.cpp:200-227)
            ftran(rho, tau);
            std::vector<double> ev(m);
            const double ap = alpha_q[p_idx], bp = beta[p_idx];
            for (int i = 0; i < m; ++i) {
                const int j = basis[i];
                x[j] = x[j] - theta_P * alpha_q[i];
                ev[i] = (i != p_idx) ? -alpha_q[i] / ap : 1 / ap;
                if (i != p_idx) { const double r = alpha_q[i] / ap; beta[i] = beta[i] - 2 * alpha_q[i] / ap * tau[i] + (r * r) * bp; }
            }
            beta[p_idx] = beta[p_idx] / (ap * ap);
            x[q] = x[q] + theta_P;
            basis[p_idx] = q; nonbasis[q_idx] = p; is_basic[q] = 1; is_basic[p] = 0;
            eta.push_back(std::move(ev)); eta_p.push_back(p_idx);
            for (int j : low) x[j] = ub[j];
            for (int j : up) x[j] = lb[j];
            obj += theta * delta;
            if (std::fabs(theta) < EPS_A) cycle += 1;
            ++pivots;
            record(p, q, theta);
        }
        return status == ST_OPTIMAL;
    }
    // presolve + solve + postProcess (tpp:123-180), with the optional cleanup
    void run() {
        try {
            refactor();  // initDualSimplex: B <- slack basis, LU (sequentialDualSimplex.cpp:4-25)
            Phase1Out st = presolve();
            if (st == P1_DUALINF) { status = ST_DUAL_INF; return; }
            bool ok = phase2();
            for (int round = 0; round < 3 && perturbed; ++round) {
                costs = original_costs;
                dual_simplex_init();
                if (!ok || opt.strict_reference || dual_feasible()) break;
                // cleanup: the perturbed optimum is dual infeasible for the true costs
                status = ST_UNSOLVED;
                refactor(); Phase1Out s1 = phase1();
                if (s1 == P1_DUALINF) { status = ST_DUAL_INF; return; }
                set_primal_vars();
                ok = phase2();
            }
        } catch (const Stop&) {
            if (status == ST_UNSOLVED || status == ST_OPTIMAL) status = ST_ERROR;
        }
    }
};

}  // namespace

extern "C" {

void or_default_options(or_options* o) {
    o->refactor_interval = 100;
    o->max_iterations = 2000000;
    o->strict_reference = 0;
    o->seed = 12345;
    o->gpu_control_flow = 1;
    o->verbose = 0;
    o->var_weight = nullptr;
    o->harris = 0;
    o->block_lu = 0;
    o->rt_rel_tol = 0.0;
    o->col_rel_tol = 0.0;
    o->pivot_abs_tol = 0.0;
    o->shift_costs = 0;
}

int or_solve_typed(int m, int n, const int* row_ptr, const int* col_idx, const double* val,
                   const double* c, const int* col_type, const double* col_lb, const double* col_ub,
                   const int* row_type, const double* row_lb, const double* row_ub,
                   const or_options* opt, or_result* res, double* x_out, double* d_out,
                   int* basis_out, int* trace_p, int* trace_q, double* trace_theta,
                   double* trace_obj, int trace_cap, int* trace_count) {
    if (m <= 0 || n <= 0 || !row_ptr || !res) return -1;
    if (m > n) return -4;  // Problem::checkConstraints (problem.tpp:230-239)
    Oracle o;
    if (opt) o.opt = *opt; else or_default_options(&o.opt);
    o.load(m, n, row_ptr, col_idx, val, c, col_type, col_lb, col_ub, row_type, row_lb, row_ub);
    o.tp = trace_p; o.tq = trace_q; o.tth = trace_theta; o.tob = trace_obj; o.tcap = trace_cap;
    o.run();
    res->status = o.status;
    res->iterations = o.iteration;
    res->phase1_iterations = o.phase1_iters;
    res->refactors = o.refactors;
    res->restarts = o.restarts;
    res->perturbed = o.perturbed;
    res->bfrt_flips = o.flips;
    res->bump_size = o.k;
    double z = 0; for (int j = 0; j < n; ++j) z += (o.perturbed ? o.original_costs[j] : o.costs[j]) * o.x[j];
    res->objective = z;
    res->obj_incremental = o.obj;
    res->min_pivot = o.min_pivot; res->min_pivot_rel = o.min_pivot_rel; res->max_step = o.max_step;
    res->refused_pivots = o.refused_pivots;
    if (x_out) std::memcpy(x_out, o.x.data(), sizeof(double) * o.N);
    if (d_out) std::memcpy(d_out, o.d.data(), sizeof(double) * o.N);
    if (basis_out) std::memcpy(basis_out, o.basis.data(), sizeof(int) * m);
    if (trace_count) *trace_count = o.tcount;
    return 0;
}

int or_dse_pricing(int m, const int* basis, const double* x, const double* lb, const double* ub,
                   const int* type, const double* beta, int* p, int* p_idx, double* delta,
                   int* is_lower, int* primal_feasible) {
    // Same code path as the solver: a tiny Oracle holding only the vectors.
    Oracle o;
    int N = 0;
    for (int i = 0; i < m; ++i) N = std::max(N, basis[i] + 1);
    (void)N;
    o.m = m;
    // DSEPricing (tpp:470-501) on caller vectors
    double maxw = 0, dl = 0; int pp = -1, pi = -1; bool il = false;
    auto infeas = [&](int i) -> std::pair<bool, double> {
        switch (type[i]) {
            case LOWER: if (x[i] < lb[i] - EPS_BOUND) return {true, x[i] - lb[i]}; [[fallthrough]];
            case UPPER: if (x[i] > ub[i] + EPS_BOUND) return {true, x[i] - ub[i]}; [[fallthrough]];
            case FIXED: if (std::fabs(x[i] - lb[i]) < EPS_BOUND) return {true, x[i] - lb[i]}; [[fallthrough]];
            case BOXED:
                if (x[i] > ub[i] + EPS_BOUND) return {true, x[i] - ub[i]};
                else if (x[i] < lb[i] - EPS_BOUND) return {true, x[i] - lb[i]};
        }
        return {false, 0.0};
    };
    for (int i = 0; i < m; ++i) {
        auto [inf, dt] = infeas(basis[i]);
        if (inf && std::fabs(dt) > 1e-8) {
            const double w = (dt * dt) / beta[i];
            if (w > maxw) { pp = basis[i]; pi = i; dl = dt; maxw = w; il = dt < 0; }
        }
    }
    *p = pp; *p_idx = pi; *delta = dl; *is_lower = il;
    bool feas = true;
    for (int ii = 0; ii < m && feas; ++ii) {
        const int i = basis[ii];
        switch (type[i]) {
            case FIXED: if (std::fabs(x[i] - lb[i]) > EPS_BOUND) { feas = false; break; } [[fallthrough]];
            case FREE: break;
            case BOXED:
                if (x[i] > ub[i] + EPS_R * std::fabs(ub[i]) + EPS_BOUND || x[i] < lb[i] - EPS_R * std::fabs(lb[i]) - EPS_BOUND) { feas = false; break; }
                [[fallthrough]];
            case UPPER: if (x[i] > ub[i] + EPS_R * std::fabs(ub[i]) + EPS_BOUND) { feas = false; break; } [[fallthrough]];
            case LOWER: if (x[i] < lb[i] - EPS_R * std::fabs(lb[i]) - EPS_BOUND) { feas = false; break; }
        }
    }
    *primal_feasible = feas;
    return 0;
}

int or_ratio_test(int n, const int* nonbasis, const double* alpha_in, double delta_in, int is_lower,
                  const double* x, const double* d, const double* lb, const double* ub,
                  const int* type, int* q_out, int* q_idx_out, double* theta_out, double* delta_out,
                  int* num_candidates) {
    std::vector<double> alpha(alpha_in, alpha_in + n);
    double delta = std::fabs(delta_in);
    const int sgn = is_lower ? -1 : 1;
    if (is_lower) for (double& a : alpha) a = -a;
    std::vector<int> F;
    for (int i = 0; i < n; ++i) {
        bool cond = false;
        const double a = alpha[i];
        const int j = nonbasis[i];
        if (a > EPS_A) cond = std::fabs(x[j] - lb[j]) < EPS_Z && (type[j] == LOWER || type[j] == BOXED);
        else if (a < -EPS_A) cond = std::fabs(x[j] - ub[j]) < EPS_Z && (type[j] == UPPER || type[j] == BOXED);
        else cond = type[j] == FREE;
        if (cond) F.push_back(i);
    }
    *num_candidates = (int)F.size();
    int q = -1, q_idx = -1;
    auto scan = [&]() {
        q = -1; q_idx = -1;
        double theta = INF;
        for (int i : F) {
            const int j = nonbasis[i];
            const double tt = d[j] / alpha[i];
            if (tt < theta) { theta = tt; q = j; q_idx = i; }
            else if (q_idx >= 0 && std::fabs(tt - theta) < EPS_Z) {
                if (std::fabs(alpha[i]) > std::fabs(alpha[q_idx])) { theta = tt; q = j; q_idx = i; }
            }
        }
    };
    while (!F.empty()) {
        scan();
        if (q < 0) break;
        if (type[q] == BOXED) {
            if (delta - (ub[q] - lb[q]) * std::fabs(alpha[q_idx]) <= 0) break;
            delta -= (ub[q] - lb[q]) * std::fabs(alpha[q_idx]);
            F.erase(std::remove(F.begin(), F.end(), q_idx), F.end());
        } else break;
    }
    *q_out = q; *q_idx_out = q_idx;
    if (q >= 0) {
        *theta_out = d[q] / alpha_in[q_idx];
    } else {
        *theta_out = 0;
    }
    *delta_out = sgn * delta;
    return 0;
}

int or_pivot_row(int m, int n, const int* csc_ptr, const int* csc_row, const double* csc_val,
                 const int* nonbasis, const double* rho, double* alpha) {
    (void)m;
    for (int i = 0; i < n; ++i) {
        const int j = nonbasis[i];
        double acc = 0.0;
        if (j < n) {
            for (int e = csc_ptr[j]; e < csc_ptr[j + 1]; ++e) acc += csc_val[e] * rho[csc_row[e]] * 1.0;
        } else {
            acc += 1.0 * rho[j - n] * 1.0;
        }
        alpha[i] = acc;
    }
    return 0;
}

int or_pfi_apply(int m, int T, const double* etav, const int* pos, const double* rhs, double* sol,
                 int transpose) {
    std::vector<double> s(rhs, rhs + m);
    if (!transpose) {
        for (int t = 0; t < T; ++t) {
            const int kk = pos[t]; const double* ev = etav + (size_t)t * m;
            const double sk = s[kk];
            for (int i = 0; i < m; ++i) s[i] = s[i] + sk * ev[i];
            s[kk] = sk * ev[kk];
        }
    } else {
        for (int t = T - 1; t >= 0; --t) {
            const int kk = pos[t]; const double* ev = etav + (size_t)t * m;
            double acc = 0.0;
            for (int i = 0; i < m; ++i) acc += ev[i] * s[i];
            s[kk] = acc;
        }
    }
    std::memcpy(sol, s.data(), sizeof(double) * m);
    return 0;
}

int or_dense_solve(int n, const int* csr_ptr, const int* csr_col, const double* csr_val,
                   const double* rhs, double* sol, int transpose) {
    std::vector<double> A((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i)
        for (int e = csr_ptr[i]; e < csr_ptr[i + 1]; ++e) A[(size_t)i * n + csr_col[e]] = csr_val[e];
    if (transpose)
        for (int i = 0; i < n; ++i) for (int j = i + 1; j < n; ++j) std::swap(A[(size_t)i * n + j], A[(size_t)j * n + i]);
    std::vector<double> b(rhs, rhs + n);
    for (int c = 0; c < n; ++c) {
        int pr = c; double best = std::fabs(A[(size_t)c * n + c]);
        for (int r = c + 1; r < n; ++r) if (std::fabs(A[(size_t)r * n + c]) > best) { best = std::fabs(A[(size_t)r * n + c]); pr = r; }
        if (!(best > 0)) return -5;
        if (pr != c) { for (int j = 0; j < n; ++j) std::swap(A[(size_t)c * n + j], A[(size_t)pr * n + j]); std::swap(b[c], b[pr]); }
        for (int r = c + 1; r < n; ++r) {
            const double l = A[(size_t)r * n + c] / A[(size_t)c * n + c];
            for (int j = c; j < n; ++j) A[(size_t)r * n + j] -= l * A[(size_t)c * n + j];
            b[r] -= l * b[c];
        }
    }
    for (int r = n - 1; r >= 0; --r) {
        double s = b[r];
        for (int j = r + 1; j < n; ++j) s -= A[(size_t)r * n + j] * sol[j];
        sol[r] = s / A[(size_t)r * n + r];
    }
    return 0;
}

}  // extern "C"
