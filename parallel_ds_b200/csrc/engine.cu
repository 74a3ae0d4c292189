// Host driver of the B200 dual simplex engine and the ds_* C ABI.
//
// The control flow restates CudaDualSimplex / BaseDualSimplex of
// veret-v/parallel_ds (src/gpu/cudaDualSimplex.cpp, src/common/baseDualSimplex.tpp);
// every numeric step of an iteration runs on the device.  Phase 2 runs as a
// CUDA graph of one iteration launched back to back; the host synchronises
// only every few iterations (or when a kernel raises an event) and then
// handles the event exactly where the reference's loop would.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <stdexcept>
#include <string>
#include <unordered_set>
#include <vector>

#include "../../include/ds_api.h"
#include "engine.cuh"
#include "kernels.cuh"
#include "mlp.cuh"

namespace ds {

struct CudaError : std::runtime_error {
    int code;
    CudaError(const std::string& s, int c) : std::runtime_error(s), code(c) {}
};

#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            throw CudaError(std::string(#call) + ": " + cudaGetErrorString(e_), DS_ERR_CUDA); \
    } while (0)

constexpr double PERTURB_RATIO = 0.25;
constexpr double PSI = 1e-5;
constexpr double EPS_COSTS = 1e-8;
constexpr double INF_OBJ = 1e25;
constexpr int BATCH_ITERS = 32;

template <typename T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    void alloc(size_t count) {
        free();
        if (count == 0) count = 1;
        CK(cudaMalloc(&p, count * sizeof(T)));
        n = count;
    }
    void ensure(size_t count) { if (count > n) alloc(count); }
    void free() { if (p) cudaFree(p); p = nullptr; n = 0; }
    ~DBuf() { free(); }
};

struct Engine {
    ds_options opt;
    std::string err;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    bool loaded = false;

    // host copy of the LP (computational form: N = n + m, slacks implicit in A)
    int m = 0, n = 0, N = 0;
    std::vector<int> h_cptr, h_crow, h_rptr, h_rcol;
    std::vector<double> h_cval, h_rval, h_lb, h_ub, h_cost, h_cost_orig;
    std::vector<unsigned char> h_type;

    // device buffers
    DBuf<int> d_cptr, d_crow, d_rptr, d_rcol;
    DBuf<double> d_cval, d_rval, d_lb, d_ub, d_cost;
    DBuf<unsigned char> d_type, d_blocked, d_cand, d_flip;
    DBuf<double> d_x, d_d, d_beta, d_f;
    DBuf<int> d_basis, d_nonbasis, d_var_pos;
    DBuf<int> d_s_pos, d_s_var, d_rp_row, d_pos_kidx, d_row_slackpos, d_row_kidx;
    DBuf<int> d_cpl_ptr, d_cpl_col;
    DBuf<double> d_cpl_val, d_Kinv, d_S, d_Pan, d_Wk, d_Winv;
    DBuf<int> d_rowpiv, d_piv_rows, d_ferr;
    DBuf<double> d_eta, d_Mtri;
    DBuf<int> d_eta_pos, d_ybt_pos;
    DBuf<double> d_rho, d_alpha, d_theta, d_ybt, d_btr_rhs, d_aq, d_cc, d_alpha_q, d_tau, d_dxb;
    DBuf<double> d_y0[MAX_FTRAN_RHS];
    DBuf<double> d_part, d_seta, d_red;
    DBuf<int> d_redi, d_flip_list, d_trace;
    DBuf<double> d_trace_d;
    DBuf<unsigned> d_tile_tickets;
    DBuf<double> d_tmp_rows, d_tmp_rows2, d_tmp_pos, d_tmp_pos2, d_h;
    DBuf<Ctl> d_ctl;
    DBuf<float> d_feat, d_score;
    DBuf<int> d_row_cnt;

    Ctl* hc = nullptr;          // pinned host mirror of Ctl
    Dev D{};
    cudaGraphExec_t gexec = nullptr;
    int cap = 0;
    int k = 0;
    size_t k_alloc = 0;

    // solver state kept on the host
    int status = DS_STATUS_UNSOLVED;
    bool perturbed = false;
    std::mt19937 gen;
    int trace_cap = 0;
    std::vector<int> trace_pq;
    std::vector<double> trace_td;
    ds_stats st{};
    double objective = 0.0;
    std::vector<double> x_out, d_out;
    std::vector<int> basis_out;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, evr0 = nullptr, evr1 = nullptr;
    MlpModel* mlp = nullptr;    // learned pricing (not owned)

    // --------------------------------------------------------------- setup
    explicit Engine(const ds_options& o) : opt(o) {
        CK(cudaSetDevice(opt.device));
        if (opt.stream) stream = (cudaStream_t)opt.stream;
        else { CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking)); own_stream = true; }
        CK(cudaMallocHost(&hc, sizeof(Ctl)));
        CK(cudaEventCreate(&ev0)); CK(cudaEventCreate(&ev1));
        CK(cudaEventCreate(&evr0)); CK(cudaEventCreate(&evr1));
    }
    ~Engine() {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (hc) cudaFreeHost(hc);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (evr0) cudaEventDestroy(evr0);
        if (evr1) cudaEventDestroy(evr1);
        if (own_stream && stream) cudaStreamDestroy(stream);
    }

    template <typename T>
    void up(DBuf<T>& b, const std::vector<T>& v) {
        b.alloc(v.size());
        if (!v.empty()) CK(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, stream));
    }

    void load(int m_, int n_, const int* row_ptr, const int* col_idx, const double* val, const double* c,
              const int* col_type, const double* col_lb, const double* col_ub, const int* row_type,
              const double* row_lb, const double* row_ub) {
        m = m_; n = n_; N = n + m;
        const int nnz = row_ptr[m];
        h_rptr.assign(row_ptr, row_ptr + m + 1);
        h_rcol.assign(col_idx, col_idx + nnz);
        h_rval.assign(val, val + nnz);
        // structural CSC by walking rows in order (rows ascending in each column),
        // Matrix::genSparseReprs (matrix.cpp:99-146)
        h_cptr.assign(n + 1, 0);
        for (int e = 0; e < nnz; ++e) {
            if (col_idx[e] < 0 || col_idx[e] >= n) throw CudaError("column index out of range", DS_ERR_ARG);
            h_cptr[col_idx[e] + 1]++;
        }
        for (int j = 0; j < n; ++j) h_cptr[j + 1] += h_cptr[j];
        h_crow.resize(nnz); h_cval.resize(nnz);
        std::vector<int> cur(h_cptr.begin(), h_cptr.end() - 1);
        for (int i = 0; i < m; ++i)
            for (int e = row_ptr[i]; e < row_ptr[i + 1]; ++e) { const int p = cur[col_idx[e]]++; h_crow[p] = i; h_cval[p] = val[e]; }
        // bounds, types, costs: transformToComputeForm (problem.tpp:176-226)
        h_lb.resize(N); h_ub.resize(N); h_cost.resize(N); h_type.resize(N);
        for (int j = 0; j < n; ++j) { h_lb[j] = col_lb[j]; h_ub[j] = col_ub[j]; h_cost[j] = c[j]; h_type[j] = (unsigned char)col_type[j]; }
        for (int i = 0; i < m; ++i) {
            h_ub[n + i] = -row_lb[i];
            h_lb[n + i] = -row_ub[i];
            h_cost[n + i] = 0;
            unsigned char t;
            switch (row_type[i]) {
                case DS_FIXED: t = FIXED; break;
                case DS_BOXED: t = BOXED; break;
                case DS_LOWER: t = UPPER; break;
                case DS_UPPER: t = LOWER; break;
                default: t = FREE; break;
            }
            h_type[n + i] = t;
        }
        h_cost_orig = h_cost;
        up(d_rptr, h_rptr); up(d_rcol, h_rcol); up(d_rval, h_rval);
        up(d_cptr, h_cptr); up(d_crow, h_crow); up(d_cval, h_cval);
        up(d_lb, h_lb); up(d_ub, h_ub); up(d_cost, h_cost); up(d_type, h_type);
        // iteration state
        d_x.alloc(N); d_d.alloc(N); d_beta.alloc(m); d_f.alloc(m);
        d_basis.alloc(m); d_nonbasis.alloc(n); d_var_pos.alloc(N); d_blocked.alloc(N);
        d_s_pos.alloc(m); d_s_var.alloc(m); d_rp_row.alloc(m); d_pos_kidx.alloc(m);
        d_row_slackpos.alloc(m); d_row_kidx.alloc(m);
        d_cpl_ptr.alloc(m + 1); d_cpl_col.alloc(std::max(nnz, 1)); d_cpl_val.alloc(std::max(nnz, 1));
        cap = std::min(std::max(opt.refactor_interval, 1), 240) + 5;
        d_eta.alloc((size_t)cap * m); d_Mtri.alloc((size_t)cap * cap); d_eta_pos.alloc(cap); d_ybt_pos.alloc(cap + 1);
        d_rho.alloc(m); d_alpha.alloc(n); d_theta.alloc(n); d_cand.alloc(n); d_ybt.alloc(m);
        d_btr_rhs.alloc(m); d_aq.alloc(m); d_cc.alloc(m); d_alpha_q.alloc(m); d_tau.alloc(m); d_dxb.alloc(m);
        for (auto& b : d_y0) b.alloc(m);
        d_seta.alloc((size_t)MAX_FTRAN_RHS * cap);
        const int nb = std::max((m + 255) / 256, (n + 255) / 256) + 8;
        d_red.alloc(2 * nb); d_redi.alloc(2 * nb);
        d_flip.alloc(n); d_flip_list.alloc(n);
        d_tmp_rows.alloc(m); d_tmp_rows2.alloc(m); d_tmp_pos.alloc(m); d_tmp_pos2.alloc(m); d_h.alloc(cap);
        d_ctl.alloc(1);
        d_Winv.alloc(16 * 16); d_ferr.alloc(1);
        d_trace.alloc(2); d_trace_d.alloc(2);
        d_feat.alloc((size_t)m * 12); d_score.alloc(m);
        std::vector<int> rc(m);
        for (int i = 0; i < m; ++i) rc[i] = h_rptr[i + 1] - h_rptr[i];
        up(d_row_cnt, rc);
        CK(cudaMemsetAsync(d_ybt.p, 0, sizeof(double) * m, stream));
        CK(cudaMemsetAsync(d_aq.p, 0, sizeof(double) * m, stream));
        CK(cudaMemsetAsync(d_Mtri.p, 0, sizeof(double) * cap * cap, stream));
        CK(cudaStreamSynchronize(stream));
        loaded = true;
        status = DS_STATUS_UNSOLVED;
    }

    void sync_dev() {
        D.m = m; D.n = n; D.N = N; D.cap = cap; D.k = k;
        D.cptr = d_cptr.p; D.crow = d_crow.p; D.cval = d_cval.p;
        D.rptr = d_rptr.p; D.rcol = d_rcol.p; D.rval = d_rval.p;
        D.lb = d_lb.p; D.ub = d_ub.p; D.type = d_type.p; D.cost = d_cost.p;
        D.x = d_x.p; D.d = d_d.p; D.beta = d_beta.p; D.f = d_f.p;
        D.basis = d_basis.p; D.nonbasis = d_nonbasis.p; D.var_pos = d_var_pos.p; D.blocked = d_blocked.p;
        D.s_pos = d_s_pos.p; D.s_var = d_s_var.p; D.rp_row = d_rp_row.p; D.pos_kidx = d_pos_kidx.p;
        D.row_slackpos = d_row_slackpos.p;
        D.cpl_ptr = d_cpl_ptr.p; D.cpl_col = d_cpl_col.p; D.cpl_val = d_cpl_val.p;
        D.Kinv = d_Kinv.p;
        D.eta = d_eta.p; D.eta_pos = d_eta_pos.p; D.Mtri = d_Mtri.p;
        D.rho = d_rho.p; D.alpha = d_alpha.p; D.theta_arr = d_theta.p; D.cand = d_cand.p;
        D.ybt = d_ybt.p; D.ybt_pos = d_ybt_pos.p; D.btr_rhs = d_btr_rhs.p;
        D.aq_dense = d_aq.p; D.cc = d_cc.p; D.alpha_q = d_alpha_q.p; D.tau = d_tau.p; D.dxb = d_dxb.p;
        for (int r = 0; r < MAX_FTRAN_RHS; ++r) D.y0[r] = d_y0[r].p;
        D.frhs[0] = d_aq.p; D.frhs[1] = d_rho.p; D.frhs[2] = d_cc.p;
        D.fout[0] = d_alpha_q.p; D.fout[1] = d_tau.p; D.fout[2] = d_dxb.p;
        D.ftr_part = d_part.p; D.s_eta = d_seta.p; D.red = d_red.p; D.redi = d_redi.p;
        D.flip = d_flip.p; D.flip_list = d_flip_list.p;
        D.trace = d_trace.p; D.trace_d = d_trace_d.p;
        D.mlp_w = nullptr; D.feat = d_feat.p; D.score = d_score.p; D.feat_row_cnt = d_row_cnt.p;
        D.ctl = d_ctl.p;
        D.tile_tickets = d_tile_tickets.p;
    }

    // Ctl round trips (the host mirror is authoritative only right after pull()).
    void pull() {
        CK(cudaMemcpyAsync(hc, d_ctl.p, sizeof(Ctl), cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
    }
    void push() {
        CK(cudaMemcpyAsync(d_ctl.p, hc, sizeof(Ctl), cudaMemcpyHostToDevice, stream));
        CK(cudaStreamSynchronize(stream));   // hc may be written again right after
    }
    void clear_event() { hc->event = EV_NONE; hc->halt = 0; hc->event_stage = 0; }

    // ------------------------------------------------------- refactorisation
    // reFactorize (cudaDualSimplex.cpp:229-238): eta file reset, B0 <- A[:, basis],
    // factorisation of the structural block.
    void refactor() {
        auto t0 = std::chrono::steady_clock::now();
        pull();
        std::vector<int> basis(m);
        CK(cudaMemcpyAsync(basis.data(), d_basis.p, sizeof(int) * m, cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        std::vector<int> s_pos, s_var, rp_row, row_slackpos(m, -1), pos_kidx(m, -1), row_kidx(m, -1), kcol(n, -1);
        for (int i = 0; i < m; ++i) {
            const int v = basis[i];
            if (v < 0 || v >= N) throw CudaError("corrupt basis", DS_ERR_NUMERIC);
            if (v < n) { pos_kidx[i] = (int)s_pos.size(); kcol[v] = (int)s_pos.size(); s_pos.push_back(i); s_var.push_back(v); }
            else row_slackpos[v - n] = i;
        }
        for (int r = 0; r < m; ++r) if (row_slackpos[r] < 0) { row_kidx[r] = (int)rp_row.size(); rp_row.push_back(r); }
        k = (int)s_pos.size();
        if ((int)rp_row.size() != k) throw CudaError("basis is structurally singular", DS_ERR_NUMERIC);
        // coupling rows: A[r, S] for rows r whose slack is basic, CSR column order
        std::vector<int> cptr(m + 1, 0), ccol; std::vector<double> cval;
        for (int r = 0; r < m; ++r) {
            if (row_slackpos[r] >= 0)
                for (int e = h_rptr[r]; e < h_rptr[r + 1]; ++e) {
                    const int j = kcol[h_rcol[e]];
                    if (j >= 0) { ccol.push_back(j); cval.push_back(h_rval[e]); }
                }
            cptr[r + 1] = (int)ccol.size();
        }
        auto put = [&](DBuf<int>& b, const std::vector<int>& v) {
            if (!v.empty()) CK(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(int), cudaMemcpyHostToDevice, stream));
        };
        put(d_s_pos, s_pos); put(d_s_var, s_var); put(d_rp_row, rp_row);
        put(d_row_slackpos, row_slackpos); put(d_pos_kidx, pos_kidx); put(d_row_kidx, row_kidx);
        put(d_cpl_ptr, cptr); put(d_cpl_col, ccol);
        if (!cval.empty()) CK(cudaMemcpyAsync(d_cpl_val.p, cval.data(), cval.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
        const size_t kk = (size_t)std::max(k, 1) * std::max(k, 1);
        if (kk > k_alloc) {
            d_Kinv.alloc(kk); d_S.alloc(kk); k_alloc = kk;
        }
        d_Pan.ensure((size_t)std::max(k, 1) * 16); d_Wk.ensure((size_t)std::max(k, 1) * 16);
        d_rowpiv.ensure(std::max(k, 1)); d_piv_rows.ensure(std::max(k, 1));
        // FTRAN launch geometry for this k
        const int tile = 256;
        const int ntile = std::max(1, (k + tile - 1) / tile);
        int chunk = std::max(64, (k + std::max(1, 296 / ntile) - 1) / std::max(1, 296 / ntile));
        const int nchunk = std::max(1, (k + chunk - 1) / chunk);
        D.ftr_tile = tile; D.ftr_chunk = chunk; D.ftr_ntile = ntile; D.ftr_nchunk = nchunk;
        d_part.ensure((size_t)nchunk * MAX_FTRAN_RHS * std::max(k, 1));
        d_tile_tickets.ensure(ntile);
        CK(cudaMemsetAsync(d_tile_tickets.p, 0, sizeof(unsigned) * ntile, stream));
        sync_dev();
        FactorBufs F{d_S.p, d_Pan.p, d_Wk.p, d_rowpiv.p, d_piv_rows.p, d_Winv.p, d_ferr.p, d_s_var.p, d_row_kidx.p};
        CK(cudaEventRecord(evr0, stream));
        CK(factor_bump(F, D, k, stream));
        CK(cudaEventRecord(evr1, stream));
        int ferr = 0;
        CK(cudaMemcpyAsync(&ferr, d_ferr.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        float ms = 0; cudaEventElapsedTime(&ms, evr0, evr1);
        st.refactor_ms += ms;
        if (k > 0 && ferr) throw CudaError("singular basis in refactorisation", DS_ERR_NUMERIC);
        hc->T = 0;
        hc->k = k;
        push();
        st.refactors++;
        st.bump_size = k;
        invalidate_graph();
        (void)t0;
    }

    void invalidate_graph() {
        if (gexec) { cudaGraphExecDestroy(gexec); gexec = nullptr; }
    }
    void ensure_graph() {
        if (gexec) return;
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t le = launch_iteration(D, stream);
        cudaError_t ce = cudaStreamEndCapture(stream, &g);
        CK(le); CK(ce);
        CK(cudaGraphInstantiate(&gexec, g, 0));
        cudaGraphDestroy(g);
    }

    // -------------------------------------------------------------- solves
    // FTRAN of one dense row vector: out = B^-1 rhs (solveLinSys, transpose=false)
    void ftran1(const double* rhs, double* out) {
        Dev E = D;
        E.frhs[0] = rhs; E.fout[0] = out;
        CK(launch_ftran(E, 1, 0, 1, stream));
    }
    void ftran2(const double* r0, double* o0, const double* r1, double* o1) {
        Dev E = D;
        E.frhs[0] = r0; E.fout[0] = o0; E.frhs[1] = r1; E.fout[1] = o1;
        CK(launch_ftran(E, 2, 0, 1, stream));
    }
    // BTRAN of a dense position vector: y = B^-T c (rows)
    void btran_dense(const double* c0, double* y) {
        CK(launch_btran_dense_eta(D, c0, d_h.p, hc->T, stream));
        CK(launch_btran_b0(D, y, 1, stream));
    }

    // initReducedCosts (cudaDualSimplex.cpp:186-209)
    void init_reduced_costs() {
        CK(launch_gather_basic_cost(D, d_tmp_pos.p, stream));
        btran_dense(d_tmp_pos.p, d_tmp_rows2.p);
        CK(launch_reduced_costs(D, d_tmp_rows2.p, stream));
    }
    // dualSimplexInit (cudaDualSimplex.cpp:312-336)
    void dual_simplex_init() {
        CK(launch_set_primal_vars(D, stream));
        CK(launch_xb_rhs(D, d_tmp_rows.p, stream));
        ftran1(d_tmp_rows.p, d_tmp_pos2.p);
        CK(launch_scatter_basic(D, d_tmp_pos2.p, d_x.p, stream));
        init_reduced_costs();
        CK(launch_dot_cost_x(D, &d_ctl.p->obj, stream));
        pull();
    }
    // initBetaWeights (tpp:34-70)
    void init_beta(bool ibasis) {
        if (ibasis) {
            std::vector<double> ones(m, 1.0);
            CK(cudaMemcpyAsync(d_beta.p, ones.data(), sizeof(double) * m, cudaMemcpyHostToDevice, stream));
            CK(cudaStreamSynchronize(stream));
            return;
        }
        for (int i = 0; i < m; ++i) {
            CK(launch_btran_unit(D, i, stream));
            CK(launch_btran_b0(D, d_tmp_rows.p, 1, stream));
            CK(launch_norm2(d_tmp_rows.p, m, d_beta.p + i, stream));
        }
        pull();
    }
    // checkPerturbNeed (tpp:223-234) with std::unique's compare-to-kept semantics
    bool perturb_needed() const {
        std::vector<double> c(h_cost);
        std::sort(c.begin(), c.end());
        int uniq = c.empty() ? 0 : 1;
        double last = c.empty() ? 0 : c[0];
        for (size_t i = 1; i < c.size(); ++i) if (!(std::fabs(last - c[i]) < EPS_COSTS)) { last = c[i]; ++uniq; }
        return uniq < PERTURB_RATIO * (double)N;
    }
    // perturbCosts (tpp:238-275): seeded generator in place of std::random_device
    void perturb() {
        std::uniform_real_distribution<> dist(0.0, 1.0);
        double mean = 0; for (double v : h_cost) mean += v; mean /= (double)N;
        const double min_p = std::min(1e-2 * EPS_D, PSI);
        const double max_p = std::max(1e+3 * EPS_D, PSI * 10 * mean);
        static const double w[10] = {0.01, 0.1, 1, 2, 5, 10, 20, 30, 40, 100};
        for (int i = 0; i < N; ++i) {
            const double mag = 100 * EPS_D + PSI * h_cost[i];
            double pert;
            if (h_type[i] != LOWER && h_type[i] != FREE) pert = -0.5 * mag * (1 + dist(gen));
            pert = 0.5 * mag * (1 + dist(gen));
            const int nz = (i < n) ? (h_cptr[i + 1] - h_cptr[i]) : 1;
            const int kk = (nz > 10) ? 9 : (nz == 0 ? 0 : nz - 1);
            pert = w[kk] * pert;
            while (std::fabs(pert) > std::fabs(max_p) || std::fabs(pert) < std::fabs(min_p)) {
                if (std::fabs(pert) > std::fabs(max_p)) pert = 0.1 * pert;
                else if (std::fabs(pert) < std::fabs(min_p)) pert = 10 * pert;
            }
            h_cost[i] += pert;
        }
        perturbed = true;
        st.perturbed = 1;
        CK(cudaMemcpyAsync(d_cost.p, h_cost.data(), sizeof(double) * N, cudaMemcpyHostToDevice, stream));
        pull();
        hc->perturbed = 1;
        push();
    }
    bool dual_feasible() {
        pull();
        hc->dual_infeas = 0;
        push();
        CK(launch_dual_check(D, stream));
        pull();
        return hc->dual_infeas == 0;
    }
    void tick_host() {
        if (hc->iteration > hc->max_iter) { status = DS_STATUS_ITER_LIMIT; throw CudaError("iteration limit", 0); }
    }

    // -------------------------------------------------------------- phase 1
    void phase1_init() {
        init_reduced_costs();
        CK(launch_phase1_init(D, d_tmp_rows.p, stream));
        ftran1(d_tmp_rows.p, d_f.p);
        pull();
    }
    // minimizeDualInfeasibility (tpp:799-934), one synchronised step per iteration
    int phase1() {
        pull();
        const int saved_cycle = hc->cycle;
        hc->phase = 1; hc->cycle = 0; push();
        phase1_init();
        bool blocked_any = false;
        CK(cudaMemsetAsync(d_blocked.p, 0, N, stream));
        int result = EV_P1_DONE;
        int pivots_at_nop = -1;
        while (true) {
            pull();
            hc->iteration += 1; st.phase1_iterations++;
            push();
            tick_host();
            if (!perturbed && hc->cycle > MAX_CYCLE) { perturb(); phase1_init(); }
            pull();
            if (hc->cycle > NEED_RESTART || hc->z_phase1 > INF_OBJ || std::isnan(hc->z_phase1)) phase1_init();
            if (hc->iteration % hc->R == 0) refactor();
            pull(); clear_event(); push();
            CK(launch_count_dual_inf(D, stream));
            CK(launch_body(D, ST_PRICING, stream));
            pull();
            const int ev = hc->event;
            if (ev == EV_P1_DONE || ev == EV_P1_DUALINF) { result = ev; break; }
            if (ev == EV_P1_RESTART) {
                // no leaving row with infeasibilities left, twice without a pivot:
                // dual infeasible (see the oracle; the reference restarts forever)
                if (!opt.strict_reference && !hc->p1_found && hc->p1_dinf > 0 && hc->z_phase1 < -EPS_A &&
                    pivots_at_nop == hc->pivots) { result = EV_P1_DUALINF; break; }
                if (!hc->p1_found) pivots_at_nop = hc->pivots;
                clear_event(); push();
                refactor(); phase1_init(); init_beta(false);
                if (blocked_any) { CK(cudaMemsetAsync(d_blocked.p, 0, N, stream)); blocked_any = false; }
                st.restarts++;
                continue;
            }
            if (ev == EV_P1_BLOCK) {
                const unsigned char one = 1;
                CK(cudaMemcpyAsync(d_blocked.p + hc->p, &one, 1, cudaMemcpyHostToDevice, stream));
                blocked_any = true;
                clear_event(); push();
                refactor(); phase1_init();
                st.restarts++;
                continue;
            }
            if (ev == EV_MISMATCH) { handle_mismatch(); pull(); }
            if (hc->event == EV_ETA_FULL) { clear_event(); push(); refactor(); pull(); }
            if (hc->event == EV_ERROR) throw CudaError("phase 1: no takeable ratio-test candidate", DS_ERR_NUMERIC);
            if (hc->event != EV_NONE) throw CudaError("phase 1: unexpected event", DS_ERR_NUMERIC);
            if (blocked_any) { CK(cudaMemsetAsync(d_blocked.p, 0, N, stream)); blocked_any = false; }
        }
        pull();
        clear_event();
        hc->phase = 2; hc->cycle = saved_cycle;
        push();
        return result;
    }

    // After FTRAN: refactor, then redo tau (and the BFRT FTRAN) with the new factor
    // and finish the iteration (cudaDualSimplex.cpp:555-560 then :595-623).
    void handle_mismatch() {
        pull();
        clear_event(); push();
        const int nr = hc->nrhs;
        refactor();
        if (nr > 2) ftran2(d_rho.p, d_tau.p, d_cc.p, d_dxb.p);
        else ftran1(d_rho.p, d_tau.p);
        CK(launch_update_forced(D, stream));
    }

    // -------------------------------------------------------------- phase 2
    // Launch graph iterations until an event is raised.
    int run_until_event() {
        while (true) {
            ensure_graph();
            const int it = hc->iteration;
            const int R = hc->R;
            int batch = R - (it % R);
            if (batch > BATCH_ITERS) batch = BATCH_ITERS;
            if (batch < 1) batch = 1;
            for (int b = 0; b < batch; ++b) CK(cudaGraphLaunch(gexec, stream));
            st.kernel_launches += batch * 13;
            pull();
            if (hc->halt) return hc->event;
        }
    }

    // remaining top-of-loop steps after a refactor at iteration it (reference order)
    void top_after_refactor() {
        pull();
        if (hc->iteration % NEED_RESTART == 0 && !dual_feasible()) {
            refactor(); phase1(); dual_simplex_init(); st.restarts++;
        }
        pull();
        if (!perturbed && hc->cycle > MAX_CYCLE) { perturb(); refactor(); dual_simplex_init(); }
    }

    // Run the rest of the current iteration from pricing on (after a top event).
    int run_body_once() {
        pull(); clear_event(); push();
        CK(launch_body(D, ST_PRICING, stream));
        pull();
        return hc->halt ? hc->event : EV_NONE;
    }

    // callDualSolver (cudaDualSimplex.cpp:396-655)
    bool phase2() {
        refactor();
        dual_simplex_init();
        pull();
        hc->cycle = 0; hc->unbound_checked = 0; clear_event();
        push();
        int pivots_at_nop = -1;
        int ev = run_until_event();
        while (true) {
            switch (ev) {
                case EV_NONE: ev = run_until_event(); continue;
                case EV_ITER_LIMIT: status = DS_STATUS_ITER_LIMIT; return false;
                case EV_REFACTOR_DUE:
                    clear_event(); push();
                    refactor(); top_after_refactor();
                    ev = run_body_once();
                    continue;
                case EV_DUALINF:
                    clear_event(); push();
                    refactor(); phase1(); dual_simplex_init(); st.restarts++;
                    pull();
                    if (!perturbed && hc->cycle > MAX_CYCLE) { perturb(); refactor(); dual_simplex_init(); }
                    ev = run_body_once();
                    continue;
                case EV_PERTURB:
                    clear_event(); push();
                    perturb(); refactor(); dual_simplex_init();
                    ev = run_body_once();
                    continue;
                case EV_OPTIMAL: status = DS_STATUS_OPTIMAL; return true;
                case EV_NO_P: {
                    pull();
                    if (!opt.strict_reference && pivots_at_nop == hc->pivots) { status = DS_STATUS_OPTIMAL; return true; }
                    pivots_at_nop = hc->pivots;
                    clear_event(); push();
                    refactor(); init_beta(false); phase1(); dual_simplex_init(); st.restarts++;
                    ev = run_until_event();
                    continue;
                }
                case EV_UNBOUNDED: {
                    pull();
                    if (hc->unbound_checked) { status = DS_STATUS_PRIMAL_INFEASIBLE; return false; }
                    hc->unbound_checked = 1; clear_event(); push();
                    refactor(); init_beta(false); phase1(); dual_simplex_init(); st.restarts++;
                    pull(); hc->unbound_checked = 1; push();
                    ev = run_until_event();
                    continue;
                }
                case EV_MISMATCH:
                    handle_mismatch();
                    pull();
                    if (hc->halt && hc->event == EV_ETA_FULL) { clear_event(); push(); refactor(); }
                    else if (hc->halt) { ev = hc->event; continue; }
                    ev = run_until_event();
                    continue;
                case EV_ETA_FULL:
                    clear_event(); push(); refactor();
                    ev = run_until_event();
                    continue;
                case EV_ERROR:
                default:
                    throw CudaError("numerical failure in the iteration (event " + std::to_string(ev) + ")", DS_ERR_NUMERIC);
            }
        }
    }

    // presolve + solve + postProcess (tpp:5-30, 123-180) with the cleanup guard
    void solve() {
        if (!loaded) throw CudaError("solve before load", DS_ERR_STATE);
        st = ds_stats{};
        status = DS_STATUS_UNSOLVED;
        perturbed = false;
        h_cost = h_cost_orig;
        gen.seed((unsigned)(opt.seed & 0xffffffffu) ^ (unsigned)(opt.seed >> 32));
        CK(cudaMemcpyAsync(d_cost.p, h_cost.data(), sizeof(double) * N, cudaMemcpyHostToDevice, stream));
        // slack basis (tpp:184-204)
        std::vector<int> basis(m), nonbasis(n), var_pos(N);
        for (int i = 0; i < n; ++i) { nonbasis[i] = i; var_pos[i] = -(i + 1); }
        for (int i = 0; i < m; ++i) { basis[i] = n + i; var_pos[n + i] = i; }
        CK(cudaMemcpyAsync(d_basis.p, basis.data(), sizeof(int) * m, cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(d_nonbasis.p, nonbasis.data(), sizeof(int) * n, cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(d_var_pos.p, var_pos.data(), sizeof(int) * N, cudaMemcpyHostToDevice, stream));
        CK(cudaMemsetAsync(d_x.p, 0, sizeof(double) * N, stream));
        CK(cudaMemsetAsync(d_d.p, 0, sizeof(double) * N, stream));
        CK(cudaMemsetAsync(d_blocked.p, 0, N, stream));
        d_trace.alloc(2 * std::max(trace_cap, 1)); d_trace_d.alloc(2 * std::max(trace_cap, 1));
        std::memset(hc, 0, sizeof(Ctl));
        hc->max_iter = opt.max_iterations; hc->R = std::min(std::max(opt.refactor_interval, 1), cap - 5);
        hc->phase = 2; hc->prev_q = -1; hc->ybt_n = -1; hc->trace_cap = trace_cap;
        sync_dev();
        push();
        CK(cudaEventRecord(ev0, stream));
        try {
            refactor();                      // initDualSimplex (cudaDualSimplex.cpp:20-81)
            if (perturb_needed()) perturb();  // presolve (tpp:5-30)
            init_beta(true);
            const int p1 = phase1();
            if (p1 == EV_P1_DUALINF) {
                status = DS_STATUS_DUAL_INFEASIBLE;
            } else {
                CK(launch_set_primal_vars(D, stream));
                bool ok = phase2();
                for (int round = 0; round < 3 && perturbed; ++round) {
                    h_cost = h_cost_orig;
                    CK(cudaMemcpyAsync(d_cost.p, h_cost.data(), sizeof(double) * N, cudaMemcpyHostToDevice, stream));
                    dual_simplex_init();
                    if (!ok || opt.strict_reference || dual_feasible()) break;
                    status = DS_STATUS_UNSOLVED;
                    refactor();
                    if (phase1() == EV_P1_DUALINF) { status = DS_STATUS_DUAL_INFEASIBLE; break; }
                    CK(launch_set_primal_vars(D, stream));
                    ok = phase2();
                }
            }
        } catch (const CudaError& e) {
            if (e.code == 0) {
                // iteration limit: state is consistent, fall through to the results
            } else {
                status = DS_STATUS_ERROR;
                err = e.what();
                if (e.code == DS_ERR_CUDA) throw;
            }
        }
        CK(cudaEventRecord(ev1, stream));
        CK(cudaStreamSynchronize(stream));
        float ms = 0; cudaEventElapsedTime(&ms, ev0, ev1);
        st.solve_ms = ms;
        pull();
        st.iterations = hc->iteration;
        st.learned_used = hc->learned_used;
        st.learned_fallback = hc->learned_fallback;
        x_out.resize(N); d_out.resize(N); basis_out.resize(m);
        CK(cudaMemcpyAsync(x_out.data(), d_x.p, sizeof(double) * N, cudaMemcpyDeviceToHost, stream));
        CK(cudaMemcpyAsync(d_out.data(), d_d.p, sizeof(double) * N, cudaMemcpyDeviceToHost, stream));
        CK(cudaMemcpyAsync(basis_out.data(), d_basis.p, sizeof(int) * m, cudaMemcpyDeviceToHost, stream));
        const int tn = std::min(hc->trace_n, trace_cap);
        trace_pq.resize(2 * tn); trace_td.resize(2 * tn);
        if (tn > 0) {
            CK(cudaMemcpyAsync(trace_pq.data(), d_trace.p, sizeof(int) * 2 * tn, cudaMemcpyDeviceToHost, stream));
            CK(cudaMemcpyAsync(trace_td.data(), d_trace_d.p, sizeof(double) * 2 * tn, cudaMemcpyDeviceToHost, stream));
        }
        CK(cudaStreamSynchronize(stream));
        double z = 0;
        for (int j = 0; j < n; ++j) z += h_cost_orig[j] * x_out[j];
        objective = z;
    }
};

}  // namespace ds

// ======================================================================= C ABI
using ds::Engine;

struct ds_solver {
    Engine* e;
    std::string last_error;
};

static int fail(ds_solver* s, int code, const std::string& msg) {
    if (s) s->last_error = msg;
    return code;
}

#define GUARD(s, body)                                                        \
    try { body }                                                              \
    catch (const ds::CudaError& ex) { return fail(s, ex.code ? ex.code : DS_ERR_NUMERIC, ex.what()); } \
    catch (const std::exception& ex) { return fail(s, DS_ERR_ARG, ex.what()); }

extern "C" {

void ds_default_options(ds_options* o) {
    if (!o) return;
    o->refactor_interval = 100;
    o->max_iterations = 2000000;
    o->pricing = DS_PRICING_DSE;
    o->strict_reference = 0;
    o->seed = 12345;
    o->device = 0;
    o->stream = nullptr;
    o->learned_margin = 0.0;
    o->verbose = 0;
}

const char* ds_version(void) { return "ds_b200 1.0 (sm_100a)"; }

int ds_create(const ds_options* opts, ds_solver** out) {
    if (!out) return DS_ERR_ARG;
    *out = nullptr;
    ds_options o;
    ds_default_options(&o);
    if (opts) o = *opts;
    if (o.refactor_interval < 1 || o.refactor_interval > 240) return DS_ERR_ARG;
    auto* s = new ds_solver{nullptr, ""};
    try {
        s->e = new Engine(o);
    } catch (const std::exception& ex) {
        delete s;
        return DS_ERR_CUDA;
    }
    *out = s;
    return DS_OK;
}

int ds_destroy(ds_solver* s) {
    if (!s) return DS_ERR_ARG;
    delete s->e;
    delete s;
    return DS_OK;
}

static int check_lp_args(int m, int n, const int* row_ptr, const int* col_idx, const double* val,
                         const double* c) {
    if (m <= 0 || n <= 0 || !row_ptr || !c) return DS_ERR_ARG;
    if (row_ptr[0] != 0 || row_ptr[m] < 0) return DS_ERR_ARG;
    for (int i = 0; i < m; ++i) if (row_ptr[i + 1] < row_ptr[i]) return DS_ERR_ARG;
    if (row_ptr[m] > 0 && (!col_idx || !val)) return DS_ERR_ARG;
    if (m > n) return DS_ERR_SHAPE;   // Problem::checkConstraints (problem.tpp:230-239)
    return DS_OK;
}

int ds_load_typed(ds_solver* s, int m, int n, const int* row_ptr, const int* col_idx, const double* val,
                  const double* c, const int* col_type, const double* col_lb, const double* col_ub,
                  const int* row_type, const double* row_lb, const double* row_ub) {
    if (!s) return DS_ERR_ARG;
    int rc = check_lp_args(m, n, row_ptr, col_idx, val, c);
    if (rc) return fail(s, rc, rc == DS_ERR_SHAPE ? "Incorrect constraint size (m > n)" : "bad LP arguments");
    if (!col_type || !col_lb || !col_ub || !row_type || !row_lb || !row_ub) return fail(s, DS_ERR_ARG, "null bounds");
    for (int j = 0; j < n; ++j) if (col_type[j] < 0 || col_type[j] > 4) return fail(s, DS_ERR_ARG, "bad column type");
    for (int i = 0; i < m; ++i) if (row_type[i] < 0 || row_type[i] > 4) return fail(s, DS_ERR_ARG, "bad row type");
    GUARD(s, { s->e->load(m, n, row_ptr, col_idx, val, c, col_type, col_lb, col_ub, row_type, row_lb, row_ub); return DS_OK; })
}

static int bound_type(double lo, double hi) {
    const bool li = (lo > 1e100 || lo < -1e100), hi_inf = (hi > 1e100 || hi < -1e100);
    if (li && hi_inf) return DS_FREE;
    if (li) return DS_UPPER;
    if (hi_inf) return DS_LOWER;
    if (lo == hi) return DS_FIXED;
    return DS_BOXED;
}

int ds_load_csr(ds_solver* s, int m, int n, const int* row_ptr, const int* col_idx, const double* val,
                const double* c, const double* col_lb, const double* col_ub, const double* row_lb,
                const double* row_ub) {
    if (!s || !col_lb || !col_ub || !row_lb || !row_ub || m <= 0 || n <= 0) return DS_ERR_ARG;
    std::vector<int> ct(n), rt(m);
    for (int j = 0; j < n; ++j) ct[j] = bound_type(col_lb[j], col_ub[j]);
    for (int i = 0; i < m; ++i) rt[i] = bound_type(row_lb[i], row_ub[i]);
    return ds_load_typed(s, m, n, row_ptr, col_idx, val, c, ct.data(), col_lb, col_ub, rt.data(), row_lb, row_ub);
}

int ds_solve(ds_solver* s) {
    if (!s) return DS_ERR_ARG;
    GUARD(s, {
        s->e->solve();
        if (s->e->status == DS_STATUS_ERROR) return fail(s, DS_ERR_NUMERIC, s->e->err);
        return DS_OK;
    })
}

int ds_get_status(const ds_solver* s) { return s ? s->e->status : DS_STATUS_ERROR; }
double ds_get_objective(const ds_solver* s) { return s ? s->e->objective : NAN; }

int ds_get_primal(const ds_solver* s, double* x, double* slacks) {
    if (!s || !x) return DS_ERR_ARG;
    const Engine* e = s->e;
    if (e->x_out.empty()) return DS_ERR_STATE;
    std::memcpy(x, e->x_out.data(), sizeof(double) * e->n);
    if (slacks) std::memcpy(slacks, e->x_out.data() + e->n, sizeof(double) * e->m);
    return DS_OK;
}

int ds_get_dual(const ds_solver* s, double* y) {
    if (!s || !y) return DS_ERR_ARG;
    const Engine* e = s->e;
    if (e->d_out.empty()) return DS_ERR_STATE;
    for (int i = 0; i < e->m; ++i) y[i] = -e->d_out[e->n + i];
    return DS_OK;
}

int ds_get_reduced_costs(const ds_solver* s, double* d) {
    if (!s || !d) return DS_ERR_ARG;
    const Engine* e = s->e;
    if (e->d_out.empty()) return DS_ERR_STATE;
    std::memcpy(d, e->d_out.data(), sizeof(double) * e->n);
    return DS_OK;
}

int ds_get_iterations(const ds_solver* s) { return s ? s->e->st.iterations : -1; }

int ds_get_stats(const ds_solver* s, ds_stats* st) {
    if (!s || !st) return DS_ERR_ARG;
    *st = s->e->st;
    return DS_OK;
}

int ds_get_basis(const ds_solver* s, int* basis) {
    if (!s || !basis) return DS_ERR_ARG;
    if (s->e->basis_out.empty()) return DS_ERR_STATE;
    std::memcpy(basis, s->e->basis_out.data(), sizeof(int) * s->e->m);
    return DS_OK;
}

const char* ds_last_error(const ds_solver* s) { return s ? s->last_error.c_str() : "null handle"; }

int ds_set_trace(ds_solver* s, int cap) {
    if (!s || cap < 0) return DS_ERR_ARG;
    s->e->trace_cap = cap;
    return DS_OK;
}

int ds_get_trace(const ds_solver* s, int* p, int* q, double* theta, double* obj, int* count) {
    if (!s || !count) return DS_ERR_ARG;
    const Engine* e = s->e;
    const int tn = (int)e->trace_pq.size() / 2;
    for (int t = 0; t < tn; ++t) {
        if (p) p[t] = e->trace_pq[2 * t];
        if (q) q[t] = e->trace_pq[2 * t + 1];
        if (theta) theta[t] = e->trace_td[2 * t];
        if (obj) obj[t] = e->trace_td[2 * t + 1];
    }
    *count = tn;
    return DS_OK;
}

}  // extern "C"
