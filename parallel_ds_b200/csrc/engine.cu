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
#include <mutex>
#include <random>
#include <stdexcept>
#include <string>
#include <unordered_set>
#include <vector>

#include "../../include/ds_api.h"
#include "engine.cuh"
#include "host_util.cuh"
#include "kernels.cuh"
#include "mlp.cuh"
#include "pdhg.cuh"
#include "sparse_factor.cuh"

namespace ds {

constexpr double PERTURB_RATIO = 0.25;
constexpr double PSI = 1e-5;
constexpr double EPS_COSTS = 1e-8;
constexpr double INF_OBJ = 1e25;
// Iteration graphs enqueued per host synchronisation.  A batch never crosses
// the refactor boundary; an event raised earlier in the batch halts the
// iteration and the batch's remaining launches return at once (a few
// microseconds each), so long batches cost little and save host round trips.
constexpr int BATCH_ITERS = 100;
// Iterations per launch of the unrolled iteration graph: inside one graph the
// kernels of consecutive iterations are chained by programmatic dependencies,
// so the boundary between iterations costs no graph launch.
constexpr int GRAPH_UNROLL = 8;
// Dense mode: largest probe residual of B^-1 (relative to 1 + |B^-1 v|) at
// which the periodic rebuild is skipped.
constexpr double DENSE_PROBE_TOL = 1e-10;

// Blocks freed to the device's default memory pool stay cached for reuse
// (release threshold: unlimited) instead of going back to the driver at each
// synchronisation.  Once per device, per process.
static void keep_pool_memory(int dev) {
    static std::mutex mu;
    static std::vector<int> done;
    std::lock_guard<std::mutex> lk(mu);
    if (std::find(done.begin(), done.end(), dev) != done.end()) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    done.push_back(dev);
}

struct Engine {
    ds_options opt;
    std::string err;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    bool loaded = false;
    bool binv_valid = false;   // dense mode: B^-1 was built for this LP at least once

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
    DBuf<unsigned long long> d_probe;
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
    SparseLU sflu;                         // eta-file mode's sparse factor of B0
    SfInfo sfi;                            // its last factorisation
    DBuf<float> d_score, d_ftr_feat;
    // first-order warm-start evidence (pdhg.cu)
    DBuf<double> d_pd_c, d_pd_lo, d_pd_hi, d_pd_L, d_pd_U, d_pd_tau, d_pd_sigma;
    DBuf<double> d_pd_x, d_pd_xbar, d_pd_xsum, d_pd_y, d_pd_ysum;
    DBuf<float> d_pd_gap, d_pd_dual;
    // dense mode: explicit B^-1
    bool dense = false;
    DBuf<double> d_Binv, d_binv_part;
    DBuf<unsigned> d_binv_tickets;
    static constexpr int BINV_RC = 32;    // rows of B^-1 per chunk of the tiled kernels
    PdhgDev PD{};
    PdhgClusterGeom pd_geom{0, 0, 0, 0, 0, 0};
    cudaGraphExec_t pd_gexec = nullptr;
    static constexpr int PDHG_RESTART = 500;
    cudaEvent_t evp0 = nullptr, evp1 = nullptr;
    // The PDHG warm start runs on its own stream, overlapping the start of the
    // solve; the main stream waits for it (pd_done) only before the first
    // iteration the network prices (learn_start), so the pivot sequence does not
    // depend on timing.
    cudaStream_t pd_stream = nullptr;
    cudaEvent_t pd_done = nullptr, pd_go = nullptr;
    bool pd_pending = false;
    int learn_start = 0;
    DBuf<int> d_row_nnz, d_enter_cnt, d_entered_at, d_ftr_meta;

    Ctl* hc = nullptr;          // pinned host mirror of Ctl
    Dev D{};
    cudaGraphExec_t gexec = nullptr;     // one iteration
    cudaGraphExec_t gexec_u = nullptr;   // GRAPH_UNROLL iterations
    int cap = 0;
    int k = 0;

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
    int ftr_every = 0, ftr_cap = 0;   // feature trace settings
    int ftr_total = 0;                // candidates seen by the last traced solve
    std::vector<float> ftr_feat;      // kept records, sorted by (iteration, position)
    std::vector<int> ftr_meta;
    bool model_wait_timeout = false;  // a scoring launch gave up waiting on its MMAs
    long long graph_nodes = 0;  // kernel nodes in the iteration graph
    long long nnz_S = 0, nnz_cpl = 0;   // structural nonzeros in the basis / coupling rows
    // per-kernel profiling (ds_profile_solve)
    bool prof = false;
    double prof_us[S_NSTEPS] = {}, prof_bytes[S_NSTEPS] = {};
    long long prof_n[S_NSTEPS] = {};
    cudaEvent_t pev[2 * S_NSTEPS] = {};

    // --------------------------------------------------------------- setup
    explicit Engine(const ds_options& o) : opt(o) {
        CK(cudaSetDevice(opt.device));
        if (opt.stream) stream = (cudaStream_t)opt.stream;
        else { CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking)); own_stream = true; }
        CK(cudaMallocHost(&hc, sizeof(Ctl)));
        keep_pool_memory(opt.device);
        CK(cudaEventCreate(&ev0)); CK(cudaEventCreate(&ev1));
        CK(cudaEventCreate(&evp0)); CK(cudaEventCreate(&evp1));
        CK(cudaStreamCreateWithFlags(&pd_stream, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&pd_done, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&pd_go, cudaEventDisableTiming));
        CK(cudaEventCreate(&evr0)); CK(cudaEventCreate(&evr1));
    }
    ~Engine() {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (gexec_u) cudaGraphExecDestroy(gexec_u);
        if (hc) cudaFreeHost(hc);
        if (ev0) cudaEventDestroy(ev0);
        if (evp0) cudaEventDestroy(evp0);
        if (evp1) cudaEventDestroy(evp1);
        if (pd_done) cudaEventDestroy(pd_done);
        if (pd_go) cudaEventDestroy(pd_go);
        if (pd_stream) cudaStreamDestroy(pd_stream);
        if (pd_gexec) cudaGraphExecDestroy(pd_gexec);
        if (ev1) cudaEventDestroy(ev1);
        if (evr0) cudaEventDestroy(evr0);
        if (evr1) cudaEventDestroy(evr1);
        for (auto& e : pev) if (e) cudaEventDestroy(e);
        if (own_stream && stream) cudaStreamDestroy(stream);
    }

    template <typename T>
    void up(DBuf<T>& b, const std::vector<T>& v) {
        b.ensure(stream, v.size());
        if (!v.empty()) CK(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, stream));
    }

    void load(int m_, int n_, const int* row_ptr, const int* col_idx, const double* val, const double* c,
              const int* col_type, const double* col_lb, const double* col_ub, const int* row_type,
              const double* row_lb, const double* row_ub) {
        m = m_; n = n_; N = n + m;
        const int nnz = row_ptr[m];
        // non-finite input would poison every later step (the reference has no
        // check and iterates on NaN): matrix entries and costs must be finite,
        // bounds may be infinite but not NaN
        for (int e = 0; e < nnz; ++e)
            if (!std::isfinite(val[e])) throw CudaError("matrix entry is not finite", DS_ERR_ARG);
        for (int j = 0; j < n; ++j) {
            if (!std::isfinite(c[j])) throw CudaError("cost is not finite", DS_ERR_ARG);
            if (std::isnan(col_lb[j]) || std::isnan(col_ub[j])) throw CudaError("column bound is NaN", DS_ERR_ARG);
        }
        for (int i = 0; i < m; ++i)
            if (std::isnan(row_lb[i]) || std::isnan(row_ub[i])) throw CudaError("row bound is NaN", DS_ERR_ARG);
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
        setup_pdhg();
        up(d_rptr, h_rptr); up(d_rcol, h_rcol); up(d_rval, h_rval);
        up(d_cptr, h_cptr); up(d_crow, h_crow); up(d_cval, h_cval);
        up(d_lb, h_lb); up(d_ub, h_ub); up(d_cost, h_cost); up(d_type, h_type);
        // iteration state
        d_x.ensure(stream, N); d_d.ensure(stream, N); d_beta.ensure(stream, m); d_f.ensure(stream, m);
        d_basis.ensure(stream, m); d_nonbasis.ensure(stream, n); d_var_pos.ensure(stream, N); d_blocked.ensure(stream, N);
        d_s_pos.ensure(stream, m); d_s_var.ensure(stream, m); d_rp_row.ensure(stream, m); d_pos_kidx.ensure(stream, m);
        d_row_slackpos.ensure(stream, m); d_row_kidx.ensure(stream, m);
        d_cpl_ptr.ensure(stream, m + 1); d_cpl_col.ensure(stream, std::max(nnz, 1)); d_cpl_val.ensure(stream, std::max(nnz, 1));
        cap = std::min(std::max(opt.refactor_interval, 1), 200) + 5;
        CK(init_kernel_attributes(cap));
        d_eta.ensure(stream, (size_t)cap * m); d_Mtri.ensure(stream, (size_t)cap * cap); d_eta_pos.ensure(stream, cap); d_ybt_pos.ensure(stream, cap + 1);
        d_rho.ensure(stream, m); d_alpha.ensure(stream, n); d_theta.ensure(stream, n); d_cand.ensure(stream, n); d_ybt.ensure(stream, m);
        d_btr_rhs.ensure(stream, m); d_aq.ensure(stream, m); d_cc.ensure(stream, m); d_alpha_q.ensure(stream, m); d_tau.ensure(stream, m); d_dxb.ensure(stream, m);
        for (auto& b : d_y0) b.ensure(stream, m);
        d_seta.ensure(stream, (size_t)MAX_FTRAN_RHS * cap);
        // per-block partials: 256-wide grids over m or n, and the 16-CTA clusters
        const int nb = std::max(std::max((m + 255) / 256, (n + 255) / 256), 16) + 8;
        d_red.ensure(stream, 2 * nb); d_redi.ensure(stream, 4 * nb);
        d_flip.ensure(stream, n); d_flip_list.ensure(stream, n);
        d_tmp_rows.ensure(stream, m); d_tmp_rows2.ensure(stream, m); d_tmp_pos.ensure(stream, m); d_tmp_pos2.ensure(stream, m); d_h.ensure(stream, cap);
        d_ctl.ensure(stream, 1);
        d_Winv.ensure(stream, 16 * 16); d_ferr.ensure(stream, 1); d_probe.ensure(stream, 2);
        d_trace.ensure(stream, 2); d_trace_d.ensure(stream, 2);
        d_score.ensure(stream, m); d_enter_cnt.ensure(stream, N); d_entered_at.ensure(stream, N);
        dense = opt.dense_max_m > 0 && m <= opt.dense_max_m;
        if (dense) {
            const int chunks = (m + BINV_RC - 1) / BINV_RC;
            d_Binv.ensure(stream, (size_t)m * m);
            d_binv_part.ensure(stream, (size_t)chunks * m);
            // one ticket per 32-position slice (k_binv_update) covers the
            // 256-position tiles of k_dense_colsum too
            d_binv_tickets.ensure(stream, (size_t)(m + 31) / 32 + 1);
            CK(cudaMemsetAsync(d_binv_tickets.p, 0, sizeof(unsigned) * ((m + 31) / 32 + 1), stream));
        }
        std::vector<int> rc(m);
        for (int i = 0; i < m; ++i) rc[i] = h_rptr[i + 1] - h_rptr[i];
        up(d_row_nnz, rc);
        CK(cudaMemsetAsync(d_ybt.p, 0, sizeof(double) * m, stream));
        CK(cudaMemsetAsync(d_aq.p, 0, sizeof(double) * m, stream));
        CK(cudaMemsetAsync(d_Mtri.p, 0, sizeof(double) * cap * cap, stream));
        CK(cudaStreamSynchronize(stream));
        loaded = true;
        binv_valid = false;
        status = DS_STATUS_UNSOLVED;
    }

    // PDHG data of the loaded LP: bounds by variable type (FIXED pins both
    // sides to lb), row activity bounds from the slack s = -A x, step sizes.
    void setup_pdhg() {
        const double inf = INFINITY;
        auto lower_of = [&](int v) {
            const int t = h_type[v];
            return (t == FIXED || t == BOXED || t == LOWER) ? h_lb[v] : -inf;
        };
        auto upper_of = [&](int v) {
            const int t = h_type[v];
            return t == FIXED ? h_lb[v] : (t == BOXED || t == UPPER) ? h_ub[v] : inf;
        };
        std::vector<double> lo(n), hi(n), L(m), U(m), tau(n), sig(m), c(h_cost_orig.begin(), h_cost_orig.begin() + n);
        for (int j = 0; j < n; ++j) {
            lo[j] = lower_of(j); hi[j] = upper_of(j);
            double a = 0;
            for (int e = h_cptr[j]; e < h_cptr[j + 1]; ++e) a += std::fabs(h_cval[e]);
            tau[j] = a > 0 ? 1.0 / a : 1.0;
        }
        for (int i = 0; i < m; ++i) {
            L[i] = -upper_of(n + i); U[i] = -lower_of(n + i);
            double a = 0;
            for (int e = h_rptr[i]; e < h_rptr[i + 1]; ++e) a += std::fabs(h_rval[e]);
            sig[i] = a > 0 ? 1.0 / a : 1.0;
        }
        up(d_pd_c, c); up(d_pd_lo, lo); up(d_pd_hi, hi); up(d_pd_L, L); up(d_pd_U, U);
        up(d_pd_tau, tau); up(d_pd_sigma, sig);
        d_pd_x.ensure(stream, n); d_pd_xbar.ensure(stream, n); d_pd_xsum.ensure(stream, n); d_pd_y.ensure(stream, m); d_pd_ysum.ensure(stream, m);
        d_pd_gap.ensure(stream, N); d_pd_dual.ensure(stream, N);
        if (pd_gexec) { cudaGraphExecDestroy(pd_gexec); pd_gexec = nullptr; }
        pd_geom = opt.pdhg_cluster ? pdhg_cluster_geometry(m, n, h_cptr.data(), h_rptr.data())
                                   : PdhgClusterGeom{0, 0, 0, 0, 0, 0};
    }

    // ceil(iters / PDHG_RESTART) restart periods of PDHG from the zero start,
    // then the per-variable evidence arrays.
    void run_pdhg(int iters) { run_pdhg_on(iters, stream); }
    void run_pdhg_on(int iters, cudaStream_t ps) {
        PD = PdhgDev{m, n, PDHG_RESTART, d_cptr.p, d_crow.p, d_cval.p, d_rptr.p, d_rcol.p, d_rval.p,
                     d_pd_c.p, d_pd_lo.p, d_pd_hi.p, d_pd_L.p, d_pd_U.p, d_pd_tau.p, d_pd_sigma.p,
                     d_pd_x.p, d_pd_xbar.p, d_pd_xsum.p, d_pd_y.p, d_pd_ysum.p};
        CK(launch_pdhg_init(PD, ps));
        if (!pd_gexec) {
            cudaGraph_t g;
            CK(cudaStreamBeginCapture(ps, cudaStreamCaptureModeThreadLocal));
            set_launch_counting(false);
            cudaError_t le = launch_pdhg_period(PD, ps);
            set_launch_counting(true);
            cudaError_t ce = cudaStreamEndCapture(ps, &g);
            CK(le); CK(ce);
            CK(cudaGraphInstantiate(&pd_gexec, g, 0));
            cudaGraphDestroy(g);
        }
        const int periods = (iters + PDHG_RESTART - 1) / PDHG_RESTART;
        if (!launch_pdhg_cluster(PD, pd_geom, periods, ps)) {   // fallback: graph of 1000 launches per period
            for (int p = 0; p < periods; ++p) CK(cudaGraphLaunch(pd_gexec, ps));
            count_launch(periods * 2 * PDHG_RESTART);
            CK(launch_pdhg_finish(PD, ps));
        }
        CK(launch_pdhg_evidence(PD, d_pd_gap.p, d_pd_dual.p, ps));
    }

    void pdhg_estimate(int iters, double* x, double* y) {
        run_pdhg(iters);
        CK(cudaMemcpyAsync(x, d_pd_x.p, sizeof(double) * n, cudaMemcpyDeviceToHost, stream));
        CK(cudaMemcpyAsync(y, d_pd_y.p, sizeof(double) * m, cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
    }

    // Make the main stream wait for the PDHG evidence before launches whose
    // iterations reach learn_start.
    void pd_wait_before(int last_iteration) {
        if (pd_pending && last_iteration >= learn_start) {
            CK(cudaStreamWaitEvent(stream, pd_done, 0));
            pd_pending = false;
        }
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
        D.learned = (opt.pricing == DS_PRICING_LEARNED && mlp) ? 1 : 0;
        D.learn_mix = opt.learned_mix;
        D.learn_margin = opt.learned_margin;
        D.learn_start = learn_start;
        D.mlp_w1 = D.mlp_w2 = nullptr; D.mlp_p = nullptr; D.mlp_err = nullptr;
        if (mlp) model_pointers(mlp, &D.mlp_w1, &D.mlp_w2, &D.mlp_p, &D.mlp_err);
        D.score = d_score.p; D.row_nnz = d_row_nnz.p;
        D.enter_count = d_enter_cnt.p; D.entered_at = d_entered_at.p;
        D.ftr_every = ftr_every; D.ftr_cap = ftr_cap;
        D.ftr_feat = d_ftr_feat.p; D.ftr_meta = d_ftr_meta.p;
        D.pd_gap = d_pd_gap.p; D.pd_dual = d_pd_dual.p;
        D.dense = dense ? 1 : 0;
        D.Binv = d_Binv.p; D.binv_part = d_binv_part.p; D.binv_tickets = d_binv_tickets.p;
        D.binv_rc = BINV_RC; D.binv_chunks = (m + BINV_RC - 1) / BINV_RC;
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
        nnz_S = 0;
        for (int v : s_var) nnz_S += h_cptr[v + 1] - h_cptr[v];
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
        nnz_cpl = (long long)ccol.size();
        put(d_cpl_ptr, cptr); put(d_cpl_col, ccol);
        if (!cval.empty()) CK(cudaMemcpyAsync(d_cpl_val.p, cval.data(), cval.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
        const bool sparse = !dense && opt.factor_mode == DS_FACTOR_SPARSE && k > 0;
        if (!sparse) {
            const size_t kk = (size_t)std::max(k, 1) * std::max(k, 1);
            d_Kinv.ensure(stream, kk); d_S.ensure(stream, kk);
            d_Pan.ensure(stream, (size_t)std::max(k, 1) * 16); d_Wk.ensure(stream, (size_t)std::max(k, 1) * 16);
            d_rowpiv.ensure(stream, std::max(k, 1)); d_piv_rows.ensure(stream, std::max(k, 1));
        }
        // FTRAN launch geometry for this k
        const int tile = 256;
        const int ntile = std::max(1, (k + tile - 1) / tile);
        // about four blocks per SM: chunks of at least 16 rows of Kinv per block
        const int want = std::max(1, 592 / ntile);
        int chunk = std::max(16, (k + want - 1) / want);
        const int nchunk = std::max(1, (k + chunk - 1) / chunk);
        D.ftr_tile = tile; D.ftr_chunk = chunk; D.ftr_ntile = ntile; D.ftr_nchunk = nchunk;
        d_part.ensure(stream, (size_t)nchunk * MAX_FTRAN_RHS * std::max(k, 1));
        d_tile_tickets.ensure(stream, ntile);
        CK(cudaMemsetAsync(d_tile_tickets.p, 0, sizeof(unsigned) * ntile, stream));
        D.sf.on = 0;
        sync_dev();
        int ferr = 0;
        float ms = 0;
        if (sparse) {
            // sparse LU: host triangularisation, device kernel LU, solve programs
            SfInput in{m, n, k, h_cptr.data(), h_crow.data(), h_cval.data(), (long long)h_cptr[n],
                       s_var.data(), s_pos.data(), rp_row.data(), row_kidx.data()};
            const auto h0 = std::chrono::steady_clock::now();
            SfInfo fi = sflu.factor(in, d_cval.p, stream, &D.sf);
            sfi = fi;
            const double host_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - h0).count();
            st.refactor_ms += host_ms;   // the whole factorisation, host stages included
            st.lu_kernel = fi.km; st.lu_dense = fi.kd; st.lu_rounds = fi.rounds;
            st.lu_levels = fi.lev_ft + fi.lev_bt;
            if (opt.verbose >= 1)
                fprintf(stderr, "[ds] sparse LU it %d: k %d kernel %d (sparse pivots %d in %d rounds, dense %d%s), "
                        "L %d U %d, levels %d/%d, entries %lld/%lld, %.2f ms (device %.2f)\n", hc->iteration, k, fi.km,
                        fi.ks, fi.rounds, fi.kd, fi.dense_fallback ? ", dense fallback" : "", fi.lnnz, fi.unnz,
                        fi.lev_ft, fi.lev_bt, fi.ent_ft, fi.ent_bt, host_ms, fi.kernel_ms);
            if (fi.singular) {
                char msg[320];
                snprintf(msg, sizeof(msg), "singular basis in refactorisation (iteration %d, k %d): %s", hc->iteration, k, fi.msg);
                throw CudaError(msg, DS_ERR_NUMERIC);
            }
            sync_dev();
        } else {
            FactorBufs F{d_S.p, d_Pan.p, d_Wk.p, d_rowpiv.p, d_piv_rows.p, d_Winv.p, d_ferr.p, d_s_var.p, d_row_kidx.p};
            CK(cudaEventRecord(evr0, stream));
            CK(factor_bump(F, D, k, stream));
            CK(cudaEventRecord(evr1, stream));
            CK(cudaMemcpyAsync(&ferr, d_ferr.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
            CK(cudaStreamSynchronize(stream));
            cudaEventElapsedTime(&ms, evr0, evr1);
            st.refactor_ms += ms;
        }
        if (k > 0 && ferr) {
            // diagnostics: duplicate basic variables, K columns without an R' entry
            std::vector<int> seen(N, 0);
            int dups = 0, empty_cols = 0;
            for (int v : basis) if (seen[v]++) ++dups;
            for (int j = 0; j < k; ++j) {
                bool any = false;
                for (int e = h_cptr[s_var[j]]; e < h_cptr[s_var[j] + 1]; ++e) any |= row_kidx[h_crow[e]] >= 0;
                if (!any) ++empty_cols;
            }
            char msg[256];
            snprintf(msg, sizeof(msg), "singular basis in refactorisation (iteration %d, k %d, pivot column %d, "
                     "duplicate basics %d, empty K columns %d)", hc->iteration, k, ferr - 1, dups, empty_cols);
            throw CudaError(msg, DS_ERR_NUMERIC);
        }
        if (opt.verbose >= 3 && k > 0 && !sparse) {
            // debug: || Kinv K - I ||_max on the host
            std::vector<double> Ki((size_t)k * k), Kd((size_t)k * k, 0.0);
            CK(cudaMemcpyAsync(Ki.data(), d_Kinv.p, sizeof(double) * k * k, cudaMemcpyDeviceToHost, stream));
            CK(cudaStreamSynchronize(stream));
            for (int j = 0; j < k; ++j)
                for (int e = h_cptr[s_var[j]]; e < h_cptr[s_var[j] + 1]; ++e)
                    if (row_kidx[h_crow[e]] >= 0) Kd[(size_t)row_kidx[h_crow[e]] + (size_t)j * k] = h_cval[e];
            double worst = 0;
            for (int i = 0; i < k; ++i)
                for (int j = 0; j < k; ++j) {
                    double s2 = 0;
                    for (int t = 0; t < k; ++t) s2 += Ki[(size_t)i + (size_t)t * k] * Kd[(size_t)t + (size_t)j * k];
                    worst = std::max(worst, std::fabs(s2 - (i == j ? 1.0 : 0.0)));
                }
            fprintf(stderr, "[ds-check] refactor it %d k %d |Kinv K - I| %.3e (%.2f ms)\n", hc->iteration, k, worst, ms);
        }
        if (dense) { CK(launch_binv_build(D, stream)); binv_valid = true; }   // B^-1 of the new B0 (D.k set by sync_dev above)
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
        if (gexec_u) { cudaGraphExecDestroy(gexec_u); gexec_u = nullptr; }
    }
    // Capture `iters` consecutive iterations into one executable graph.
    cudaGraphExec_t capture_iterations(int iters, long long* nodes) {
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        set_launch_counting(false);
        cudaError_t le = cudaSuccess;
        for (int u = 0; u < iters && le == cudaSuccess; ++u) le = launch_iteration(D, stream);
        set_launch_counting(true);
        cudaError_t ce = cudaStreamEndCapture(stream, &g);
        CK(le); CK(ce);
        size_t nn = 0;
        CK(cudaGraphGetNodes(g, nullptr, &nn));
        if (nodes) *nodes = (long long)nn;
        cudaGraphExec_t ge = nullptr;
        CK(cudaGraphInstantiate(&ge, g, 0));
        cudaGraphDestroy(g);
        return ge;
    }
    void ensure_graph() {
        if (gexec) return;
        gexec = capture_iterations(1, &graph_nodes);
        gexec_u = capture_iterations(GRAPH_UNROLL, nullptr);
    }

    // -------------------------------------------------------------- solves
    // FTRAN of one dense row vector: out = B^-1 rhs (solveLinSys, transpose=false)
    void ftran1(const double* rhs, double* out) {
        if (dense) { CK(launch_dense_ftran_vec(D, rhs, out, stream)); return; }
        Dev E = D;
        E.frhs[0] = rhs; E.fout[0] = out;
        CK(launch_ftran(E, 1, 0, 1, stream));
    }
    void ftran2(const double* r0, double* o0, const double* r1, double* o1) {
        if (dense) {
            CK(launch_dense_ftran_vec(D, r0, o0, stream));
            CK(launch_dense_ftran_vec(D, r1, o1, stream));
            return;
        }
        Dev E = D;
        E.frhs[0] = r0; E.fout[0] = o0; E.frhs[1] = r1; E.fout[1] = o1;
        CK(launch_ftran(E, 2, 0, 1, stream));
    }
    // BTRAN of a dense position vector: y = B^-T c (rows)
    void btran_dense(const double* c0, double* y) {
        if (dense) { CK(launch_dense_btran_vec(D, c0, y, stream)); return; }
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
        if (dense) {                 // exact weights from the explicit inverse
            CK(launch_dense_beta(D, stream));
            CK(cudaStreamSynchronize(stream));
            return;
        }
        pull();
        if (hc->T == 0 && !D.sf.on) {   // every caller refactors first: B = B0 (explicit Kinv)
            CK(launch_beta_exact(D, stream));
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
            if (hc->iteration % hc->R == 0) refresh();
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
                refresh(); phase1_init(); init_beta(false);
                if (blocked_any) { CK(cudaMemsetAsync(d_blocked.p, 0, N, stream)); blocked_any = false; }
                st.restarts++;
                continue;
            }
            if (ev == EV_P1_BLOCK) {
                const unsigned char one = 1;
                CK(cudaMemcpyAsync(d_blocked.p + hc->p, &one, 1, cudaMemcpyHostToDevice, stream));
                blocked_any = true;
                clear_event(); push();
                refresh(); phase1_init();
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
        if (dense) {
            // rebuild B^-1 for the current basis, then redo rho, the FTRAN and the
            // update of this iteration with it
            refactor();
            CK(launch_dense_rho(D, hc->p_idx, stream));
            CK(launch_ftran_dense(D, 0, 1, stream));
            CK(launch_update_forced(D, stream));
            CK(launch_binv_update(D, 1, stream));
            return;
        }
        refactor();
        if (nr > 2) ftran2(d_rho.p, d_tau.p, d_cc.p, d_dxb.p);
        else ftran1(d_rho.p, d_tau.p);
        CK(launch_update_forced(D, stream));
    }

    // -------------------------------------------------------------- phase 2
    // Launch graph iterations until an event is raised.
    // Algorithmic bytes moved by one launch of each iteration kernel (FP64 = 8 B,
    // int32 = 4 B), with T the eta count at the start of the iteration.
    double step_bytes(int st, int T, int nrhs, bool dual_check) const {
        const double M = m, Nn = n, K = k, Tt = T, R = nrhs;
        switch (st) {
            case S_SCORE: return 69 * M + 10248.0 * ((m + 127) / 128);
            case S_CHUZR: return 37 * M + 8 * Tt + 4 * Tt * Tt + (dual_check ? 13 * Nn : 0);
            case S_BTRAN_RHS: return 24.0 * nnz_S + 20 * K;
            case S_BTRAN_GEMV:
                if (D.sf.on)   // program entries (coefficient + slot), ops (slot, range, divisor), dense block, gather/scatter
                    return 12.0 * sfi.ent_bt + 16.0 * sfi.op_bt + 8.0 * sfi.kd * sfi.kd + 24 * K + 12 * (M - K);
                return 8 * K * K + 8 * K + 12 * M;
            case S_PIVOT_ROW: return 12.0 * ((double)h_rptr[m] - nnz_S) + 8 * K + 4 * Nn + 8 * (Nn - K) + 8 * M + 50 * Nn;
            case S_DUAL_UPDATE: return 30 * Nn + (dense ? (12.0 + 8 * M) * ((double)h_rptr[m] / n) + 8 * M : 0.0);
            case S_FTRAN_K:
                if (D.sf.on) return R * (12.0 * sfi.ent_ft + 16.0 * sfi.op_ft + 8.0 * sfi.kd * sfi.kd + 24 * K);
                return 8 * K * K + 16 * R * K + 8 * R * K * D.ftr_nchunk;
            case S_FTRAN_ASM: return 20.0 * nnz_cpl + (M - K) * (4 + 16 * R) + 8 * R * Tt;
            case S_ETA_APPLY: return 8 * Tt * M + 16 * R * M;
            case S_UPDATE: return dense ? 44 * M : 60 * M + 8 * Tt + 4 * Tt * Tt;
            case S_FTRAN_DENSE: return (12.0 + 8 * M) * ((double)h_rptr[m] / n) + 8 * M;
            case S_BINV: return 16 * M * M + 16 * M + 8 * M * ((M + BINV_ROWS - 1) / BINV_ROWS);
        }
        return 0;
    }

    // Debug self-check (verbose >= 3): residuals of this iteration's solves
    // against the basis it started from, computed on the host in O(nnz).
    std::vector<int> dbg_basis;
    void debug_check_iteration() {
        std::vector<double> aq(m), rho(m), tau(m), x(N);
        CK(cudaMemcpyAsync(aq.data(), d_alpha_q.p, sizeof(double) * m, cudaMemcpyDeviceToHost, stream));
        CK(cudaMemcpyAsync(rho.data(), d_rho.p, sizeof(double) * m, cudaMemcpyDeviceToHost, stream));
        CK(cudaMemcpyAsync(tau.data(), d_tau.p, sizeof(double) * m, cudaMemcpyDeviceToHost, stream));
        CK(cudaMemcpyAsync(x.data(), d_x.p, sizeof(double) * N, cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        auto col_axpy = [&](int v, double a, std::vector<double>& out) {
            if (v < n) { for (int e = h_cptr[v]; e < h_cptr[v + 1]; ++e) out[h_crow[e]] += a * h_cval[e]; }
            else out[v - n] += a;
        };
        auto col_dot = [&](int v, const std::vector<double>& y) {
            double s = 0;
            if (v < n) { for (int e = h_cptr[v]; e < h_cptr[v + 1]; ++e) s += h_cval[e] * y[h_crow[e]]; }
            else s = y[v - n];
            return s;
        };
        const std::vector<int>& B = dbg_basis;
        std::vector<double> r1(m, 0.0), r3(m, 0.0);
        for (int i = 0; i < m; ++i) { col_axpy(B[i], aq[i], r1); col_axpy(B[i], tau[i], r3); }
        col_axpy(hc->q, -1.0, r1);
        double e1 = 0, e2 = 0, e3 = 0, nr = 0;
        for (int r = 0; r < m; ++r) { e1 = std::max(e1, std::fabs(r1[r])); e3 = std::max(e3, std::fabs(r3[r] - rho[r])); nr = std::max(nr, std::fabs(rho[r])); }
        for (int i = 0; i < m; ++i) e2 = std::max(e2, std::fabs(col_dot(B[i], rho) - (i == hc->p_idx ? 1.0 : 0.0)));
        // primal residual with the new basis: A x + s = 0 over all columns
        std::vector<double> rp(m, 0.0);
        for (int j = 0; j < N; ++j) if (x[j] != 0.0) col_axpy(j, x[j], rp);
        double e4 = 0; for (double v : rp) e4 = std::max(e4, std::fabs(v));
        if (e1 > 1e-8 || e2 > 1e-8 || e3 > 1e-8 * (1 + nr) || e4 > 1e-7)
            fprintf(stderr, "[ds-check] it %d k %d T %d p_idx %d q %d |B aq - a_q| %.3e |B^T rho - e_p| %.3e |B tau - rho| %.3e |Ax+s| %.3e\n",
                    hc->iteration, k, hc->T, hc->p_idx, hc->q, e1, e2, e3, e4);
    }

    // Debug: does B0 + the eta file still represent the current basis?  FTRAN and
    // BTRAN of random vectors checked against the basis read back from the device.
    void debug_check_representation(const char* where) {
        std::vector<int> B(m);
        CK(cudaMemcpyAsync(B.data(), d_basis.p, sizeof(int) * m, cudaMemcpyDeviceToHost, stream));
        std::vector<double> r(m), y(m), c(m), z(m);
        uint64_t st2 = 0x9E3779B97F4A7C15ull ^ (uint64_t)hc->iteration;
        for (int i = 0; i < m; ++i) { st2 = st2 * 6364136223846793005ull + 1442695040888963407ull; r[i] = (double)(st2 >> 11) * 0x1.0p-53 - 0.5; c[i] = r[(i * 7) % m]; }
        CK(cudaMemcpyAsync(d_tmp_rows.p, r.data(), sizeof(double) * m, cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(d_tmp_pos.p, c.data(), sizeof(double) * m, cudaMemcpyHostToDevice, stream));
        ftran1(d_tmp_rows.p, d_tmp_pos2.p);
        btran_dense(d_tmp_pos.p, d_tmp_rows2.p);
        CK(cudaMemcpyAsync(y.data(), d_tmp_pos2.p, sizeof(double) * m, cudaMemcpyDeviceToHost, stream));
        CK(cudaMemcpyAsync(z.data(), d_tmp_rows2.p, sizeof(double) * m, cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        std::vector<double> By(m, 0.0);
        double e1 = 0, e2 = 0;
        for (int i = 0; i < m; ++i) {
            const int v = B[i];
            if (v < n) { for (int e = h_cptr[v]; e < h_cptr[v + 1]; ++e) By[h_crow[e]] += h_cval[e] * y[i]; }
            else By[v - n] += y[i];
            double d2 = 0;
            if (v < n) { for (int e = h_cptr[v]; e < h_cptr[v + 1]; ++e) d2 += h_cval[e] * z[h_crow[e]]; }
            else d2 = z[v - n];
            e2 = std::max(e2, std::fabs(d2 - c[i]));
        }
        for (int i = 0; i < m; ++i) e1 = std::max(e1, std::fabs(By[i] - r[i]));
        if (e1 > 1e-9 || e2 > 1e-9)
            fprintf(stderr, "[ds-rep] %s it %d k %d T %d |B FTRAN(r) - r| %.3e |B^T BTRAN(c) - c| %.3e\n",
                    where, hc->iteration, k, hc->T, e1, e2);
    }

    void debug_check_x(const char* where) {
        std::vector<double> x(N);
        CK(cudaMemcpyAsync(x.data(), d_x.p, sizeof(double) * N, cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        std::vector<double> rp(m, 0.0);
        for (int j = 0; j < N; ++j) {
            if (x[j] == 0.0) continue;
            if (j < n) { for (int e = h_cptr[j]; e < h_cptr[j + 1]; ++e) rp[h_crow[e]] += h_cval[e] * x[j]; }
            else rp[j - n] += x[j];
        }
        double e4 = 0; for (double v : rp) e4 = std::max(e4, std::fabs(v));
        fprintf(stderr, "[ds-x] %s it %d |Ax+s| %.3e\n", where, hc->iteration, e4);
    }

    // Profiling: one iteration at a time, every kernel bracketed by CUDA events.
    int run_until_event_profiled() {
        if (!pev[0]) for (auto& e : pev) CK(cudaEventCreate(&e));
        while (true) {
            pull();
            if (opt.verbose >= 3) {
                dbg_basis.resize(m);
                CK(cudaMemcpyAsync(dbg_basis.data(), d_basis.p, sizeof(int) * m, cudaMemcpyDeviceToHost, stream));
                CK(cudaStreamSynchronize(stream));
            }
            const int T0 = hc->T;
            pd_wait_before(hc->iteration + 1);
            bool ran[S_NSTEPS] = {};
            for (int stp = 0; stp < S_NSTEPS; ++stp) {
                if (!step_active(D, stp)) continue;
                CK(cudaEventRecord(pev[2 * stp], stream));
                CK(launch_step(D, stp, stream));
                CK(cudaEventRecord(pev[2 * stp + 1], stream));
                ran[stp] = true;
            }
            pull();
            if (hc->halt) return hc->event;
            if (opt.verbose >= 3) { debug_check_iteration(); debug_check_representation("graph"); pull(); }
            const bool dchk = (hc->iteration % NEED_RESTART) == 0;
            for (int stp = 0; stp < S_NSTEPS; ++stp) {
                if (!ran[stp]) continue;
                float ms = 0;
                CK(cudaEventElapsedTime(&ms, pev[2 * stp], pev[2 * stp + 1]));
                prof_us[stp] += 1000.0 * ms;
                prof_bytes[stp] += step_bytes(stp, T0, hc->nrhs, dchk);
                prof_n[stp] += 1;
            }
        }
    }

    int run_until_event() {
        if (prof || opt.verbose >= 3) return run_until_event_profiled();
        while (true) {
            ensure_graph();
            const int it = hc->iteration;
            const int R = hc->R;
            int batch = R - (it % R);
            if (batch > BATCH_ITERS) batch = BATCH_ITERS;
            if (batch < 1) batch = 1;
            pd_wait_before(it + batch);
            int b = 0;
            for (; b + GRAPH_UNROLL <= batch; b += GRAPH_UNROLL) CK(cudaGraphLaunch(gexec_u, stream));
            for (; b < batch; ++b) CK(cudaGraphLaunch(gexec, stream));
            count_launch((int)(batch * graph_nodes));
            pull();
            if (hc->halt) return hc->event;
        }
    }

    // Dense mode, at the periodic rebuild: is the maintained B^-1 still accurate?
    // The rank-1 updates drift slowly, so the rebuild (a k x k inversion, some
    // milliseconds) is skipped while the probe residual |B (B^-1 v) - v|_max stays
    // below DENSE_PROBE_TOL (1 + |B^-1 v|_max).  The per-iteration pivot check
    // still forces a rebuild on any visible drift.  The eta-file path and
    // strict_reference rebuild on every period, as the reference does.
    bool inverse_accurate() {
        if (!dense || opt.strict_reference) return false;
        unsigned long long bits[2] = {0, 0};
        CK(launch_binv_probe(D, d_tmp_rows.p, d_tmp_pos.p, d_probe.p, stream));
        CK(cudaMemcpyAsync(bits, d_probe.p, sizeof(bits), cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        double res, ymax;
        std::memcpy(&res, &bits[0], sizeof(double));
        std::memcpy(&ymax, &bits[1], sizeof(double));
        if (opt.verbose)
            fprintf(stderr, "[ds] it %d inverse probe residual %.3e |B^-1 v| %.3e\n", hc->iteration, res, ymax);
        return res <= DENSE_PROBE_TOL * (1.0 + ymax);
    }

    // A refactorisation wherever the solve only needs an accurate B^-1 for the
    // current basis (periodic, restarts, phase changes): in dense mode it is
    // skipped while the maintained inverse passes the probe.  A pivot mismatch
    // and the explicit basis solves always refactorise.
    void refresh() {
        if (binv_valid && inverse_accurate()) return;
        refactor();
    }

    // remaining top-of-loop steps after a refactor at iteration it (reference order)
    void top_after_refactor() {
        pull();
        if (hc->iteration % NEED_RESTART == 0 && !dual_feasible()) {
            refresh(); phase1(); dual_simplex_init(); st.restarts++;
        }
        pull();
        if (!perturbed && hc->cycle > MAX_CYCLE) { perturb(); refresh(); dual_simplex_init(); perturb_guard(); }
    }

    // Perturbing the basic costs moves y = B^-T c_B and can leave nonbasic reduced
    // costs of the wrong sign; the reference then takes a step of the wrong sign
    // until its next NEED_RESTART check.  Restore dual feasibility at once.
    void perturb_guard() {
        if (opt.strict_reference || dual_feasible()) return;
        refresh(); phase1(); dual_simplex_init(); st.restarts++;
    }

    // Run the rest of the current iteration from pricing on (after a top event).
    int run_body_once() {
        pull(); clear_event(); hc->top_done = 1; push();
        if (opt.verbose >= 3) {
            debug_check_representation("before-body");
            dbg_basis.resize(m);
            CK(cudaMemcpyAsync(dbg_basis.data(), d_basis.p, sizeof(int) * m, cudaMemcpyDeviceToHost, stream));
            CK(cudaStreamSynchronize(stream));
            debug_check_x("before-body");
        }
        pd_wait_before(hc->iteration);
        CK(launch_body(D, ST_PRICING, stream));
        pull();
        if (opt.verbose >= 3 && !hc->halt) {
            fprintf(stderr, "[ds-body] it %d p %d p_idx %d q %d q_idx %d theta %.6e delta %.6e nrhs %d T %d\n", hc->iteration,
                    hc->p, hc->p_idx, hc->q, hc->q_idx, hc->theta, hc->delta_bfrt, hc->nrhs, hc->T);
            debug_check_iteration(); debug_check_representation("after-body"); pull();
        }
        return hc->halt ? hc->event : EV_NONE;
    }

    // callDualSolver (cudaDualSimplex.cpp:396-655)
    bool phase2() {
        refresh();
        dual_simplex_init();
        pull();
        hc->cycle = 0; hc->unbound_checked = 0; clear_event();
        push();
        int pivots_at_nop = -1;
        int ev = run_until_event();
        while (true) {
            if (opt.verbose) {
                fprintf(stderr, "[ds] it %d event %d stage %d k %d T %d obj %.12g cycle %d pert %d\n", hc->iteration, ev,
                        hc->event_stage, k, hc->T, hc->obj, hc->cycle, (int)perturbed);
            }
            switch (ev) {
                case EV_NONE: ev = run_until_event(); continue;
                case EV_ITER_LIMIT: status = DS_STATUS_ITER_LIMIT; return false;
                case EV_REFACTOR_DUE:
                    clear_event(); push();
                    refresh();
                    top_after_refactor();
                    ev = run_body_once();
                    continue;
                case EV_DUALINF:
                    clear_event(); push();
                    refresh(); phase1(); dual_simplex_init(); st.restarts++;
                    pull();
                    if (!perturbed && hc->cycle > MAX_CYCLE) { perturb(); refresh(); dual_simplex_init(); perturb_guard(); }
                    ev = run_body_once();
                    continue;
                case EV_PERTURB:
                    clear_event(); push();
                    perturb(); refresh(); dual_simplex_init();
                    perturb_guard();
                    ev = run_body_once();
                    continue;
                case EV_OPTIMAL: status = DS_STATUS_OPTIMAL; return true;
                case EV_NO_P: {
                    pull();
                    if (!opt.strict_reference && pivots_at_nop == hc->pivots) { status = DS_STATUS_OPTIMAL; return true; }
                    pivots_at_nop = hc->pivots;
                    clear_event(); push();
                    refresh(); init_beta(false); phase1(); dual_simplex_init(); st.restarts++;
                    ev = run_until_event();
                    continue;
                }
                case EV_UNBOUNDED: {
                    pull();
                    if (hc->unbound_checked) { status = DS_STATUS_PRIMAL_INFEASIBLE; return false; }
                    hc->unbound_checked = 1; clear_event(); push();
                    refresh(); init_beta(false); phase1(); dual_simplex_init(); st.restarts++;
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

    // Factorise the given basis and apply B^-1 (rows -> positions) or B^-T
    // (positions -> rows) to nr dense vectors.
    void basis_solve(const int* basis, const double* rhs, double* out, int nr, int transpose) {
        if (!loaded) throw CudaError("basis_solve before load", DS_ERR_STATE);
        std::vector<int> b(basis, basis + m), nb, vp(N, 0), seen(N, 0);
        for (int v : b) { if (v < 0 || v >= N || seen[v]++) throw CudaError("bad basis", DS_ERR_ARG); }
        for (int j = 0; j < N; ++j) if (!seen[j]) nb.push_back(j);
        if ((int)nb.size() != n) throw CudaError("bad basis", DS_ERR_ARG);
        for (int i = 0; i < m; ++i) vp[b[i]] = i;
        for (int s2 = 0; s2 < n; ++s2) vp[nb[s2]] = -(s2 + 1);
        std::memset(hc, 0, sizeof(Ctl));
        hc->max_iter = 1; hc->R = 1; hc->phase = 2; hc->prev_q = -1; hc->ybt_n = -1;
        sync_dev(); push();
        CK(cudaMemcpyAsync(d_basis.p, b.data(), sizeof(int) * m, cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(d_nonbasis.p, nb.data(), sizeof(int) * n, cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(d_var_pos.p, vp.data(), sizeof(int) * N, cudaMemcpyHostToDevice, stream));
        refactor();
        DBuf<double> in, o;
        in.alloc(stream, (size_t)nr * m); o.alloc(stream, (size_t)nr * m);
        CK(cudaMemcpyAsync(in.p, rhs, sizeof(double) * nr * m, cudaMemcpyHostToDevice, stream));
        for (int r0 = 0; r0 < nr; r0 += (transpose ? 1 : MAX_FTRAN_RHS)) {
            if (transpose) {
                btran_dense(in.p + (size_t)r0 * m, o.p + (size_t)r0 * m);
            } else {
                Dev E = D;
                const int cnt = std::min(MAX_FTRAN_RHS, nr - r0);
                for (int q = 0; q < cnt; ++q) { E.frhs[q] = in.p + (size_t)(r0 + q) * m; E.fout[q] = o.p + (size_t)(r0 + q) * m; }
                CK(launch_ftran(E, cnt, 0, 1, stream));
            }
        }
        CK(cudaMemcpyAsync(out, o.p, sizeof(double) * nr * m, cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
    }

    // Copy the feature trace back, ordered by (iteration, position): the device
    // appends records in completion order.
    void fetch_feature_trace() {
        ftr_total = hc->ftr_n;
        const int kept = std::min(hc->ftr_n, ftr_cap);
        std::vector<float> f((size_t)kept * DS_NUM_FEATURES);
        std::vector<int> mt((size_t)kept * 3);
        if (kept > 0) {
            CK(cudaMemcpyAsync(f.data(), d_ftr_feat.p, sizeof(float) * f.size(), cudaMemcpyDeviceToHost, stream));
            CK(cudaMemcpyAsync(mt.data(), d_ftr_meta.p, sizeof(int) * mt.size(), cudaMemcpyDeviceToHost, stream));
            CK(cudaStreamSynchronize(stream));
        }
        std::vector<int> ord(kept);
        for (int r = 0; r < kept; ++r) ord[r] = r;
        std::sort(ord.begin(), ord.end(), [&](int a, int b) {
            if (mt[3 * a] != mt[3 * b]) return mt[3 * a] < mt[3 * b];
            return mt[3 * a + 1] < mt[3 * b + 1];
        });
        ftr_feat.resize(f.size()); ftr_meta.resize(mt.size());
        for (int r = 0; r < kept; ++r) {
            std::copy(f.begin() + (size_t)ord[r] * DS_NUM_FEATURES, f.begin() + (size_t)(ord[r] + 1) * DS_NUM_FEATURES,
                      ftr_feat.begin() + (size_t)r * DS_NUM_FEATURES);
            std::copy(mt.begin() + 3 * (size_t)ord[r], mt.begin() + 3 * (size_t)(ord[r] + 1), ftr_meta.begin() + 3 * (size_t)r);
        }
    }

    // presolve + solve + postProcess (tpp:5-30, 123-180) with the cleanup guard
    // A nonbasic free structural with a nonzero reduced cost is dual infeasible,
    // and the reference's phase 1 can leave one behind (the solve then ends
    // "optimal" at a dual infeasible basis).  Unless strict_reference is set,
    // each free structural column (at most CRASH_MAX) first takes the place of a
    // slack whose row has a finite bound, chosen by partial pivoting on the
    // columns eliminated so far: largest |entry|, lowest row on ties, pivots below
    // 1e-9 of the column's largest entry refused, so the structural block stays
    // nonsingular.  A free basic variable never leaves the basis.
    static constexpr int CRASH_MAX = 512;
    void crash_free_columns(std::vector<int>& basis, std::vector<int>& nonbasis, std::vector<int>& var_pos) {
        std::vector<int> cols;
        for (int j = 0; j < n && (int)cols.size() < CRASH_MAX; ++j)
            if (h_type[j] == FREE && h_cptr[j + 1] > h_cptr[j]) cols.push_back(j);
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
            for (int e = h_cptr[j]; e < h_cptr[j + 1]; ++e) {
                const int i = h_crow[e];
                w[i] = h_cval[e];
                if (!mark[i]) { mark[i] = 1; touched.push_back(i); }
                vmax = std::max(vmax, std::fabs(h_cval[e]));
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
                if (used[i] || h_type[n + i] == FREE) continue;
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
                basis[r] = j; var_pos[j] = r;
                nonbasis[j] = n + r; var_pos[n + r] = -(j + 1);
            }
            for (int i : touched) { w[i] = 0.0; mark[i] = 0; }
        }
    }

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
        if (!opt.strict_reference) crash_free_columns(basis, nonbasis, var_pos);
        CK(cudaMemcpyAsync(d_basis.p, basis.data(), sizeof(int) * m, cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(d_nonbasis.p, nonbasis.data(), sizeof(int) * n, cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(d_var_pos.p, var_pos.data(), sizeof(int) * N, cudaMemcpyHostToDevice, stream));
        CK(cudaMemsetAsync(d_x.p, 0, sizeof(double) * N, stream));
        CK(cudaMemsetAsync(d_d.p, 0, sizeof(double) * N, stream));
        CK(cudaMemsetAsync(d_blocked.p, 0, N, stream));
        CK(cudaMemsetAsync(d_aq.p, 0, sizeof(double) * m, stream));
        CK(cudaMemsetAsync(d_enter_cnt.p, 0, sizeof(int) * N, stream));
        CK(cudaMemsetAsync(d_entered_at.p, 0, sizeof(int) * N, stream));
        d_trace.alloc(stream, 2 * std::max(trace_cap, 1)); d_trace_d.alloc(stream, 2 * std::max(trace_cap, 1));
        if (opt.pricing == DS_PRICING_LEARNED && !mlp)
            throw CudaError("learned pricing needs a model (ds_set_model)", DS_ERR_STATE);
        if (mlp && model_device(mlp) != opt.device)
            throw CudaError("model lives on another device", DS_ERR_STATE);
        if (ftr_every > 0) {
            d_ftr_feat.ensure(stream, (size_t)ftr_cap * DS_NUM_FEATURES);
            d_ftr_meta.ensure(stream, (size_t)ftr_cap * 3);
        }
        invalidate_graph();   // launch parameters may have changed
        const bool want_pd = (opt.pricing == DS_PRICING_LEARNED) || ftr_every > 0;
        learn_start = 0;
        if (opt.pricing == DS_PRICING_LEARNED && ftr_every == 0)
            // default 7m/20: at m = 2000 the 700 DSE iterations take about as long as
            // the 4000 PDHG iterations beside them, so the evidence is ready when
            // learned pricing starts (measured best of m/8 .. 2m/5 on B200)
            learn_start = opt.learned_start_iteration >= 0 ? opt.learned_start_iteration : (7 * m) / 20;
        std::memset(hc, 0, sizeof(Ctl));
        hc->max_iter = opt.max_iterations;
        // dense mode has no eta file: a rebuild only resets rounding, so it runs on
        // its own (longer) interval unless the reference's cadence is asked for
        hc->R = (dense && !opt.strict_reference) ? std::max(opt.dense_refactor_interval, 1)
                                                 : std::min(std::max(opt.refactor_interval, 1), cap - 5);
        hc->phase = 2; hc->prev_q = -1; hc->ybt_n = -1; hc->trace_cap = trace_cap;
        sync_dev();
        push();
        const long long launches0 = launch_count();
        CK(cudaEventRecord(ev0, stream));
        pd_pending = false;
        if (want_pd && opt.learned_pdhg_iters > 0) {
            // warm-start evidence for the scorer's features, on its own stream
            CK(cudaEventRecord(pd_go, stream));
            CK(cudaStreamWaitEvent(pd_stream, pd_go, 0));
            CK(cudaEventRecord(evp0, pd_stream));
            run_pdhg_on(opt.learned_pdhg_iters, pd_stream);
            CK(cudaEventRecord(evp1, pd_stream));
            CK(cudaEventRecord(pd_done, pd_stream));
            pd_pending = true;
            if (learn_start == 0) { CK(cudaStreamWaitEvent(stream, pd_done, 0)); pd_pending = false; }
        } else {
            CK(cudaEventRecord(evp0, stream));
            CK(cudaMemsetAsync(d_pd_gap.p, 0, sizeof(float) * N, stream));
            CK(cudaMemsetAsync(d_pd_dual.p, 0, sizeof(float) * N, stream));
            CK(cudaEventRecord(evp1, stream));
        }
        try {
            refresh();                       // initDualSimplex (cudaDualSimplex.cpp:20-81)
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
                    refresh();
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
        if (pd_pending) { CK(cudaStreamWaitEvent(stream, pd_done, 0)); pd_pending = false; }   // count all launched work
        CK(cudaEventRecord(ev1, stream));
        CK(cudaStreamSynchronize(stream));
        float ms = 0; cudaEventElapsedTime(&ms, ev0, ev1);
        st.solve_ms = ms;
        float pms = 0; cudaEventElapsedTime(&pms, evp0, evp1);
        st.pdhg_ms = pms;
        st.kernel_launches = (int)(launch_count() - launches0);
        pull();
        st.iterations = hc->iteration;
        st.learned_used = hc->learned_used;
        st.learned_fallback = hc->learned_fallback;
        st.bfrt_flips = hc->flips_total;
        if (ftr_every > 0) fetch_feature_trace();
        model_wait_timeout = false;
        if (D.learned && D.mlp_err) {
            int fe = 0;
            CK(cudaMemcpyAsync(&fe, D.mlp_err, sizeof(int), cudaMemcpyDeviceToHost, stream));
            CK(cudaStreamSynchronize(stream));
            model_wait_timeout = fe != 0;
        }
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
    o->learned_margin = 0.5;
    o->verbose = 0;
    o->learned_mix = 0.05;
    o->learned_pdhg_iters = 4000;
    o->dense_max_m = 4096;
    o->dense_refactor_interval = 400;
    o->learned_start_iteration = -1;
    o->pdhg_cluster = 1;
    o->factor_mode = DS_FACTOR_SPARSE;
}

const char* ds_version(void) { return "ds_b200 1.0 (sm_100a)"; }

int ds_create(const ds_options* opts, ds_solver** out) {
    if (!out) return DS_ERR_ARG;
    *out = nullptr;
    ds_options o;
    ds_default_options(&o);
    if (opts) o = *opts;
    if (o.refactor_interval < 1 || o.refactor_interval > 200) return DS_ERR_ARG;
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
        if (s->e->model_wait_timeout)
            return fail(s, DS_ERR_DEVICE_WAIT, "a network scoring launch timed out waiting for its MMAs "
                                               "(those iterations used DSE pricing)");
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

long long ds_kernel_launch_count(void) { return ds::launch_count(); }

int ds_basis_solve(ds_solver* s, const int* basis, const double* rhs, double* out, int nrhs, int transpose) {
    if (!s || !basis || !rhs || !out || nrhs <= 0) return DS_ERR_ARG;
    GUARD(s, { s->e->basis_solve(basis, rhs, out, nrhs, transpose); return DS_OK; })
}

int ds_profile_solve(ds_solver* s, char* json, int len) {
    if (!s || !json || len <= 0) return DS_ERR_ARG;
    Engine* e = s->e;
    GUARD(s, {
        for (int i = 0; i < ds::S_NSTEPS; ++i) { e->prof_us[i] = 0; e->prof_bytes[i] = 0; e->prof_n[i] = 0; }
        e->prof = true;
        try { e->solve(); } catch (...) { e->prof = false; throw; }
        e->prof = false;
        double tot = 0;
        for (int i = 0; i < ds::S_NSTEPS; ++i) tot += e->prof_us[i];
        std::string out = "{\"iterations\": " + std::to_string(e->st.iterations) + ", \"kernels\": [";
        bool first = true;
        for (int i = 0; i < ds::S_NSTEPS; ++i) {
            if (e->prof_n[i] == 0) continue;
            char buf[512];
            const double avg_us = e->prof_us[i] / e->prof_n[i];
            const double avg_b = e->prof_bytes[i] / e->prof_n[i];
            snprintf(buf, sizeof(buf),
                     "%s{\"name\": \"%s\", \"launches\": %lld, \"total_us\": %.3f, \"avg_us\": %.4f, "
                     "\"bytes\": %.1f, \"gbs\": %.2f, \"share\": %.5f}",
                     first ? "" : ", ", ds::kStepNames[i], e->prof_n[i], e->prof_us[i], avg_us, avg_b,
                     avg_b / (avg_us * 1e-6) / 1e9, tot > 0 ? e->prof_us[i] / tot : 0.0);
            out += buf;
            first = false;
        }
        out += "]}";
        if ((int)out.size() + 1 > len) return fail(s, DS_ERR_CAPACITY, "profile buffer too small");
        std::memcpy(json, out.c_str(), out.size() + 1);
        return DS_OK;
    })
}

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

int ds_set_model(ds_solver* s, ds_model* m) {
    if (!s) return DS_ERR_ARG;
    s->e->mlp = m ? ds_model_impl(m) : nullptr;
    s->e->invalidate_graph();
    return DS_OK;
}

int ds_pdhg_estimate(ds_solver* s, int iters, double* x, double* y) {
    if (!s || iters <= 0 || !x || !y) return DS_ERR_ARG;
    if (!s->e->loaded) return fail(s, DS_ERR_STATE, "no LP loaded");
    GUARD(s, {
        s->e->pdhg_estimate(iters, x, y);
        return DS_OK;
    })
}

int ds_set_feature_trace(ds_solver* s, int every, int cap) {
    if (!s || every < 0 || cap < 0 || (every > 0 && cap == 0)) return DS_ERR_ARG;
    s->e->ftr_every = every;
    s->e->ftr_cap = every > 0 ? cap : 0;
    s->e->invalidate_graph();
    return DS_OK;
}

int ds_get_feature_trace(const ds_solver* s, float* feat, int* meta, int* count, int* total) {
    if (!s || !count) return DS_ERR_ARG;
    const Engine* e = s->e;
    const int kept = (int)e->ftr_meta.size() / 3;
    if (feat) std::copy(e->ftr_feat.begin(), e->ftr_feat.end(), feat);
    if (meta) std::copy(e->ftr_meta.begin(), e->ftr_meta.end(), meta);
    *count = kept;
    if (total) *total = e->ftr_total;
    return DS_OK;
}

}  // extern "C"
