// ds_kernel_*: run one engine kernel on caller-supplied host vectors.
//
// These exist for index-selection parity: the same device code that runs
// inside ds_solve is fed identical input vectors to the reference's routines
// (DSEPricing, the ratio test with its bound-flipping loop, dotUpdate, the PFI
// eta file) and its output is compared bit for bit.
#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/ds_api.h"
#include "engine.cuh"
#include "kernels.cuh"

namespace {

using namespace ds;

struct Scratch {
    std::vector<void*> ptrs;
    ~Scratch() { for (void* p : ptrs) cudaFree(p); }
    template <typename T>
    T* alloc(size_t n) {
        void* p = nullptr;
        if (cudaMalloc(&p, (n ? n : 1) * sizeof(T)) != cudaSuccess) return nullptr;
        ptrs.push_back(p);
        cudaMemset(p, 0, (n ? n : 1) * sizeof(T));
        return (T*)p;
    }
    template <typename T>
    T* copy(const T* h, size_t n) {
        T* d = alloc<T>(n);
        if (d && h && n) cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice);
        return d;
    }
};

Ctl* new_ctl(Scratch& s) {
    Ctl* c = s.alloc<Ctl>(1);
    Ctl h;
    std::memset(&h, 0, sizeof(h));
    h.phase = 2; h.ybt_n = -1; h.prev_q = -1; h.max_iter = 1 << 30; h.R = 100; h.top_done = 1;
    cudaMemcpy(c, &h, sizeof(Ctl), cudaMemcpyHostToDevice);
    return c;
}

std::vector<unsigned char> types_u8(const int* t, int n) {
    std::vector<unsigned char> v(n);
    for (int i = 0; i < n; ++i) v[i] = (unsigned char)t[i];
    return v;
}

// Device time of the kernels the last timed ds_kernel_* call launched (this thread).
thread_local double g_last_ms = -1.0;

struct KernelTimer {
    cudaEvent_t a = nullptr, b = nullptr;
    KernelTimer() { cudaEventCreate(&a); cudaEventCreate(&b); cudaEventRecord(a, 0); }
    void stop() {
        cudaEventRecord(b, 0);
        float ms = -1.0f;
        if (cudaEventSynchronize(b) == cudaSuccess && cudaEventElapsedTime(&ms, a, b) == cudaSuccess) g_last_ms = ms;
    }
    ~KernelTimer() { if (a) cudaEventDestroy(a); if (b) cudaEventDestroy(b); }
};

int finish(cudaError_t e) {
    if (e != cudaSuccess) return DS_ERR_CUDA;
    e = cudaDeviceSynchronize();
    return e == cudaSuccess ? DS_OK : DS_ERR_CUDA;
}

}  // namespace

extern "C" {

int ds_kernel_dse_pricing(int m, int N, const int* basis, const double* x, const double* lb,
                          const double* ub, const int* type, const double* beta, int* p, int* p_idx,
                          double* delta, int* is_lower, int* primal_feasible) {
    if (m <= 0 || N < m || !basis || !x || !lb || !ub || !type || !beta) return DS_ERR_ARG;
    Scratch s;
    Dev D{};
    D.m = m; D.n = N - m; D.N = N; D.cap = 8; D.k = 0;
    auto t8 = types_u8(type, N);
    D.basis = s.copy(basis, m);
    D.x = s.copy(x, N); D.lb = s.copy(lb, N); D.ub = s.copy(ub, N);
    D.type = s.copy(t8.data(), N);
    D.beta = s.copy(beta, m);
    const int nbk = (std::max(m, N - m) + 255) / 256 + 8;
    D.red = s.alloc<double>(2 * nbk); D.redi = s.alloc<int>(4 * nbk);
    D.ybt = s.alloc<double>(m); D.ybt_pos = s.alloc<int>(D.cap + 1);
    D.eta = s.alloc<double>(1); D.eta_pos = s.alloc<int>(1); D.Mtri = s.alloc<double>(1);
    D.ctl = new_ctl(s);
    if (init_kernel_attributes(D.cap) != cudaSuccess) return DS_ERR_CUDA;
    if (!D.ctl || !D.ybt) return DS_ERR_CUDA;
    int rc = finish(launch_chuzr_only(D, 0));
    if (rc) return rc;
    Ctl h;
    cudaMemcpy(&h, D.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost);
    *p = h.p; *p_idx = h.p_idx; *delta = h.p_idx >= 0 ? h.delta : 0.0;
    *is_lower = h.p_idx >= 0 ? h.is_lower : 0;
    *primal_feasible = h.primal_feasible;
    return DS_OK;
}

int ds_kernel_pivot_row(int m, int n, const int* csc_ptr, const int* csc_row, const double* csc_val,
                        const int* nonbasis, const double* rho, double* alpha) {
    if (m <= 0 || n <= 0 || !csc_ptr || !nonbasis || !rho || !alpha) return DS_ERR_ARG;
    Scratch s;
    Dev D{};
    D.m = m; D.n = n; D.N = n + m;
    const int nnz = csc_ptr[n];
    D.cptr = s.copy(csc_ptr, n + 1); D.crow = s.copy(csc_row, nnz); D.cval = s.copy(csc_val, nnz);
    D.nonbasis = s.copy(nonbasis, n);
    D.rho = s.copy(rho, m);
    D.alpha = s.alloc<double>(n);
    D.redi = s.alloc<int>(n / 256 + 8);
    D.ctl = new_ctl(s);
    cudaDeviceSynchronize();
    KernelTimer tm;
    cudaError_t le = launch_pivot_row_mode(D, 1, 0);
    tm.stop();
    int rc = finish(le);
    if (rc) return rc;
    cudaMemcpy(alpha, D.alpha, sizeof(double) * n, cudaMemcpyDeviceToHost);
    return DS_OK;
}

int ds_kernel_ratio_test(int n, int N, const int* nonbasis, const double* alpha, double delta,
                         int is_lower, const double* x, const double* d, const double* lb,
                         const double* ub, const int* type, int* q, int* q_idx, double* theta,
                         double* delta_out, int* num_candidates) {
    if (n <= 0 || N < n || !nonbasis || !alpha || !x || !d || !lb || !ub || !type) return DS_ERR_ARG;
    Scratch s;
    Dev D{};
    D.n = n; D.N = N; D.m = N - n;
    auto t8 = types_u8(type, N);
    D.nonbasis = s.copy(nonbasis, n);
    D.alpha = s.copy(alpha, n);
    D.x = s.copy(x, N); D.d = s.copy(d, N); D.lb = s.copy(lb, N); D.ub = s.copy(ub, N);
    D.type = s.copy(t8.data(), N);
    D.theta_arr = s.alloc<double>(n); D.cand = s.alloc<unsigned char>(n);
    D.red = s.alloc<double>(2 * (n / 256 + 8));
    D.redi = s.alloc<int>(2 * (n / 256 + 8));
    D.ctl = new_ctl(s);
    Ctl h;
    cudaMemcpy(&h, D.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost);
    h.delta = delta; h.is_lower = is_lower ? 1 : 0;
    cudaMemcpy(D.ctl, &h, sizeof(Ctl), cudaMemcpyHostToDevice);
    int rc = finish(launch_pivot_row_mode(D, 2, 0));
    if (rc) return rc;
    cudaMemcpy(&h, D.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost);
    *num_candidates = h.ncand;
    if (h.event == EV_UNBOUNDED || h.event == EV_ERROR || h.ncand == 0) {
        *q = -1; *q_idx = -1; *theta = 0.0; *delta_out = (is_lower ? -1.0 : 1.0) * (delta < 0 ? -delta : delta);
        return DS_OK;
    }
    *q = h.q; *q_idx = h.q_idx; *theta = h.theta; *delta_out = h.delta_bfrt;
    return DS_OK;
}

int ds_kernel_pfi_apply(int m, int T, const double* eta, const int* pos, const double* rhs, double* sol,
                        int transpose) {
    if (m <= 0 || T < 0 || T > 200 || !rhs || !sol || (T > 0 && (!eta || !pos))) return DS_ERR_ARG;
    Scratch s;
    Dev D{};
    D.m = m; D.n = 1; D.N = m + 1; D.k = 0; D.cap = T + 1;
    D.eta = s.copy(eta, (size_t)T * m);
    D.eta_pos = s.copy(pos, T);
    D.Mtri = s.alloc<double>((size_t)D.cap * D.cap);
    std::vector<int> ident(m), zeros(m + 1, 0);
    for (int i = 0; i < m; ++i) ident[i] = i;
    D.row_slackpos = s.copy(ident.data(), m);
    D.cpl_ptr = s.copy(zeros.data(), m + 1);
    D.cpl_col = s.alloc<int>(1); D.cpl_val = s.alloc<double>(1);
    D.s_pos = s.alloc<int>(1);
    D.ybt = s.alloc<double>(m); D.ybt_pos = s.alloc<int>(D.cap + 1);
    D.s_eta = s.alloc<double>((size_t)MAX_FTRAN_RHS * D.cap);
    D.red = s.alloc<double>(m / 256 + 8); D.redi = s.alloc<int>(m / 256 + 8);
    double* d_rhs = s.copy(rhs, m);
    double* d_out = s.alloc<double>(m);
    double* d_y0 = s.alloc<double>(m);
    double* d_h = s.alloc<double>(D.cap);
    D.y0[0] = d_y0; D.frhs[0] = d_rhs; D.fout[0] = d_out;
    D.ctl = new_ctl(s);
    if (init_kernel_attributes(D.cap) != cudaSuccess) return DS_ERR_CUDA;
    cudaError_t e = launch_build_mtri(D, T, 0);   // the eta file's G, kept between iterations by the engine
    cudaDeviceSynchronize();
    KernelTimer tm;
    if (e == cudaSuccess) {
        if (!transpose) e = launch_ftran(D, 1, 0, 1, 0);
        else {
            e = launch_btran_dense_eta(D, d_rhs, d_h, T, 0);
            if (e == cudaSuccess) e = launch_btran_b0(D, d_out, 1, 0);
        }
    }
    tm.stop();
    int rc = finish(e);
    if (rc) return rc;
    cudaMemcpy(sol, d_out, sizeof(double) * m, cudaMemcpyDeviceToHost);
    return DS_OK;
}

int ds_kernel_last_time(double* ms) {
    if (!ms) return DS_ERR_ARG;
    *ms = g_last_ms;
    return g_last_ms >= 0.0 ? DS_OK : DS_ERR_STATE;
}

}  // extern "C"
