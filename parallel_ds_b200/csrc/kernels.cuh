// Launchers of the engine's kernels (host-callable, stream ordered).
#pragma once
#include <cuda_runtime.h>

#include "engine.cuh"

namespace ds {

struct FactorBufs {
    double* S;        // k*k work array (in-place inverse before the final gather)
    double* Pan;      // k * NB panel copy
    double* Wk;       // k * NB working panel
    int* rowpiv;      // k
    int* piv_rows;    // k
    double* Winv;     // NB * NB
    int* err;         // 1
    int* s_var;       // k (device copy)
    int* row_kidx;    // m: row -> K row index or -1
};

cudaError_t factor_bump(const FactorBufs& F, const Dev& D, int k, cudaStream_t s);
// Gauss-Jordan inverse of the k x k column-major matrix already in F.S, written to out.
cudaError_t gj_inverse(const FactorBufs& F, int k, double* out, cudaStream_t s);

// Kernels of one iteration, in launch order.
// PFI mode runs S_BTRAN_RHS .. S_ETA_APPLY; dense mode runs S_FTRAN_DENSE and S_BINV
// instead (step_active tells which).
enum Step : int { S_SCORE = 0, S_CHUZR, S_BTRAN_RHS, S_BTRAN_GEMV, S_PIVOT_ROW, S_DUAL_UPDATE,
                  S_FTRAN_K, S_FTRAN_ASM, S_ETA_APPLY, S_FTRAN_DENSE, S_UPDATE, S_BINV, S_NSTEPS };
bool step_active(const Dev& D, int step);
extern const char* const kStepNames[S_NSTEPS];
cudaError_t launch_step(const Dev& D, int step, cudaStream_t s);
// S_SCORE: network scores (learned pricing) and/or the feature trace; no
// launch when neither is on (mlp.cu).
bool score_step_active(const Dev& D);
cudaError_t launch_score(const Dev& D, cudaStream_t s);

// Programmatic dependent launch: the iteration kernels are launched with
// programmatic stream serialisation, so a kernel's CTAs become resident while
// its predecessor still runs and start the moment it completes (its memory
// visible).  Each such kernel begins with pdl_enter(); launched without the
// attribute, the two instructions do nothing.
// k_binv_update tiling: rows of B^-1 per warp and per 256-thread block.
constexpr int BINV_RW = 32;
constexpr int BINV_ROWS = 8 * BINV_RW;

#ifdef __CUDACC__
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}
#endif
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              Args... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// Kernel launch accounting (graph replays are added by the caller).
void count_launch(int nk);
void set_launch_counting(bool on);
long long launch_count();

cudaError_t init_kernel_attributes(int cap);
cudaError_t launch_body(const Dev& D, int from_stage, cudaStream_t s);
cudaError_t launch_iteration(const Dev& D, cudaStream_t s);
cudaError_t launch_update_forced(const Dev& D, cudaStream_t s);
cudaError_t launch_dual_check(const Dev& D, cudaStream_t s);
cudaError_t launch_count_dual_inf(const Dev& D, cudaStream_t s);
cudaError_t launch_btran_b0(const Dev& D, double* out, int force, cudaStream_t s);
cudaError_t launch_ftran(const Dev& D, int nr_fixed, int check, int force, cudaStream_t s);
cudaError_t launch_set_primal_vars(const Dev& D, cudaStream_t s);
cudaError_t launch_xb_rhs(const Dev& D, double* rhs, cudaStream_t s);
cudaError_t launch_scatter_basic(const Dev& D, const double* xb, double* dst, cudaStream_t s);
cudaError_t launch_gather_basic_cost(const Dev& D, double* cb, cudaStream_t s);
cudaError_t launch_reduced_costs(const Dev& D, const double* y, cudaStream_t s);
cudaError_t launch_btran_dense_eta(const Dev& D, const double* c0, double* h, int T, cudaStream_t s);
cudaError_t launch_btran_unit(const Dev& D, int p_idx, cudaStream_t s);
cudaError_t launch_norm2(const double* v, int n, double* out, cudaStream_t s);
// Exact DSE weights of B0 (valid with an empty eta file).
cudaError_t launch_beta_exact(const Dev& D, cudaStream_t s);
cudaError_t launch_dot_cost_x(const Dev& D, double* out, cudaStream_t s);
cudaError_t launch_phase1_init(const Dev& D, double* cc, cudaStream_t s);

// Single-kernel entry points used by the ds_kernel_* C ABI (kernel_api.cu).
cudaError_t launch_chuzr_only(const Dev& D, cudaStream_t s);
// mode bit 1: compute alpha from rho (else alpha is given); bit 2: run CHUZC.
cudaError_t launch_pivot_row_mode(const Dev& D, int mode, cudaStream_t s);
cudaError_t launch_build_mtri(const Dev& D, int T, cudaStream_t s);

// Dense mode (explicit B^-1).
cudaError_t launch_binv_build(const Dev& D, cudaStream_t s);             // after factor_bump
cudaError_t launch_dense_rho(const Dev& D, int p_idx, cudaStream_t s);   // rho = row p_idx of B^-1
cudaError_t launch_ftran_dense(const Dev& D, int check, int force, cudaStream_t s);
cudaError_t launch_binv_update(const Dev& D, int force, cudaStream_t s);
cudaError_t launch_dense_ftran_vec(const Dev& D, const double* v, double* y, cudaStream_t s);  // y = B^-1 v
// out[0] = max |B (B^-1 v) - v| for a fixed probe v, out[1] = max |B^-1 v| (bit patterns of doubles)
cudaError_t launch_binv_probe(const Dev& D, double* v, double* y, unsigned long long* out, cudaStream_t s);
cudaError_t launch_dense_btran_vec(const Dev& D, const double* c, double* y, cudaStream_t s);  // y = B^-T c
cudaError_t launch_dense_beta(const Dev& D, cudaStream_t s);             // exact DSE weights

}  // namespace ds
