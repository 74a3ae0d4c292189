// Sparse LU of the basis's structural block (eta-file mode), the counterpart of
// the reference's cuDSS factorisation (cudaSparseMatrix.cpp:502-567, called by
// CudaDualSimplex::reFactorize, cudaDualSimplex.cpp:229-238) and of its solves
// (cudaSparseMatrix.cpp:570-605).
#pragma once
#include <vector>

#include <cuda_runtime.h>

#include "engine.cuh"
#include "host_util.cuh"

namespace ds {

struct SfInput {
    int m, n, k;
    // host copy of the structural CSC of A (the device holds the same arrays)
    const int* cptr; const int* crow; const double* cval;
    long long nnzA;
    const int* s_var;      // k: K column -> variable
    const int* s_pos;      // k: K column -> basis position
    const int* rp_row;     // k: K row -> constraint row
    const int* row_kidx;   // m: constraint row -> K row or -1
};

struct SfInfo {
    int singular = 0;          // 1: the bump is singular (structurally or numerically)
    int km = 0;                // kernel order after the singleton triangularisation
    int ks = 0;                // kernel pivots taken by the sparse Markowitz rounds
    int kd = 0;                // order of the dense block that remained
    int rounds = 0;            // Markowitz rounds
    int lnnz = 0, unnz = 0;    // kernel L and U entries
    int dense_fallback = 0;    // 1: the kernel's work area overflowed and it was factorised dense
    int lev_ft = 0, lev_bt = 0;
    long long ent_ft = 0, ent_bt = 0, op_ft = 0, op_bt = 0;
    float kernel_ms = 0.f;     // device time of the kernel factorisation and the dense block inverse
    char msg[160] = {0};
};

// Singleton triangularisation of the bump's pattern (sparse_factor.cu).
struct Triangular {
    std::vector<int> u1_t, u1_j, u1_e;   // column singletons: row, column, CSC entry (pivot order)
    std::vector<int> u3_t, u3_j, u3_e;   // row singletons: row, column, CSR entry (peel order)
    std::vector<char> rdone, cdone;      // rows / columns pivoted (the rest is the kernel)
};
const char* triangularise(int k, const int* kc_ptr, const int* kc_row, const int* kr_ptr, const int* kr_col,
                          Triangular& T);

class SparseLU {
public:
    SparseLU() = default;
    SparseLU(const SparseLU&) = delete;
    SparseLU& operator=(const SparseLU&) = delete;
    ~SparseLU() {
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
    }
    // Factorise the bump given by `in` (values from d_cval, the device CSC
    // values of A) and fill `out` with the solve programs.  Synchronises `s`.
    SfInfo factor(const SfInput& in, const double* d_cval, cudaStream_t s, SfDev* out);

private:
    // kernel Markowitz work area
    DBuf<int> k_row_ptr, k_row_col, k_r_start, k_r_len, k_r_cap, k_c_ptr, k_c_cur, k_c_row;
    DBuf<long long> k_row_src;
    DBuf<int> k_pool_col, k_cand_row, k_cand_cost, k_col_piv, k_row_piv;
    DBuf<double> k_pool_val, k_cand_val, k_L_val;
    DBuf<unsigned char> k_cand_ok;
    DBuf<unsigned long long> k_row_key;
    DBuf<int> k_piv_row, k_piv_col, k_piv_uidx, k_piv_ulen, k_L_row, k_L_piv, k_dense_row, k_dense_col, k_out;
    // dense block (Gauss-Jordan)
    DBuf<double> g_S, g_Pan, g_Wk, g_Winv, g_Sinv, g_SinvT;
    DBuf<int> g_rowpiv, g_pivrows, g_err;
    // programs
    DBuf<int> p_slot_row, p_slot_kcol, p_slot_pos;
    DBuf<int> p_lvl_ptr[2], p_lvl_kind[2], p_op_slot[2], p_op_ptr[2], p_ent_slot[2];
    DBuf<long long> p_diag_src[2], p_ent_src[2];
    DBuf<double> p_op_diag[2], p_ent_coef[2];
    DBuf<double> p_gvec, p_gtmp;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    long long pool_hint = 0;   // work-area size the last overflowing factorisation grew to
};

}  // namespace ds
