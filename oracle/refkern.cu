// TEST INFRASTRUCTURE ONLY: a timing harness for two of the reference's own GPU
// kernels, built for sm_100a from the reference's source file
// (src/gpu/cudaKernels.cu, compiled where it lies by oracle/Makefile into
// oracle/_ref/librefkern.so; nothing of it is copied here).  It gives the
// same-box per-kernel baseline for the engine's replacements:
//
//   spmvUpdateTKernel (cudaKernels.cu:108-157), launched as
//     spmvUpdateInc does for the pivot row (utillities.cu:86-169):
//     256-thread blocks, grid (rows + 255) / 256, alpha = 1, beta = 0;
//   etaSolveKernel (cudaKernels.cu:266-322), launched as PFIfactor's solve
//     does (utillities.cu:320-345): one block of the largest power of two
//     <= min(1024, m) threads.
//
// Each rk_* call copies the inputs to the device, runs `warm` untimed launches,
// then times `reps` launches with CUDA events and returns the mean per launch.
#include <cuda_runtime.h>

// Signatures of the reference kernels (defined in the reference's cudaKernels.cu).
__global__ void spmvUpdateTKernel(double* sol, const double* vec1, const double* vec2, const double* val_csr,
                                  const int* id_csr, const int* ptr_csr, const int* cols_idx, double* buff,
                                  const int cols_idx_size, const int nnz, const int major_dim, const double alpha,
                                  const double beta, const bool set);
__global__ void etaSolveKernel(double* y, const double* x, const double* values, const int* col_id, int size,
                               int col_len, bool transpose);

namespace {

template <typename T>
T* dcopy(const T* h, size_t n) {
    T* d = nullptr;
    if (cudaMalloc(&d, (n ? n : 1) * sizeof(T)) != cudaSuccess) return nullptr;
    if (h && n) cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice);
    else cudaMemset(d, 0, (n ? n : 1) * sizeof(T));
    return d;
}

}  // namespace

extern "C" {

// alpha_N: for the `ncols` target columns of the CSC matrix [A | I] (N columns,
// ptr/idx/val), out[c] = rho^T column(cols[c]).
int rk_pivot_row(int m, int N, const int* ptr, const int* idx, const double* val, const double* rho,
                 const int* cols, int ncols, double* out, int warm, int reps, float* ms) {
    const int nnz = ptr[N];
    int* d_ptr = dcopy(ptr, (size_t)N + 1);
    int* d_idx = dcopy(idx, (size_t)nnz);
    double* d_val = dcopy(val, (size_t)nnz);
    double* d_rho = dcopy(rho, (size_t)m);
    int* d_cols = dcopy(cols, (size_t)ncols);
    double* d_vec2 = dcopy<double>(nullptr, (size_t)N);
    double* d_buff = dcopy<double>(nullptr, (size_t)N);
    double* d_sol = dcopy<double>(nullptr, (size_t)ncols);
    if (!d_ptr || !d_idx || !d_val || !d_rho || !d_cols || !d_vec2 || !d_buff || !d_sol) return -1;
    const int block = 256, grid = (m + block - 1) / block;
    cudaEvent_t a, b;
    cudaEventCreate(&a); cudaEventCreate(&b);
    for (int r = 0; r < warm; ++r)
        spmvUpdateTKernel<<<grid, block>>>(d_sol, d_rho, d_vec2, d_val, d_idx, d_ptr, d_cols, d_buff, ncols, nnz, N,
                                           1.0, 0.0, false);
    cudaEventRecord(a);
    for (int r = 0; r < reps; ++r)
        spmvUpdateTKernel<<<grid, block>>>(d_sol, d_rho, d_vec2, d_val, d_idx, d_ptr, d_cols, d_buff, ncols, nnz, N,
                                           1.0, 0.0, false);
    cudaEventRecord(b);
    cudaError_t e = cudaEventSynchronize(b);
    float t = 0.f;
    cudaEventElapsedTime(&t, a, b);
    *ms = reps > 0 ? t / reps : 0.f;
    if (e == cudaSuccess) e = cudaMemcpy(out, d_sol, sizeof(double) * ncols, cudaMemcpyDeviceToHost);
    cudaEventDestroy(a); cudaEventDestroy(b);
    cudaFree(d_ptr); cudaFree(d_idx); cudaFree(d_val); cudaFree(d_rho); cudaFree(d_cols);
    cudaFree(d_vec2); cudaFree(d_buff); cudaFree(d_sol);
    return e == cudaSuccess ? 0 : -2;
}

// The PFI eta file (T dense columns of m doubles, pivots pos) applied to x,
// forwards (transpose = 0) or backwards (transpose = 1), result in y.
int rk_eta_solve(int m, int T, const double* eta, const int* pos, const double* x, int transpose, double* y,
                 int warm, int reps, float* ms) {
    double* d_eta = dcopy(eta, (size_t)T * m);
    int* d_pos = dcopy(pos, (size_t)T);
    double* d_x = dcopy(x, (size_t)m);
    double* d_y = dcopy<double>(nullptr, (size_t)m);
    if (!d_eta || !d_pos || !d_x || !d_y) return -1;
    const int max_size = m < 1024 ? m : 1024;
    int block = 1;
    while (block * 2 <= max_size) block *= 2;
    cudaEvent_t a, b;
    cudaEventCreate(&a); cudaEventCreate(&b);
    for (int r = 0; r < warm; ++r) etaSolveKernel<<<1, block>>>(d_y, d_x, d_eta, d_pos, T, m, transpose != 0);
    cudaEventRecord(a);
    for (int r = 0; r < reps; ++r) etaSolveKernel<<<1, block>>>(d_y, d_x, d_eta, d_pos, T, m, transpose != 0);
    cudaEventRecord(b);
    cudaError_t e = cudaEventSynchronize(b);
    float t = 0.f;
    cudaEventElapsedTime(&t, a, b);
    *ms = reps > 0 ? t / reps : 0.f;
    if (e == cudaSuccess) e = cudaMemcpy(y, d_y, sizeof(double) * m, cudaMemcpyDeviceToHost);
    cudaEventDestroy(a); cudaEventDestroy(b);
    cudaFree(d_eta); cudaFree(d_pos); cudaFree(d_x); cudaFree(d_y);
    return e == cudaSuccess ? 0 : -2;
}

}  // extern "C"
