// Refactorisation of the basis on the device (replaces the reference's cuDSS LU,
// cudaSparseMatrix.cpp:502-567, called from CudaDualSimplex::reFactorize,
// cudaDualSimplex.cpp:229-238).
//
// The basis B0 = [A_S | I_R] has unit columns for its basic slacks, so only the
// structural block K = A[R', S] (k x k, R' = rows whose slack is nonbasic) needs
// a factorisation.  K is inverted in place by blocked Gauss-Jordan elimination
// with partial pivoting, NB columns per panel:
//   k_gj_panel   one block: tall-skinny LU of the panel over the not-yet-pivoted
//                rows picks the NB pivot rows; W^-1 of the pivot block
//   k_gj_rows    pivot rows of the other columns:  S[P, J] <- W^-1 S[P, J]
//   k_gj_update  rank-NB update of the other rows:  S[I, J] -= Pan[I, :] S[P, J],
//                and the panel columns become the inverse's columns
// No rows are swapped physically; a final gather (k_gj_permute) writes Kinv in
// natural order.
#include <cmath>
#include <mutex>

#include "engine.cuh"
#include "kernels.cuh"

namespace ds {

constexpr int GJ_NB = 16;

__global__ void k_fill_zero(double* p, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] = 0.0;
}

// K[t + j k] = A[rp_row[t], s_var[j]] using row_kidx (row -> t or -1).
__global__ void k_build_K(const int* cptr, const int* crow, const double* cval, const int* s_var,
                          const int* row_kidx, int k, double* S) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= k) return;
    const int v = s_var[j];
    for (int e = cptr[v]; e < cptr[v + 1]; ++e) {
        const int t = row_kidx[crow[e]];
        if (t >= 0) S[(size_t)t + (size_t)j * k] = cval[e];
    }
}

// One block.  Pan <- S[:, c0:c0+w]; LU of a working copy over the rows not yet
// pivoted picks the pivot rows; Winv <- (Pan[pivot rows, :])^-1 by unpivoted
// Gauss-Jordan (its pivots are the LU's, hence the partial-pivoting choices).
// SMEM: the working copy (k x w) and the pivoted-row flags live in shared
// memory (k <= GJ_SMEM_ROWS); otherwise in global memory.
constexpr int GJ_SMEM_ROWS = 1600;
template <int BS, bool SMEM>
__global__ void k_gj_panel(double* S, int k, int c0, int w, double* Pan, double* Wk_g, int* rowpiv,
                           int* piv_rows, double* Winv, int* err) {
    if (*(volatile int*)err) return;   // an earlier panel found the matrix singular
    extern __shared__ double sh[];
    __shared__ double red_v[BS / 32];
    __shared__ int red_i[BS / 32];
    __shared__ int s_r;
    __shared__ double prow[GJ_NB];
    __shared__ double W[GJ_NB][GJ_NB + 1];
    __shared__ double Wi[GJ_NB][GJ_NB + 1];
    double* Wk = SMEM ? sh : Wk_g;
    unsigned char* piv = SMEM ? (unsigned char*)(sh + (size_t)k * GJ_NB) : nullptr;
    for (int r = threadIdx.x; r < k; r += BS) {
        if (SMEM) piv[r] = rowpiv[r] >= 0 ? 1 : 0;
        double v[GJ_NB];
#pragma unroll
        for (int a = 0; a < GJ_NB; ++a) v[a] = (a < w) ? S[(size_t)r + (size_t)(c0 + a) * k] : 0.0;
#pragma unroll
        for (int a = 0; a < GJ_NB; ++a)
            if (a < w) { Pan[(size_t)r + (size_t)a * k] = v[a]; Wk[(size_t)r + (size_t)a * k] = v[a]; }
    }
    __syncthreads();
    for (int a = 0; a < w; ++a) {
        double best = -1.0; int bi = -1;
        for (int r = threadIdx.x; r < k; r += BS) {
            if (SMEM ? piv[r] : (rowpiv[r] >= 0)) continue;
            const double v = fabs(Wk[(size_t)r + (size_t)a * k]);
            if (v > best || (v == best && bi >= 0 && r < bi)) { best = v; bi = r; }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_down_sync(0xffffffffu, best, o);
            const int oi = __shfl_down_sync(0xffffffffu, bi, o);
            if (ov > best || (ov == best && oi >= 0 && (bi < 0 || oi < bi))) { best = ov; bi = oi; }
        }
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        if (lane == 0) { red_v[wid] = best; red_i[wid] = bi; }
        __syncthreads();
        if (threadIdx.x == 0) {
            double bv = -1.0; int b = -1;
            for (int u = 0; u < BS / 32; ++u)
                if (red_v[u] > bv || (red_v[u] == bv && red_i[u] >= 0 && (b < 0 || red_i[u] < b))) { bv = red_v[u]; b = red_i[u]; }
            if (b < 0 || !(bv > 1e-300)) { *err = c0 + a + 1; b = -1; }
            else {
                rowpiv[b] = c0 + a; piv_rows[c0 + a] = b;
                if (SMEM) piv[b] = 1;
            }
            s_r = b;
        }
        __syncthreads();
        const int pr = s_r;
        if (pr < 0) return;
        if (threadIdx.x < w) prow[threadIdx.x] = Wk[(size_t)pr + (size_t)threadIdx.x * k];
        __syncthreads();
        const double pv = prow[a];
        for (int r = threadIdx.x; r < k; r += BS) {
            if (SMEM ? piv[r] : (rowpiv[r] >= 0)) continue;
            const double l = Wk[(size_t)r + (size_t)a * k] / pv;
            if (l != 0.0)
                for (int b = a + 1; b < w; ++b) Wk[(size_t)r + (size_t)b * k] -= l * prow[b];
        }
        __syncthreads();
    }
    // W = Pan[pivot rows, :], Gauss-Jordan in shared memory
    for (int e = threadIdx.x; e < w * w; e += BS) {
        const int a = e / w, b = e % w;
        W[a][b] = Pan[(size_t)piv_rows[c0 + a] + (size_t)b * k];
        Wi[a][b] = (a == b) ? 1.0 : 0.0;
    }
    __syncthreads();
    for (int a = 0; a < w; ++a) {
        const double pv = W[a][a];
        __syncthreads();
        if (threadIdx.x < w) { W[a][threadIdx.x] /= pv; }
        else if (threadIdx.x < 2 * w) { Wi[a][threadIdx.x - w] /= pv; }
        __syncthreads();
        for (int e = threadIdx.x; e < w * w; e += BS) {
            const int r = e / w, b = e % w;
            if (r == a) continue;
            const double f = W[r][a];
            if (b != a) W[r][b] -= f * W[a][b];
            Wi[r][b] -= f * Wi[a][b];
        }
        __syncthreads();
        for (int r = threadIdx.x; r < w; r += BS) if (r != a) W[r][a] = 0.0;
        __syncthreads();
    }
    for (int e = threadIdx.x; e < w * w; e += BS) {
        const int a = e / w, b = e % w;
        Winv[a * GJ_NB + b] = Wi[a][b];
    }
}

// S[P, j] <- Winv S[P, j] for every column j outside the panel: a group of
// GJ_NB threads per column, thread a loading pivot row a's entry and forming
// row a of the product (the sum over b in order, as a single thread would).
__global__ void k_gj_rows(double* S, int k, int c0, int w, const int* piv_rows, const double* Winv, const int* err) {
    if (*err) return;   // singular: the pivot rows of this panel were not all chosen
    const int j = (int)((blockIdx.x * blockDim.x + threadIdx.x) / GJ_NB);
    const int a = (int)(threadIdx.x % GJ_NB);
    const unsigned mask = 0xffffu << (threadIdx.x & 16);   // this column's half-warp
    if (j >= k || (j >= c0 && j < c0 + w)) return;        // whole groups leave together
    double* col = S + (size_t)j * k;
    const int pr = (a < w) ? piv_rows[c0 + a] : 0;
    const double va = (a < w) ? col[pr] : 0.0;
    double s = 0.0;
    for (int b = 0; b < w; ++b) s += Winv[a * GJ_NB + b] * __shfl_sync(mask, va, b, GJ_NB);
    if (a < w) col[pr] = s;
}

// 32 x 32 tiles: rows on threadIdx.x (coalesced in column-major S), columns on y.
__global__ void k_gj_update(double* S, int k, int c0, int w, const double* Pan, const int* rowpiv,
                            const int* piv_rows, const double* Winv, const int* err) {
    if (*err) return;
    __shared__ double sp[32][GJ_NB + 1];   // Pan rows of the tile
    __shared__ double sq[GJ_NB][33];       // S[P, tile columns] or Winv
    const int i = blockIdx.x * 32 + threadIdx.x;
    const int j = blockIdx.y * 32 + threadIdx.y;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    for (int e = tid; e < 32 * w; e += 1024) {
        const int rr = e % 32, a = e / 32;
        const int gi = blockIdx.x * 32 + rr;
        sp[rr][a] = (gi < k) ? Pan[(size_t)gi + (size_t)a * k] : 0.0;
    }
    for (int e = tid; e < 32 * w; e += 1024) {
        const int cc = e % 32, a = e / 32;
        const int gj = blockIdx.y * 32 + cc;
        double v = 0.0;
        if (gj < k) {
            if (gj >= c0 && gj < c0 + w) v = Winv[a * GJ_NB + (gj - c0)];
            else v = S[(size_t)piv_rows[c0 + a] + (size_t)gj * k];
        }
        sq[a][cc] = v;
    }
    __syncthreads();
    if (i >= k || j >= k) return;
    const int rp = rowpiv[i];
    const bool pivot_row_now = (rp >= c0 && rp < c0 + w);
    const bool panel_col = (j >= c0 && j < c0 + w);
    double* dst = S + (size_t)i + (size_t)j * k;
    if (pivot_row_now) {
        if (panel_col) *dst = sq[rp - c0][threadIdx.y];   // Winv[a][b]
        return;                                           // other columns set by k_gj_rows
    }
    double s = 0.0;
    for (int a = 0; a < w; ++a) s += sp[threadIdx.x][a] * sq[a][threadIdx.y];
    if (panel_col) *dst = -s;
    else *dst = *dst - s;
}

// Kinv(c, piv_rows[c2]) = S(piv_rows[c], c2)
__global__ void k_gj_permute(const double* S, int k, const int* piv_rows, double* Kinv, const int* err) {
    if (*err) return;
    const int c = blockIdx.x * 32 + threadIdx.x;
    const int c2 = blockIdx.y * 32 + threadIdx.y;
    if (c >= k || c2 >= k) return;
    Kinv[(size_t)c + (size_t)piv_rows[c2] * k] = S[(size_t)piv_rows[c] + (size_t)c2 * k];
}

// Gauss-Jordan inverse of the k x k matrix in F.S (column major), written to out.
cudaError_t gj_inverse(const FactorBufs& F, int k, double* out, cudaStream_t s) {
    if (k == 0) return cudaSuccess;
    cudaMemsetAsync(F.rowpiv, 0xff, sizeof(int) * k, s);
    cudaMemsetAsync(F.piv_rows, 0, sizeof(int) * k, s);   // in range even where a singular panel stops early
    cudaMemsetAsync(F.err, 0, sizeof(int), s);
    const bool smem = k <= GJ_SMEM_ROWS;
    const size_t psh = smem ? (size_t)k * GJ_NB * sizeof(double) + (size_t)k : 0;
    if (smem) {
        // process-wide attribute: raised once to the largest panel (other threads launch concurrently)
        static std::once_flag once;
        static cudaError_t attr = cudaSuccess;
        std::call_once(once, [] {
            attr = cudaFuncSetAttribute(k_gj_panel<512, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)((size_t)GJ_SMEM_ROWS * GJ_NB * sizeof(double) + GJ_SMEM_ROWS));
        });
        if (attr != cudaSuccess) return attr;
    }
    for (int c0 = 0; c0 < k; c0 += GJ_NB) {
        const int w = (k - c0 < GJ_NB) ? (k - c0) : GJ_NB;
        if (smem) k_gj_panel<512, true><<<1, 512, psh, s>>>(F.S, k, c0, w, F.Pan, F.Wk, F.rowpiv, F.piv_rows, F.Winv, F.err);
        else k_gj_panel<512, false><<<1, 512, 0, s>>>(F.S, k, c0, w, F.Pan, F.Wk, F.rowpiv, F.piv_rows, F.Winv, F.err);
        k_gj_rows<<<(k * GJ_NB + 255) / 256, 256, 0, s>>>(F.S, k, c0, w, F.piv_rows, F.Winv, F.err);
        dim3 g((k + 31) / 32, (k + 31) / 32), b(32, 32);
        k_gj_update<<<g, b, 0, s>>>(F.S, k, c0, w, F.Pan, F.rowpiv, F.piv_rows, F.Winv, F.err);
    }
    dim3 g((k + 31) / 32, (k + 31) / 32), b(32, 32);
    k_gj_permute<<<g, b, 0, s>>>(F.S, k, F.piv_rows, out, F.err);
    count_launch(1 + 3 * ((k + GJ_NB - 1) / GJ_NB));
    return cudaGetLastError();
}

cudaError_t factor_bump(const FactorBufs& F, const Dev& D, int k, cudaStream_t s) {
    if (k == 0) return cudaSuccess;
    const size_t kk = (size_t)k * k;
    k_fill_zero<<<1184, 256, 0, s>>>(F.S, kk);
    k_build_K<<<(k + 255) / 256, 256, 0, s>>>(D.cptr, D.crow, D.cval, F.s_var, F.row_kidx, k, F.S);
    count_launch(2);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return gj_inverse(F, k, D.Kinv, s);
}

}  // namespace ds
