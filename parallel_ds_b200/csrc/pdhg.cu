// First-order estimate of an optimal primal-dual pair, the warm-start evidence
// of the learned leaving-row scorer.  No counterpart in the reference.
//
// Primal-dual hybrid gradient (Chambolle & Pock 2011) for
//     min c^T x   s.t.  L <= A x <= U,  lo <= x <= hi
// with the diagonal step sizes of Pock & Chambolle (ICCV 2011, alpha = 1):
// tau_j = 1 / sum_i |A_ij|, sigma_i = 1 / sum_j |A_ij|, and a restart to the
// running average every R iterations:
//     x+   = clip(x - tau (c + A^T y), lo, hi)
//     xbar = 2 x+ - x
//     v    = y + sigma (A xbar)
//     y+   = v - sigma clip(v / sigma, L, U)        (Moreau identity)
// Bounds follow the variable types (a type without a lower or upper bound
// gets -inf / +inf).  Row activity bounds come from the slack s = -A x.
//
// One warp per column (A^T y over the CSC) and one warp per row (A xbar over
// the CSR); lanes stride the nonzeros and reduce with shuffles in a fixed
// order, so results are deterministic.  One restart period (2R kernels) is
// captured once per LP as a CUDA graph and replayed; the restart itself sits
// at the period's ends (x restarts in the first primal step, y in the last
// dual step), so every replay is the same graph.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>

#include "../../include/ds_api.h"
#include "engine.cuh"
#include "kernels.cuh"
#include "pdhg.cuh"

namespace ds {

constexpr int PD_BS = 256;
constexpr int PD_WARPS = PD_BS / 32;

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double clipd(double v, double lo, double hi) { return fmin(fmax(v, lo), hi); }

// Primal step for column j (one warp).  restart: x <- xsum / R first.
__global__ void __launch_bounds__(PD_BS) k_pdhg_primal(PdhgDev P, int restart) {
    const int j = blockIdx.x * PD_WARPS + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (j >= P.n) return;
    double acc = 0.0;
    for (int e = P.cptr[j] + lane; e < P.cptr[j + 1]; e += 32) acc += P.cval[e] * P.y[P.crow[e]];
    acc = warp_sum(acc);
    if (lane == 0) {
        double x = P.x[j];
        if (restart) { x = P.xsum[j] / P.R; P.xsum[j] = 0.0; }
        const double xn = clipd(x - P.tau[j] * (P.c[j] + acc), P.lo[j], P.hi[j]);
        P.xbar[j] = 2.0 * xn - x;
        P.x[j] = xn;
        P.xsum[j] += xn;
    }
}

// Dual step for row r (one warp).  restart: y <- ysum / R afterwards.
__global__ void __launch_bounds__(PD_BS) k_pdhg_dual(PdhgDev P, int restart) {
    const int r = blockIdx.x * PD_WARPS + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (r >= P.m) return;
    double acc = 0.0;
    for (int e = P.rptr[r] + lane; e < P.rptr[r + 1]; e += 32) acc += P.rval[e] * P.xbar[P.rcol[e]];
    acc = warp_sum(acc);
    if (lane == 0) {
        const double s = P.sigma[r];
        const double v = P.y[r] + s * acc;
        double yn = v - s * clipd(v / s, P.L[r], P.U[r]);
        const double sum = P.ysum[r] + yn;
        if (restart) { yn = sum / P.R; P.ysum[r] = 0.0; }
        else P.ysum[r] = sum;
        P.y[r] = yn;
    }
}

// Start point: x = clip(0, lo, hi) with xsum = R x (so the first restart is a
// no-op), y = 0.
__global__ void k_pdhg_init(PdhgDev P) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < P.n) {
        const double x0 = clipd(0.0, P.lo[i], P.hi[i]);
        P.x[i] = x0; P.xbar[i] = x0; P.xsum[i] = P.R * x0;
    }
    if (i < P.m) { P.y[i] = 0.0; P.ysum[i] = 0.0; }
}

__global__ void k_pdhg_finish(PdhgDev P) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < P.n) { P.x[j] = P.xsum[j] / P.R; P.xsum[j] = 0.0; }
}

// Per-variable evidence for the scorer: the distance to the nearest finite
// bound (structural: x_j; slack of row r: the row activity) and the dual
// magnitude (structural: |c_j + A_j^T y|; slack: |y_r|), one warp per variable.
__global__ void __launch_bounds__(PD_BS) k_pdhg_evidence(PdhgDev P, float* gap, float* dual) {
    const int v = blockIdx.x * PD_WARPS + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (v >= P.n + P.m) return;
    double acc = 0.0;
    if (v < P.n) {
        for (int e = P.cptr[v] + lane; e < P.cptr[v + 1]; e += 32) acc += P.cval[e] * P.y[P.crow[e]];
    } else {
        const int r = v - P.n;
        for (int e = P.rptr[r] + lane; e < P.rptr[r + 1]; e += 32) acc += P.rval[e] * P.x[P.rcol[e]];
    }
    acc = warp_sum(acc);
    if (lane) return;
    double val, lo, hi, du;
    if (v < P.n) { val = P.x[v]; lo = P.lo[v]; hi = P.hi[v]; du = P.c[v] + acc; }
    else { const int r = v - P.n; val = acc; lo = P.L[r]; hi = P.U[r]; du = P.y[r]; }
    const double g = fmin(val - lo, hi - val);      // +inf when both bounds are infinite
    gap[v] = (float)fmin(g, 1e30);
    dual[v] = (float)fabs(du);
}

// ---------------------------------------------------------------- one cluster
// The whole PDHG run in one thread-block cluster of CL CTAs when the LP fits its
// shared memory: CTA r owns columns [r nc, (r+1) nc) and rows [r nr, (r+1) nr)
// with their CSC / CSR slices, steps and bounds, and keeps a replica of all of
// xbar and y.  After its half step a CTA writes its new values into every
// replica (distributed shared memory stores), then a hardware cluster barrier
// separates the half steps.  Same iteration and restarts as the graph path;
// each column / row is summed by one thread in storage order.
namespace cg = cooperative_groups;

__host__ __device__ inline size_t pdhg_cluster_smem(int m, int n, int nc, int nr, int nzc_cap, int nzr_cap) {
    return 8 * ((size_t)n + m + 6 * (size_t)nc + 4 * (size_t)nr + nzc_cap + nzr_cap) +
           4 * ((size_t)nc + 1 + nzc_cap + (size_t)nr + 1 + nzr_cap);
}

template <int BS>
__global__ void __launch_bounds__(BS) k_pdhg_cluster(PdhgDev P, PdhgClusterGeom G, int periods) {
    cg::cluster_group cl = cg::this_cluster();
    const int r = (int)cl.block_rank();
    const int CL = G.CL, nc = G.nc, nr = G.nr, m = P.m, n = P.n, R = P.R;
    extern __shared__ double sm[];
    double* xbar = sm;                  // n: replica of xbar
    double* yf = xbar + n;              // m: replica of y
    double* x = yf + m;                 // own columns
    double* xs = x + nc;
    double* tau = xs + nc;
    double* lo = tau + nc;
    double* hi = lo + nc;
    double* cv = hi + nc;               // costs
    double* ys = cv + nc;               // own rows
    double* sig = ys + nr;
    double* Lr = sig + nr;
    double* Ur = Lr + nr;
    double* aval = Ur + nr;             // CSC values of own columns (nzc_cap)
    double* rval = aval + G.nzc_cap;    // CSR values of own rows (nzr_cap)
    int* cpl = reinterpret_cast<int*>(rval + G.nzr_cap);   // nc + 1
    int* crw = cpl + nc + 1;                                 // nzc_cap
    int* rpl = crw + G.nzc_cap;                              // nr + 1
    int* rcl = rpl + nr + 1;                                 // nzr_cap
    const int j0 = min(n, r * nc), j1 = min(n, j0 + nc), i0 = min(m, r * nr), i1 = min(m, i0 + nr);
    const int nj = j1 - j0, ni = i1 - i0;
    const int t = threadIdx.x;
    // ---- load the slices and the start point
    const int ec = P.cptr[j0], er = P.rptr[i0];
    for (int k = t; k <= nj; k += BS) cpl[k] = P.cptr[j0 + k] - ec;
    for (int k = t; k < P.cptr[j1] - ec; k += BS) { crw[k] = P.crow[ec + k]; aval[k] = P.cval[ec + k]; }
    for (int k = t; k <= ni; k += BS) rpl[k] = P.rptr[i0 + k] - er;
    for (int k = t; k < P.rptr[i1] - er; k += BS) { rcl[k] = P.rcol[er + k]; rval[k] = P.rval[er + k]; }
    for (int k = t; k < nj; k += BS) {
        const int j = j0 + k;
        tau[k] = P.tau[j]; lo[k] = P.lo[j]; hi[k] = P.hi[j]; cv[k] = P.c[j];
        const double x0 = clipd(0.0, lo[k], hi[k]);
        x[k] = x0; xs[k] = R * x0;
    }
    for (int k = t; k < ni; k += BS) { sig[k] = P.sigma[i0 + k]; Lr[k] = P.L[i0 + k]; Ur[k] = P.U[i0 + k]; ys[k] = 0.0; }
    for (int k = t; k < m; k += BS) yf[k] = 0.0;
    cl.sync();
    for (int pp = 0; pp < periods; ++pp) {
        for (int it = 0; it < R; ++it) {
            for (int k = t; k < nj; k += BS) {        // primal half step, own columns
                double acc = 0.0;
                for (int e = cpl[k]; e < cpl[k + 1]; ++e) acc += aval[e] * yf[crw[e]];
                double xo = x[k];
                if (it == 0) { xo = xs[k] / R; xs[k] = 0.0; }
                const double xn = clipd(xo - tau[k] * (cv[k] + acc), lo[k], hi[k]);
                const double xb = 2.0 * xn - xo;
                x[k] = xn;
                xs[k] += xn;
                for (int q = 0; q < CL; ++q) *cl.map_shared_rank(&xbar[j0 + k], q) = xb;
            }
            cl.sync();
            for (int k = t; k < ni; k += BS) {        // dual half step, own rows
                double acc = 0.0;
                for (int e = rpl[k]; e < rpl[k + 1]; ++e) acc += rval[e] * xbar[rcl[e]];
                const double s = sig[k];
                const double v = yf[i0 + k] + s * acc;
                double yn = v - s * clipd(v / s, Lr[k], Ur[k]);
                const double sum = ys[k] + yn;
                if (it == R - 1) { yn = sum / R; ys[k] = 0.0; }
                else ys[k] = sum;
                for (int q = 0; q < CL; ++q) *cl.map_shared_rank(&yf[i0 + k], q) = yn;
            }
            cl.sync();
        }
    }
    // the pending restart of x, and the results for the evidence kernel
    for (int k = t; k < nj; k += BS) { P.x[j0 + k] = xs[k] / R; P.xsum[j0 + k] = 0.0; }
    for (int k = t; k < ni; k += BS) P.y[i0 + k] = yf[i0 + k];
}

constexpr int PD_CL = 16;
constexpr int PD_CL_BS = 256;
constexpr size_t PD_CL_SMEM_MAX = 220 * 1024;

// Cluster geometry of an LP, or CL = 0 when it does not fit.
PdhgClusterGeom pdhg_cluster_geometry(int m, int n, const int* cptr, const int* rptr) {
    PdhgClusterGeom G{0, 0, 0, 0, 0, 0};
    const int nc = (n + PD_CL - 1) / PD_CL, nr = (m + PD_CL - 1) / PD_CL;
    if (nc > PD_CL_BS * 4 || nr > PD_CL_BS * 4) return G;
    int zc = 0, zr = 0;
    for (int r = 0; r < PD_CL; ++r) {
        const int j0 = std::min(n, r * nc), j1 = std::min(n, j0 + nc);
        const int i0 = std::min(m, r * nr), i1 = std::min(m, i0 + nr);
        zc = std::max(zc, cptr[j1] - cptr[j0]);
        zr = std::max(zr, rptr[i1] - rptr[i0]);
    }
    const size_t smem = pdhg_cluster_smem(m, n, nc, nr, zc, zr);
    if (smem > PD_CL_SMEM_MAX) return G;
    G = PdhgClusterGeom{PD_CL, nc, nr, zc, zr, smem};
    return G;
}

// The cluster run: false (nothing launched) when the device cannot place the cluster.
bool launch_pdhg_cluster(const PdhgDev& P, const PdhgClusterGeom& G, int periods, cudaStream_t s) {
    if (G.CL == 0) return false;
    auto kern = k_pdhg_cluster<PD_CL_BS>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G.smem) != cudaSuccess) return false;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) return false;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(G.CL);
    cfg.blockDim = dim3(PD_CL_BS);
    cfg.dynamicSmemBytes = G.smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = G.CL;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg) != cudaSuccess || clusters < 1) {
        cudaGetLastError();
        return false;
    }
    if (cudaLaunchKernelEx(&cfg, kern, P, G, periods) != cudaSuccess) { cudaGetLastError(); return false; }
    count_launch(1);
    return true;
}

cudaError_t launch_pdhg_init(const PdhgDev& P, cudaStream_t s) {
    const int nmax = P.n > P.m ? P.n : P.m;
    k_pdhg_init<<<(nmax + 255) / 256, 256, 0, s>>>(P);
    count_launch(1);
    return cudaGetLastError();
}

// One restart period: R primal/dual pairs.
cudaError_t launch_pdhg_period(const PdhgDev& P, cudaStream_t s) {
    const int gp = (P.n + PD_WARPS - 1) / PD_WARPS, gd = (P.m + PD_WARPS - 1) / PD_WARPS;
    for (int t = 0; t < P.R; ++t) {
        k_pdhg_primal<<<gp, PD_BS, 0, s>>>(P, t == 0 ? 1 : 0);
        k_pdhg_dual<<<gd, PD_BS, 0, s>>>(P, t == P.R - 1 ? 1 : 0);
    }
    count_launch(2 * P.R);
    return cudaGetLastError();
}

cudaError_t launch_pdhg_finish(const PdhgDev& P, cudaStream_t s) {
    k_pdhg_finish<<<(P.n + 255) / 256, 256, 0, s>>>(P);
    count_launch(1);
    return cudaGetLastError();
}

cudaError_t launch_pdhg_evidence(const PdhgDev& P, float* gap, float* dual, cudaStream_t s) {
    const int nv = P.n + P.m;
    k_pdhg_evidence<<<(nv + PD_WARPS - 1) / PD_WARPS, PD_BS, 0, s>>>(P, gap, dual);
    count_launch(1);
    return cudaGetLastError();
}

}  // namespace ds
