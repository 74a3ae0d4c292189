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
