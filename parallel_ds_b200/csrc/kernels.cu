// Per-iteration kernels of the dual simplex hot loop (sm_100a, FP64).
//
// One iteration (reference: CudaDualSimplex::callDualSolver,
// cudaDualSimplex.cpp:417-648) is this launch sequence, captured once per
// factor as a CUDA graph:
//
//   k_chuzr        loop bookkeeping (iteration++, refactor / restart / perturb,
//                  checkDualFeasible every NEED_RESTART), CHUZR (DSE pricing +
//                  optimality test), then the eta part of BTRAN for e_p
//   k_btran_rhs    BTRAN through the basis's slack rows
//   k_btran_gemv   BTRAN through Kinv^T -> rho
//   k_pivot_row    alpha_N = rho^T A_N fused with CHUZC part 1; the last block
//                  runs CHUZC part 2 (ordered tie scan) and the BFRT loop
//   k_dual_update  d_N -= theta alpha_N, bound-flip set, BFRT column change
//   k_ftran_k      FTRAN through Kinv for [a_q, rho, column_change] at once
//   k_ftran_assemble  FTRAN through the slack rows; eta-chain scalars s = M g
//   k_eta_apply    y = y0 + sum_t s_t (eta_t - e_{p_t}) in one streaming pass
//   k_update       x_B, DSE weights, eta append, basis swap, flips, objective
//
// A kernel that needs a decision reads it from Ctl; any kernel may raise an
// event, after which every later kernel of the iteration returns at once and
// the host handles the event.  "Last block" finishing uses a ticket counter
// (threadfence + atomicAdd); all reductions are in a fixed order, so results
// do not depend on scheduling.
//
// Arithmetic that decides indices follows the reference's operation order
// exactly and the file is compiled with -fmad=false.
#include <atomic>
#include <cfloat>
#include <mutex>
#include <climits>
#include <cmath>

#include <cooperative_groups.h>
#include <math_constants.h>

#include "engine.cuh"
#include "kernels.cuh"

namespace ds {

namespace cg = cooperative_groups;

__device__ __forceinline__ bool halted(const Ctl* c) { return *(volatile const int*)&c->halt != 0; }

__device__ __forceinline__ void raise_ev(Ctl* c, int ev, int stage) {
    c->event = ev;
    c->event_stage = stage;
    c->halt = 1;
    __threadfence();
}

// True in exactly one block: the last one to arrive.  All blocks must call it.
__device__ bool last_block(unsigned* ticket) {
    __shared__ bool is_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned nb = gridDim.x * gridDim.y;
        const unsigned t = atomicAdd(ticket, 1u);
        is_last = (t == nb - 1);
        if (is_last) *ticket = 0u;
    }
    __syncthreads();
    if (is_last) __threadfence();
    return is_last;
}

// ---------------------------------------------------------------- reductions
struct ArgMax { double w; int i; };
__device__ __forceinline__ ArgMax better_max(ArgMax a, ArgMax b) {  // larger w, then smaller i
    if (b.w > a.w || (b.w == a.w && b.i < a.i)) return b;
    return a;
}
struct ArgMin { double t; int i; };
__device__ __forceinline__ ArgMin better_min(ArgMin a, ArgMin b) {  // smaller t, then smaller i
    if (b.t < a.t || (b.t == a.t && b.i < a.i)) return b;
    return a;
}

template <int BS>
__device__ ArgMax block_argmax(ArgMax v) {
    __shared__ double sw[BS / 32];
    __shared__ int si[BS / 32];
    for (int o = 16; o > 0; o >>= 1) {
        ArgMax u{__shfl_down_sync(0xffffffffu, v.w, o), __shfl_down_sync(0xffffffffu, v.i, o)};
        v = better_max(v, u);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { sw[wid] = v.w; si[wid] = v.i; }
    __syncthreads();
    if (wid == 0) {
        v = (lane < BS / 32) ? ArgMax{sw[lane], si[lane]} : ArgMax{-1.0, INT_MAX};
        for (int o = 16; o > 0; o >>= 1) {
            ArgMax u{__shfl_down_sync(0xffffffffu, v.w, o), __shfl_down_sync(0xffffffffu, v.i, o)};
            v = better_max(v, u);
        }
    }
    __syncthreads();
    return v;  // valid in thread 0
}

template <int BS>
__device__ ArgMin block_argmin(ArgMin v) {
    __shared__ double st[BS / 32];
    __shared__ int si[BS / 32];
    for (int o = 16; o > 0; o >>= 1) {
        ArgMin u{__shfl_down_sync(0xffffffffu, v.t, o), __shfl_down_sync(0xffffffffu, v.i, o)};
        v = better_min(v, u);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { st[wid] = v.t; si[wid] = v.i; }
    __syncthreads();
    if (wid == 0) {
        v = (lane < BS / 32) ? ArgMin{st[lane], si[lane]} : ArgMin{CUDART_INF, INT_MAX};
        for (int o = 16; o > 0; o >>= 1) {
            ArgMin u{__shfl_down_sync(0xffffffffu, v.t, o), __shfl_down_sync(0xffffffffu, v.i, o)};
            v = better_min(v, u);
        }
    }
    __syncthreads();
    return v;
}

// The smallest (t, i) pair and the second smallest t value.
struct Min2 { double t1; int i1; double t2; };
__device__ __forceinline__ Min2 comb_min2(Min2 a, Min2 b) {
    if (b.t1 < a.t1 || (b.t1 == a.t1 && b.i1 < a.i1)) return Min2{b.t1, b.i1, fmin(b.t2, a.t1)};
    return Min2{a.t1, a.i1, fmin(a.t2, b.t1)};
}
template <int BS>
__device__ Min2 block_min2(Min2 v) {
    __shared__ double s1[BS / 32], s2[BS / 32];
    __shared__ int si[BS / 32];
    for (int o = 16; o > 0; o >>= 1) {
        Min2 u{__shfl_down_sync(0xffffffffu, v.t1, o), __shfl_down_sync(0xffffffffu, v.i1, o),
               __shfl_down_sync(0xffffffffu, v.t2, o)};
        v = comb_min2(v, u);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { s1[wid] = v.t1; si[wid] = v.i1; s2[wid] = v.t2; }
    __syncthreads();
    if (wid == 0) {
        v = (lane < BS / 32) ? Min2{s1[lane], si[lane], s2[lane]} : Min2{CUDART_INF, INT_MAX, CUDART_INF};
        for (int o = 16; o > 0; o >>= 1) {
            Min2 u{__shfl_down_sync(0xffffffffu, v.t1, o), __shfl_down_sync(0xffffffffu, v.i1, o),
                   __shfl_down_sync(0xffffffffu, v.t2, o)};
            v = comb_min2(v, u);
        }
    }
    __syncthreads();
    return v;   // valid in thread 0
}

template <int BS>
__device__ int block_sum_int(int v) {
    __shared__ int s[BS / 32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) s[wid] = v;
    __syncthreads();
    if (wid == 0) {
        v = (lane < BS / 32) ? s[lane] : 0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    __syncthreads();
    return v;
}

template <int BS>
__device__ double block_sum(double v) {
    __shared__ double s[BS / 32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) s[wid] = v;
    __syncthreads();
    if (wid == 0) {
        v = (lane < BS / 32) ? s[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    __syncthreads();
    return v;
}

// ------------------------------------------------------------ per-variable rules
// checkDualFeasible (tpp:362-385) for one nonbasic variable.
__device__ __forceinline__ bool var_dual_bad(unsigned char t, double d) {
    switch (t) {
        case FREE: return fabs(d) < EPS_D || isnan(d);
        case UPPER: return d > EPS_D || isnan(d);
        case LOWER: return d < -EPS_D || isnan(d);
        default: return false;
    }
}

// simpleRatioTestPart1 candidate rule (cudaDualSimplex.cpp:367-394).
__device__ __forceinline__ bool rt_candidate(double a, unsigned char t, double x, double l, double u) {
    if (a > EPS_A) return fabs(x - l) < EPS_Z && (t == LOWER || t == BOXED);
    if (a < -EPS_A) return fabs(x - u) < EPS_Z && (t == UPPER || t == BOXED);
    return t == FREE;
}

// checkDualFeasible over the nonbasic slots; also used standalone (force=1).
template <int BS>
__global__ void k_dual_check(Dev D, int force) {
    Ctl* c = D.ctl;
    if (!force && (halted(c) || !c->need_dual_check)) return;
    const int i = blockIdx.x * BS + threadIdx.x;
    int bad = 0;
    if (i < D.n) {
        const int j = D.nonbasis[i];
        bad = var_dual_bad(D.type[j], D.d[j]) ? 1 : 0;
    }
    bad = block_sum_int<BS>(bad);
    if (threadIdx.x == 0 && bad) atomicAdd(&c->dual_infeas, bad);
    if (last_block(&c->tickets[1]) && threadIdx.x == 0) {
        if (force) return;
        c->need_dual_check = 0;
        if (atomicAdd(&c->dual_infeas, 0) > 0) raise_ev(c, EV_DUALINF, ST_TOP);
        else if (!c->perturbed && c->cycle > MAX_CYCLE) raise_ev(c, EV_PERTURB, ST_TOP);
    }
}

// ================================================================ eta chain
// G[t][u] = eta_u[p_t] - [p_u == p_t] (u < t) couples the product-form factors.
// FTRAN needs s_t = g_t + sum_{u<t} G[t][u] s_u (s_t is the pivot entry the
// sequential product form reads before applying eta t); BTRAN needs
// d_t = h_t + sum_{u>t} G[u][t] d_u.  The block first stages G's strict lower
// triangle in shared memory (packed by rows, row t at t(t-1)/2); then one warp
// walks the chain, each step's dot product spread over the lanes and reduced by
// shuffles in a fixed order.
__device__ __forceinline__ int pk(int t, int u) { return (t * (t - 1)) / 2 + u; }

template <int BS>
__device__ void stage_G(const Dev& D, double* Gs, int T) {
    // one element per thread per row (T <= cap <= 205 < BS); the unrolled row
    // loop keeps eight independent loads in flight per thread
    const int u = threadIdx.x;
#pragma unroll 8
    for (int t = 1; t < T; ++t)
        if (u < t) Gs[pk(t, u)] = __ldcg(&D.Mtri[(size_t)t * D.cap + u]);
}
// The chain recurrences, one warp, in blocks of 32 unknowns: each lane owns one
// unknown of the block, first sums the contributions of the blocks already
// solved (its own dot product, no shuffles), then the block's triangle is
// walked one unknown at a time, the finished value broadcast by a shuffle and
// folded into the lanes still open.  T sequential steps of a shuffle and a
// fused update instead of T warp-wide reductions.
__device__ void eta_forward(const double* Gs, const double* g, double* s, int T) {
    const int lane = threadIdx.x & 31;
    for (int b0 = 0; b0 < T; b0 += 32) {
        const int t = b0 + lane;
        double v = 0.0;
        if (t < T) {
            const double* Gr = Gs + pk(t, 0);
            double a0 = 0.0, a1 = 0.0;
            int u = 0;
            for (; u + 1 < b0; u += 2) { a0 += Gr[u] * s[u]; a1 += Gr[u + 1] * s[u + 1]; }
            if (u < b0) a0 += Gr[u] * s[u];
            v = g[t] + (a0 + a1);
        }
        const int nb = min(32, T - b0);
        for (int j = 0; j < nb; ++j) {
            const double sj = __shfl_sync(0xffffffffu, v, j);
            if (lane > j && t < T) v += Gs[pk(t, b0 + j)] * sj;
        }
        if (t < T) s[t] = v;
        __syncwarp();
    }
}
__device__ void eta_backward(const double* Gs, const double* h, double* dl, int T) {
    const int lane = threadIdx.x & 31;
    for (int b1 = T - 1; b1 >= 0; b1 -= 32) {
        const int t = b1 - lane;
        double v = 0.0;
        if (t >= 0) {
            double a0 = 0.0, a1 = 0.0;
            int u = b1 + 1;
            for (; u + 1 < T; u += 2) { a0 += Gs[pk(u, t)] * dl[u]; a1 += Gs[pk(u + 1, t)] * dl[u + 1]; }
            if (u < T) a0 += Gs[pk(u, t)] * dl[u];
            v = h[t] + (a0 + a1);
        }
        const int nb = min(32, b1 + 1);
        for (int j = 0; j < nb; ++j) {
            const double dj = __shfl_sync(0xffffffffu, v, j);
            if (lane > j && t >= 0) v += Gs[pk(b1 - j, t)] * dj;
        }
        if (t >= 0) dl[t] = v;
        __syncwarp();
    }
}

// y[p_t] += dl[t] for every eta t, duplicates summed in eta order by the thread
// holding their first occurrence (deterministic, no atomics).
template <int BS>
__device__ void scatter_pivots(const Dev& D, double* y, const double* dl, int T) {
    for (int t = threadIdx.x; t < T; t += BS) {
        const int pt = D.eta_pos[t];
        bool first = true;
        for (int u = 0; u < t; ++u) first &= (D.eta_pos[u] != pt);
        if (!first) continue;
        double acc = y[pt];
        for (int u = t; u < T; ++u) if (D.eta_pos[u] == pt) acc = acc + dl[u];
        y[pt] = acc;
    }
}

// ====================================================================== CHUZR
// Eta part of BTRAN for the unit vector e_p, run by one block:
//   h_t = eta_t[p] - [p_t == p],  d = (I - G^T)^-1 h,  y = e_p + sum_t d_t e_{p_t}.
template <int BS>
__device__ void btran_unit_eta(const Dev& D, int p_idx, double* Gs) {
    Ctl* c = D.ctl;
    __shared__ double h[256];
    __shared__ double dl[256];
    const int T = c->T;
    // clear what the previous BTRAN left in ybt
    const int nprev = c->ybt_n;
    if (nprev < 0) {
        for (int i = threadIdx.x; i < D.m; i += BS) D.ybt[i] = 0.0;
    } else {
        for (int u = threadIdx.x; u < nprev; u += BS) D.ybt[D.ybt_pos[u]] = 0.0;
    }
    for (int t = threadIdx.x; t < T; t += BS)
        h[t] = D.eta[(size_t)t * D.m + p_idx] - (D.eta_pos[t] == p_idx ? 1.0 : 0.0);
    stage_G<BS>(D, Gs, T);
    __syncthreads();
    if (threadIdx.x < 32) eta_backward(Gs, h, dl, T);
    __syncthreads();
    if (threadIdx.x == 0) D.ybt[p_idx] = 1.0;
    for (int t = threadIdx.x; t < T; t += BS) D.ybt_pos[t + 1] = D.eta_pos[t];
    __syncthreads();
    scatter_pivots<BS>(D, D.ybt, dl, T);
    if (threadIdx.x == 0) { D.ybt_pos[0] = p_idx; c->ybt_n = T + 1; }
    __syncthreads();
}

// Loop bookkeeping of the reference's while loop (cudaDualSimplex.cpp:419-446:
// iteration++, refactor every R, dual check every NEED_RESTART, perturbation),
// then DSEPricing (tpp:470-501) + checkPrimalFeasible (tpp:296-324), or
// phase1Pricing (tpp:746-772) when Ctl::phase == 1.  Threads cover max(m, n):
// positions for pricing, nonbasic slots for the dual check.
// Loop bookkeeping at the top of the reference's iteration (cudaDualSimplex.cpp:419-446).
__device__ __forceinline__ void chuzr_top(const Ctl* c, bool do_top, int* it, int* top_ev, bool* dual_chk) {
    *it = c->iteration;
    *top_ev = EV_NONE;
    *dual_chk = false;
    if (do_top) {
        *it += 1;
        if (*it > c->max_iter) *top_ev = EV_ITER_LIMIT;
        else if (*it % c->R == 0) *top_ev = EV_REFACTOR_DUE;
        else {
            *dual_chk = (*it % NEED_RESTART == 0);
            if (!*dual_chk && !c->perturbed && c->cycle > MAX_CYCLE) *top_ev = EV_PERTURB;
        }
    }
}

// One basis position of DSEPricing (phase 2) or phase1Pricing (phase 1).
__device__ __forceinline__ void chuzr_row(const Dev& D, int i, int phase, bool learned, ArgMax& best, ArgMax& bestL,
                                          int& infeas) {
    const int j = D.basis[i];
    const unsigned char t = D.type[j];
    if (phase == 2) {
        const double x = D.x[j], l = D.lb[j], u = D.ub[j];
        double dt;
        if (var_infeas(t, x, l, u, &dt) && fabs(dt) > 1e-8) {
            const double w = (dt * dt) / D.beta[i];
            if (w > 0.0) {
                best = better_max(best, ArgMax{w, i});   // strict '>' against max_weight = 0; NaN never wins
                if (learned) {
                    const double sg = 1.0 / (1.0 + exp(-(double)D.score[i]));
                    const double v = w * (D.learn_mix + (1.0 - D.learn_mix) * sg);
                    if (v > 0.0) bestL = better_max(bestL, ArgMax{v, i});
                }
            }
        }
        infeas += var_primal_ok(t, x, l, u) ? 0 : 1;
    } else {
        const double fi = D.f[i];
        if ((t == LOWER && fi > EPS_F) || (t == UPPER && fi < -EPS_F) || t == BOXED || t == FIXED) {
            const double w = (fi * fi) / D.beta[i];
            if (w > 0.0 && !D.blocked[j]) best = better_max(best, ArgMax{w, i});
        }
    }
}

// Thread 0's decision after the reductions of CHUZR: loop bookkeeping events,
// the dual check, the optimality test, the leaving row (DSE or learned) or the
// phase-1 outcome.  Returns the leaving position for the eta part of BTRAN, or -1.
// What the decision needs of a winning row, recorded by the thread that scanned
// it (cluster CHUZR), so that the deciding thread does not load it again.
struct RowInfo { int j; double dt, be, sg; };

__device__ int chuzr_decide(const Dev& D, Ctl* c, ArgMax v, ArgMax vL, int tot, int dtot, int top_ev, bool dual_chk,
                            bool do_top, int it, bool learned, int phase, const RowInfo* iw = nullptr,
                            const RowInfo* il = nullptr) {
    int s_pidx = -1;
    if (do_top) c->iteration = it;
    c->top_done = 0;
    int pidx = (v.i == INT_MAX || v.w <= 0.0) ? -1 : v.i;
    // Learned pricing: take the network's row when it is a valid leaving
    // row (a primal infeasible position) whose sigmoid score reaches the
    // margin; otherwise fall back to the DSE row.
    if (learned && top_ev == EV_NONE && !(dual_chk && dtot > 0) && pidx >= 0) {
        const int pl = (vL.i == INT_MAX || !(vL.w > 0.0)) ? -1 : vL.i;
        const double sg = pl < 0 ? 0.0 : il ? il->sg : 1.0 / (1.0 + exp(-(double)D.score[pl]));
        if (pl >= 0 && sg >= D.learn_margin) { pidx = pl; c->learned_used += 1; }
        else c->learned_fallback += 1;
    }
    if (top_ev != EV_NONE) {
        raise_ev(c, top_ev, ST_TOP);
    } else if (dual_chk && dtot > 0) {
        raise_ev(c, EV_DUALINF, ST_TOP);
    } else if (dual_chk && !c->perturbed && c->cycle > MAX_CYCLE) {
        raise_ev(c, EV_PERTURB, ST_TOP);
    } else if (phase == 2) {
        c->primal_feasible = (tot == 0);
        c->ninfeas = tot;
        c->p = -1; c->p_idx = -1;
        if (pidx >= 0) {
            const RowInfo* ri = (iw && pidx == v.i) ? iw : (il && pidx == vL.i) ? il : nullptr;
            int j;
            double dt, be;
            if (ri) {
                j = ri->j; dt = ri->dt; be = ri->be;
            } else {
                j = D.basis[pidx];
                var_infeas(D.type[j], D.x[j], D.lb[j], D.ub[j], &dt);
                be = D.beta[pidx];
            }
            c->p = j; c->p_idx = pidx; c->delta = dt; c->is_lower = dt < 0;
            c->beta_p = be;
        }
        if (tot == 0) raise_ev(c, EV_OPTIMAL, ST_PRICING);
        else if (pidx < 0) raise_ev(c, EV_NO_P, ST_PRICING);
        else s_pidx = pidx;
    } else {
        const int found = pidx >= 0;
        c->p1_found = found;
        const int dinf = c->p1_dinf;
        const double Z = c->z_phase1;
        int ev = EV_NONE;
        if (!found || !dinf) {
            if (fabs(Z) < EPS_A || !dinf) ev = EV_P1_DONE;
            else if (Z > 0) ev = EV_P1_DUALINF;
        }
        if (ev == EV_NONE && pidx < 0) ev = EV_P1_RESTART;
        if (ev == EV_NONE && Z > EPS_BOUND) ev = EV_P1_RESTART;
        if (ev != EV_NONE) raise_ev(c, ev, ST_PRICING);
        else {
            c->p = D.basis[pidx]; c->p_idx = pidx; c->f_p = D.f[pidx];
            c->beta_p = D.beta[pidx];
            s_pidx = pidx;
        }
    }
    return s_pidx;
}

template <int BS>
__global__ void k_chuzr(Dev D) {
    pdl_enter();
    extern __shared__ double Gs[];
    Ctl* c = D.ctl;
    if (halted(c)) return;
    const int phase = c->phase;
    const bool do_top = (phase == 2 && !c->top_done);
    int it, top_ev;
    bool dual_chk;
    chuzr_top(c, do_top, &it, &top_ev, &dual_chk);
    const int i = blockIdx.x * BS + threadIdx.x;
    const bool learned = D.learned && phase == 2 && it >= D.learn_start;
    ArgMax best{-1.0, INT_MAX};
    ArgMax bestL{-1.0, INT_MAX};   // learned ranking: DSE weight x network score
    int infeas = 0, dbad = 0;
    if (top_ev == EV_NONE) {
        if (i < D.m) chuzr_row(D, i, phase, learned, best, bestL, infeas);
        if (dual_chk && i < D.n) dbad = var_dual_bad(D.type[D.nonbasis[i]], D.d[D.nonbasis[i]]) ? 1 : 0;
    }
    best = block_argmax<BS>(best);
    if (learned) bestL = block_argmax<BS>(bestL);
    infeas = block_sum_int<BS>(infeas);
    dbad = block_sum_int<BS>(dbad);
    if (threadIdx.x == 0) {
        D.red[blockIdx.x] = best.w;
        D.redi[blockIdx.x] = best.i;
        D.redi[gridDim.x + blockIdx.x] = infeas;
        D.redi[2 * gridDim.x + blockIdx.x] = dbad;
        if (learned) {
            D.red[gridDim.x + blockIdx.x] = bestL.w;
            D.redi[3 * gridDim.x + blockIdx.x] = bestL.i;
        }
    }
    if (!last_block(&c->tickets[2])) return;
    // ---- last block: combine the partials in block order
    __shared__ int s_pidx;
    ArgMax v{-1.0, INT_MAX}, vL{-1.0, INT_MAX};
    int tot = 0, dtot = 0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += BS) {
        v = better_max(v, ArgMax{__ldcg(&D.red[b]), __ldcg(&D.redi[b])});
        tot += __ldcg(&D.redi[gridDim.x + b]);
        dtot += __ldcg(&D.redi[2 * gridDim.x + b]);
        if (learned) vL = better_max(vL, ArgMax{__ldcg(&D.red[gridDim.x + b]), __ldcg(&D.redi[3 * gridDim.x + b])});
    }
    v = block_argmax<BS>(v);
    if (learned) vL = block_argmax<BS>(vL);
    tot = block_sum_int<BS>(tot);
    dtot = block_sum_int<BS>(dtot);
    if (threadIdx.x == 0)
        s_pidx = chuzr_decide(D, c, v, vL, tot, dtot, top_ev, dual_chk, do_top, it, learned, phase);
    __syncthreads();
    if (s_pidx >= 0) {
        if (D.dense) {
            // rho = B^-T e_p = row p of the explicit inverse (strided gather,
            // unrolled so that the loads of one thread are in flight together)
            const double* src = D.Binv + s_pidx;
            const size_t M = D.m;
#pragma unroll 8
            for (int r = threadIdx.x; r < D.m; r += BS) D.rho[r] = src[(size_t)r * M];
        } else {
            btran_unit_eta<BS>(D, s_pidx, Gs);
        }
    }
}

// CHUZR over one thread-block cluster of CZ_CL CTAs (dense mode).  Each CTA
// scans its share of the positions (loads issued together) and the dual-check
// slots, reduces them in one fused block reduction, and stores its winners,
// counts and the scanning threads' data of the winning rows into rank 0's
// shared memory; after a hardware cluster barrier rank 0 combines the CZ_CL
// partials (selections and integer sums: order-independent), decides, and
// stores the leaving position into every CTA's shared memory; after a second
// barrier all CTAs gather their share of rho = row p of B^-1.  Spreading the
// scattered loads of the scan and the gather over CZ_CL SMs is the point: one
// SM's L2 bandwidth bounds the single-CTA form.  Ctl is written in this kernel
// only by rank 0 after the first barrier, so the early exit below is taken by
// every CTA alike and no CTA misses a barrier.
constexpr int CZ_CL = 8, CZ_BS = 256;
template <int BS>
__global__ void __launch_bounds__(BS) k_chuzr_cluster(Dev D) {
    pdl_enter();
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    Ctl* c = D.ctl;
    if (halted(c)) return;
    const int phase = c->phase;
    const bool do_top = (phase == 2 && !c->top_done);
    int it, top_ev;
    bool dual_chk;
    chuzr_top(c, do_top, &it, &top_ev, &dual_chk);
    const bool learned = D.learned && phase == 2 && it >= D.learn_start;
    constexpr int STRIDE = CZ_CL * BS;
    const int t0 = rank * BS + (int)threadIdx.x;
    ArgMax best{-1.0, INT_MAX}, bestL{-1.0, INT_MAX};
    RowInfo rw{-1, 0.0, 0.0, 0.0}, rl{-1, 0.0, 0.0, 0.0};
    int infeas = 0, dbad = 0;
    if (top_ev == EV_NONE) {
        if (phase == 2) {
            constexpr int RPT = 2;
            const double mix = D.learn_mix;
            for (int i0 = 0; i0 < D.m; i0 += STRIDE * RPT) {
                int ii[RPT], jj[RPT];
                double be[RPT];
                float sc[RPT];
#pragma unroll
                for (int u = 0; u < RPT; ++u) {
                    ii[u] = i0 + u * STRIDE + t0;
                    const int ic = min(ii[u], D.m - 1);
                    jj[u] = D.basis[ic];
                    be[u] = D.beta[ic];
                    sc[u] = learned ? D.score[ic] : 0.f;
                }
                unsigned char tt[RPT];
                double xx[RPT], ll[RPT], uu[RPT];
#pragma unroll
                for (int u = 0; u < RPT; ++u) { tt[u] = D.type[jj[u]]; xx[u] = D.x[jj[u]]; ll[u] = D.lb[jj[u]]; uu[u] = D.ub[jj[u]]; }
#pragma unroll
                for (int u = 0; u < RPT; ++u) {
                    if (ii[u] >= D.m) continue;
                    // DSEPricing (tpp:470-501) + checkPrimalFeasible, as chuzr_row
                    double dt;
                    if (var_infeas(tt[u], xx[u], ll[u], uu[u], &dt) && fabs(dt) > 1e-8) {
                        const double w = (dt * dt) / be[u];
                        if (w > 0.0) {   // strict '>' against max_weight = 0
                            if (better_max(best, ArgMax{w, ii[u]}).i == ii[u]) {
                                best = ArgMax{w, ii[u]};
                                rw = RowInfo{jj[u], dt, be[u], 0.0};
                            }
                            if (learned) {
                                const double sg = 1.0 / (1.0 + exp(-(double)sc[u]));
                                const double v = w * (mix + (1.0 - mix) * sg);
                                if (v > 0.0 && better_max(bestL, ArgMax{v, ii[u]}).i == ii[u]) {
                                    bestL = ArgMax{v, ii[u]};
                                    rl = RowInfo{jj[u], dt, be[u], sg};
                                }
                            }
                        }
                    }
                    infeas += var_primal_ok(tt[u], xx[u], ll[u], uu[u]) ? 0 : 1;
                }
            }
        } else {
            for (int i = t0; i < D.m; i += STRIDE) chuzr_row(D, i, phase, learned, best, bestL, infeas);
        }
        if (dual_chk)
            for (int i = t0; i < D.n; i += STRIDE) dbad += var_dual_bad(D.type[D.nonbasis[i]], D.d[D.nonbasis[i]]) ? 1 : 0;
    }
    const int my_i = best.i, my_il = bestL.i;
    // fused block reduction
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __shared__ double s_w[BS / 32], s_wl[BS / 32];
    __shared__ int s_i[BS / 32], s_il[BS / 32], s_inf[BS / 32], s_db[BS / 32];
    __shared__ int s_win, s_winl, s_pidx;
    // rank 0's cluster partials
    __shared__ ArgMax c_b[CZ_CL], c_bl[CZ_CL];
    __shared__ int c_inf[CZ_CL], c_db[CZ_CL];
    __shared__ RowInfo c_rw[CZ_CL], c_rl[CZ_CL];
    for (int o = 16; o > 0; o >>= 1) {
        best = better_max(best, ArgMax{__shfl_down_sync(FULL, best.w, o), __shfl_down_sync(FULL, best.i, o)});
        bestL = better_max(bestL, ArgMax{__shfl_down_sync(FULL, bestL.w, o), __shfl_down_sync(FULL, bestL.i, o)});
        infeas += __shfl_down_sync(FULL, infeas, o);
        dbad += __shfl_down_sync(FULL, dbad, o);
    }
    if (lane == 0) { s_w[wid] = best.w; s_i[wid] = best.i; s_wl[wid] = bestL.w; s_il[wid] = bestL.i; s_inf[wid] = infeas; s_db[wid] = dbad; }
    __syncthreads();
    if (wid == 0) {
        const bool in = lane < BS / 32;
        best = in ? ArgMax{s_w[lane], s_i[lane]} : ArgMax{-1.0, INT_MAX};
        bestL = in ? ArgMax{s_wl[lane], s_il[lane]} : ArgMax{-1.0, INT_MAX};
        infeas = in ? s_inf[lane] : 0;
        dbad = in ? s_db[lane] : 0;
        for (int o = 16; o > 0; o >>= 1) {
            best = better_max(best, ArgMax{__shfl_down_sync(FULL, best.w, o), __shfl_down_sync(FULL, best.i, o)});
            bestL = better_max(bestL, ArgMax{__shfl_down_sync(FULL, bestL.w, o), __shfl_down_sync(FULL, bestL.i, o)});
            infeas += __shfl_down_sync(FULL, infeas, o);
            dbad += __shfl_down_sync(FULL, dbad, o);
        }
        if (lane == 0) {
            s_win = best.i; s_winl = bestL.i;
            *cl.map_shared_rank(&c_b[rank], 0) = best;
            *cl.map_shared_rank(&c_bl[rank], 0) = bestL;
            *cl.map_shared_rank(&c_inf[rank], 0) = infeas;
            *cl.map_shared_rank(&c_db[rank], 0) = dbad;
        }
    }
    __syncthreads();
    // the threads that scanned this CTA's winning rows hand their data to rank 0
    if (my_i != INT_MAX && my_i == s_win) *cl.map_shared_rank(&c_rw[rank], 0) = rw;
    if (my_il != INT_MAX && my_il == s_winl) *cl.map_shared_rank(&c_rl[rank], 0) = rl;
    cl.sync();
    if (rank == 0 && threadIdx.x == 0) {
        ArgMax v{-1.0, INT_MAX}, vL{-1.0, INT_MAX};
        int tot = 0, dtot = 0, rv = -1, rvl = -1;
        for (int r = 0; r < CZ_CL; ++r) {
            if (better_max(v, c_b[r]).i != v.i) { v = c_b[r]; rv = r; }
            if (better_max(vL, c_bl[r]).i != vL.i) { vL = c_bl[r]; rvl = r; }
            tot += c_inf[r];
            dtot += c_db[r];
        }
        const bool info = phase == 2 && top_ev == EV_NONE;
        const int pidx = chuzr_decide(D, c, v, vL, tot, dtot, top_ev, dual_chk, do_top, it, learned, phase,
                                      (info && v.i != INT_MAX && rv >= 0) ? &c_rw[rv] : nullptr,
                                      (info && learned && vL.i != INT_MAX && rvl >= 0) ? &c_rl[rvl] : nullptr);
        for (int r = 0; r < CZ_CL; ++r) *cl.map_shared_rank(&s_pidx, r) = pidx;
    }
    cl.sync();
    const int p = s_pidx;
    if (p >= 0) {
        const double* src = D.Binv + p;
        const size_t M = D.m;
        for (int r = t0; r < D.m; r += STRIDE) D.rho[r] = src[(size_t)r * M];
    }
}

// Accuracy probe of the explicit inverse (dense mode): v_r = 1 + (r mod 7) / 8,
// y = B^-1 v (k_dense_colsum), then the max-norm residual max_r |(B y)_r - v_r|
// with B's columns taken at the basic positions (var_pos), each row summed in
// CSR order; out[0] gets the residual and out[1] max_i |y_i|, as the bit
// patterns of non-negative doubles (which order as integers; NaN counts as inf).
__global__ void k_probe_fill(double* v, int m) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < m) v[r] = 1.0 + (double)(r % 7) * 0.125;
}
template <int BS>
__global__ void k_basis_residual(Dev D, const double* y, const double* v, unsigned long long* out) {
    const int r = blockIdx.x * BS + threadIdx.x;
    double e = 0.0, a = 0.0;
    if (r < D.m) {
        double s = 0.0;
        for (int k = D.rptr[r]; k < D.rptr[r + 1]; ++k) {
            const int p = D.var_pos[D.rcol[k]];
            if (p >= 0) s += D.rval[k] * y[p];
        }
        const int ps = D.var_pos[D.n + r];
        if (ps >= 0) s += y[ps];
        e = fabs(s - v[r]);
        a = fabs(y[r]);
        if (!(e <= CUDART_INF)) e = CUDART_INF;
        if (!(a <= CUDART_INF)) a = CUDART_INF;
    }
    for (int o = 16; o > 0; o >>= 1) {
        e = fmax(e, __shfl_down_sync(0xffffffffu, e, o));
        a = fmax(a, __shfl_down_sync(0xffffffffu, a, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&out[0], (unsigned long long)__double_as_longlong(e));
        atomicMax(&out[1], (unsigned long long)__double_as_longlong(a));
    }
}

// Standalone eta part of BTRAN for e_{p_idx} (exact DSE weight recomputation).
template <int BS>
__global__ void k_btran_unit(Dev D, int p_idx) {
    extern __shared__ double Gs[];
    btran_unit_eta<BS>(D, p_idx, Gs);
}

// ====================================================================== BTRAN
// rhs_j = y[s_pos[j]] - sum_{r in col(s_var[j]), r in R} a_rj * y[slackpos(r)]
template <int BS>
__global__ void k_btran_rhs(Dev D, int force) {
    pdl_enter();
    if (!force && halted(D.ctl)) return;
    const int j = blockIdx.x * BS + threadIdx.x;
    if (j >= D.k) return;
    const int v = D.s_var[j];
    double s = D.ybt[D.s_pos[j]];
    for (int e = D.cptr[v]; e < D.cptr[v + 1]; ++e) {
        const int sp = D.row_slackpos[D.crow[e]];
        if (sp >= 0) s -= D.cval[e] * D.ybt[sp];
    }
    D.btr_rhs[j] = s;
}

// rho[rp_row[t]] = sum_j Kinv(j, t) rhs_j (one warp per t), rho[r] = y[slackpos(r)] for r in R.
template <int BS>
__global__ void k_btran_gemv(Dev D, double* out, int force) {
    pdl_enter();
    if (!force && halted(D.ctl)) return;
    const int warps_per_block = BS / 32;
    const int nb_warp = (D.k + warps_per_block - 1) / warps_per_block;
    if ((int)blockIdx.x < nb_warp) {
        const int t = blockIdx.x * warps_per_block + (threadIdx.x >> 5);
        const int lane = threadIdx.x & 31;
        if (t >= D.k) return;
        const double* col = D.Kinv + (size_t)t * D.k;
        double s = 0.0;
        for (int j = lane; j < D.k; j += 32) s += col[j] * D.btr_rhs[j];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) out[D.rp_row[t]] = s;
    } else {
        const int r = (blockIdx.x - nb_warp) * BS + threadIdx.x;
        if (r >= D.m) return;
        const int sp = D.row_slackpos[r];
        if (sp >= 0) out[r] = D.ybt[sp];
    }
}

// ============================================= sparse factor solves
// B0 solves through the sparse LU of the bump (sparse_factor.cu): a program of
// levels over one vector of k slots, in shared memory when it fits.  The ops
// of a level are independent (the program builder puts every op above the ops
// it reads), so one barrier per level orders them.
constexpr int SF_BS = 1024;

// One op's program data: its slot, divisor, entry range and first entries.
// The data of a thread's first op of the next level is loaded before the
// level barrier (it does not depend on the vector), so each level pays only
// the barrier and the shared-memory arithmetic, not a chain of L2 loads.
constexpr int SF_PRE = 4;
constexpr int SF_MAXLEV = 512;   // level bounds staged in shared memory up to this many levels
struct SfOp { int s, e0, e1; double dg; int es[SF_PRE]; double cf[SF_PRE]; };
__device__ __forceinline__ void sf_load_op(const SfProg& P, int o, SfOp& q) {
    q.s = P.op_slot[o]; q.e0 = P.op_ptr[o]; q.e1 = P.op_ptr[o + 1]; q.dg = P.op_diag[o];
#pragma unroll
    for (int u = 0; u < SF_PRE; ++u) {
        const bool in = q.e0 + u < q.e1;
        q.es[u] = in ? P.ent_slot[q.e0 + u] : 0;
        q.cf[u] = in ? P.ent_coef[q.e0 + u] : 0.0;
    }
}

template <int BS>
__device__ __forceinline__ void sf_run(const SfDev& F, const SfProg& P, double* v, double* tmp) {
    __shared__ int s_lp[SF_MAXLEV + 1];
    __shared__ int s_lk[SF_MAXLEV];
    const bool staged = P.nlev <= SF_MAXLEV;
    if (staged) {
        for (int L = threadIdx.x; L <= P.nlev; L += BS) s_lp[L] = P.lvl_ptr[L];
        for (int L = threadIdx.x; L < P.nlev; L += BS) s_lk[L] = P.lvl_kind[L];
    }
    __syncthreads();
    const int* lp = staged ? s_lp : P.lvl_ptr;
    const int* lk = staged ? s_lk : P.lvl_kind;
    SfOp q;
    bool have = false;
    if (P.nlev > 0 && lk[0] == 0 && lp[0] + (int)threadIdx.x < lp[1]) { sf_load_op(P, lp[0] + threadIdx.x, q); have = true; }
    for (int L = 0; L < P.nlev; ++L) {
        const int kind = lk[L];
        if (kind == 0) {
            const int o0 = lp[L] + threadIdx.x, o1 = lp[L + 1];
            for (int o = o0; o < o1; o += BS) {
                SfOp c;
                if (o == o0 && have) c = q;
                else sf_load_op(P, o, c);
                double acc = v[c.s];
#pragma unroll
                for (int u = 0; u < SF_PRE; ++u)
                    if (c.e0 + u < c.e1) acc -= c.cf[u] * v[c.es[u]];
                for (int e = c.e0 + SF_PRE; e < c.e1; ++e) acc -= P.ent_coef[e] * v[P.ent_slot[e]];
                v[c.s] = acc / c.dg;
            }
        } else {   // dense block: v[d0 + o] = sum_i M[o + i kd] v[d0 + i]
            const double* M = (kind == 1) ? F.Sinv : F.SinvT;
            const int kd = F.kd, d0 = F.d0;
            for (int o = threadIdx.x; o < kd; o += BS) {
                double acc = 0.0;
                for (int i = 0; i < kd; ++i) acc += M[o + (size_t)i * kd] * v[d0 + i];
                tmp[o] = acc;
            }
            __syncthreads();
            for (int o = threadIdx.x; o < kd; o += BS) v[d0 + o] = tmp[o];
        }
        have = false;
        if (L + 1 < P.nlev && lk[L + 1] == 0 && lp[L + 1] + (int)threadIdx.x < lp[L + 2]) {
            sf_load_op(P, lp[L + 1] + threadIdx.x, q);
            have = true;
        }
        __syncthreads();
    }
}

// FTRAN through B0's bump for the nr right-hand sides (one CTA each): slot s
// starts as the rhs entry of its pivot row and ends as the solution entry of
// its pivot column, written to y0 at that column's basis position.
template <int BS>
__global__ void __launch_bounds__(BS) k_sf_ftran(Dev D, int nr_fixed, int force) {
    pdl_enter();
    Ctl* c = D.ctl;
    if (!force && halted(c)) return;
    const int nr = nr_fixed > 0 ? nr_fixed : c->nrhs;
    const int r = blockIdx.x;
    if (r >= nr) return;
    extern __shared__ double sf_vec[];
    const SfDev& F = D.sf;
    double* v = F.smem ? sf_vec : F.gvec + (size_t)r * F.k;
    double* tmp = F.gtmp + (size_t)r * (F.kd > 0 ? F.kd : 1);
    const double* rhs = D.frhs[r];
    for (int s = threadIdx.x; s < F.k; s += BS) v[s] = rhs[F.slot_row[s]];
    __syncthreads();
    sf_run<BS>(F, F.ft, v, tmp);
    double* y0 = D.y0[r];
    for (int s = threadIdx.x; s < F.k; s += BS) y0[F.slot_pos[s]] = v[s];
}

// BTRAN through B0's bump (block 0: rho at the rows of R' from btr_rhs) and
// the basis's slack rows (the other blocks: rho[r] = y[slackpos(r)]).
template <int BS>
__global__ void __launch_bounds__(BS) k_sf_btran(Dev D, double* out, int force) {
    pdl_enter();
    if (!force && halted(D.ctl)) return;
    if (blockIdx.x == 0) {
        extern __shared__ double sf_vec[];
        const SfDev& F = D.sf;
        double* v = F.smem ? sf_vec : F.gvec;
        for (int s = threadIdx.x; s < F.k; s += BS) v[s] = D.btr_rhs[F.slot_kcol[s]];
        __syncthreads();
        sf_run<BS>(F, F.bt, v, F.gtmp);
        for (int s = threadIdx.x; s < F.k; s += BS) out[F.slot_row[s]] = v[s];
    } else {
        const int r = (blockIdx.x - 1) * BS + threadIdx.x;
        if (r >= D.m) return;
        const int sp = D.row_slackpos[r];
        if (sp >= 0) out[r] = D.ybt[sp];
    }
}

static size_t sf_smem(const Dev& D) { return D.sf.smem ? sizeof(double) * (size_t)D.sf.k : 0; }
static int sf_btran_blocks(const Dev& D) { return 1 + (D.m + SF_BS - 1) / SF_BS; }

// ================================================================ pivot row
// Full sequential ratio scan over F in slot order (simpleRatioTest, tpp:546-572):
// the fallback when the tie window could not be shown exact.
__device__ void rt_full_scan(const Dev& D, double sgn_a, int* q_idx_out) {
    double theta = INF_THETA;
    int q_idx = -1;
    for (int i = 0; i < D.n; ++i) {
        if (!__ldcg(&D.cand[i])) continue;
        const double th = __ldcg(&D.theta_arr[i]);
        if (isnan(th)) continue;   // removed by BFRT or not takeable
        const double a = sgn_a * __ldcg(&D.alpha[i]);
        if (th < theta) { theta = th; q_idx = i; }
        else if (q_idx >= 0 && fabs(th - theta) < EPS_Z) {
            if (fabs(a) > fabs(sgn_a * __ldcg(&D.alpha[q_idx]))) { theta = th; q_idx = i; }
        }
    }
    *q_idx_out = q_idx;
}

// CHUZC part 2 from the first minimiser (theta*, i*): the sequential scan's state
// after i* is (theta*, i*) whatever came before, and later candidates can only be
// taken through the EPS_Z tie branch, i.e. from a chain starting at theta*.  The
// chain is followed over the candidates inside [theta*, theta* + RT_WINDOW]; if it
// stayed at least 2 EPS_Z below the window edge no outside candidate could have
// joined it and the result equals the full scan; otherwise the full scan runs.
template <int BS>
__device__ int rt_select(const Dev& D, double sgn_a) {
    __shared__ double s_tmin[BS / 32];
    __shared__ int s_imin[BS / 32];
    __shared__ int list[2048];
    __shared__ int nlist, overflow, result;
    __shared__ double s_bound;
    // global first minimiser over takeable candidates
    ArgMin v{CUDART_INF, INT_MAX};
    for (int i = threadIdx.x; i < D.n; i += BS) {
        const double th = __ldcg(&D.theta_arr[i]);
        if (__ldcg(&D.cand[i]) && !isnan(th)) v = better_min(v, ArgMin{th, i});
    }
    (void)s_tmin; (void)s_imin;
    v = block_argmin<BS>(v);
    if (threadIdx.x == 0) {
        nlist = 0; overflow = 0; result = (v.i == INT_MAX) ? -1 : v.i;
        s_bound = v.t + RT_WINDOW;
        s_tmin[0] = v.t;
    }
    __syncthreads();
    if (result < 0) return -1;
    const int istar = result;
    const double B = s_bound;
    // ordered collection of window members after i*
    for (int base = istar + 1; base < D.n; base += BS) {
        const int i = base + threadIdx.x;
        bool mem = false;
        if (i < D.n && __ldcg(&D.cand[i])) {
            const double th = __ldcg(&D.theta_arr[i]);
            mem = !isnan(th) && th <= B;
        }
        const unsigned ball = __ballot_sync(0xffffffffu, mem);
        __shared__ int wcount[BS / 32];
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        if (lane == 0) wcount[wid] = __popc(ball);
        __syncthreads();
        if (threadIdx.x == 0) {
            int acc = nlist;
            for (int w = 0; w < BS / 32; ++w) { const int cnt = wcount[w]; wcount[w] = acc; acc += cnt; }
            if (acc > 2048) overflow = 1;
            nlist = acc > 2048 ? 2048 : acc;
        }
        __syncthreads();
        if (mem) {
            const int slot = wcount[wid] + __popc(ball & ((1u << lane) - 1u));
            if (slot < 2048) list[slot] = i;
        }
        __syncthreads();
        if (overflow) break;
    }
    if (threadIdx.x == 0) {
        int q = istar;
        double theta = __ldcg(&D.theta_arr[istar]);
        double maxrun = theta;
        bool exact = !overflow;
        if (exact) {
            for (int u = 0; u < nlist; ++u) {
                const int i = list[u];
                const double th = __ldcg(&D.theta_arr[i]);
                const double a = sgn_a * __ldcg(&D.alpha[i]);
                if (th < theta) { theta = th; q = i; }
                else if (fabs(th - theta) < EPS_Z) {
                    if (fabs(a) > fabs(sgn_a * __ldcg(&D.alpha[q]))) { theta = th; q = i; }
                }
                if (theta > maxrun) maxrun = theta;
            }
            exact = (B - maxrun) >= 2.0 * EPS_Z;
        }
        if (!exact) {
            atomicAdd(&D.ctl->window_fallbacks, 1);
            rt_full_scan(D, sgn_a, &q);
        }
        result = q;
    }
    __syncthreads();
    return result;
}

// Last block of the pivot-row kernels: combine the per-block candidate counts
// and (t1, i1, t2) minima in block order, then CHUZC part 2 + the BFRT loop
// (cudaDualSimplex.cpp:484-549), writing q, theta and delta_bfrt to Ctl.
template <int BS>
__device__ void pivot_row_finish(const Dev& D, Ctl* c, int phase, double sgn_a) {
    __shared__ int s_tot, s_q, s_fast;
    int tot = 0;
    Min2 g{CUDART_INF, INT_MAX, CUDART_INF};
    for (int b = threadIdx.x; b < (int)gridDim.x; b += BS) {
        tot += __ldcg(&D.redi[b]);
        g = comb_min2(g, Min2{__ldcg(&D.red[2 * b]), __ldcg(&D.redi[gridDim.x + b]), __ldcg(&D.red[2 * b + 1])});
    }
    tot = block_sum_int<BS>(tot);
    g = block_min2<BS>(g);
    if (threadIdx.x == 0) {
        s_tot = tot;
        c->ncand = tot;
        if (tot == 0) raise_ev(c, phase == 2 ? EV_UNBOUNDED : EV_P1_BLOCK, ST_RATIO);
        else if (phase == 2) c->unbound_checked = 0;
        // fast path: no second candidate within the tie window of the first
        // minimiser, so the ordered scan (rt_select) would return it unchanged
        s_fast = (g.i1 != INT_MAX && g.t2 > g.t1 + RT_WINDOW) ? g.i1 : -1;
    }
    __syncthreads();
    if (s_tot == 0) return;
    // CHUZC part 2 + BFRT
    double delta = fabs(c->delta);
    int remaining = s_tot;
    int q_idx = -1;
    bool first_pass = true;
    while (true) {
        const int qi = (first_pass && s_fast >= 0) ? s_fast : rt_select<BS>(D, sgn_a);
        first_pass = false;
        if (threadIdx.x == 0) s_q = qi;
        __syncthreads();
        if (s_q < 0) break;          // nothing takeable (reference: uninitialised q)
        q_idx = s_q;
        if (phase != 2) break;
        const int qv = D.nonbasis[q_idx];
        if (D.type[qv] != BOXED) break;
        const double span = (D.ub[qv] - D.lb[qv]) * fabs(sgn_a * __ldcg(&D.alpha[q_idx]));
        if (delta - span <= 0) break;
        delta -= span;
        __syncthreads();
        if (threadIdx.x == 0) __stcg(&D.theta_arr[q_idx], CUDART_NAN);   // F.erase(q_idx)
        --remaining;
        __syncthreads();
        if (remaining == 0) break;
    }
    if (threadIdx.x == 0) {
        if (q_idx < 0) { c->err = 1; raise_ev(c, EV_ERROR, ST_RATIO); return; }
        const int qv = D.nonbasis[q_idx];
        c->q = qv; c->q_idx = q_idx;
        c->theta = D.d[qv] / __ldcg(&D.alpha[q_idx]);
        c->delta_bfrt = (c->is_lower ? -1.0 : 1.0) * delta;
        if (phase == 1) {
            // infisibilityCorr(q) (tpp:614-625) on d before the update
            const unsigned char t = D.type[qv];
            const double dq = D.d[qv];
            double corr = 0;
            if ((t == UPPER || t == FREE) && dq > EPS_D) corr = 1;
            else if ((t == LOWER || t == FREE) && dq < -EPS_D) corr = -1;
            c->dz = corr;   // phase 1 reuses dz for the correction term
        }
    }
}

// One nonbasic slot i of the pivot row: alpha_i = sum_e a_e rho[row_e] in CSC
// order (matrix.cpp:273-286, mode bit 1) and the ratio-test candidate test
// (mode bit 2), accumulated into the thread's count and (t1, i1, t2) minimum.
__device__ __forceinline__ void pivot_row_slot(const Dev& D, int i, int mode, int phase, double sgn_a, int& ncand,
                                               Min2& mm) {
    const int j = D.nonbasis[i];
    // the candidate test's operands depend only on j: load them with the dot's
    unsigned char tj = 0;
    double dj = 0.0, xj = 0.0, lj = 0.0, uj = 0.0;
    if (mode & 2) { dj = D.d[j]; tj = D.type[j]; xj = D.x[j]; lj = D.lb[j]; uj = D.ub[j]; }
    double acc = 0.0;
    if (mode & 1) {
        if (j < D.n) {
            // the CSC order of the reference's dot (matrix.cpp:273-286), with the
            // loads of sixteen nonzeros (the last batch predicated) issued before
            // their products are summed
            const int e1 = D.cptr[j + 1];
            for (int e = D.cptr[j]; e < e1; e += 16) {
                int rr[16];
                double vv[16], pp[16];
#pragma unroll
                for (int u = 0; u < 16; ++u) {
                    const bool ok = e + u < e1;
                    rr[u] = ok ? D.crow[e + u] : 0;
                    vv[u] = ok ? D.cval[e + u] : 0.0;
                }
#pragma unroll
                for (int u = 0; u < 16; ++u) pp[u] = D.rho[rr[u]];
#pragma unroll
                for (int u = 0; u < 16; ++u)
                    if (e + u < e1) acc += vv[u] * pp[u];
            }
        } else {
            acc += 1.0 * D.rho[j - D.n];
        }
        D.alpha[i] = acc;
    } else {
        acc = D.alpha[i];
    }
    if (mode & 2) {
        const double a = sgn_a * acc;
        bool cand;
        if (phase == 2) cand = rt_candidate(a, tj, xj, lj, uj);
        else cand = (dj >= 0 && a > EPS_A) || (dj <= 0 && a < -EPS_A);
        double th = CUDART_NAN;
        if (cand) {
            ncand += 1;
            const double tt = dj / a;
            if (tt < INF_THETA) { th = tt; mm = comb_min2(mm, Min2{tt, i, CUDART_INF}); }   // NaN / >= INF never taken
        }
        D.theta_arr[i] = th;
        D.cand[i] = cand ? 1 : 0;
    }
}

// alpha_i = sum_e a_e rho[row_e] in CSC order (matrix.cpp:273-286), fused with the
// candidate test; the last block selects q (CHUZC) and runs the BFRT loop
// (cudaDualSimplex.cpp:484-549).  Phase 1 uses phase1SetRatioTestCandidates.
template <int BS>
__global__ void k_pivot_row(Dev D, int mode) {
    pdl_enter();
    Ctl* c = D.ctl;
    if (halted(c)) return;
    const int phase = c->phase;
    const double sgn_a = (phase == 2) ? (c->is_lower ? -1.0 : 1.0) : (c->f_p > 0 ? -1.0 : 1.0);
    const int i = blockIdx.x * BS + threadIdx.x;
    int ncand = 0;
    Min2 mm{CUDART_INF, INT_MAX, CUDART_INF};
    if (i < D.n) pivot_row_slot(D, i, mode, phase, sgn_a, ncand, mm);
    ncand = block_sum_int<BS>(ncand);
    if (!(mode & 2)) return;
    mm = block_min2<BS>(mm);
    if (threadIdx.x == 0) {
        D.redi[blockIdx.x] = ncand;
        D.redi[gridDim.x + blockIdx.x] = mm.i1;
        D.red[2 * blockIdx.x] = mm.t1;
        D.red[2 * blockIdx.x + 1] = mm.t2;
    }
    if (!last_block(&c->tickets[3])) return;
    pivot_row_finish<BS>(D, c, phase, sgn_a);
}

// The pivot row of the iteration step in one thread-block cluster of PR_CL
// CTAs (n <= PR_CL_MAX_N): the same slot work as k_pivot_row over a strided
// slot range, per-CTA partials in global memory, then a hardware cluster
// barrier instead of the last-block ticket, and rank 0 runs CHUZC + BFRT.  Ctl
// is not written before the barrier, so every CTA takes the early exit alike.
constexpr int PR_CL = 16, PR_BS = 256, PR_CL_MAX_N = 2 * PR_CL * PR_BS;
template <int BS>
__global__ void __launch_bounds__(BS) k_pivot_row_cluster(Dev D) {
    pdl_enter();
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    Ctl* c = D.ctl;
    if (halted(c)) return;
    const int phase = c->phase;
    const double sgn_a = (phase == 2) ? (c->is_lower ? -1.0 : 1.0) : (c->f_p > 0 ? -1.0 : 1.0);
    int ncand = 0;
    Min2 mm{CUDART_INF, INT_MAX, CUDART_INF};
    for (int i = rank * BS + (int)threadIdx.x; i < D.n; i += PR_CL * BS) pivot_row_slot(D, i, 3, phase, sgn_a, ncand, mm);
    ncand = block_sum_int<BS>(ncand);
    mm = block_min2<BS>(mm);
    if (threadIdx.x == 0) {
        D.redi[rank] = ncand;
        D.redi[PR_CL + rank] = mm.i1;
        D.red[2 * rank] = mm.t1;
        D.red[2 * rank + 1] = mm.t2;
    }
    cl.sync();
    if (rank != 0) return;
    pivot_row_finish<BS>(D, c, phase, sgn_a);
}

// Serial part of the dual update, in one CTA once every slot is updated: the
// dense-mode FTRAN/BTRAN pivot check, d_p = -theta, d_q = 0, the ordered flip
// list, the column change and delta_z, and the eta-mode entering column.  tot:
// flips found by the slot pass (valid in thread 0).
template <int BS>
__device__ void dual_update_finish(const Dev& D, Ctl* c, int phase, double theta, int tot) {
    if (D.dense && threadIdx.x == 0) {
        // the reference's FTRAN/BTRAN pivot check (cudaDualSimplex.cpp:555)
        const double aqp = __ldcg(&D.alpha_q[c->p_idx]);
        const double apq = D.alpha[c->q_idx];
        if (!(fabs(aqp) > 0.0) || isnan(aqp)) raise_ev(c, EV_ERROR, ST_FTRAN);
        else if (fabs(aqp - apq) > EPS_R * (1 + fabs(aqp))) raise_ev(c, EV_MISMATCH, ST_FTRAN);
    }
    __shared__ int s_nf;
    if (threadIdx.x == 0) {
        s_nf = tot;
        c->nflips = tot;
        D.d[c->p] = -theta;
        D.d[c->q] = 0.0;
        if (phase == 1) c->z_phase1 = c->z_phase1 - theta * c->f_p;
    }
    __syncthreads();
    // entering column a_q as a dense row vector (clear the previous one first);
    // the eta-file FTRAN reads it, dense mode does not
    const int pq = D.dense ? -1 : c->prev_q;
    if (pq >= 0) {
        if (pq < D.n) { for (int e = D.cptr[pq] + threadIdx.x; e < D.cptr[pq + 1]; e += BS) D.aq_dense[D.crow[e]] = 0.0; }
        else if (threadIdx.x == 0) D.aq_dense[pq - D.n] = 0.0;
    }
    __syncthreads();
    const int q = c->q;
    if (!D.dense) {
        if (q < D.n) { for (int e = D.cptr[q] + threadIdx.x; e < D.cptr[q + 1]; e += BS) D.aq_dense[D.crow[e]] = D.cval[e]; }
        else if (threadIdx.x == 0) D.aq_dense[q - D.n] = 1.0;
    }
    if (threadIdx.x == 0) { c->prev_q = q; c->nrhs = (s_nf > 0) ? 3 : 2; }
    if (s_nf == 0) { if (threadIdx.x == 0) c->dz = (phase == 2) ? 0.0 : c->dz; return; }
    // ---- flips (rare): ordered lists, column change and delta_z in slot order
    for (int r = threadIdx.x; r < D.m; r += BS) D.cc[r] = 0.0;
    __syncthreads();
    __shared__ int nlist;
    if (threadIdx.x == 0) {
        double dz = 0.0;
        int nl = 0;
        for (int s = 0; s < D.n; ++s) {
            const unsigned char fl = __ldcg(&D.flip[s]);
            if (!fl) continue;
            const int j = D.nonbasis[s];
            const double span = D.ub[j] - D.lb[j];
            if (fl == 1) dz += D.cost[j] * span; else dz -= D.cost[j] * span;
            D.flip_list[nl++] = (fl == 1) ? j : -(j + 1);
        }
        c->dz = dz;
        nlist = nl;
    }
    __syncthreads();
    // addSparseCol(low, +1) then addSparseCol(up, -1) (matrix.cpp:606-616)
    for (int pass = 0; pass < 2; ++pass) {
        for (int u = 0; u < nlist; ++u) {
            const int code = D.flip_list[u];
            const bool low = code >= 0;
            if ((pass == 0) != low) continue;
            const int j = low ? code : -code - 1;
            const double span = D.ub[j] - D.lb[j];
            const double mult = low ? 1.0 : -1.0;
            if (j < D.n) {
                for (int e = D.cptr[j] + threadIdx.x; e < D.cptr[j + 1]; e += BS)
                    D.cc[D.crow[e]] += D.cval[e] * span * mult;
            } else if (threadIdx.x == 0) {
                D.cc[j - D.n] += 1.0 * span * mult;
            }
            __syncthreads();
        }
    }
}

// ================================================================ dual update
// Eta-file mode (dense mode runs k_dual_update_cluster): d_j -= theta alpha_j
// over the nonbasic slots and the BFRT flip test (cudaDualSimplex.cpp:564-593).
// Last block: d_p = -theta, d_q = 0, the ordered flip list, the column change
// and delta_z, and the dense entering column.
template <int BS>
__global__ void k_dual_update(Dev D) {
    pdl_enter();
    Ctl* c = D.ctl;
    if (halted(c)) return;
    const int phase = c->phase;
    const double theta = c->theta;
    const int i = blockIdx.x * BS + threadIdx.x;
    int nf = 0;
    if (i < D.n) {
        const int j = D.nonbasis[i];
        const double dj = D.d[j] - theta * D.alpha[i];
        D.d[j] = dj;
        unsigned char fl = 0;
        if (phase == 2 && D.type[j] == BOXED) {
            const double x = D.x[j];
            if (fabs(x - D.lb[j]) < EPS_Z && dj < -EPS_D) fl = 1;
            else if (fabs(x - D.ub[j]) < EPS_Z && dj > EPS_D) fl = 2;
        }
        D.flip[i] = fl;
        nf = fl ? 1 : 0;
    }
    nf = block_sum_int<BS>(nf);
    if (threadIdx.x == 0) D.redi[blockIdx.x] = nf;
    if (!last_block(&c->tickets[4])) return;
    int tot = 0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += BS) tot += __ldcg(&D.redi[b]);
    tot = block_sum_int<BS>(tot);
    dual_update_finish<BS>(D, c, phase, theta, tot);
}

// ====================================================================== FTRAN
// xs_r[j] = sum_t Kinv(j, t) rhs_r[rp_row[t]] for the nr right-hand sides: the
// t range is split over blockIdx.y chunks; the last chunk block of each j tile
// adds the partials in chunk order and writes y0 at the structural positions.
// Tile-wise variant of last_block: arrivals counted per tile over gridDim.y blocks.
__device__ bool last_in_tile(unsigned* ticket) {
    __shared__ bool is_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned t = atomicAdd(ticket, 1u);
        is_last = (t == gridDim.y - 1);
        if (is_last) *ticket = 0u;
    }
    __syncthreads();
    if (is_last) __threadfence();
    return is_last;
}

template <int BS>
__global__ void k_ftran_k2(Dev D, int nr_fixed, int force) {
    pdl_enter();
    Ctl* c = D.ctl;
    if (!force && halted(c)) return;
    const int nr = nr_fixed > 0 ? nr_fixed : c->nrhs;
    const int k = D.k;
    const int j = blockIdx.x * BS + threadIdx.x;
    const int t0 = blockIdx.y * D.ftr_chunk;
    const int t1 = min(k, t0 + D.ftr_chunk);
    extern __shared__ double sh[];
    for (int u = threadIdx.x; u < (t1 - t0); u += BS) {
        const int row = D.rp_row[t0 + u];
        for (int r = 0; r < nr; ++r) sh[r * D.ftr_chunk + u] = D.frhs[r][row];
    }
    __syncthreads();
    if (j < k) {
        double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0;
        const double* col = D.Kinv + (size_t)t0 * k + j;
        const int len = t1 - t0;
        const int C = D.ftr_chunk;
        if (nr == 1) {
#pragma unroll 8
            for (int t = 0; t < len; ++t) acc0 += col[(size_t)t * k] * sh[t];
        } else if (nr == 2) {
#pragma unroll 8
            for (int t = 0; t < len; ++t) {
                const double kv = col[(size_t)t * k];
                acc0 += kv * sh[t];
                acc1 += kv * sh[C + t];
            }
        } else {
#pragma unroll 8
            for (int t = 0; t < len; ++t) {
                const double kv = col[(size_t)t * k];
                acc0 += kv * sh[t];
                acc1 += kv * sh[C + t];
                acc2 += kv * sh[2 * C + t];
            }
        }
        double* part = D.ftr_part + (size_t)blockIdx.y * MAX_FTRAN_RHS * k;
        part[j] = acc0;
        if (nr > 1) part[k + j] = acc1;
        if (nr > 2) part[2 * k + j] = acc2;
    }
    if (!last_in_tile(&D.tile_tickets[blockIdx.x])) return;
    if (j < k) {
        const int pos = D.s_pos[j];
        for (int r = 0; r < nr; ++r) {
            double s = 0.0;
            for (int ch = 0; ch < (int)gridDim.y; ++ch) s += __ldcg(&D.ftr_part[(size_t)ch * MAX_FTRAN_RHS * k + r * k + j]);
            D.y0[r][pos] = s;
        }
    }
}

// Slack rows of B0: y0[slackpos(r)] = rhs[r] - sum_{coupling row r} a * xs.  The
// last block gathers g_t = y0[p_t] and solves s = Mtri g for the eta chain.
template <int BS>
__global__ void k_ftran_assemble(Dev D, int nr_fixed, int force) {
    pdl_enter();
    extern __shared__ double Gs[];
    Ctl* c = D.ctl;
    if (!force && halted(c)) return;
    const int nr = nr_fixed > 0 ? nr_fixed : c->nrhs;
    const int r = blockIdx.x * BS + threadIdx.x;
    if (r < D.m) {
        const int sp = D.row_slackpos[r];
        if (sp >= 0) {
            for (int q = 0; q < nr; ++q) {
                double s = D.frhs[q][r];
                for (int e = D.cpl_ptr[r]; e < D.cpl_ptr[r + 1]; ++e)
                    s -= D.cpl_val[e] * D.y0[q][D.s_pos[D.cpl_col[e]]];
                D.y0[q][sp] = s;
            }
        }
    }
    if (!last_block(&c->tickets[5])) return;
    const int T = c->T;
    __shared__ double g[MAX_FTRAN_RHS][256];
    __shared__ double sv[MAX_FTRAN_RHS][256];
    for (int t = threadIdx.x; t < T; t += BS)
        for (int q = 0; q < nr; ++q) g[q][t] = __ldcg(&D.y0[q][D.eta_pos[t]]);
    stage_G<BS>(D, Gs, T);
    __syncthreads();
    const int w = threadIdx.x >> 5;
    if (w < nr) eta_forward(Gs, g[w], sv[w], T);
    __syncthreads();
    for (int t = threadIdx.x; t < T; t += BS)
        for (int q = 0; q < nr; ++q) D.s_eta[q * D.cap + t] = sv[q][t];
}

// y = y0 + sum_t s_t eta_t, streaming over the eta file: a block covers ROWS
// rows with ETA_SPLIT thread groups, group g summing its contiguous share of
// the etas (more loads in flight per row than one thread could keep), the
// partials added in group order.  The last block applies the -s_t e_{p_t}
// terms (duplicated positions summed in eta order by the thread owning the
// first occurrence) and, for the iteration FTRAN, the pivot check
// |alpha_q[p] - alpha_p[q]| > EPS_R (1 + |alpha_q[p]|)  (cudaDualSimplex.cpp:555).
constexpr int ETA_SPLIT = 4;
template <int ROWS>
__global__ void __launch_bounds__(ROWS * ETA_SPLIT) k_eta_apply(Dev D, int nr_fixed, int check, int force) {
    constexpr int BS = ROWS * ETA_SPLIT;
    pdl_enter();
    Ctl* c = D.ctl;
    if (!force && halted(c)) return;
    const int nr = nr_fixed > 0 ? nr_fixed : c->nrhs;
    const int T = c->T;
    const int r = threadIdx.x % ROWS, g = threadIdx.x / ROWS;
    const int i = blockIdx.x * ROWS + r;
    __shared__ double s[MAX_FTRAN_RHS][256];
    __shared__ double part[ETA_SPLIT][MAX_FTRAN_RHS][ROWS];
    for (int q = 0; q < nr; ++q)
        for (int t = threadIdx.x; t < T; t += BS) s[q][t] = D.s_eta[q * D.cap + t];
    __syncthreads();
    const int chunk = (T + ETA_SPLIT - 1) / ETA_SPLIT;
    const int t0 = g * chunk, t1 = min(T, t0 + chunk);
    if (i < D.m) {
        const double* e = D.eta + i;
        const size_t M = D.m;
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        if (nr == 1) {
            double b0 = 0.0;
            int t = t0;
#pragma unroll 4
            for (; t + 1 < t1; t += 2) { a0 += s[0][t] * e[t * M]; b0 += s[0][t + 1] * e[(t + 1) * M]; }
            if (t < t1) a0 += s[0][t] * e[t * M];
            a0 += b0;
        } else {
#pragma unroll 8
            for (int t = t0; t < t1; ++t) {
                const double ev = e[t * M];
                a0 += s[0][t] * ev;
                a1 += s[1][t] * ev;
                if (nr > 2) a2 += s[2][t] * ev;
            }
        }
        part[g][0][r] = a0; part[g][1][r] = a1; part[g][2][r] = a2;
    }
    __syncthreads();
    if (g == 0 && i < D.m) {
        for (int q = 0; q < nr; ++q) {
            double acc = D.y0[q][i];
            for (int gg = 0; gg < ETA_SPLIT; ++gg) acc += part[gg][q][r];
            D.fout[q][i] = acc;
        }
    }
    if (!last_block(&c->tickets[6])) return;
    for (int t = threadIdx.x; t < T; t += BS) {
        const int pt = D.eta_pos[t];
        bool first = true;
        for (int u = 0; u < t; ++u) first &= (D.eta_pos[u] != pt);
        if (!first) continue;
        for (int q = 0; q < nr; ++q) {
            double acc = __ldcg(&D.fout[q][pt]);
            for (int u = t; u < T; ++u) if (D.eta_pos[u] == pt) acc = acc - s[q][u];
            D.fout[q][pt] = acc;
        }
    }
    __syncthreads();
    if (check && threadIdx.x == 0) {
        const double aqp = __ldcg(&D.fout[0][c->p_idx]);
        const double apq = D.alpha[c->q_idx];
        if (!(fabs(aqp) > 0.0) || isnan(aqp)) raise_ev(c, EV_ERROR, ST_FTRAN);
        else if (fabs(aqp - apq) > EPS_R * (1 + fabs(aqp))) raise_ev(c, EV_MISMATCH, ST_FTRAN);
    }
}

// ===================================================================== update
// updateAndChangeBasis (cudaDualSimplex.cpp:254-282) / phase1UpdateAndChangeBasis
// (:285-309), BFRT x_B correction (:595-617), flips and objective (:618-634).
struct UpdArgs {
    int phase, p_idx, T, nflips;
    double ap, bp, theta_P;
};
__device__ __forceinline__ UpdArgs update_args(const Dev& D, const Ctl* c) {
    UpdArgs u;
    u.phase = c->phase; u.p_idx = c->p_idx; u.T = c->T; u.nflips = c->nflips;
    u.ap = __ldcg(&D.alpha_q[u.p_idx]);
    u.bp = c->beta_p;
    u.theta_P = (u.phase == 2) ? c->delta_bfrt / u.ap : c->f_p / u.ap;
    return u;
}

// Basis position i: x_B (phase 2) or f (phase 1), and in eta-file mode the new
// eta entry and the DSE weight.  Returns the objective correction of flips.
__device__ double update_position(const Dev& D, const UpdArgs& u, int i) {
    const int j = D.basis[i];
    const double aqi = D.alpha_q[i];
    double dzc = 0.0;
    if (u.phase == 2) {
        double xj = D.x[j];
        if (u.nflips > 0) {
            double dx;
            if (D.dense) {   // dx_B = B^-1 column_change (bound flips, rare)
                dx = 0.0;
                for (int r = 0; r < D.m; ++r) {
                    const double v = D.cc[r];
                    if (v != 0.0) dx += D.Binv[(size_t)r * D.m + i] * v;
                }
            } else {
                dx = D.dxb[i];
            }
            xj = xj - dx;
            dzc = D.cost[j] * dx;
        }
        xj = xj - u.theta_P * aqi;
        D.x[j] = xj;
    } else if (i != u.p_idx) {
        D.f[i] = D.f[i] - aqi * u.theta_P;
    }
    if (!D.dense) {   // dense mode: B^-1 and exact DSE weights are updated by k_binv_update
        D.eta[(size_t)u.T * D.m + i] = (i != u.p_idx) ? -aqi / u.ap : 1 / u.ap;
        if (i != u.p_idx) {
            const double r = aqi / u.ap;
            D.beta[i] = D.beta[i] - 2 * aqi / u.ap * D.tau[i] + (r * r) * u.bp;
        }
    }
    return dzc;
}

// One thread, after every position: objective, entering value, basis swap,
// flips, cycle counter, trace.  nred: number of flip-objective partials in red.
__device__ void update_tail(const Dev& D, Ctl* c, const UpdArgs& u, int nred) {
    const int p = c->p, q = c->q, q_idx = c->q_idx, p_idx = u.p_idx;
    if (!D.dense) D.beta[p_idx] = u.bp / (u.ap * u.ap);
    if (u.phase == 2) {
        double dz = c->dz;
        if (u.nflips > 0) for (int b = 0; b < nred; ++b) dz -= __ldcg(&D.red[b]);
        c->obj += dz;
        D.x[q] = D.x[q] + u.theta_P;
    } else {
        D.f[p_idx] = D.f[p_idx] / u.ap + c->dz;   // + infisibilityCorr
    }
    D.basis[p_idx] = q;
    D.nonbasis[q_idx] = p;
    D.var_pos[q] = p_idx;
    D.var_pos[p] = -(q_idx + 1);
    if (D.enter_count) { D.enter_count[q] += 1; D.entered_at[q] = c->iteration; }
    if (u.phase == 2 && u.nflips > 0) {
        c->flips_total += u.nflips;
        for (int k = 0; k < D.n; ++k) {
            const int code = D.flip_list[k];
            if (k >= u.nflips) break;
            if (code >= 0) D.x[code] = D.ub[code];
            else D.x[-code - 1] = D.lb[-code - 1];
        }
    }
    const double theta = c->theta;
    if (u.phase == 2) {
        c->obj += theta * c->delta_bfrt;
        if (fabs(theta) < EPS_A) c->cycle += 1;
    } else {
        c->cycle = (fabs(theta) < EPS_A) ? c->cycle + 1 : 0;
    }
    if (!D.dense) D.eta_pos[u.T] = p_idx;
    c->pivots += 1;
    if (u.phase == 2 && c->trace_n < c->trace_cap) {
        const int tn = c->trace_n;
        D.trace[2 * tn] = p; D.trace[2 * tn + 1] = q;
        D.trace_d[2 * tn] = theta; D.trace_d[2 * tn + 1] = c->obj;
    }
    if (u.phase == 2) c->trace_n += 1;
}

template <int BS>
__global__ void k_update(Dev D, int force) {
    pdl_enter();
    Ctl* c = D.ctl;
    if (!force && halted(c)) return;
    const UpdArgs u = update_args(D, c);
    const int i = blockIdx.x * BS + threadIdx.x;
    double dzc = 0.0;
    if (i < D.m) dzc = update_position(D, u, i);
    if (u.phase == 2 && u.nflips > 0) {
        dzc = block_sum<BS>(dzc);
        if (threadIdx.x == 0) D.red[blockIdx.x] = dzc;
    }
    if (!last_block(&c->tickets[7])) return;
    __shared__ double g[1024];
    if (threadIdx.x == 0) update_tail(D, c, u, (int)gridDim.x);
    if (D.dense) return;   // no eta file in dense mode
    const int T = u.T, p_idx = u.p_idx;
    // new row of G: G[T][u] = eta_u[p_T] - [p_u == p_T]
    for (int v = threadIdx.x; v < T; v += BS)
        g[v] = D.eta[(size_t)v * D.m + p_idx] - (D.eta_pos[v] == p_idx ? 1.0 : 0.0);
    __syncthreads();
    for (int v = threadIdx.x; v < T; v += BS) D.Mtri[(size_t)T * D.cap + v] = g[v];
    __syncthreads();
    if (threadIdx.x == 0) {
        c->T = T + 1;
        if (c->T >= D.cap) raise_ev(c, EV_ETA_FULL, ST_UPDATE);
    }
}

// Dense-mode dual update and primal update in one thread-block cluster of
// DU_CL CTAs (replaces k_dual_update + k_update there).  Pass 1: d_j -= theta
// alpha_j and the BFRT flip test over the nonbasic slots
// (cudaDualSimplex.cpp:564-593), and alpha_q = B^-1 a_q over the positions (the
// entering column staged in shared memory).  Cluster barrier; rank 0 runs the
// serial part (pivot check, flips, column change).  Cluster barrier; unless
// that part raised an event, pass 2 updates x_B (or f in phase 1) over the
// positions (cudaDualSimplex.cpp:254-309, :595-617).  Cluster barrier; rank 0
// runs the bookkeeping tail (basis swap, objective, flips, trace).  The
// barriers replace the global-memory tickets of the two-kernel form.  Ctl is
// written here only by rank 0 between barriers, and every CTA reads what
// decides an early exit right after a barrier, so all CTAs exit alike.
constexpr int DU_CL = 16, DU_BS = 256;
template <int BS>
__global__ void __launch_bounds__(BS) k_dual_update_cluster(Dev D) {
    pdl_enter();
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    Ctl* c = D.ctl;
    if (halted(c)) return;
    const int phase = c->phase;
    const double theta = c->theta;
    constexpr int STRIDE = DU_CL * BS;
    const int t0 = rank * BS + (int)threadIdx.x;
    int nf = 0;
    for (int i = t0; i < D.n; i += STRIDE) {
        const int j = D.nonbasis[i];
        const double dj = D.d[j] - theta * D.alpha[i];
        D.d[j] = dj;
        unsigned char fl = 0;
        if (phase == 2 && D.type[j] == BOXED) {
            const double x = D.x[j];
            if (fabs(x - D.lb[j]) < EPS_Z && dj < -EPS_D) fl = 1;
            else if (fabs(x - D.ub[j]) < EPS_Z && dj > EPS_D) fl = 2;
        }
        D.flip[i] = fl;
        nf += fl ? 1 : 0;
    }
    {   // alpha_q = B^-1 a_q, sixteen B^-1 loads in flight per thread
        __shared__ int s_r[BS + 16];   // rows past the column's end read row 0 (not summed)
        __shared__ double s_v[BS];
        const int q = c->q;
        const size_t M = D.m;
        if (threadIdx.x < 16) s_r[BS + threadIdx.x] = 0;
        for (int ib = rank * BS; ib < D.m; ib += STRIDE) {   // block-uniform
            const int i = ib + (int)threadIdx.x;
            double sq = 0.0;
            if (q < D.n) {
                const int e0 = D.cptr[q], e1 = D.cptr[q + 1];
                for (int eb = e0; eb < e1; eb += BS) {
                    const int cnt = min(BS, e1 - eb);
                    __syncthreads();
                    const bool in = (int)threadIdx.x < cnt;
                    s_r[threadIdx.x] = in ? D.crow[eb + threadIdx.x] : 0;
                    if (in) s_v[threadIdx.x] = D.cval[eb + threadIdx.x];
                    __syncthreads();
                    if (i < D.m) {
                        for (int u0 = 0; u0 < cnt; u0 += 16) {
                            double bv[16];
#pragma unroll
                            for (int u = 0; u < 16; ++u) bv[u] = D.Binv[(size_t)s_r[u0 + u] * M + i];
#pragma unroll
                            for (int u = 0; u < 16; ++u)
                                if (u0 + u < cnt) sq += bv[u] * s_v[u0 + u];
                        }
                    }
                }
            } else if (i < D.m) {
                sq = D.Binv[(size_t)(q - D.n) * M + i];
            }
            if (i < D.m) D.alpha_q[i] = sq;
        }
    }
    __shared__ int c_nf[DU_CL];
    nf = block_sum_int<BS>(nf);
    if (threadIdx.x == 0) *cl.map_shared_rank(&c_nf[rank], 0) = nf;
    cl.sync();
    if (rank == 0) {
        int tot = 0;
        if (threadIdx.x == 0) for (int r = 0; r < DU_CL; ++r) tot += c_nf[r];
        dual_update_finish<BS>(D, c, phase, theta, tot);
    }
    cl.sync();
    if (halted(c)) return;   // pivot check failed: the host redoes this iteration's update
    const UpdArgs u = update_args(D, c);
    double dzc = 0.0;
    for (int i = t0; i < D.m; i += STRIDE) dzc += update_position(D, u, i);
    if (u.phase == 2 && u.nflips > 0) {
        dzc = block_sum<BS>(dzc);
        if (threadIdx.x == 0) D.red[rank] = dzc;
    }
    cl.sync();
    if (rank == 0 && threadIdx.x == 0) update_tail(D, c, u, DU_CL);
}

// ================================================================ init helpers
// setPrimalVars (tpp:74-101)
__global__ void k_set_primal_vars(Dev D) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.n) return;
    const int j = D.nonbasis[i];
    double v;
    switch (D.type[j]) {
        case FIXED: v = D.lb[j]; break;
        case FREE: v = 0; break;
        case BOXED: v = (D.d[j] > 0) ? D.lb[j] : D.ub[j]; break;
        case UPPER: v = D.ub[j]; break;
        default: v = D.lb[j]; break;
    }
    D.x[j] = v;
}

// rhs_i = RHS_i * 1 + sum_e (a_e * x_e) * -1 over nonbasic columns of row i, the
// slack entry last (dotUpdate UPDATE, matrix.cpp:330-341).
__global__ void k_xb_rhs(Dev D, double* rhs) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= D.m) return;
    double s = 0.0 * 1.0;
    for (int e = D.rptr[r]; e < D.rptr[r + 1]; ++e) {
        const int cidx = D.rcol[e];
        const double b = (D.var_pos[cidx] < 0) ? D.x[cidx] : 0.0;
        s += D.rval[e] * b * -1.0;
    }
    const int sl = D.n + r;
    s += 1.0 * ((D.var_pos[sl] < 0) ? D.x[sl] : 0.0) * -1.0;
    rhs[r] = s;
}

__global__ void k_scatter_basic(Dev D, const double* xb, double* dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.m) return;
    dst[D.basis[i]] = xb[i];
}

__global__ void k_gather_basic_cost(Dev D, double* cb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.m) return;
    cb[i] = D.cost[D.basis[i]];
}

// d_j = sum_e (a_e * y_e) * -1 + c_j for nonbasic j (dotUpdate UPDATE_T, alpha=-1, beta=1).
__global__ void k_reduced_costs(Dev D, const double* y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.n) return;
    const int j = D.nonbasis[i];
    double acc = 0.0;
    if (j < D.n) {
        for (int e = D.cptr[j]; e < D.cptr[j + 1]; ++e) acc += D.cval[e] * y[D.crow[e]] * -1.0;
    } else {
        acc += 1.0 * y[j - D.n] * -1.0;
    }
    D.d[j] = acc + D.cost[j] * 1.0;
}

// General BTRAN eta pass for a dense position vector c0:
//   h_t = eta_t . c0 - c0[p_t]  (one block per t)
template <int BS>
__global__ void k_eta_dots(Dev D, const double* c0, double* h) {
    const int t = blockIdx.x;
    const double* e = D.eta + (size_t)t * D.m;
    double s = 0.0;
    for (int i = threadIdx.x; i < D.m; i += BS) s += e[i] * c0[i];
    s = block_sum<BS>(s);
    if (threadIdx.x == 0) h[t] = s - c0[D.eta_pos[t]];
}

// ybt = c0 + sum_t (Mtri^T h)_t e_{p_t}; marks ybt as dense for the next clear.
template <int BS>
__global__ void k_btran_dense_fix(Dev D, const double* c0, const double* h) {
    extern __shared__ double Gs[];
    __shared__ double dl[256];
    __shared__ double hs[256];
    const int T = D.ctl->T;
    for (int i = threadIdx.x; i < D.m; i += BS) D.ybt[i] = c0[i];
    for (int t = threadIdx.x; t < T; t += BS) hs[t] = h[t];
    stage_G<BS>(D, Gs, T);
    __syncthreads();
    if (threadIdx.x < 32) eta_backward(Gs, hs, dl, T);
    __syncthreads();
    scatter_pivots<BS>(D, D.ybt, dl, T);
    if (threadIdx.x == 0) D.ctl->ybt_n = -1;
}

// Exact DSE weights right after a refactorisation (no etas): beta_i is the
// squared norm of row i of B0^-1 (initBetaWeights(false), tpp:53-67, computes
// the same norms one BTRAN at a time).  Structural position s_pos[j]: row j of
// Kinv.  Slack position of row r: e_r - (A[r,S] Kinv) on the R' rows.
template <int BS>
__global__ void k_beta_exact_struct(Dev D) {
    const int j = blockIdx.x * BS + threadIdx.x;
    if (j >= D.k) return;
    double s = 0.0;
    for (int t = 0; t < D.k; ++t) { const double v = D.Kinv[(size_t)j + (size_t)t * D.k]; s += v * v; }
    D.beta[D.s_pos[j]] = s;
}
template <int BS>
__global__ void k_beta_exact_slack(Dev D) {
    const int r = blockIdx.x;
    const int sp = D.row_slackpos[r];
    if (sp < 0) return;
    const int e0 = D.cpl_ptr[r], e1 = D.cpl_ptr[r + 1];
    double acc = 0.0;
    for (int t = threadIdx.x; t < D.k; t += BS) {
        double v = 0.0;
        for (int e = e0; e < e1; ++e) v += D.cpl_val[e] * D.Kinv[(size_t)D.cpl_col[e] + (size_t)t * D.k];
        acc += v * v;
    }
    acc = block_sum<BS>(acc);
    if (threadIdx.x == 0) D.beta[sp] = 1.0 + acc;
}

template <int BS>
__global__ void k_norm2(const double* v, int n, double* out) {
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += BS) s += v[i] * v[i];
    s = block_sum<BS>(s);
    if (threadIdx.x == 0) *out = s;
}

// obj = c . x over all N (deterministic two-level sum)
template <int BS>
__global__ void k_dot_cost_x(Dev D, double* out) {
    double s = 0.0;
    for (int j = threadIdx.x; j < D.N; j += BS) s += D.cost[j] * D.x[j];
    s = block_sum<BS>(s);
    if (threadIdx.x == 0) *out = s;
}

// Phase 1 initialisation (tpp:776-795, cudaDualSimplex.cpp:212-226): classify the
// nonbasic slots, Z, and the column sum of the dual infeasible columns, one block
// in slot order.
template <int BS>
__global__ void k_phase1_init(Dev D, double* cc) {
    for (int r = threadIdx.x; r < D.m; r += BS) cc[r] = 0.0;
    // 1) the dual infeasible slots in slot order, compacted by a block scan into
    //    flip_list (scratch here): +(i+1) for inf_l, -(i+1) for inf_u
    __shared__ int s_cnt, s_warp[BS / 32];
    int* list = D.flip_list;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_cnt = 0;
    __syncthreads();
    for (int i0 = 0; i0 < D.n; i0 += BS) {
        const int i = i0 + (int)threadIdx.x;
        int code = 0;
        if (i < D.n) {
            const int j = D.nonbasis[i];
            const unsigned char t = D.type[j];
            const double dj = D.d[j];
            const bool up = (t == UPPER || t == FREE) && dj > EPS_D;
            const bool lo = !up && (t == LOWER || t == FREE) && dj < -EPS_D;
            code = lo ? i + 1 : up ? -(i + 1) : 0;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, code != 0);
        if (lane == 0) s_warp[wid] = __popc(bal);
        __syncthreads();
        int before = s_cnt;
        for (int w = 0; w < wid; ++w) before += s_warp[w];
        if (code != 0) list[before + __popc(bal & ((1u << lane) - 1u))] = code;
        __syncthreads();
        if (threadIdx.x == 0) for (int w = 0; w < BS / 32; ++w) s_cnt += s_warp[w];
        __syncthreads();
    }
    // 2) Z and the column sum in slot order, inf_l (+1) first, then inf_u (-1)
    __shared__ double Zs;
    if (threadIdx.x == 0) Zs = 0.0;
    __syncthreads();
    const int cnt = s_cnt;
    for (int pass = 0; pass < 2; ++pass) {
        for (int u = 0; u < cnt; ++u) {
            const int code = list[u];
            if ((pass == 0) != (code > 0)) continue;   // block-uniform
            const int j = D.nonbasis[(code > 0 ? code : -code) - 1];
            const double dj = D.d[j];
            const double mult = (pass == 0) ? 1.0 : -1.0;
            if (threadIdx.x == 0) Zs = (pass == 0) ? Zs + dj : Zs - dj;
            if (j < D.n) {
                for (int e = D.cptr[j] + threadIdx.x; e < D.cptr[j + 1]; e += BS) cc[D.crow[e]] += D.cval[e] * mult;
            } else if (threadIdx.x == 0) {
                cc[j - D.n] += mult;
            }
            __syncthreads();
        }
    }
    if (threadIdx.x == 0) D.ctl->z_phase1 = Zs;
}

// counterDualInfeasible into Ctl::p1_dinf (phase 1 pricing needs the count)
template <int BS>
__global__ void k_count_dual_inf(Dev D) {
    Ctl* c = D.ctl;
    const int i = blockIdx.x * BS + threadIdx.x;
    int bad = 0;
    if (i < D.n) { const int j = D.nonbasis[i]; bad = var_dual_bad(D.type[j], D.d[j]) ? 1 : 0; }
    bad = block_sum_int<BS>(bad);
    if (threadIdx.x == 0) D.redi[blockIdx.x] = bad;
    if (!last_block(&c->tickets[8])) return;
    int tot = 0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += BS) tot += __ldcg(&D.redi[b]);
    tot = block_sum_int<BS>(tot);
    if (threadIdx.x == 0) c->p1_dinf = tot;
}

// G for an eta file given column by column (one block, rows in order).
template <int BS>
__global__ void k_build_mtri(Dev D, int T) {
    __shared__ double g[1024];
    for (int t = 0; t < T; ++t) {
        const int pt = D.eta_pos[t];
        for (int u = threadIdx.x; u < t; u += BS)
            g[u] = D.eta[(size_t)u * D.m + pt] - (D.eta_pos[u] == pt ? 1.0 : 0.0);
        __syncthreads();
        for (int u = threadIdx.x; u < t; u += BS) D.Mtri[(size_t)t * D.cap + u] = g[u];
        __syncthreads();
    }
    if (threadIdx.x == 0) D.ctl->T = T;
}

// ================================================================= launchers
constexpr int BS = 256;
constexpr int BS_ETA = 64;   // eta streaming: narrow blocks spread small m over many SMs
// Shared memory for G's packed lower triangle (eta chains) at capacity cap.
static size_t g_smem_bytes(int cap) { return sizeof(double) * (size_t)cap * (size_t)(cap - 1) / 2; }

static std::atomic<long long> g_launches{0};
static thread_local bool g_counting_off = false;
void count_launch(int nk) { if (!g_counting_off) g_launches.fetch_add(nk, std::memory_order_relaxed); }
void set_launch_counting(bool on) { g_counting_off = !on; }
long long launch_count() { return g_launches.load(); }
static inline int nblk(int n) { return (n + BS - 1) / BS; }

#define LAUNCH_OK() do { cudaError_t e_ = cudaGetLastError(); if (e_ != cudaSuccess) return e_; } while (0)

cudaError_t launch_dual_check(const Dev& D, cudaStream_t s) {
    k_dual_check<BS><<<nblk(D.n), BS, 0, s>>>(D, 1);
    count_launch(1);
    LAUNCH_OK();
    return cudaSuccess;
}

cudaError_t launch_count_dual_inf(const Dev& D, cudaStream_t s) {
    k_count_dual_inf<BS><<<nblk(D.n), BS, 0, s>>>(D);
    count_launch(1);
    LAUNCH_OK();
    return cudaSuccess;
}

cudaError_t launch_btran_b0(const Dev& D, double* out, int force, cudaStream_t s) {
    if (D.k > 0) k_btran_rhs<BS><<<nblk(D.k), BS, 0, s>>>(D, force);
    if (D.sf.on && D.k > 0) {
        k_sf_btran<SF_BS><<<sf_btran_blocks(D), SF_BS, sf_smem(D), s>>>(D, out, force);
    } else {
        const int nbw = (D.k + BS / 32 - 1) / (BS / 32);
        k_btran_gemv<BS><<<nbw + nblk(D.m), BS, 0, s>>>(D, out, force);
    }
    count_launch((D.k > 0 ? 1 : 0) + 1);
    LAUNCH_OK();
    return cudaSuccess;
}

cudaError_t launch_ftran(const Dev& D, int nr_fixed, int check, int force, cudaStream_t s) {
    if (D.k > 0 && D.sf.on) {
        k_sf_ftran<SF_BS><<<MAX_FTRAN_RHS, SF_BS, sf_smem(D), s>>>(D, nr_fixed, force);
    } else if (D.k > 0) {
        dim3 g(D.ftr_ntile, D.ftr_nchunk);
        const size_t sh = (size_t)D.ftr_chunk * MAX_FTRAN_RHS * sizeof(double);
        k_ftran_k2<BS><<<g, BS, sh, s>>>(D, nr_fixed, force);
    }
    k_ftran_assemble<BS><<<nblk(D.m), BS, g_smem_bytes(D.cap), s>>>(D, nr_fixed, force);
    k_eta_apply<BS_ETA><<<(D.m + BS_ETA - 1) / BS_ETA, BS_ETA * ETA_SPLIT, 0, s>>>(D, nr_fixed, check, force);
    count_launch((D.k > 0 ? 1 : 0) + 2);
    LAUNCH_OK();
    return cudaSuccess;
}

// One kernel of the iteration sequence (profiling launches them one by one).
const char* const kStepNames[S_NSTEPS] = {"k_mlp_score", "k_chuzr", "k_btran_rhs", "k_btran_gemv", "k_pivot_row",
                                          "k_dual_update", "k_ftran_k", "k_ftran_assemble", "k_eta_apply",
                                          "k_ftran_dense", "k_update", "k_binv_update"};

bool step_active(const Dev& D, int step) {
    switch (step) {
        case S_SCORE: return score_step_active(D);
        case S_BTRAN_RHS: case S_FTRAN_K: return !D.dense && D.k > 0;
        case S_BTRAN_GEMV: case S_FTRAN_ASM: case S_ETA_APPLY: return !D.dense;
        case S_FTRAN_DENSE: return false;   // dense FTRAN runs inside the dual update (mismatch path: launch_ftran_dense)
        case S_UPDATE: return !D.dense;     // dense mode: inside k_dual_update_cluster (mismatch path: launch_update_forced)
        case S_BINV: return D.dense != 0;
        default: return true;
    }
}


static cudaError_t set_kernel_attributes(int cap);

// The dynamic shared memory limits are process-wide function attributes, so
// they are raised once to the largest size any handle can request (cap 205)
// rather than per call (solver handles on other threads launch concurrently).
cudaError_t init_kernel_attributes(int cap) {
    static std::once_flag once;
    static cudaError_t result = cudaSuccess;
    (void)cap;
    std::call_once(once, [] { result = set_kernel_attributes(205); });
    return result;
}

static cudaError_t set_kernel_attributes(int cap) {
    const int bytes = (int)g_smem_bytes(cap);
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k_chuzr<BS>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_btran_unit<BS>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_ftran_assemble<BS>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_btran_dense_fix<BS>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)) != cudaSuccess) return e;
    const int sf_bytes = (int)(sizeof(double) * SF_SMEM_SLOTS);
    if ((e = cudaFuncSetAttribute(k_sf_ftran<SF_BS>, cudaFuncAttributeMaxDynamicSharedMemorySize, sf_bytes)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_sf_btran<SF_BS>, cudaFuncAttributeMaxDynamicSharedMemorySize, sf_bytes)) != cudaSuccess) return e;
    // a 16-CTA cluster is above the portable size of 8
    if ((e = cudaFuncSetAttribute(k_dual_update_cluster<DU_BS>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1)) != cudaSuccess)
        return e;
    if ((e = cudaFuncSetAttribute(k_pivot_row_cluster<PR_BS>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1)) != cudaSuccess)
        return e;
    return cudaSuccess;
}

// The dense CHUZR cluster, chained to the previous kernel like launch_pdl.
static cudaError_t launch_chuzr_cluster(const Dev& D, cudaStream_t s) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(CZ_CL);
    cfg.blockDim = dim3(CZ_BS);
    cfg.stream = s;
    cudaLaunchAttribute at[2];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = CZ_CL;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 2;
    return cudaLaunchKernelEx(&cfg, k_chuzr_cluster<CZ_BS>, D);
}

// The pivot-row cluster, chained to the previous kernel like launch_pdl.
static cudaError_t launch_pivot_row_cluster(const Dev& D, cudaStream_t s) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(PR_CL);
    cfg.blockDim = dim3(PR_BS);
    cfg.stream = s;
    cudaLaunchAttribute at[2];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = PR_CL;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 2;
    return cudaLaunchKernelEx(&cfg, k_pivot_row_cluster<PR_BS>, D);
}

// The dense dual/primal update cluster, chained to the previous kernel like launch_pdl.
static cudaError_t launch_dual_update_cluster(const Dev& D, cudaStream_t s) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(DU_CL);
    cfg.blockDim = dim3(DU_BS);
    cfg.stream = s;
    cudaLaunchAttribute at[2];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = DU_CL;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 2;
    return cudaLaunchKernelEx(&cfg, k_dual_update_cluster<DU_BS>, D);
}

cudaError_t launch_step(const Dev& D, int step, cudaStream_t s) {
    if (step != S_SCORE && !step_active(D, step)) return cudaSuccess;
    switch (step) {
        case S_FTRAN_DENSE: return launch_ftran_dense(D, 1, 0, s);
        case S_BINV: return launch_binv_update(D, 0, s);
        case S_SCORE: return launch_score(D, s);
        case S_CHUZR:
            if (D.dense) { cudaError_t e = launch_chuzr_cluster(D, s); if (e) return e; }
            else { cudaError_t e = launch_pdl(k_chuzr<BS>, dim3(nblk(D.m > D.n ? D.m : D.n)), dim3(BS), g_smem_bytes(D.cap), s, D); if (e) return e; }
            break;
        case S_BTRAN_RHS: { cudaError_t e = launch_pdl(k_btran_rhs<BS>, dim3(nblk(D.k)), dim3(BS), 0, s, D, 0); if (e) return e; break; }
        case S_BTRAN_GEMV: {
            cudaError_t e;
            if (D.sf.on && D.k > 0) {
                e = launch_pdl(k_sf_btran<SF_BS>, dim3(sf_btran_blocks(D)), dim3(SF_BS), sf_smem(D), s, D, D.rho, 0);
            } else {
                const int nbw = (D.k + BS / 32 - 1) / (BS / 32);
                e = launch_pdl(k_btran_gemv<BS>, dim3(nbw + nblk(D.m)), dim3(BS), 0, s, D, D.rho, 0);
            }
            if (e) return e;
            break;
        }
        case S_PIVOT_ROW: {
            cudaError_t e = (D.n <= PR_CL_MAX_N) ? launch_pivot_row_cluster(D, s)
                                                 : launch_pdl(k_pivot_row<BS>, dim3(nblk(D.n)), dim3(BS), 0, s, D, 3);
            if (e) return e;
            break;
        }
        case S_DUAL_UPDATE: {
            cudaError_t e = D.dense ? launch_dual_update_cluster(D, s)
                                    : launch_pdl(k_dual_update<BS>, dim3(nblk(D.n)), dim3(BS), 0, s, D);
            if (e) return e;
            break;
        }
        case S_FTRAN_K:
            if (D.k > 0 && D.sf.on) {
                cudaError_t e = launch_pdl(k_sf_ftran<SF_BS>, dim3(MAX_FTRAN_RHS), dim3(SF_BS), sf_smem(D), s, D, 0, 0);
                if (e) return e;
            } else if (D.k > 0) {
                dim3 g(D.ftr_ntile, D.ftr_nchunk);
                const size_t sh = (size_t)D.ftr_chunk * MAX_FTRAN_RHS * sizeof(double);
                cudaError_t e = launch_pdl(k_ftran_k2<BS>, g, dim3(BS), sh, s, D, 0, 0);
                if (e) return e;
            } else {
                return cudaSuccess;
            }
            break;
        case S_FTRAN_ASM: { cudaError_t e = launch_pdl(k_ftran_assemble<BS>, dim3(nblk(D.m)), dim3(BS), g_smem_bytes(D.cap), s, D, 0, 0); if (e) return e; break; }
        case S_ETA_APPLY: { cudaError_t e = launch_pdl(k_eta_apply<BS_ETA>, dim3((D.m + BS_ETA - 1) / BS_ETA), dim3(BS_ETA * ETA_SPLIT), 0, s, D, 0, 1, 0); if (e) return e; break; }
        case S_UPDATE: { cudaError_t e = launch_pdl(k_update<BS>, dim3(nblk(D.m)), dim3(BS), 0, s, D, 0); if (e) return e; break; }
        default: return cudaErrorInvalidValue;
    }
    count_launch(1);
    return cudaGetLastError();
}

cudaError_t launch_body(const Dev& D, int from_stage, cudaStream_t s) {
    const int first = (from_stage <= ST_PRICING) ? S_SCORE : S_UPDATE;
    for (int st = first; st < S_NSTEPS; ++st) {
        cudaError_t e = launch_step(D, st, s);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_update_forced(const Dev& D, cudaStream_t s) {
    k_update<BS><<<nblk(D.m), BS, 0, s>>>(D, 1);
    count_launch(1);
    LAUNCH_OK();
    return cudaSuccess;
}

cudaError_t launch_iteration(const Dev& D, cudaStream_t s) {
    for (int st = S_SCORE; st < S_NSTEPS; ++st) {
        cudaError_t e = launch_step(D, st, s);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_set_primal_vars(const Dev& D, cudaStream_t s) {
    k_set_primal_vars<<<nblk(D.n), BS, 0, s>>>(D);
    count_launch(1);
    LAUNCH_OK();
    return cudaSuccess;
}

cudaError_t launch_xb_rhs(const Dev& D, double* rhs, cudaStream_t s) {
    k_xb_rhs<<<nblk(D.m), BS, 0, s>>>(D, rhs);
    count_launch(1);
    LAUNCH_OK();
    return cudaSuccess;
}

cudaError_t launch_scatter_basic(const Dev& D, const double* xb, double* dst, cudaStream_t s) {
    k_scatter_basic<<<nblk(D.m), BS, 0, s>>>(D, xb, dst);
    count_launch(1);
    LAUNCH_OK();
    return cudaSuccess;
}

cudaError_t launch_gather_basic_cost(const Dev& D, double* cb, cudaStream_t s) {
    k_gather_basic_cost<<<nblk(D.m), BS, 0, s>>>(D, cb);
    count_launch(1);
    LAUNCH_OK();
    return cudaSuccess;
}

cudaError_t launch_reduced_costs(const Dev& D, const double* y, cudaStream_t s) {
    k_reduced_costs<<<nblk(D.n), BS, 0, s>>>(D, y);
    count_launch(1);
    LAUNCH_OK();
    return cudaSuccess;
}

cudaError_t launch_btran_dense_eta(const Dev& D, const double* c0, double* h, int T, cudaStream_t s) {
    if (T > 0) k_eta_dots<BS><<<T, BS, 0, s>>>(D, c0, h);
    k_btran_dense_fix<BS><<<1, BS, g_smem_bytes(D.cap), s>>>(D, c0, h);
    count_launch((T > 0 ? 1 : 0) + 1);
    LAUNCH_OK();
    return cudaSuccess;
}

cudaError_t launch_btran_unit(const Dev& D, int p_idx, cudaStream_t s) {
    k_btran_unit<BS><<<1, BS, g_smem_bytes(D.cap), s>>>(D, p_idx);
    count_launch(1);
    LAUNCH_OK();
    return cudaSuccess;
}

cudaError_t launch_beta_exact(const Dev& D, cudaStream_t s) {
    if (D.k > 0) k_beta_exact_struct<BS><<<nblk(D.k), BS, 0, s>>>(D);
    k_beta_exact_slack<128><<<D.m, 128, 0, s>>>(D);
    count_launch((D.k > 0 ? 1 : 0) + 1);
    LAUNCH_OK();
    return cudaSuccess;
}

cudaError_t launch_norm2(const double* v, int n, double* out, cudaStream_t s) {
    k_norm2<BS><<<1, BS, 0, s>>>(v, n, out);
    count_launch(1);
    LAUNCH_OK();
    return cudaSuccess;
}

cudaError_t launch_dot_cost_x(const Dev& D, double* out, cudaStream_t s) {
    k_dot_cost_x<BS><<<1, BS, 0, s>>>(D, out);
    count_launch(1);
    LAUNCH_OK();
    return cudaSuccess;
}

cudaError_t launch_build_mtri(const Dev& D, int T, cudaStream_t s) {
    k_build_mtri<BS><<<1, BS, 0, s>>>(D, T);
    count_launch(1);
    LAUNCH_OK();
    return cudaSuccess;
}

cudaError_t launch_chuzr_only(const Dev& D, cudaStream_t s) {
    k_chuzr<BS><<<nblk(D.m > D.n ? D.m : D.n), BS, g_smem_bytes(D.cap), s>>>(D);
    count_launch(1);
    LAUNCH_OK();
    return cudaSuccess;
}

cudaError_t launch_pivot_row_mode(const Dev& D, int mode, cudaStream_t s) {
    k_pivot_row<BS><<<nblk(D.n), BS, 0, s>>>(D, mode);
    count_launch(1);
    LAUNCH_OK();
    return cudaSuccess;
}

cudaError_t launch_phase1_init(const Dev& D, double* cc, cudaStream_t s) {
    k_phase1_init<BS><<<1, BS, 0, s>>>(D, cc);
    count_launch(1);
    LAUNCH_OK();
    return cudaSuccess;
}

// ================================================================ dense mode
// The explicit inverse replaces the eta file for m up to ds_options.dense_max_m:
// Binv[r * m + i] = (B^-1)_{i r} (constraint row r, basis position i), so an
// FTRAN gathers whole columns (coalesced over positions) and the rank-1 update
// streams B^-1 once per iteration across every SM.

// B^-1 from the factor of B0 = P [K 0; C I]:  for a K row kr (constraint row
// r = rp_row[kr]) column r holds Kinv[:, kr] at the structural positions and
// -C Kinv[:, kr] at the slack positions; a slack row's column is a unit vector.
template <int BS>
__global__ void k_binv_struct(Dev D) {
    const int kr = blockIdx.x, k = D.k;
    const size_t r = (size_t)D.rp_row[kr];
    for (int c = threadIdx.x; c < k; c += BS) D.Binv[r * D.m + D.s_pos[c]] = D.Kinv[(size_t)kr * k + c];
}
template <int BS>
__global__ void k_binv_coupling(Dev D) {
    const int kr = blockIdx.x, k = D.k;
    const int rr = blockIdx.y * BS + threadIdx.x;
    if (rr >= D.m) return;
    const int sp = D.row_slackpos[rr];
    if (sp < 0) return;
    const double* kc = D.Kinv + (size_t)kr * k;
    double s = 0.0;
    for (int e = D.cpl_ptr[rr]; e < D.cpl_ptr[rr + 1]; ++e) s += D.cpl_val[e] * kc[D.cpl_col[e]];
    D.Binv[(size_t)D.rp_row[kr] * D.m + sp] = -s;
}
__global__ void k_binv_unit(Dev D) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= D.m) return;
    const int sp = D.row_slackpos[r];
    if (sp >= 0) D.Binv[(size_t)r * D.m + sp] = 1.0;
}

__global__ void k_dense_rho(Dev D, int p_idx) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < D.m) D.rho[r] = D.Binv[(size_t)r * D.m + p_idx];
}

// Iteration FTRAN: alpha_q = B^-1 a_q (a_q: CSC column or unit slack column) and,
// with bound flips, dx_B = B^-1 column_change; then the pivot check of k_eta_apply.
template <int BS>
__global__ void k_ftran_dense(Dev D, int check, int force) {
    Ctl* c = D.ctl;
    if (!force && halted(c)) return;
    const int q = c->q, nr = c->nrhs;
    const int i = blockIdx.x * BS + threadIdx.x;
    const size_t M = D.m;
    if (i < D.m) {
        double s = 0.0;
        if (q < D.n) {
#pragma unroll 4
            for (int e = D.cptr[q]; e < D.cptr[q + 1]; ++e) s += D.Binv[(size_t)D.crow[e] * M + i] * D.cval[e];
        } else {
            s = D.Binv[(size_t)(q - D.n) * M + i];
        }
        D.alpha_q[i] = s;
        if (nr > 2) {
            double t = 0.0;
            for (int r = 0; r < D.m; ++r) {
                const double v = D.cc[r];
                if (v != 0.0) t += D.Binv[(size_t)r * M + i] * v;
            }
            D.dxb[i] = t;
        }
    }
    if (!last_block(&c->tickets[6])) return;
    if (check && threadIdx.x == 0) {
        const double aqp = __ldcg(&D.alpha_q[c->p_idx]);
        const double apq = D.alpha[c->q_idx];
        if (!(fabs(aqp) > 0.0) || isnan(aqp)) raise_ev(c, EV_ERROR, ST_FTRAN);
        else if (fabs(aqp - apq) > EPS_R * (1 + fabs(aqp))) raise_ev(c, EV_MISMATCH, ST_FTRAN);
    }
}

// B^-1 <- E B^-1 with E the eta of (alpha_q, p): row p scaled by 1/alpha_p, row i
// minus alpha_q[i]/alpha_p times row p; fused with the exact DSE weights
// beta_i = ||row i of B^-1||^2 (chunk partials, summed in chunk order by the
// last block of each column tile).  Grid: (position tiles, row chunks).  Runs
// after k_update, whose bound-flip correction still needs the old B^-1.
// Sum of the chunk partials part[y * M + i], y = 0..ny-1, in chunk order, with
// sixteen loads in flight per batch.
__device__ __forceinline__ double sum_chunk_parts(const double* part, size_t M, int i, int ny) {
    double b = 0.0;
    for (int y0 = 0; y0 < ny; y0 += 16) {
        double t[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) t[k] = (y0 + k < ny) ? __ldcg(&part[(size_t)(y0 + k) * M + i]) : 0.0;
#pragma unroll
        for (int k = 0; k < 16; ++k)
            if (y0 + k < ny) b += t[k];
    }
    return b;
}

// B^-1 <- E B^-1 for the pivot (p, alpha_q) (Binv[r * m + i] = (B^-1)_{i,r}),
// with beta_i = ||row i of B^-1||^2 summed from the updated values.  A block
// covers 32 positions i (a lane each: one coalesced 256-byte segment per row)
// and BINV_ROWS rows r, BINV_RW per warp; the warps' sums are added in warp
// order in shared memory, and the last of a slice's row-chunk blocks adds the
// chunk partials in chunk order (8 for m = 2000), so beta is deterministic.
template <int BS>
__global__ void __launch_bounds__(BS) k_binv_update(Dev D, int force) {
    static_assert(BS == 8 * 32, "eight warps per block");
    pdl_enter();
    Ctl* c = D.ctl;
    if (!force && halted(c)) return;
    const int p = c->p_idx;
    const size_t M = D.m;
    const double inv = 1.0 / __ldcg(&D.alpha_q[p]);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int i = blockIdx.x * 32 + lane;
    const int r0 = blockIdx.y * BINV_ROWS + warp * BINV_RW, r1 = min(D.m, r0 + BINV_RW);
    double acc = 0.0;
    if (i < D.m) {
        const double f = D.alpha_q[i];
        const bool isp = (i == p);
        double* col = D.Binv + i;
        int r = r0;
        for (; r + 8 <= r1; r += 8) {
            double v[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) v[k] = col[(size_t)(r + k) * M];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const double piv = D.rho[r + k] * inv;
                const double nv = isp ? piv : v[k] - f * piv;
                col[(size_t)(r + k) * M] = nv;
                acc += nv * nv;
            }
        }
        for (; r < r1; ++r) {
            const double piv = D.rho[r] * inv;
            const double nv = isp ? piv : col[(size_t)r * M] - f * piv;
            col[(size_t)r * M] = nv;
            acc += nv * nv;
        }
    }
    __shared__ double s_acc[8][32];
    s_acc[warp][lane] = acc;
    __syncthreads();
    if (warp == 0 && i < D.m) {
        double b = 0.0;
#pragma unroll
        for (int w = 0; w < 8; ++w) b += s_acc[w][lane];
        D.binv_part[(size_t)blockIdx.y * M + i] = b;
    }
    if (!last_in_tile(&D.binv_tickets[blockIdx.x])) return;
    if (warp == 0 && i < D.m) D.beta[i] = sum_chunk_parts(D.binv_part, M, i, (int)gridDim.y);
}

// y = B^-1 v (mode 0) or y_i = ||row i of B^-1||^2 (mode 1), same tiling.
template <int BS>
__global__ void k_dense_colsum(Dev D, const double* v, double* y, int mode) {
    const size_t M = D.m;
    const int i = blockIdx.x * BS + threadIdx.x;
    const int r0 = blockIdx.y * D.binv_rc, r1 = min(D.m, r0 + D.binv_rc);
    if (i < D.m) {
        double acc = 0.0;
        for (int r = r0; r < r1; ++r) {
            const double b = D.Binv[(size_t)r * M + i];
            acc += mode ? b * b : b * v[r];
        }
        D.binv_part[(size_t)blockIdx.y * M + i] = acc;
    }
    if (!last_in_tile(&D.binv_tickets[blockIdx.x])) return;
    if (i < D.m) y[i] = sum_chunk_parts(D.binv_part, M, i, (int)gridDim.y);
}

// y = B^-T c: one warp per constraint row r, a contiguous dot over positions.
__global__ void k_dense_btran_vec(Dev D, const double* cpos, double* y) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= D.m) return;
    const double* col = D.Binv + (size_t)w * D.m;
    double s = 0.0;
    for (int i = lane; i < D.m; i += 32) s += col[i] * cpos[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) y[w] = s;
}

cudaError_t launch_binv_build(const Dev& D, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(D.Binv, 0, sizeof(double) * (size_t)D.m * D.m, s);
    if (e != cudaSuccess) return e;
    if (D.k > 0) {
        k_binv_struct<BS><<<D.k, BS, 0, s>>>(D);
        k_binv_coupling<BS><<<dim3(D.k, nblk(D.m)), BS, 0, s>>>(D);
        count_launch(2);
    }
    k_binv_unit<<<nblk(D.m), BS, 0, s>>>(D);
    count_launch(1);
    LAUNCH_OK();
    return cudaSuccess;
}

cudaError_t launch_dense_rho(const Dev& D, int p_idx, cudaStream_t s) {
    k_dense_rho<<<nblk(D.m), BS, 0, s>>>(D, p_idx);
    count_launch(1);
    LAUNCH_OK();
    return cudaSuccess;
}

cudaError_t launch_ftran_dense(const Dev& D, int check, int force, cudaStream_t s) {
    k_ftran_dense<BS><<<nblk(D.m), BS, 0, s>>>(D, check, force);
    count_launch(1);
    LAUNCH_OK();
    return cudaSuccess;
}

cudaError_t launch_binv_update(const Dev& D, int force, cudaStream_t s) {
    cudaError_t e = launch_pdl(k_binv_update<BS>, dim3((D.m + 31) / 32, (D.m + BINV_ROWS - 1) / BINV_ROWS), dim3(BS), 0, s,
                               D, force);
    if (e != cudaSuccess) return e;
    count_launch(1);
    LAUNCH_OK();
    return cudaSuccess;
}

cudaError_t launch_dense_ftran_vec(const Dev& D, const double* v, double* y, cudaStream_t s) {
    k_dense_colsum<BS><<<dim3(nblk(D.m), D.binv_chunks), BS, 0, s>>>(D, v, y, 0);
    count_launch(1);
    LAUNCH_OK();
    return cudaSuccess;
}

cudaError_t launch_binv_probe(const Dev& D, double* v, double* y, unsigned long long* out, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(out, 0, 2 * sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    k_probe_fill<<<nblk(D.m), BS, 0, s>>>(v, D.m);
    k_dense_colsum<BS><<<dim3(nblk(D.m), D.binv_chunks), BS, 0, s>>>(D, v, y, 0);
    k_basis_residual<BS><<<nblk(D.m), BS, 0, s>>>(D, y, v, out);
    count_launch(3);
    LAUNCH_OK();
    return cudaSuccess;
}

cudaError_t launch_dense_btran_vec(const Dev& D, const double* c, double* y, cudaStream_t s) {
    k_dense_btran_vec<<<(D.m * 32 + BS - 1) / BS, BS, 0, s>>>(D, c, y);
    count_launch(1);
    LAUNCH_OK();
    return cudaSuccess;
}

cudaError_t launch_dense_beta(const Dev& D, cudaStream_t s) {
    k_dense_colsum<BS><<<dim3(nblk(D.m), D.binv_chunks), BS, 0, s>>>(D, nullptr, D.beta, 1);
    count_launch(1);
    LAUNCH_OK();
    return cudaSuccess;
}

}  // namespace ds
