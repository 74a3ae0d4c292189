// Internal declarations of the B200 dual simplex engine.
//
// Layout in HBM (structure of arrays, all device resident for the whole solve):
//   LP (immutable):  structural A in CSC (column walks: pivot row, FTRAN rhs,
//                    basis build) and CSR (row walks: x_B init, coupling);
//                    lb/ub/type/cost per variable (n structurals + m slacks).
//   State:           x, d (N), beta (m), basis (m), nonbasis (n), var_pos (N).
//   Factor of B0:    the basis's structural block K = A[R', S] (k x k) kept as
//                    an explicit inverse Kinv (column major); slack columns of
//                    the basis are unit vectors and are eliminated exactly.
//   Eta file:        up to cap dense columns of m doubles + pivot positions, and
//                    G (cap x cap, G[t][u] = eta_u[p_t] - [p_u == p_t]): the
//                    chain's pivot values come from a small triangular solve,
//                    after which the eta columns are applied in one streaming pass.
//   Control:         a small Ctl block; every kernel of an iteration reads the
//                    decisions of the previous kernels from it and returns at
//                    once when a previous kernel raised an event.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace ds {

// Tolerances and constants of the reference, baseDualSimplex.hpp:23-46.
constexpr double EPS_BOUND = 1e-10;
constexpr double EPS_D = 1e-7;
constexpr double EPS_A = 1e-5;
constexpr double EPS_Z = 1e-10;
constexpr double EPS_R = 1e-9;
constexpr double EPS_F = 1e-10;
constexpr double INF_THETA = 1e25;   // INF
constexpr int MAX_CYCLE = 5;
constexpr int NEED_RESTART = 40;
constexpr double RT_WINDOW = 1e-9;   // CHUZC tie window (10 x EPS_Z), exactness checked

enum VarType : unsigned char { FIXED = 0, FREE = 1, BOXED = 2, UPPER = 3, LOWER = 4 };

enum Event : int {
    EV_NONE = 0,
    EV_ITER_LIMIT = 1,
    EV_REFACTOR_DUE = 2,   // iteration % R == 0 (top of loop)
    EV_DUALINF = 3,        // iteration % 40 == 0 and !checkDualFeasible
    EV_PERTURB = 4,        // !perturbed && cycle_num > MAX_CYCLE
    EV_OPTIMAL = 5,        // checkPrimalFeasible
    EV_NO_P = 6,           // DSEPricing found no row
    EV_UNBOUNDED = 7,      // ratio-test set F empty
    EV_MISMATCH = 8,       // |alpha_q[p] - alpha_p[q]| too large after FTRAN
    EV_ETA_FULL = 9,       // eta file at capacity after the append
    EV_ERROR = 10,         // no takeable ratio-test candidate / NaN pivot
    EV_P1_DONE = 11,       // phase 1: solved
    EV_P1_DUALINF = 12,    // phase 1: dual infeasible
    EV_P1_RESTART = 13,    // phase 1: soft restart (p < 0 or Z > 0)
    EV_P1_BLOCK = 14,      // phase 1: F empty -> block p and restart
};

// Stage labels for events and timing (reference TimeProfiler buckets, types.hpp:12-27).
enum Stage : int { ST_TOP = 0, ST_PRICING, ST_BTRAN, ST_PIVOTROW, ST_RATIO, ST_UPDRED,
                   ST_FTRAN, ST_UPDATE, ST_NSTAGES };

constexpr int TICKETS = 16;
constexpr int MAX_FTRAN_RHS = 3;

struct Ctl {
    int iteration, max_iter, R, event, halt, event_stage, phase;
    int p, p_idx, is_lower, primal_feasible, nop;
    double delta, beta_p;
    int q, q_idx, ncand, unbound_checked;
    double theta, delta_bfrt;
    int nflips, prev_q, nrhs, T;
    double dz, obj;
    int cycle, perturbed, need_dual_check, dual_infeas, k;
    int top_done;               // the host already ran this iteration's loop bookkeeping
    double f_p;                 // phase 1: f[p_idx]
    double z_phase1;            // phase 1 objective (obj_func_val)
    int p1_found, p1_dinf;
    int ybt_n;                  // positions set in the BTRAN work vector
    int pivots;                 // basis changes (both phases)
    int trace_n, trace_cap;
    int learned_used, learned_fallback;
    int window_fallbacks;       // CHUZC tie-window scans that needed the full scan
    int ftr_n;                  // feature-trace records written (may exceed the capacity)
    int ninfeas;                // primal infeasible positions at the last pricing
    int flips_total;            // bound flips of the BFRT ratio test, whole solve
    int err;
    unsigned tickets[TICKETS];
};

// Sparse LU of the structural bump K (eta-file mode, sparse_factor.cu).  The
// factor is a sequence of k pivots ("slots"): K's column singletons, the
// Markowitz pivots of its kernel, a small dense block, then K's row singletons,
// which puts K in block upper triangular form.  A B0 solve runs a program of
// levels over one vector of k slots: the ops of a level are independent, and
// each sets v[slot] = (v[slot] - sum_e coef_e * v[src_e]) / diag.
struct SfProg {
    int nlev;
    const int* lvl_ptr;        // nlev + 1: op ranges
    const int* lvl_kind;       // nlev: 0 sparse ops, 1 dense block (Sinv), 2 dense block (SinvT)
    const int* op_slot;        // per op: the slot it sets
    const int* op_ptr;         // nop + 1: entry ranges
    const double* op_diag;     // per op: divisor (1.0 for ops that only subtract)
    const int* ent_slot;       // per entry: source slot
    const double* ent_coef;    // per entry: coefficient
};
struct SfDev {
    int on;                    // 1: B0 solves use this factor instead of Kinv
    int k;                     // slots (bump size)
    int d0, kd;                // dense block: first slot, order
    int smem;                  // 1: the slot vector fits in shared memory
    const double* Sinv;        // kd x kd inverse of the dense block (column major)
    const double* SinvT;       // its transpose
    const int* slot_row;       // constraint row of the slot's pivot row
    const int* slot_kcol;      // K column of the slot's pivot column
    const int* slot_pos;       // basis position of the slot's pivot column
    SfProg ft, bt;             // FTRAN and BTRAN programs
    double* gvec;              // MAX_FTRAN_RHS * k slot vectors (when smem == 0)
    double* gtmp;              // MAX_FTRAN_RHS * kd dense-block scratch
};
constexpr int SF_SMEM_SLOTS = 26624;   // 208 KB of doubles: slot vectors up to this size live in shared memory

struct Dev {
    int m, n, N, cap;            // cap = eta file capacity
    int k;                       // bump size of the current factor
    // LP
    const int* cptr; const int* crow; const double* cval;      // structural CSC
    const int* rptr; const int* rcol; const double* rval;      // structural CSR
    const double* lb; const double* ub; const unsigned char* type;
    double* cost;
    // state
    double* x; double* d; double* beta; double* f;             // f: phase-1 vector (m)
    int* basis; int* nonbasis; int* var_pos;                   // var_pos: pos >= 0 or -(slot+1)
    unsigned char* blocked;                                     // phase 1 blocked rows (per var)
    // factor of B0
    int* s_pos; int* s_var; int* rp_row;                        // k each
    int* pos_kidx;                                              // m: position -> K column, -1 for slack
    int* row_slackpos;                                          // m: row -> slack position, -1 if in R'
    int* cpl_ptr; int* cpl_col; double* cpl_val;                // coupling A[R, S] by rows
    double* Kinv;                                               // k*k column major (dense factor)
    SfDev sf;                                                   // sparse factor (eta-file mode)
    // eta file
    double* eta; int* eta_pos; double* Mtri;                    // Mtri holds G (row t: G[t][0..t-1])
    // work vectors
    double* rho;        // m (rows)
    double* alpha;      // n (nonbasic slots), un-negated pivot row
    double* theta_arr;  // n; NaN where not a takeable candidate
    unsigned char* cand;// n; 1 if in F
    double* ybt;        // m (positions): BTRAN work vector after the eta pass
    int* ybt_pos;       // cap+1 positions touched in ybt
    double* btr_rhs;    // k
    double* aq_dense;   // m (rows): entering column
    double* cc;         // m (rows): BFRT column change
    double* alpha_q; double* tau; double* dxb;                  // m (positions)
    double* y0[MAX_FTRAN_RHS];                                  // m (positions)
    const double* frhs[MAX_FTRAN_RHS];                          // FTRAN right-hand sides (rows)
    double* fout[MAX_FTRAN_RHS];                                // FTRAN outputs (positions)
    double* ftr_part;   // nchunk * 3 * k partial sums
    double* s_eta;      // 3 * cap
    double* red;        // block partial scratch (doubles)
    int* redi;          // block partial scratch (ints)
    unsigned char* flip;// n slot flags: 1 low->ub, 2 up->lb
    int* flip_list;     // n
    int* trace;         // 2 * trace_cap ints (p, q)
    double* trace_d;    // 2 * trace_cap doubles (theta, obj)
    // learned pricing (mlp.cu)
    int learned;                // 1: CHUZR ranks rows by DSE weight x network score
    int learn_start;            // first iteration priced by the network (DSE before it)
    double learn_mix;           // score = w * (mix + (1 - mix) * sigmoid(logit))
    double learn_margin;        // minimum sigmoid(logit) of the network's row
    const void* mlp_w1;         // bf16 W1 (64 x 12), row major
    const void* mlp_w2;         // bf16 W2 (64 x 64), row major
    const float* mlp_p;         // fp32 parameters (biases, w3, b3)
    int* mlp_err;               // set when an MMA completion wait timed out
    float* score;               // m logits (-inf where the row is not a candidate)
    int* row_nnz;               // m: nonzeros of each row
    int* enter_count;           // N: times each variable entered the basis
    int* entered_at;            // N: iteration of its last entry
    // feature trace (training data): candidate rows every ftr_every iterations
    int ftr_every;              // 0: off
    int ftr_cap;                // records
    float* ftr_feat;            // ftr_cap x DS_NUM_FEATURES
    int* ftr_meta;              // ftr_cap x 3: iteration, position, variable
    const float* pd_gap;        // N: PDHG estimate's distance to the nearest bound
    const float* pd_dual;       // N: PDHG estimate's dual magnitude
    // dense mode (m <= ds_options.dense_max_m): explicit B^-1, column r (constraint
    // row r) contiguous over basis positions: Binv[r * m + i] = (B^-1)_{i r}
    int dense;
    double* Binv;               // m * m
    double* binv_part;          // binv_chunks * m partial sums (exact DSE weights, dense FTRAN)
    unsigned* binv_tickets;     // one per column tile of BS positions
    int binv_rc, binv_chunks;   // rows of B^-1 per chunk, chunk count
    Ctl* ctl;
    // launch geometry (set per factor)
    int ftr_tile, ftr_chunk, ftr_ntile, ftr_nchunk;
    unsigned* tile_tickets; // ftr_ntile
};

#ifdef __CUDACC__
// ------------------------------------------------------------ per-variable rules
// checkVarIsInfeas (baseDualSimplex.tpp:443-466) with its case fallthrough.
__device__ __forceinline__ bool var_infeas(unsigned char t, double x, double l, double u, double* delta) {
    switch (t) {
        case LOWER:
            if (x < l - EPS_BOUND) { *delta = x - l; return true; }
            [[fallthrough]];
        case UPPER:
            if (x > u + EPS_BOUND) { *delta = x - u; return true; }
            [[fallthrough]];
        case FIXED:
            if (fabs(x - l) < EPS_BOUND) { *delta = x - l; return true; }
            [[fallthrough]];
        case BOXED:
            if (x > u + EPS_BOUND) { *delta = x - u; return true; }
            else if (x < l - EPS_BOUND) { *delta = x - l; return true; }
    }
    *delta = 0.0;
    return false;
}

// checkPrimalFeasible (tpp:296-324) for one basic variable, fallthrough kept.
__device__ __forceinline__ bool var_primal_ok(unsigned char t, double x, double l, double u) {
    switch (t) {
        case FIXED:
            if (fabs(x - l) > EPS_BOUND) return false;
            [[fallthrough]];
        case FREE: return true;
        case BOXED:
            if (x > u + EPS_R * fabs(u) + EPS_BOUND || x < l - EPS_R * fabs(l) - EPS_BOUND) return false;
            [[fallthrough]];
        case UPPER:
            if (x > u + EPS_R * fabs(u) + EPS_BOUND) return false;
            [[fallthrough]];
        case LOWER:
            if (x < l - EPS_R * fabs(l) - EPS_BOUND) return false;
    }
    return true;
}

#endif

}  // namespace ds
