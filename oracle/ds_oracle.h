/*
 * ds_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of veret-v/parallel_ds's sequential dual simplex
 * (src/cpu/sequentialDualSimplex.cpp + src/common/baseDualSimplex.tpp) used as
 * the parity checker for the CUDA engine.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg may load it; the product never does.
 *
 * The reference itself cannot be built here (it needs MKL PARDISO, COIN-OR Clp
 * and cuDSS, none of which exist in this image), so this is a port.  Its LU
 * stands in for PARDISO (matrix.cpp:530-583): a dense LU with partial pivoting
 * of the structural part of the basis; the slack part is solved exactly.
 */
#ifndef DS_ORACLE_H
#define DS_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_options {
    int refactor_interval;      /* REFACT_FREQ */
    int max_iterations;
    int strict_reference;       /* 1: no engine guards (see ds_api.h)         */
    unsigned long long seed;    /* perturbation seed                            */
    int gpu_control_flow;       /* 1: follow cudaDualSimplex.cpp's restarts     */
    int verbose;
    const double* var_weight;   /* experiments: DSE score of row i is multiplied by
                                   var_weight[basis[i]] (NULL: plain DSE)          */
    int harris;                 /* experiments: phase-2 ratio test by the two-pass
                                   Harris rule (tolerance EPS_D) instead of the
                                   reference's simpleRatioTest (0: reference)      */
    int block_lu;               /* experiments: factorise the structural block by
                                   singleton triangularisation + an LU of the
                                   kernel only: 1 dense, 2 sequential Markowitz
                                   (0: dense LU of the whole block)             */
    double rt_rel_tol;          /* experiments: phase-2 ratio-test candidates with
                                   |alpha_j| below this fraction of the largest
                                   candidate |alpha| are left out (0: reference) */
    double col_rel_tol;         /* experiments: a phase-2 pivot |alpha_q[p]| below
                                   this fraction of max_i |alpha_q[i]| is refused:
                                   the factor is rebuilt and row p is left out of
                                   pricing for 100 iterations (0: reference)    */
    double pivot_abs_tol;       /* experiments: phase-2 ratio-test candidates need
                                   |alpha_j| above this instead of EPS_A = 1e-5
                                   (0: reference)                              */
    int shift_costs;            /* experiments: once the costs are perturbed, a dual
                                   infeasible basis is repaired by shifting the
                                   wrong-signed nonbasic costs instead of phase 1 */
} or_options;

typedef struct or_result {
    int status;                 /* DS_STATUS_* values                          */
    int iterations;
    int phase1_iterations;
    int refactors;
    int restarts;
    int perturbed;
    int bfrt_flips;
    int bump_size;
    double objective;           /* c^T x over structurals (original costs)     */
    double obj_incremental;     /* reference obj_func_val after postProcess    */
    /* pivot statistics of the phase-2 basis changes (numerical diagnostics) */
    double min_pivot;           /* smallest |alpha_q[p]|                        */
    double min_pivot_rel;       /* smallest |alpha_q[p]| / max_i |alpha_q[i]|   */
    double max_step;            /* largest |theta_P| = |delta / alpha_q[p]|     */
    int refused_pivots;         /* experiments (col_rel_tol): pivots refused    */
} or_result;

void or_default_options(or_options* o);

/* Solve with explicit types (reference Problem 8-argument ctor).  x_out/d_out:
 * N = n + m values each (may be NULL).  trace_*: per phase-2 iteration p, q,
 * theta, incremental objective (may be NULL; trace_cap entries). */
int or_solve_typed(int m, int n, const int* row_ptr, const int* col_idx, const double* val,
                   const double* c, const int* col_type, const double* col_lb, const double* col_ub,
                   const int* row_type, const double* row_lb, const double* row_ub,
                   const or_options* opt, or_result* res, double* x_out, double* d_out,
                   int* basis_out, int* trace_p, int* trace_q, double* trace_theta,
                   double* trace_obj, int trace_cap, int* trace_count);

/* Vector-level restatements for index-selection parity. */
int or_dse_pricing(int m, const int* basis, const double* x, const double* lb, const double* ub,
                   const int* type, const double* beta, int* p, int* p_idx, double* delta,
                   int* is_lower, int* primal_feasible);
int or_ratio_test(int n, const int* nonbasis, const double* alpha, double delta, int is_lower,
                  const double* x, const double* d, const double* lb, const double* ub,
                  const int* type, int* q, int* q_idx, double* theta, double* delta_out,
                  int* num_candidates);
int or_pivot_row(int m, int n, const int* csc_ptr, const int* csc_row, const double* csc_val,
                 const int* nonbasis, const double* rho, double* alpha);
int or_pfi_apply(int m, int T, const double* eta, const int* pos, const double* rhs,
                 double* sol, int transpose);
/* Dense B x = b / B^T x = b with partial-pivoting LU (PARDISO phase 12/33 stand-in). */
int or_dense_solve(int n, const int* csr_ptr, const int* csr_col, const double* csr_val,
                   const double* rhs, double* sol, int transpose);

#ifdef __cplusplus
}
#endif
#endif
