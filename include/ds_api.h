/*
 * ds_api.h -- C ABI of the B200 dual simplex engine (libds_b200.so).
 *
 * The entry points replace the solver surface of veret-v/parallel_ds, which
 * is C++ only (no C ABI).  Each declaration cites the reference interface it
 * stands in for, by file:line within that project.
 *
 * Conventions
 *   - Every function returns 0 (DS_OK) on success and a negative DS_ERR_* code
 *     on failure; no C++ exception crosses this boundary.  ds_last_error()
 *     returns a message for the last failure on a handle.
 *   - Host pointers only; inputs are copied, the caller keeps ownership.
 *   - A bound with |v| > 1e100 is infinite (reference problem.hpp:31,83).
 *   - Variables are numbered like the reference's computational form
 *     (problem.tpp:176-226): columns 0..n-1 are the structurals, n..n+m-1 the
 *     row slacks, with A x + s = 0 and s in [-row_ub, -row_lb].
 *   - One handle per host thread; each handle owns a CUDA stream.
 */
#ifndef DS_API_H
#define DS_API_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- return codes ------------------------------------------------------- */
#define DS_OK               0
#define DS_ERR_ARG         -1   /* bad argument (null pointer, bad size)      */
#define DS_ERR_CUDA        -2   /* CUDA runtime failure                       */
#define DS_ERR_STATE       -3   /* call out of order (e.g. solve before load) */
#define DS_ERR_SHAPE       -4   /* m > n: reference problem.tpp:230-239       */
#define DS_ERR_NUMERIC     -5   /* singular basis / NaN in the iteration      */
#define DS_ERR_DEVICE_WAIT -6   /* a bounded device-side wait ran out         */
#define DS_ERR_CAPACITY    -7   /* a size exceeds a fixed capacity            */

/* ---- solution status (reference LPsolution.message values) ------------- */
#define DS_STATUS_UNSOLVED          0
#define DS_STATUS_OPTIMAL           1  /* "optimal solution" cudaDualSimplex.cpp:451 */
#define DS_STATUS_PRIMAL_INFEASIBLE 2  /* "dual unbounded"   cudaDualSimplex.cpp:500 */
#define DS_STATUS_DUAL_INFEASIBLE   3  /* "dual infeasible"  baseDualSimplex.tpp:851 */
#define DS_STATUS_ITER_LIMIT        4  /* reference has no limit (MAX_ITER unused)   */
#define DS_STATUS_ERROR             5

/* ---- bound types: same order as reference enum BoundaryType (types.hpp:49-57) */
#define DS_FIXED 0
#define DS_FREE  1
#define DS_BOXED 2
#define DS_UPPER 3   /* only an upper bound */
#define DS_LOWER 4   /* only a lower bound  */

/* ---- pricing rules ------------------------------------------------------ */
#define DS_PRICING_DSE     0   /* dual steepest edge, baseDualSimplex.tpp:470-501  */
#define DS_PRICING_LEARNED 1   /* MLP leaving-row scorer with DSE fallback (new)   */

typedef struct ds_options {
    int    refactor_interval;  /* REFACT_FREQ (baseDualSimplex.hpp:41 = 150); default 100 */
    int    max_iterations;     /* iteration cap -> DS_STATUS_ITER_LIMIT; default 2,000,000 */
    int    pricing;            /* DS_PRICING_*                                     */
    int    strict_reference;   /* 1: reproduce the reference's control flow with no
                                  engine guards (no post-perturbation cleanup, no
                                  restart-loop guard)                               */
    unsigned long long seed;   /* seeds the cost perturbation (the reference draws
                                  from std::random_device, baseDualSimplex.tpp:244) */
    int    device;             /* CUDA device ordinal                              */
    void*  stream;             /* cudaStream_t to use, or NULL for an own stream   */
    double learned_margin;     /* learned pricing: the network's row is taken only
                                  when sigmoid(logit) of that row reaches this
                                  value, else the DSE row is (default 0.5)        */
    int    verbose;            /* 0 silent, 1 events, 2 every iteration            */
    double learned_mix;        /* learned pricing ranks candidate rows by
                                  w_i * (mix + (1 - mix) * sigmoid(logit_i)),
                                  w_i the DSE weight (default 0.05)               */
    int    learned_pdhg_iters; /* learned pricing and feature traces: PDHG
                                  iterations of the warm-start estimate whose
                                  bound gaps and duals are network features
                                  (default 4000; 0 = off)                         */
    int    dense_max_m;        /* m <= this: keep B^-1 explicitly (m*m doubles) and
                                  update it by a rank-1 step per iteration instead of
                                  the eta file; exact DSE weights (default 4096;
                                  0 = always the eta file)                        */
    int    dense_refactor_interval; /* dense mode: iterations between accuracy checks
                                  of B^-1 (default 400): a probe residual
                                  |B (B^-1 v) - v| above 1e-10 (1 + |B^-1 v|)
                                  rebuilds it from a fresh factorisation; a pivot
                                  mismatch rebuilds it at once as well             */
    int    learned_start_iteration; /* learned pricing: iterations before this one use
                                  DSE while the PDHG warm start runs on a second
                                  stream (default -1 = 7m/20; 0 = wait for it first) */
    int    pdhg_cluster;       /* 1: run the PDHG warm start inside one 16-CTA thread-
                                  block cluster when the LP fits its shared memory
                                  (default 1); 0: always the launch-per-step graph */
    int    factor_mode;        /* eta-file mode's factorisation of B0 (the reference's
                                  cuDSS LU, cudaSparseMatrix.cpp:502-567):
                                  DS_FACTOR_SPARSE (default) a sparse LU of the
                                  structural block (singleton triangularisation,
                                  Markowitz kernel LU on the device, level-scheduled
                                  solves); DS_FACTOR_DENSE an explicit dense inverse
                                  of the structural block (Gauss-Jordan).  Dense
                                  mode (dense_max_m) always builds the dense inverse */
} ds_options;

#define DS_FACTOR_SPARSE 0
#define DS_FACTOR_DENSE  1

typedef struct ds_stats {
    int    iterations;         /* reference `iteration` counter (phase 1 + 2)      */
    int    phase1_iterations;
    int    refactors;
    int    restarts;
    int    perturbed;
    int    bfrt_flips;
    int    learned_used;       /* iterations where the network's row was taken     */
    int    learned_fallback;   /* iterations that fell back to DSE                 */
    int    bump_size;          /* structurals in the last factorised basis         */
    int    kernel_launches;    /* kernels launched by the solve                    */
    double solve_ms;           /* device time of ds_solve (CUDA events)            */
    double refactor_ms;        /* time spent refactorising: device time of the dense
                                  inverse; for the sparse LU the whole factorisation
                                  (host triangularisation and program building, device
                                  kernel LU), host wall time                       */
    double pdhg_ms;            /* device time of the PDHG warm-start estimate      */
    int    lu_kernel;          /* sparse LU, last factorisation: order of the bump's
                                  kernel left by the singleton triangularisation  */
    int    lu_dense;           /* ... order of the dense block left by the kernel's
                                  Markowitz rounds                                */
    int    lu_levels;          /* ... levels of the FTRAN plus the BTRAN program   */
    int    lu_rounds;          /* ... Markowitz rounds of the kernel LU            */
} ds_stats;

typedef struct ds_solver ds_solver;

void        ds_default_options(ds_options* opts);
const char* ds_version(void);

/* Create/destroy a solver handle.
 * Replaces CudaDualSimplex(problem) + initDualSimplex()
 * (cudaDualSimplex.hpp:83-86, cudaDualSimplex.cpp:20-81). */
int ds_create(const ds_options* opts, ds_solver** out);
int ds_destroy(ds_solver* s);

/* Load min c^T x, row_lb <= A x <= row_ub, col_lb <= x <= col_ub with A in CSR.
 * Bound types follow Problem::readMps (problem.tpp:350-395); slacks follow
 * transformToComputeForm (problem.tpp:176-226). */
int ds_load_csr(ds_solver* s, int m, int n,
                const int* row_ptr, const int* col_idx, const double* val,
                const double* c,
                const double* col_lb, const double* col_ub,
                const double* row_lb, const double* row_ub);

/* MPS input for callers without Clp: replaces Problem::readMps over
 * ClpModel::readMps (problem.tpp:332-409).  Fixed or free format; the first N
 * row is the objective (further N rows are dropped); RANGES, BOUNDS
 * UP/LO/FX/FR/MI/PL/BV/LI/UI (integrality ignored), the first RHS/RANGES/BOUNDS
 * set; |value| >= 1e30 is infinite (+-1e300 in the arrays); SC bounds and
 * OBJSENSE MAX are rejected.  obj_offset receives the RHS of the objective
 * row: reported objectives are c^T x - obj_offset, as problem.tpp:256 does with
 * ClpModel::objectiveOffset.
 * ds_mps_read: call once with the array pointers NULL for m, n and nnz, then
 * with arrays of m+1, nnz, nnz, n, n, n, m, m entries.  Parse errors return
 * DS_ERR_ARG with the message in ds_mps_last_error() (per host thread).
 * ds_load_mps: parse and ds_load_csr in one call. */
int ds_mps_read(const char* path, int* m, int* n, long long* nnz,
                int* row_ptr, int* col_idx, double* val, double* c,
                double* col_lb, double* col_ub, double* row_lb, double* row_ub,
                double* obj_offset);
int ds_load_mps(ds_solver* s, const char* path, double* obj_offset);
const char* ds_mps_last_error(void);

/* Load with explicit bound types: the reference's 8-argument Problem ctor
 * (problem.tpp:143-173) -- bound_type, range_type, costs, lower_range,
 * upper_range, lower_bound, upper_bound, A(CSR, matrix.cpp:21-36). */
int ds_load_typed(ds_solver* s, int m, int n,
                  const int* row_ptr, const int* col_idx, const double* val,
                  const double* c,
                  const int* col_type, const double* col_lb, const double* col_ub,
                  const int* row_type, const double* row_lb, const double* row_ub);

/* presolve("minInfeas") + solve() + postProcess
 * (baseDualSimplex.tpp:5-30, 164-180, 123-159; main.cpp:84-87). */
int ds_solve(ds_solver* s);

int    ds_get_status(const ds_solver* s);
/* c^T x of the final point (recomputed, not the incremental value). */
double ds_get_objective(const ds_solver* s);
/* Problem::getSolution x (problem.tpp:243-259): x[n] structurals, slacks[m] (may be NULL). */
int    ds_get_primal(const ds_solver* s, double* x, double* slacks);
/* Row duals y_i = -d_{n+i}; the reference keeps d protected (baseDualSimplex.hpp:76). */
int    ds_get_dual(const ds_solver* s, double* y);
int    ds_get_reduced_costs(const ds_solver* s, double* d);
int    ds_get_iterations(const ds_solver* s);
int    ds_get_stats(const ds_solver* s, ds_stats* st);
/* Basis as variable indices per basis position (basis_indexes, baseDualSimplex.hpp:80). */
int    ds_get_basis(const ds_solver* s, int* basis);
const char* ds_last_error(const ds_solver* s);

/* Record (p, q, theta, objective) per phase-2 iteration into caller arrays
 * (the reference prints these lines under DEBUG, cudaDualSimplex.cpp:636-641).
 * Pass cap = 0 to stop tracing. */
int ds_set_trace(ds_solver* s, int cap);
int ds_get_trace(const ds_solver* s, int* p, int* q, double* theta, double* obj, int* count);


/* ---- learned pricing ----------------------------------------------------------
 * No counterpart in the reference (its pricing is DSE only, tpp:470-501).
 * A model is an MLP DS_NUM_FEATURES -> 64 -> 64 -> 1 (ReLU) whose logit
 * estimates whether a candidate row's basic variable leaves the basis for good
 * (is nonbasic at the optimum).  Inference and training run on the tensor
 * cores (BF16 operands, FP32 accumulation); parameters are FP32 in the order
 * W1[64][DS_NUM_FEATURES], b1[64], W2[64][64], b2[64], w3[64], b3. */
#define DS_NUM_FEATURES 12
#define DS_MLP_NPARAMS (64 * DS_NUM_FEATURES + 64 + 64 * 64 + 64 + 64 + 1)
/* Features of a candidate row i with basic variable j, at iteration it:
 *  0 j is a slack            1 log10|delta|/4          2 log10(beta_i)/4
 *  3 log10(delta^2/beta)/4   4 log10(w_i / w of the previous pick)/4
 *  5 asinh(1000 g_j)/8, g_j the distance of the PDHG estimate of j (slack:
 *    of its row's activity) to its nearest finite bound
 *  6 asinh(1000 |d_j|)/8, d_j the PDHG estimate's reduced cost of j (slack:
 *    its row dual)                 7 infeasible rows at the previous pricing / m
 *  8 min(it/m, 10)/5               9 min(times j entered, 20)/5
 * 10 min((it - last entry of j)/m, 5)   11 sign(x_j) log10(1 + |x_j|)
 * (logs and asinh terms clamped; see csrc/mlp.cu) */
typedef struct ds_model ds_model;
int ds_model_create(int device, ds_model** out);
int ds_model_destroy(ds_model* m);
int ds_model_set_params(ds_model* m, const float* params, int count);
int ds_model_get_params(const ds_model* m, float* params, int count);
/* Forward pass over rows x DS_NUM_FEATURES floats: logits (rows); H1, H2 (rows x 64
 * post-ReLU activations, may be NULL). */
int ds_model_forward(ds_model* m, const float* X, int rows, float* logits, float* H1, float* H2);
/* Mean binary cross-entropy with logits over the rows and its gradient
 * (DS_MLP_NPARAMS floats, parameter order). */
int ds_model_gradients(ds_model* m, const float* X, const float* y, int rows, float* grads, float* loss);
/* Adam (lr, beta1 0.9, beta2 0.999, eps 1e-8) over epochs of shuffled
 * mini-batches (batch a multiple of 128); the rows stay on the device.
 * mean_loss: mean batch loss of the last epoch. */
int ds_model_train(ds_model* m, const float* X, const float* y, int rows, int epochs, int batch, float lr,
                   unsigned long long seed, float* mean_loss);
/* Attach a model (not owned; NULL detaches).  Required when pricing is
 * DS_PRICING_LEARNED; must live on the solver's device. */
int ds_set_model(ds_solver* s, ds_model* m);
/* Failure-path testing of the scorer's bounded waits.  No reference
 * counterpart.  polls > 0 replaces the bound of the wait for the network's
 * tensor-core MMAs by that many non-blocking polls (after which the kernel
 * still waits, bounded, for the MMAs to finish before it reads or frees their
 * TMEM columns): too short a bound makes the scoring launches time out, their
 * scores unusable (DSE prices those iterations) and ds_solve return
 * DS_ERR_DEVICE_WAIT with the solve otherwise complete.  polls = 0 restores the
 * default bound (2^26 polls).  Also clears the model's timeout flag. */
int ds_model_set_wait_limit(ds_model* m, int polls);
/* PDHG estimate of an optimal primal-dual pair of the loaded LP after iters
 * iterations (rounded up to whole restart periods of 500): x (n), row duals
 * y (m) with c + A^T y the reduced costs.  The learned scorer's warm-start
 * evidence, exposed for checking and for callers that want a crash point. */
int ds_pdhg_estimate(ds_solver* s, int iters, double* x, double* y);
/* Feature trace for training: every `every` phase-2 iterations, the features of
 * each candidate row (up to cap records per solve).  every = 0 turns it off. */
int ds_set_feature_trace(ds_solver* s, int every, int cap);
/* feat: count x DS_NUM_FEATURES floats; meta: count x 3 ints (iteration, basis
 * position, variable), ordered by iteration then position.  *count receives the
 * number of records kept (at most cap); *total (may be NULL) all candidates seen. */
int ds_get_feature_trace(const ds_solver* s, float* feat, int* meta, int* count, int* total);

/* Factorise the basis given as m variable indices (structurals 0..n-1, slacks
 * n..n+m-1) and apply B^-1 (transpose = 0: rhs by rows -> out by basis
 * positions) or B^-T (transpose = 1: positions -> rows) to nrhs vectors of m
 * doubles stored one after another.  Replaces the reference's
 * CudaDualSimplex::solveLinSys after reFactorize (cudaDualSimplex.cpp:105-151,
 * 229-238); the loaded LP supplies A. */
int ds_basis_solve(ds_solver* s, const int* basis, const double* rhs, double* out, int nrhs, int transpose);

/* Kernels launched by this library in this process so far (graph replays
 * counted per kernel node).  No reference counterpart. */
long long ds_kernel_launch_count(void);

/* Re-solve the loaded LP with every iteration kernel bracketed by CUDA events
 * (one iteration per synchronisation) and write a JSON summary: per kernel its
 * launches, total and mean device time, algorithmic bytes per launch and share.
 * Stands in for the reference's TimeProfiler report (timeProfiler.cpp:108-148). */
int ds_profile_solve(ds_solver* s, char* json, int len);

/* ---- kernel-level entry points (run one device kernel on host vectors) ----
 * For index-selection parity against the reference on identical inputs. */

/* CHUZR: BaseDualSimplex::DSEPricing + checkVarIsInfeas (baseDualSimplex.tpp:443-501)
 * with an empty blocked set; also returns checkPrimalFeasible (tpp:296-324). */
int ds_kernel_dse_pricing(int m, int N, const int* basis, const double* x,
                          const double* lb, const double* ub, const int* type,
                          const double* beta,
                          int* p, int* p_idx, double* delta, int* is_lower,
                          int* primal_feasible);

/* Pivot row: CudaSparseMatrix::dotUpdate(UPDATE_T) for alpha=1, beta=0
 * (cudaSparseMatrix.cpp:359-378; CPU order matrix.cpp:273-286).
 * A is the structural CSC (n columns); slack columns are implicit. */
int ds_kernel_pivot_row(int m, int n, const int* csc_ptr, const int* csc_row,
                        const double* csc_val, const int* nonbasis,
                        const double* rho, double* alpha);

/* CHUZC: simpleRatioTestPart1 + simpleRatioTest + the bound-flipping loop
 * (cudaDualSimplex.cpp:367-394, 484-549; baseDualSimplex.tpp:546-572).
 * alpha is the un-negated pivot row; delta the signed primal infeasibility. */
int ds_kernel_ratio_test(int n, int N, const int* nonbasis, const double* alpha,
                         double delta, int is_lower,
                         const double* x, const double* d,
                         const double* lb, const double* ub, const int* type,
                         int* q, int* q_idx, double* theta, double* delta_out,
                         int* num_candidates);

/* Ratio test that allocates no device memory.  No counterpart in the
 * reference.  For callers that cannot call cudaMalloc: a host framework that
 * owns all device memory through its own pool (a stray cudaMalloc breaks its
 * accounting and can fail under its memory cap), or a latency-critical loop
 * where cudaMalloc/cudaFree would stall the device.  Same kernel and results
 * as ds_kernel_ratio_test, but every array argument is a DEVICE pointer the
 * caller owns and the outputs are host scalars.  Note the type array: ONE BYTE
 * per variable (DS_* codes as unsigned char), where ds_kernel_ratio_test takes
 * an int per variable; passing int32 codes here is read as garbage types.
 * Scratch lives in a fixed array of about 0.6 MB that every GPU loading this
 * library holds until exit; n > DS_NOALLOC_MAX_SLOTS returns DS_ERR_CAPACITY.
 * The first call on a device looks up that array's device address and keeps
 * it for the life of the process, so make the first call before any stream
 * capture begins, and do not call it again after resetting the device
 * (cudaDeviceReset invalidates the kept address).  All calls share the array:
 * calls that overlap on the GPU (other threads, other streams) race.  stream
 * may be NULL.  The call copies its result back and synchronises its stream
 * before it returns, so it makes CUDA calls of its own: it must not be made
 * from inside a host function queued on a stream (cudaLaunchHostFunc), where
 * CUDA calls are not allowed, nor on a stream that is being captured into a
 * CUDA graph (the synchronisation ends the capture with an error). */
#define DS_NOALLOC_MAX_SLOTS 65536
int ds_kernel_ratio_test_noalloc(int n, int N, const int* nonbasis, const double* alpha,
                                 double delta, int is_lower, const double* x, const double* d,
                                 const double* lb, const double* ub, const unsigned char* type,
                                 int* q, int* q_idx, double* theta, double* delta_out,
                                 int* num_candidates, void* stream);

/* PFI eta file: linalg::PFIsolve (linalg.cpp:12-46) / etaSolveKernel
 * (cudaKernels.cu:266-322): apply T eta columns (eta[t*m + i], pivots pos[t])
 * forward (transpose=0) or backward (transpose=1) to rhs, result in sol. */
int ds_kernel_pfi_apply(int m, int T, const double* eta, const int* pos,
                        const double* rhs, double* sol, int transpose);

/* Singleton triangularisation of a k x k sparse pattern (CSC col_ptr, row_idx;
 * values not needed), the host stage of the eta-file mode's sparse LU of B0's
 * structural block (it replaces the analysis phase of the reference's cuDSS
 * factorisation, cudaSparseMatrix.cpp:502-567).  row_order and col_order (k
 * each) receive the rows and columns in pivot order: the column singletons,
 * then the kernel (rows and columns in index order), then the row singletons,
 * so that the permuted matrix is block upper triangular around the kernel.
 * *n_col1 and *n_kernel receive the counts of the first two groups.  Host
 * only (no device work).  DS_ERR_NUMERIC if the pattern is structurally
 * singular. */
int ds_sparse_triangularise(int k, const int* col_ptr, const int* row_idx, int* row_order, int* col_order,
                            int* n_col1, int* n_kernel);

/* Device time in milliseconds (CUDA events on the default stream) of the
 * kernels that the calling thread's last ds_kernel_pivot_row or
 * ds_kernel_pfi_apply call launched, host copies excluded: the per-kernel
 * figure compared with the reference's spmvUpdateTKernel and etaSolveKernel
 * (cudaKernels.cu:108-157, 266-322) on identical inputs.  No reference
 * counterpart.  DS_ERR_STATE if no timed call ran yet. */
int ds_kernel_last_time(double* ms);

/* ---- batched persistent solver -------------------------------------------------
 * No counterpart in the reference.  Many independent LPs
 *     min c^T x  s.t.  A x <= b,  x >= 0        (m <= DS_BATCH_MAX_M, any n)
 * solved in one persistent launch (CUDA graph), each by the reference's dual
 * simplex rules (DSE pricing, textbook ratio test with the EPS_Z tie rule)
 * on a dense explicit basis inverse.  The slack basis must be dual feasible
 * (c >= 0); other instances get DS_STATUS_ERROR and belong on ds_solve, which
 * has phase 1.  Statuses: DS_STATUS_OPTIMAL, DS_STATUS_PRIMAL_INFEASIBLE,
 * DS_STATUS_ITER_LIMIT (50 m iterations, at least 1000), DS_STATUS_ERROR. */
#define DS_BATCH_MAX_M 1024
typedef struct ds_batch ds_batch;
typedef struct ds_batch_stats {
    int       count;            /* instances loaded                                */
    int       buckets;          /* m-buckets of the schedule                       */
    int       block;            /* threads per CTA of the persistent launch        */
    double    solve_ms;         /* device time of the last ds_batch_solve          */
    double    tune_ms;          /* device time of the last ds_batch_tune           */
    long long total_nnz;
    char      schedule[512];    /* group size and B^-1 placement per bucket        */
} ds_batch_stats;
int ds_batch_create(int device, ds_batch** out);
int ds_batch_destroy(ds_batch* b);
const char* ds_batch_last_error(const ds_batch* b);
/* count instances, concatenated: instance i has m[i] rows, n[i] columns, column
 * pointers col_ptr (n[i]+1 entries starting at 0), row_idx/val (col_ptr[n[i]]
 * entries), rhs (m[i]) and cost (n[i]).  Inputs are copied.  m[i] above
 * DS_BATCH_MAX_M returns DS_ERR_CAPACITY.  Reloading instances of the same
 * shapes keeps the schedule (tuned or set) and the captured launch. */
int ds_batch_load(ds_batch* b, int count, const int* m, const int* n, const int* col_ptr, const int* row_idx,
                  const double* val, const double* rhs, const double* cost);
/* Generate and load count instances of the seeded generator (instance i: seed
 * + i, m ~ U{m_lo..m_hi} by ds_gen_batch_m, n = 2m, Bernoulli(density)). */
int ds_batch_generate(ds_batch* b, int count, int m_lo, int m_hi, double density, unsigned long long seed);
/* The same instances into caller arrays (the ds_batch_load layout).  Call with
 * col_ptr == NULL first: sizes[0..3] receive the lengths of col_ptr, row_idx /
 * val, rhs and cost, and m/n (count each, may be NULL) the shapes. */
long long ds_batch_gen_arrays(int count, int m_lo, int m_hi, double density, unsigned long long seed, int* m,
                              int* n, int* col_ptr, int* row_idx, double* val, double* rhs, double* cost,
                              long long* sizes);
/* Autotune the schedule: per m-bucket group size (32..512 threads) and B^-1
 * placement (shared or global memory), and the CTA size, timed on samples. */
int ds_batch_tune(ds_batch* b);
/* Set the schedule by hand: block in {128, 256, 512}; per bucket (largest m
 * first) the group size and whether B^-1 sits in shared memory. */
int ds_batch_set_schedule(ds_batch* b, int block, const int* group_size, const int* binv_in_smem, int nbuckets);
int ds_batch_num_buckets(const ds_batch* b);
int ds_batch_solve(ds_batch* b);
int ds_batch_get_results(const ds_batch* b, int* status, double* objective, int* iterations);
/* Instance i: x (n[i] structurals) and row duals y (m[i]); either may be NULL. */
int ds_batch_get_solution(const ds_batch* b, int i, double* x, double* y);
int ds_batch_get_stats(const ds_batch* b, ds_batch_stats* st);

/* ---- seeded LP generator (shared by tests, bench and the trainer) ---------- */
#define DS_GEN_DENSITY   0   /* Bernoulli(density) per entry                   */
#define DS_GEN_PER_COL   1   /* exactly per_col nonzeros per column            */
#define DS_GEN_BLOCK     2   /* block-angular: blocks + linking rows           */
typedef struct ds_gen_spec {
    int kind;
    int m, n;
    double density;
    int per_col;
    int blocks, block_m, block_n, link_rows;
    double block_density, link_density;
    unsigned long long seed;
} ds_gen_spec;
/* Writes A (CSR), b (m) and c (n) of min c^T x, A x <= b, x >= 0 with
 * A ~ N(0,1) entries, x0 ~ U[0,1], b = A x0 + U[0.1,1], c ~ U[0,1].
 * Returns nnz; when val is NULL or capacity < nnz only counts. */
long long ds_gen_lp(const ds_gen_spec* spec, int* row_ptr, int* col_idx, double* val,
                    double* b, double* c, long long capacity);
/* Row count m of batched instance i (m ~ U{m_lo..m_hi}, seeded by seed+i). */
int ds_gen_batch_m(unsigned long long seed, int i, int m_lo, int m_hi);

#ifdef __cplusplus
}
#endif
#endif /* DS_API_H */
