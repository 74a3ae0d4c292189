// Batched persistent dual simplex: thousands of small LPs
//     min c^T x   s.t.   A x <= b,  x >= 0          (one LP per instance)
// solved in one persistent launch.  No counterpart in the reference; each
// instance follows the reference's dual simplex rules (DSE pricing over primal
// infeasibilities, tpp:443-501; the textbook ratio test with the EPS_Z tie
// rule, cudaDualSimplex.cpp:367-394 + tpp:546-572) with a dense explicit basis
// inverse instead of LU + eta file, which suits m <= 1024.
//
// Work layout.  Instances are sorted by m (descending) and cut into buckets of
// similar m.  Each bucket has a schedule: a group size g (32 = one warp, or
// 64..512 threads synchronised by a named barrier) and whether B^-1 lives in
// shared memory or in a per-group slot of a global workspace (L2-resident
// while the group works on it).  One persistent launch walks the buckets in
// order; inside a bucket every group pulls instances from the bucket's atomic
// queue, so groups never wait for one another except when the CTA moves on to
// the next bucket.  The schedule is chosen by the host autotuner (ds_batch_tune).
//
// Per iteration of one instance (m rows, n structurals, N = n + m):
//   CHUZR   argmax over infeasible x_B[i] < 0 of x_B[i]^2 / beta_i (exact DSE
//           weights: beta_i = ||row i of B^-1||^2, refreshed by the update)
//   BTRAN   rho = row p of B^-1
//   pivot   alpha_j = rho . a_j for nonbasic j (CSC columns; slacks: rho_r)
//   CHUZC   min theta_j = d_j / -alpha_j over alpha_j < -EPS_A; ties within
//           EPS_Z -> larger |alpha_j|, then lower j
//   FTRAN   alpha_q = B^-1 a_q
//   update  d, x_B, basis, and B^-1 <- E B^-1 (rank-1) fused with beta
// All reductions run in a fixed order, so results do not depend on timing.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/ds_api.h"
#include "engine.cuh"
#include "kernels.cuh"

namespace ds {
namespace batch {

constexpr int MAX_M = DS_BATCH_MAX_M;      // largest instance the batch path takes
constexpr int MAX_BUCKETS = 16;
constexpr int RED_SLOTS = 16;              // warps per group at most (512 / 32)

struct Bucket {
    int start, count;       // range in the sorted order
    int g;                  // threads per group
    int mcap, ncap;         // largest m, n in the bucket
    int binv_smem;          // 1: B^-1 in shared memory
    long long ws_off;       // doubles from a CTA's workspace start (unused when binv_smem)
};

struct BatchDev {
    int count, nbuckets;
    const int* m; const int* n;
    const long long* cp_off;    // offset of instance i's local column pointers (n_i + 1 entries)
    const long long* nz_off;    // offset of its row indices / values
    const long long* m_off;     // offset into b and y
    const long long* n_off;     // offset into c and x
    const int* cptr; const int* crow; const double* cval;
    const double* b; const double* c;
    const int* order;           // instance ids sorted by m descending
    Bucket bk[MAX_BUCKETS];
    unsigned* next;             // per-bucket queue counters
    double* ws;                 // global B^-1 slots
    long long ws_per_cta;       // doubles
    int smem_per_cta;           // bytes of dynamic shared memory per CTA
    int max_iter_factor;        // iteration cap = max(1000, factor * m)
    // outputs
    int* status; double* obj; int* iters; double* x; double* y;
};

// ------------------------------------------------------------------ groups
struct Group {
    int g, t, gid, nwarps, bar;
    double* redd;   // RED_SLOTS doubles
    int* redi;      // 2 * RED_SLOTS ints
};

__device__ __forceinline__ void gsync(const Group& G) {
    if (G.g == 32) __syncwarp();
    else asm volatile("bar.sync %0, %1;" :: "r"(G.bar), "r"(G.g) : "memory");
}

struct AMax { double w; int i; };
__device__ __forceinline__ AMax amax(AMax a, AMax b) {   // larger w, then smaller i
    return (b.w > a.w || (b.w == a.w && b.i < a.i)) ? b : a;
}

// Group-wide argmax (every thread gets the result).
__device__ AMax group_argmax(const Group& G, AMax v) {
    for (int o = 16; o > 0; o >>= 1) {
        AMax u{__shfl_down_sync(0xffffffffu, v.w, o), __shfl_down_sync(0xffffffffu, v.i, o)};
        v = amax(v, u);
    }
    const int lane = G.t & 31, w = G.t >> 5;
    if (lane == 0) { G.redd[w] = v.w; G.redi[w] = v.i; }
    gsync(G);
    AMax r{G.redd[0], G.redi[0]};
    for (int k = 1; k < G.nwarps; ++k) r = amax(r, AMax{G.redd[k], G.redi[k]});
    gsync(G);
    return r;
}

__device__ double group_sum(const Group& G, double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = G.t & 31, w = G.t >> 5;
    if (lane == 0) G.redd[w] = v;
    gsync(G);
    double r = 0.0;
    for (int k = 0; k < G.nwarps; ++k) r += G.redd[k];
    gsync(G);
    return r;
}

// Group-wide minimum of a double (every thread gets it).
__device__ double group_min(const Group& G, double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, o));
    const int lane = G.t & 31, w = G.t >> 5;
    if (lane == 0) G.redd[w] = v;
    gsync(G);
    double r = G.redd[0];
    for (int k = 1; k < G.nwarps; ++k) r = fmin(r, G.redd[k]);
    gsync(G);
    return r;
}

// Shared-memory bytes of one group's vectors for an instance of at most
// (mcap, ncap), B^-1 excluded.
__host__ __device__ constexpr long long group_vec_bytes(int mcap, int ncap) {
    return 8LL * (4LL * mcap + 2LL * (ncap + mcap)) + 4LL * ((ncap + mcap) + mcap) + 256;
}

// ------------------------------------------------------------------ one LP
__device__ void solve_instance(const BatchDev& B, const Group& G, int inst, unsigned char* vsm, double* Binv) {
    const int m = B.m[inst], n = B.n[inst], N = n + m;
    const int* cp = B.cptr + B.cp_off[inst];
    const int* cr = B.crow + B.nz_off[inst];
    const double* cv = B.cval + B.nz_off[inst];
    const double* bb = B.b + B.m_off[inst];
    const double* cc = B.c + B.n_off[inst];
    // carve the group's vectors
    double* xB = reinterpret_cast<double*>(vsm);
    double* beta = xB + m;
    double* rho = beta + m;
    double* aq = rho + m;
    double* d = aq + m;
    double* alpha = d + N;
    int* pos = reinterpret_cast<int*>(alpha + N);
    int* basis = pos + N;
    const int t = G.t, g = G.g;

    // slack basis: B = I, x_B = b, d = c (structurals), 0 (slacks)
    int dual_bad = 0;
    for (int i = t; i < m; i += g) { basis[i] = n + i; xB[i] = bb[i]; beta[i] = 1.0; }
    for (int j = t; j < N; j += g) {
        pos[j] = j < n ? -1 : j - n;
        d[j] = j < n ? cc[j] : 0.0;
        if (j < n && cc[j] < -EPS_D) dual_bad = 1;
    }
    for (long long e = t; e < (long long)m * m; e += g) {
        const int k = (int)(e / m), i = (int)(e - (long long)k * m);
        Binv[e] = (i == k) ? 1.0 : 0.0;   // column major: (i, k) at k * m + i
    }
    const double bad = group_sum(G, (double)dual_bad);   // also orders the writes above
    int status = DS_STATUS_ITER_LIMIT;
    int it = 0;
    const int max_iter = max(1000, B.max_iter_factor * m);
    if (bad > 0.0) {
        status = DS_STATUS_ERROR;   // not dual feasible at the slack basis: needs phase 1 (ds_solve)
    } else {
        for (; it < max_iter; ++it) {
            // ---- CHUZR (checkVarIsInfeas: x < lb - EPS_BOUND, |delta| > 1e-8)
            AMax best{-1.0, INT_MAX};
            for (int i = t; i < m; i += g) {
                const double x = xB[i];
                if (x < -EPS_BOUND && -x > 1e-8) {
                    const double w = (x * x) / beta[i];
                    if (w > 0.0) best = amax(best, AMax{w, i});
                }
            }
            best = group_argmax(G, best);
            if (best.i == INT_MAX) { status = DS_STATUS_OPTIMAL; break; }
            const int p = best.i;
            const double delta = xB[p];
            // ---- BTRAN: rho = row p of B^-1
            for (int k = t; k < m; k += g) rho[k] = Binv[(long long)k * m + p];
            gsync(G);
            // ---- pivot row and CHUZC pass 1 (minimum ratio)
            double thmin = INFINITY;
            for (int j = t; j < N; j += g) {
                double a = 0.0;
                if (pos[j] < 0) {
                    if (j < n) { for (int e = cp[j]; e < cp[j + 1]; ++e) a += cv[e] * rho[cr[e]]; }
                    else a = rho[j - n];
                    if (a < -EPS_A) thmin = fmin(thmin, d[j] / -a);
                }
                alpha[j] = a;
            }
            thmin = group_min(G, thmin);
            if (!(thmin < INFINITY)) { status = DS_STATUS_PRIMAL_INFEASIBLE; break; }
            // ---- CHUZC pass 2: within EPS_Z of the minimum, the largest |alpha|, then the lowest j
            AMax qb{-1.0, INT_MAX};
            for (int j = t; j < N; j += g) {
                const double a = alpha[j];
                if (pos[j] < 0 && a < -EPS_A && d[j] / -a - thmin < EPS_Z) qb = amax(qb, AMax{-a, j});
            }
            qb = group_argmax(G, qb);
            if (qb.i == INT_MAX) { status = DS_STATUS_ERROR; break; }   // no finite ratio (NaN data)
            const int q = qb.i;
            const double apq = alpha[q];
            // ---- FTRAN: aq = B^-1 a_q
            for (int i = t; i < m; i += g) {
                double s = 0.0;
                if (q < n) {
#pragma unroll 4
                    for (int e = cp[q]; e < cp[q + 1]; ++e) s += Binv[(long long)cr[e] * m + i] * cv[e];
                }
                else s = Binv[(long long)(q - n) * m + i];
                aq[i] = s;
            }
            gsync(G);
            const double app = aq[p];
            if (!(fabs(app - apq) <= 1e-7 * (1.0 + fabs(app))) || !(fabs(app) > 0.0)) {
                status = DS_STATUS_ERROR;   // FTRAN / BTRAN pivot disagree: the inverse lost accuracy
                break;
            }
            // ---- dual update: d_j -= theta_D alpha_j, theta_D = d_q / alpha_pq (<= 0)
            const double thD = d[q] / apq;
            const int leave = basis[p];
            gsync(G);   // every thread has read d[q] before its owner zeroes it
            for (int j = t; j < N; j += g)
                if (pos[j] < 0) d[j] = (j == q) ? 0.0 : d[j] - thD * alpha[j];
            // ---- primal update: theta_P = delta / alpha_q[p]
            const double thP = delta / app;
            for (int i = t; i < m; i += g) xB[i] = (i == p) ? thP : xB[i] - thP * aq[i];
            // ---- B^-1 <- E B^-1 (row p scaled, the others eliminated) and exact DSE
            // weights.  Thread i owns row i and walks the columns; eight independent
            // loads per step keep enough bytes in flight to stream B^-1 from L2/HBM.
            const double inv = 1.0 / app;
            if (m <= g) {
                // one row per thread
                for (int i = t; i < m; i += g) {
                    const double f = aq[i];
                    const bool isp = (i == p);
                    double* col = Binv + i;
                    double acc = 0.0;
                    int k = 0;
                    for (; k + 8 <= m; k += 8) {
                        double v[8];
#pragma unroll
                        for (int u = 0; u < 8; ++u) v[u] = col[(long long)(k + u) * m];
#pragma unroll
                        for (int u = 0; u < 8; ++u) {
                            const double piv = rho[k + u] * inv;
                            const double nv = isp ? piv : v[u] - f * piv;
                            col[(long long)(k + u) * m] = nv;
                            acc += nv * nv;
                        }
                    }
                    for (; k < m; ++k) {
                        const double piv = rho[k] * inv;
                        const double nv = isp ? piv : col[(long long)k * m] - f * piv;
                        col[(long long)k * m] = nv;
                        acc += nv * nv;
                    }
                    beta[i] = acc;
                }
            } else
            // two rows per pass (i and i + g): sixteen independent loads in flight
            for (int i = t; i < m; i += 2 * g) {
                const int i2 = i + g;
                const bool two = i2 < m;
                const double f = aq[i], f2 = two ? aq[i2] : 0.0;
                const bool isp = (i == p), isp2 = (i2 == p);
                double* col = Binv + i;
                double acc = 0.0, acc2 = 0.0;
                int k = 0;
                for (; k + 8 <= m; k += 8) {
                    double v[8], w[8];
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        v[u] = col[(long long)(k + u) * m];
                        w[u] = two ? col[(long long)(k + u) * m + g] : 0.0;
                    }
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        const double piv = rho[k + u] * inv;
                        const double nv = isp ? piv : v[u] - f * piv;
                        col[(long long)(k + u) * m] = nv;
                        acc += nv * nv;
                        if (two) {
                            const double nw = isp2 ? piv : w[u] - f2 * piv;
                            col[(long long)(k + u) * m + g] = nw;
                            acc2 += nw * nw;
                        }
                    }
                }
                for (; k < m; ++k) {
                    const double piv = rho[k] * inv;
                    const double nv = isp ? piv : col[(long long)k * m] - f * piv;
                    col[(long long)k * m] = nv;
                    acc += nv * nv;
                    if (two) {
                        const double nw = isp2 ? piv : col[(long long)k * m + g] - f2 * piv;
                        col[(long long)k * m + g] = nw;
                        acc2 += nw * nw;
                    }
                }
                beta[i] = acc;
                if (two) beta[i2] = acc2;
            }
            gsync(G);
            if (t == 0) {
                d[leave] = -thD;
                pos[leave] = -1;
                pos[q] = p;
                basis[p] = q;
            }
            gsync(G);
        }
    }
    // ---- results: x, y = c_B^T B^-1 (row duals), objective
    double* xo = B.x + B.n_off[inst];
    double* yo = B.y + B.m_off[inst];
    double part = 0.0;
    for (int j = t; j < n; j += g) {
        const double v = pos[j] >= 0 ? xB[pos[j]] : 0.0;
        xo[j] = v;
        part += cc[j] * v;
    }
    for (int k = t; k < m; k += g) {
        double s = 0.0;
        for (int i = 0; i < m; ++i) {
            const int v = basis[i];
            if (v < n) s += cc[v] * Binv[(long long)k * m + i];
        }
        yo[k] = s;
    }
    const double z = group_sum(G, part);
    if (t == 0) {
        B.status[inst] = status;
        B.obj[inst] = z;
        B.iters[inst] = it;
    }
}

// ------------------------------------------------------------------ kernel
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_batch_solve(BatchDev B) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_idx[BLOCK / 32];
    for (int b = 0; b < B.nbuckets; ++b) {
        const Bucket bk = B.bk[b];
        const int g = bk.g;
        const int ngroups = BLOCK / g;
        const int gid = threadIdx.x / g;
        Group G;
        G.g = g; G.t = threadIdx.x - gid * g; G.gid = gid; G.nwarps = g / 32; G.bar = 1 + gid;
        const long long vb = group_vec_bytes(bk.mcap, bk.ncap);
        const long long per = (vb + (bk.binv_smem ? 8LL * bk.mcap * bk.mcap : 0) + 15) / 16 * 16;
        unsigned char* mine = smem + per * gid;
        G.redd = reinterpret_cast<double*>(mine);
        G.redi = reinterpret_cast<int*>(mine + 8 * RED_SLOTS);
        unsigned char* vsm = mine + 256;
        double* Binv = bk.binv_smem ? reinterpret_cast<double*>(mine + (vb + 15) / 16 * 16)
                                    : B.ws + B.ws_per_cta * blockIdx.x + bk.ws_off +
                                          (long long)gid * bk.mcap * bk.mcap;
        (void)ngroups;
        while (true) {
            if (G.t == 0) s_idx[gid] = (int)atomicAdd(&B.next[b], 1u);
            gsync(G);
            const int k = s_idx[gid];
            gsync(G);
            if (k >= bk.count) break;
            solve_instance(B, G, B.order[bk.start + k], vsm, Binv);
            gsync(G);
        }
        __syncthreads();   // every group leaves the bucket before the layout changes
    }
}

template <int BLOCK>
static cudaError_t launch_batch(const BatchDev& B, int grid, cudaStream_t s) {
    k_batch_solve<BLOCK><<<grid, BLOCK, B.smem_per_cta, s>>>(B);
    count_launch(1);
    return cudaGetLastError();
}

template <int BLOCK>
static cudaError_t set_batch_attr(int smem, int* grid) {
    cudaError_t e = cudaFuncSetAttribute(k_batch_solve<BLOCK>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_solve<BLOCK>, BLOCK, smem);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    *grid = std::max(1, per_sm) * sms;
    return cudaSuccess;
}

// ------------------------------------------------------------------ host side
struct HostBucket { int start, count, mlo, mhi, ncap; int g, binv_smem; };

template <typename T>
struct Buf {
    T* p = nullptr; size_t n = 0;
    bool ensure(size_t k) {
        if (k <= n) return true;
        if (p) cudaFree(p);
        p = nullptr; n = 0;
        if (cudaMalloc(&p, std::max<size_t>(k, 1) * sizeof(T)) != cudaSuccess) return false;
        n = std::max<size_t>(k, 1);
        return true;
    }
    ~Buf() { if (p) cudaFree(p); }
};

constexpr int SMEM_BUDGET = 200 * 1024;   // dynamic shared memory per CTA the schedules may use

struct Batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    std::string err;
    int count = 0;
    std::vector<int> hm, hn, order;
    std::vector<long long> cp_off, nz_off, m_off, n_off;
    Buf<int> d_m, d_n, d_cptr, d_crow, d_order, d_status, d_iters;
    Buf<long long> d_cp_off, d_nz_off, d_m_off, d_n_off;
    Buf<double> d_cval, d_b, d_c, d_obj, d_x, d_y, d_ws;
    Buf<unsigned> d_next;
    std::vector<HostBucket> buckets;
    int block = 512;
    bool tuned = false;
    double last_ms = 0.0, tune_ms = 0.0;
    std::string schedule;
    cudaGraphExec_t gexec = nullptr;
    long long total_nnz = 0;

    ~Batch() {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (stream) cudaStreamDestroy(stream);
    }

    // Bucket boundaries by m: (0,32], (32,64], (64,128], (128,256], (256,512], (512,1024].
    void make_buckets() {
        order.resize(count);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return hm[a] > hm[b]; });
        buckets.clear();
        const int edges[] = {1024, 512, 256, 128, 64, 32, 0};
        int pos = 0;
        for (int e = 0; e + 1 < 7; ++e) {
            const int hi = edges[e], lo = edges[e + 1];
            int s = pos;
            while (pos < count && hm[order[pos]] > lo) ++pos;
            if (pos > s) {
                HostBucket hb{s, pos - s, lo + 1, hi, 0, 0, 0};
                for (int k = s; k < pos; ++k) hb.ncap = std::max(hb.ncap, hn[order[k]]);
                hb.mhi = hm[order[s]];
                buckets.push_back(hb);
            }
        }
    }

    // Does group size g (with B^-1 in shared memory or not) fit a CTA of `blk` threads?
    static bool fits(int blk, int g, const HostBucket& hb, int binv_smem) {
        if (g > blk || blk % g) return false;
        const long long vb = group_vec_bytes(hb.mhi, hb.ncap);
        const long long per = (vb + (binv_smem ? 8LL * hb.mhi * hb.mhi : 0) + 15) / 16 * 16;
        return per * (blk / g) <= SMEM_BUDGET;
    }

    // Fill a device descriptor for the buckets [b0, b1) with their schedules.
    bool descriptor(int b0, int b1, BatchDev* D, int* smem_out, long long* ws_cta_out) {
        BatchDev B{};
        B.count = count;
        B.m = d_m.p; B.n = d_n.p;
        B.cp_off = d_cp_off.p; B.nz_off = d_nz_off.p; B.m_off = d_m_off.p; B.n_off = d_n_off.p;
        B.cptr = d_cptr.p; B.crow = d_crow.p; B.cval = d_cval.p; B.b = d_b.p; B.c = d_c.p;
        B.order = d_order.p;
        B.next = d_next.p;
        B.max_iter_factor = 50;
        B.status = d_status.p; B.obj = d_obj.p; B.iters = d_iters.p; B.x = d_x.p; B.y = d_y.p;
        int smem = 0;
        long long ws = 0;
        B.nbuckets = b1 - b0;
        for (int b = b0; b < b1; ++b) {
            const HostBucket& hb = buckets[b];
            Bucket k{hb.start, hb.count, hb.g, hb.mhi, hb.ncap, hb.binv_smem, 0};
            const long long vb = group_vec_bytes(hb.mhi, hb.ncap);
            const long long per = (vb + (hb.binv_smem ? 8LL * hb.mhi * hb.mhi : 0) + 15) / 16 * 16;
            smem = std::max<int>(smem, (int)(per * (block / hb.g)));
            if (!hb.binv_smem) ws = std::max(ws, (long long)(block / hb.g) * hb.mhi * hb.mhi);
            B.bk[b - b0] = k;
        }
        B.smem_per_cta = smem;
        *D = B;
        *smem_out = smem;
        *ws_cta_out = ws;
        return true;
    }

    cudaError_t run(int b0, int b1, bool timed, float* ms) {
        BatchDev B;
        int smem = 0;
        long long ws_cta = 0;
        descriptor(b0, b1, &B, &smem, &ws_cta);
        int grid = 0;
        cudaError_t e = (block == 512) ? set_batch_attr<512>(smem, &grid)
                      : (block == 256) ? set_batch_attr<256>(smem, &grid)
                                       : set_batch_attr<128>(smem, &grid);
        if (e != cudaSuccess) return e;
        if (!d_ws.ensure((size_t)std::max<long long>(ws_cta, 1) * grid)) return cudaErrorMemoryAllocation;
        B.ws = d_ws.p;
        B.ws_per_cta = ws_cta;
        // per-bucket queue counters live at the bucket's index
        B.next = d_next.p + b0;
        if ((e = cudaMemsetAsync(d_next.p + b0, 0, sizeof(unsigned) * (b1 - b0), stream)) != cudaSuccess) return e;
        if (timed) cudaEventRecord(e0, stream);
        e = (block == 512) ? launch_batch<512>(B, grid, stream)
          : (block == 256) ? launch_batch<256>(B, grid, stream)
                           : launch_batch<128>(B, grid, stream);
        if (e != cudaSuccess) return e;
        if (timed) {
            cudaEventRecord(e1, stream);
            if ((e = cudaEventSynchronize(e1)) != cudaSuccess) return e;
            cudaEventElapsedTime(ms, e0, e1);
        }
        return cudaSuccess;
    }

    // Autotuner: for every bucket, time each feasible (g, B^-1 placement) on a
    // sample of the bucket's instances for each CTA size; keep the CTA size
    // with the smallest estimated total and, per bucket, its fastest schedule.
    cudaError_t tune() {
        cudaEvent_t t0, t1;
        cudaEventCreate(&t0); cudaEventCreate(&t1);
        float t_tot = 0;
        cudaEventRecord(t0, stream);
        const int blocks[] = {128, 256, 512};
        const int gs[] = {32, 64, 128, 256, 512};
        double best_total = 1e300;
        int best_block = 512;
        std::vector<std::pair<int, int>> best_cfg(buckets.size(), {512, 0});
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        std::vector<HostBucket> saved = buckets;
        for (int blk : blocks) {
            double total = 0.0;
            std::vector<std::pair<int, int>> cfg(buckets.size(), {0, 0});
            bool ok_all = true;
            for (size_t b = 0; b < saved.size(); ++b) {
                double bt = 1e300;
                for (int g : gs)
                    for (int bs = 1; bs >= 0; --bs) {
                        // groups much wider than the rows idle; much narrower ones serialise
                        if (g > std::max(32, 2 * saved[b].mhi) || 16 * g < saved[b].mhi) continue;
                        if (!fits(blk, g, saved[b], bs)) continue;
                        // sample: enough instances to fill the GPU twice, at most the bucket
                        const int groups = sms * (blk / g);
                        HostBucket hb = saved[b];
                        hb.count = std::min(saved[b].count, std::max(groups, 64));
                        hb.g = g; hb.binv_smem = bs;
                        buckets = saved;
                        buckets[b] = hb;
                        block = blk;
                        float ms = 0;
                        cudaError_t e = run((int)b, (int)b + 1, true, &ms);
                        if (e != cudaSuccess) { buckets = saved; return e; }
                        const double est = ms * (double)saved[b].count / hb.count;
                        if (est < bt) { bt = est; cfg[b] = {g, bs}; }
                    }
                if (bt >= 1e300) { ok_all = false; break; }
                total += bt;
            }
            if (ok_all && total < best_total) { best_total = total; best_block = blk; best_cfg = cfg; }
        }
        buckets = saved;
        block = best_block;
        schedule = "block " + std::to_string(block);
        for (size_t b = 0; b < buckets.size(); ++b) {
            buckets[b].g = best_cfg[b].first;
            buckets[b].binv_smem = best_cfg[b].second;
            schedule += "; m " + std::to_string(buckets[b].mlo) + ".." + std::to_string(buckets[b].mhi) + " (" +
                        std::to_string(buckets[b].count) + " LPs): g " + std::to_string(buckets[b].g) +
                        (buckets[b].binv_smem ? ", B^-1 in shared memory" : ", B^-1 in global memory");
        }
        cudaEventRecord(t1, stream);
        cudaEventSynchronize(t1);
        cudaEventElapsedTime(&t_tot, t0, t1);
        cudaEventDestroy(t0); cudaEventDestroy(t1);
        tune_ms = t_tot;
        tuned = true;
        if (gexec) { cudaGraphExecDestroy(gexec); gexec = nullptr; }
        return cudaSuccess;
    }

    // Default schedule without tuning: the largest group that fits, B^-1 in
    // shared memory when it fits.
    void default_schedule() {
        block = 512;
        schedule = "block 512 (untuned)";
        for (auto& hb : buckets) {
            hb.g = 0;
            for (int g : {32, 64, 128, 256, 512}) {
                const int want = hb.mhi <= 64 ? 32 : hb.mhi <= 128 ? 128 : hb.mhi <= 256 ? 256 : 512;
                if (g == want) { hb.g = g; break; }
            }
            hb.binv_smem = fits(block, hb.g, hb, 1) ? 1 : 0;
            while (!fits(block, hb.g, hb, hb.binv_smem) && hb.g < 512) hb.g *= 2;
        }
    }

    // The whole batch: one persistent launch, captured once as a CUDA graph
    // (counter reset + kernel) and replayed.
    cudaError_t solve(float* ms) {
        if (!tuned && schedule.empty()) default_schedule();
        cudaError_t e;
        if (!gexec) {
            BatchDev B;
            int smem = 0;
            long long ws_cta = 0;
            descriptor(0, (int)buckets.size(), &B, &smem, &ws_cta);
            int grid = 0;
            e = (block == 512) ? set_batch_attr<512>(smem, &grid)
              : (block == 256) ? set_batch_attr<256>(smem, &grid)
                               : set_batch_attr<128>(smem, &grid);
            if (e != cudaSuccess) return e;
            if (!d_ws.ensure((size_t)std::max<long long>(ws_cta, 1) * grid)) return cudaErrorMemoryAllocation;
            B.ws = d_ws.p;
            B.ws_per_cta = ws_cta;
            cudaGraph_t g;
            if ((e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) return e;
            set_launch_counting(false);
            cudaMemsetAsync(d_next.p, 0, sizeof(unsigned) * MAX_BUCKETS, stream);
            cudaError_t le = (block == 512) ? launch_batch<512>(B, grid, stream)
                           : (block == 256) ? launch_batch<256>(B, grid, stream)
                                            : launch_batch<128>(B, grid, stream);
            set_launch_counting(true);
            cudaError_t ce = cudaStreamEndCapture(stream, &g);
            if (le != cudaSuccess) return le;
            if (ce != cudaSuccess) return ce;
            e = cudaGraphInstantiate(&gexec, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return e;
        }
        cudaEventRecord(e0, stream);
        if ((e = cudaGraphLaunch(gexec, stream)) != cudaSuccess) return e;
        count_launch(1);
        cudaEventRecord(e1, stream);
        if ((e = cudaEventSynchronize(e1)) != cudaSuccess) return e;
        float t = 0;
        cudaEventElapsedTime(&t, e0, e1);
        last_ms = t;
        if (ms) *ms = t;
        return cudaSuccess;
    }
};

}  // namespace batch
}  // namespace ds

using ds::batch::Batch;

struct ds_batch { Batch* b; };

extern "C" {

int ds_batch_create(int device, ds_batch** out) {
    if (!out) return DS_ERR_ARG;
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) return DS_ERR_CUDA;
    auto* b = new Batch();
    b->device = device;
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->e0) != cudaSuccess || cudaEventCreate(&b->e1) != cudaSuccess) {
        delete b;
        return DS_ERR_CUDA;
    }
    *out = new ds_batch{b};
    return DS_OK;
}

int ds_batch_destroy(ds_batch* h) {
    if (!h) return DS_ERR_ARG;
    cudaSetDevice(h->b->device);
    delete h->b;
    delete h;
    return DS_OK;
}

const char* ds_batch_last_error(const ds_batch* h) { return h ? h->b->err.c_str() : "null handle"; }

int ds_batch_load(ds_batch* h, int count, const int* m, const int* n, const int* col_ptr, const int* row_idx,
                  const double* val, const double* rhs, const double* cost) {
    if (!h || count <= 0 || !m || !n || !col_ptr || !rhs || !cost) return DS_ERR_ARG;
    Batch* B = h->b;
    if (cudaSetDevice(B->device) != cudaSuccess) return DS_ERR_CUDA;
    // A batch of the same shapes reuses the buffers (same device addresses),
    // so the schedule and the captured graph stay valid.
    const bool same_shape = count == B->count && std::equal(m, m + count, B->hm.begin()) &&
                            std::equal(n, n + count, B->hn.begin());
    B->count = count;
    B->hm.assign(m, m + count);
    B->hn.assign(n, n + count);
    B->cp_off.resize(count); B->nz_off.resize(count); B->m_off.resize(count); B->n_off.resize(count);
    long long cpo = 0, nzo = 0, mo = 0, no = 0;
    for (int i = 0; i < count; ++i) {
        if (m[i] <= 0 || n[i] <= 0) { B->err = "instance " + std::to_string(i) + ": m and n must be positive"; return DS_ERR_ARG; }
        if (m[i] > ds::batch::MAX_M) {
            B->err = "instance " + std::to_string(i) + ": m = " + std::to_string(m[i]) + " exceeds the batch limit " +
                     std::to_string(ds::batch::MAX_M) + " (solve it with ds_solve)";
            return DS_ERR_CAPACITY;
        }
        const int* cp = col_ptr + cpo;
        if (cp[0] != 0) { B->err = "instance " + std::to_string(i) + ": column pointers must start at 0"; return DS_ERR_ARG; }
        for (int j = 0; j < n[i]; ++j)
            if (cp[j + 1] < cp[j]) { B->err = "instance " + std::to_string(i) + ": column pointers decrease"; return DS_ERR_ARG; }
        const int nz = cp[n[i]];
        for (int e = 0; e < nz; ++e)
            if (!row_idx || row_idx[nzo + e] < 0 || row_idx[nzo + e] >= m[i]) {
                B->err = "instance " + std::to_string(i) + ": row index out of range";
                return DS_ERR_ARG;
            }
        B->cp_off[i] = cpo; B->nz_off[i] = nzo; B->m_off[i] = mo; B->n_off[i] = no;
        cpo += n[i] + 1; nzo += nz; mo += m[i]; no += n[i];
    }
    B->total_nnz = nzo;
    cudaStream_t s = B->stream;
    auto up = [&](auto& buf, const auto* src, size_t k) {
        if (!buf.ensure(k)) return false;
        return k == 0 || cudaMemcpyAsync(buf.p, src, k * sizeof(*src), cudaMemcpyHostToDevice, s) == cudaSuccess;
    };
    bool ok = up(B->d_m, m, count) && up(B->d_n, n, count) && up(B->d_cptr, col_ptr, (size_t)cpo) &&
              up(B->d_crow, row_idx, (size_t)nzo) && up(B->d_cval, val, (size_t)nzo) && up(B->d_b, rhs, (size_t)mo) &&
              up(B->d_c, cost, (size_t)no) && up(B->d_cp_off, B->cp_off.data(), count) &&
              up(B->d_nz_off, B->nz_off.data(), count) && up(B->d_m_off, B->m_off.data(), count) &&
              up(B->d_n_off, B->n_off.data(), count);
    ok = ok && B->d_status.ensure(count) && B->d_iters.ensure(count) && B->d_obj.ensure(count) &&
         B->d_x.ensure((size_t)no) && B->d_y.ensure((size_t)mo) && B->d_next.ensure(ds::batch::MAX_BUCKETS);
    if (!same_shape) B->make_buckets();
    ok = ok && up(B->d_order, B->order.data(), count);
    if (!ok) { B->err = "device allocation or copy failed"; return DS_ERR_CUDA; }
    if (!same_shape) {
        B->tuned = false;
        B->schedule.clear();
        if (B->gexec) { cudaGraphExecDestroy(B->gexec); B->gexec = nullptr; }
    }
    if (cudaStreamSynchronize(s) != cudaSuccess) return DS_ERR_CUDA;
    return DS_OK;
}

long long ds_batch_gen_arrays(int count, int m_lo, int m_hi, double density, unsigned long long seed, int* m_out,
                              int* n_out, int* col_ptr, int* row_idx, double* val, double* rhs, double* cost,
                              long long* sizes) {
    if (count <= 0 || m_lo <= 0 || m_hi < m_lo || density <= 0.0 || density > 1.0 || !sizes) return DS_ERR_ARG;
    std::vector<int> ms(count), ns(count);
    std::vector<long long> nzs(count), cpo(count + 1, 0), nzo(count + 1, 0), mo(count + 1, 0), no(count + 1, 0);
    for (int i = 0; i < count; ++i) {
        ms[i] = ds_gen_batch_m(seed, i, m_lo, m_hi);
        ns[i] = 2 * ms[i];
        ds_gen_spec sp{};
        sp.kind = DS_GEN_DENSITY; sp.m = ms[i]; sp.n = ns[i]; sp.density = density; sp.seed = seed + (unsigned long long)i;
        nzs[i] = ds_gen_lp(&sp, nullptr, nullptr, nullptr, nullptr, nullptr, 0);
        cpo[i + 1] = cpo[i] + ns[i] + 1; nzo[i + 1] = nzo[i] + nzs[i];
        mo[i + 1] = mo[i] + ms[i]; no[i + 1] = no[i] + ns[i];
    }
    sizes[0] = cpo[count]; sizes[1] = nzo[count]; sizes[2] = mo[count]; sizes[3] = no[count];
    if (m_out) std::copy(ms.begin(), ms.end(), m_out);
    if (n_out) std::copy(ns.begin(), ns.end(), n_out);
    if (!col_ptr || !row_idx || !val || !rhs || !cost) return DS_OK;
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < count; ++i) {
        const int m = ms[i], n = ns[i];
        ds_gen_spec sp{};
        sp.kind = DS_GEN_DENSITY; sp.m = m; sp.n = n; sp.density = density; sp.seed = seed + (unsigned long long)i;
        std::vector<int> rp(m + 1), ci((size_t)nzs[i]);
        std::vector<double> v((size_t)nzs[i]);
        ds_gen_lp(&sp, rp.data(), ci.data(), v.data(), rhs + mo[i], cost + no[i], nzs[i]);
        // CSR -> CSC (rows ascending inside each column)
        int* cp = col_ptr + cpo[i];
        std::fill(cp, cp + n + 1, 0);
        for (long long e = 0; e < nzs[i]; ++e) cp[ci[e] + 1]++;
        for (int j = 0; j < n; ++j) cp[j + 1] += cp[j];
        std::vector<int> cur(cp, cp + n);
        for (int r = 0; r < m; ++r)
            for (int e = rp[r]; e < rp[r + 1]; ++e) {
                const int k = cur[ci[e]]++;
                row_idx[nzo[i] + k] = r;
                val[nzo[i] + k] = v[e];
            }
    }
    return DS_OK;
}

int ds_batch_generate(ds_batch* h, int count, int m_lo, int m_hi, double density, unsigned long long seed) {
    if (!h || count <= 0 || m_lo <= 0 || m_hi < m_lo || density <= 0.0 || density > 1.0) return DS_ERR_ARG;
    if (m_hi > ds::batch::MAX_M) { h->b->err = "m_hi exceeds the batch limit"; return DS_ERR_CAPACITY; }
    long long sz[4];
    std::vector<int> ms(count), ns(count);
    int rc = (int)ds_batch_gen_arrays(count, m_lo, m_hi, density, seed, ms.data(), ns.data(), nullptr, nullptr,
                                      nullptr, nullptr, nullptr, sz);
    if (rc) return rc;
    std::vector<int> cptr((size_t)sz[0]), crow((size_t)sz[1]);
    std::vector<double> cval((size_t)sz[1]), b((size_t)sz[2]), c((size_t)sz[3]);
    rc = (int)ds_batch_gen_arrays(count, m_lo, m_hi, density, seed, nullptr, nullptr, cptr.data(), crow.data(),
                                  cval.data(), b.data(), c.data(), sz);
    if (rc) return rc;
    return ds_batch_load(h, count, ms.data(), ns.data(), cptr.data(), crow.data(), cval.data(), b.data(), c.data());
}

int ds_batch_tune(ds_batch* h) {
    if (!h) return DS_ERR_ARG;
    Batch* B = h->b;
    if (B->count == 0) { B->err = "no batch loaded"; return DS_ERR_STATE; }
    if (cudaSetDevice(B->device) != cudaSuccess) return DS_ERR_CUDA;
    if (B->tune() != cudaSuccess) { B->err = "tuning launch failed"; return DS_ERR_CUDA; }
    return DS_OK;
}

int ds_batch_set_schedule(ds_batch* h, int block, const int* group_size, const int* binv_in_smem, int nbuckets) {
    if (!h) return DS_ERR_ARG;
    Batch* B = h->b;
    if (B->count == 0) { B->err = "no batch loaded"; return DS_ERR_STATE; }
    if ((block != 128 && block != 256 && block != 512) || nbuckets != (int)B->buckets.size() || !group_size ||
        !binv_in_smem)
        return DS_ERR_ARG;
    for (int b = 0; b < nbuckets; ++b) {
        auto hb = B->buckets[b];
        if (!Batch::fits(block, group_size[b], hb, binv_in_smem[b] ? 1 : 0)) {
            B->err = "schedule for bucket " + std::to_string(b) + " does not fit a CTA";
            return DS_ERR_ARG;
        }
    }
    B->block = block;
    B->schedule = "block " + std::to_string(block) + " (set)";
    for (int b = 0; b < nbuckets; ++b) {
        B->buckets[b].g = group_size[b];
        B->buckets[b].binv_smem = binv_in_smem[b] ? 1 : 0;
    }
    B->tuned = true;
    if (B->gexec) { cudaGraphExecDestroy(B->gexec); B->gexec = nullptr; }
    return DS_OK;
}

int ds_batch_num_buckets(const ds_batch* h) { return h ? (int)h->b->buckets.size() : 0; }

int ds_batch_solve(ds_batch* h) {
    if (!h) return DS_ERR_ARG;
    Batch* B = h->b;
    if (B->count == 0) { B->err = "no batch loaded"; return DS_ERR_STATE; }
    if (cudaSetDevice(B->device) != cudaSuccess) return DS_ERR_CUDA;
    if (B->solve(nullptr) != cudaSuccess) { B->err = "batch launch failed"; return DS_ERR_CUDA; }
    return DS_OK;
}

int ds_batch_get_results(const ds_batch* h, int* status, double* objective, int* iterations) {
    if (!h) return DS_ERR_ARG;
    const Batch* B = h->b;
    if (B->count == 0) return DS_ERR_STATE;
    cudaSetDevice(B->device);
    if (status && cudaMemcpyAsync(status, B->d_status.p, sizeof(int) * B->count, cudaMemcpyDeviceToHost, B->stream)) return DS_ERR_CUDA;
    if (objective && cudaMemcpyAsync(objective, B->d_obj.p, sizeof(double) * B->count, cudaMemcpyDeviceToHost, B->stream)) return DS_ERR_CUDA;
    if (iterations && cudaMemcpyAsync(iterations, B->d_iters.p, sizeof(int) * B->count, cudaMemcpyDeviceToHost, B->stream)) return DS_ERR_CUDA;
    return cudaStreamSynchronize(B->stream) == cudaSuccess ? DS_OK : DS_ERR_CUDA;
}

int ds_batch_get_solution(const ds_batch* h, int i, double* x, double* y) {
    if (!h) return DS_ERR_ARG;
    const Batch* B = h->b;
    if (i < 0 || i >= B->count) return DS_ERR_ARG;
    cudaSetDevice(B->device);
    if (x && cudaMemcpyAsync(x, B->d_x.p + B->n_off[i], sizeof(double) * B->hn[i], cudaMemcpyDeviceToHost, B->stream)) return DS_ERR_CUDA;
    if (y && cudaMemcpyAsync(y, B->d_y.p + B->m_off[i], sizeof(double) * B->hm[i], cudaMemcpyDeviceToHost, B->stream)) return DS_ERR_CUDA;
    return cudaStreamSynchronize(B->stream) == cudaSuccess ? DS_OK : DS_ERR_CUDA;
}

int ds_batch_get_stats(const ds_batch* h, ds_batch_stats* st) {
    if (!h || !st) return DS_ERR_ARG;
    const Batch* B = h->b;
    std::memset(st, 0, sizeof(*st));
    st->count = B->count;
    st->buckets = (int)B->buckets.size();
    st->block = B->block;
    st->solve_ms = B->last_ms;
    st->tune_ms = B->tune_ms;
    st->total_nnz = B->total_nnz;
    std::snprintf(st->schedule, sizeof(st->schedule), "%s", B->schedule.c_str());
    return DS_OK;
}

}  // extern "C"
