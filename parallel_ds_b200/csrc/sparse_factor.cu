// Sparse LU of the basis's structural block K = A[R', S] (eta-file mode).
//
// Replaces the reference's cuDSS factorisation of B (cudaSparseMatrix.cpp:502-567,
// reached from CudaDualSimplex::reFactorize, cudaDualSimplex.cpp:229-238) and its
// triangular solves (cudaSparseMatrix.cpp:570-605).  Three stages:
//
//  1. Triangularisation (host, structure only).  Column singletons of the
//     active part of K are pivoted first, row singletons last; what remains is
//     the kernel.  With rows and columns in pivot order K is block upper
//     triangular:  [U1 X Y; 0 M Z; 0 0 U3], U1 and U3 triangular with K's own
//     entries (no arithmetic), M the kernel.
//  2. Kernel LU (device, FP64).  Right-looking Markowitz elimination with
//     threshold partial pivoting (|a_ij| >= 0.1 max_i |a_ij|), run in rounds
//     by one CTA: each round every active column proposes its cheapest
//     admissible pivot, a Luby-style rule keeps a set of mutually independent
//     pivots (no pivot's row meets another's column), and all of them are
//     eliminated at once, each target row updated by the one thread that owns
//     it.  When the active part turns dense it is inverted as a dense block by
//     Gauss-Jordan with partial pivoting (factor.cu).
//  3. Solve programs (host, integer work; values gathered on the device).  The
//     k pivots become slots of one vector; FTRAN and BTRAN are programs of
//     levels of independent slot updates (kernels.cu: k_sf_ftran, k_sf_btran).
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "kernels.cuh"
#include "sparse_factor.cuh"

namespace ds {

constexpr int KLU_BS = 1024;
constexpr double KLU_U = 0.1;          // threshold partial pivoting
constexpr double KLU_DENSE = 0.2;      // active density at which the rest is factorised dense
constexpr int KLU_DENSE_CAP = 1536;    // ... if the active part has at most this many rows
constexpr int KLU_MAX_ROUNDS = 8192;
constexpr int KLU_DENSE_FALLBACK = 6144;   // largest kernel factorised dense when the work area overflows

struct KluArgs {
    int km;
    const int* row_ptr; const int* row_col; const long long* row_src; const double* cval;
    int pool_cap; int* pool_col; double* pool_val;
    int* r_start; int* r_len; int* r_cap;
    int* c_ptr; int* c_cur; int* c_row;
    int* cand_row; int* cand_cost; double* cand_val; unsigned char* cand_ok;
    unsigned long long* row_key;
    int* col_piv; int* row_piv;
    int* piv_row; int* piv_col; int* piv_uidx; int* piv_ulen;
    int* L_row; int* L_piv; double* L_val; int L_cap;
    int* dense_row; int* dense_col;
    int* out;      // [0] pivots [1] L entries [2] error [3] rounds [4] pool top [5] dense order
    int sparse;    // 0: no Markowitz rounds (the whole kernel is the dense block)
};

enum KluErr : int { KLU_OK = 0, KLU_SINGULAR = 2, KLU_STALL = 3, KLU_L_FULL = 4, KLU_POOL_FULL = 5, KLU_ROUNDS = 6 };

template <int BS>
__device__ long long klu_sum(long long v, long long* sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    long long t = 0;
    for (int u = 0; u < BS / 32; ++u) t += sh[u];
    return t;
}

template <int BS>
__device__ int klu_min(int v, int* sh) {
    for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_down_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    int t = INT_MAX;
    for (int u = 0; u < BS / 32; ++u) t = min(t, sh[u]);
    return t;
}

// Exclusive scan of in[0..n) into out[0..n) (in place allowed) by one block:
// thread chunks of consecutive elements, then a scan of the chunk sums.
// Returns the total.  Callers synchronise before reading out.
template <int BS>
__device__ int klu_scan(const int* in, int* out, int n, int* sh) {
    const int per = (n + BS - 1) / BS;
    const int b0 = min(n, (int)threadIdx.x * per), b1 = min(n, b0 + per);
    int s = 0;
    for (int i = b0; i < b1; ++i) s += in[i];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = s;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    __syncthreads();
    if (lane == 31) sh[w] = x;
    __syncthreads();
    if (w == 0) {
        int t = (lane < BS / 32) ? sh[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < BS / 32) sh[lane] = t;
    }
    __syncthreads();
    int run = (w > 0 ? sh[w - 1] : 0) + x - s;
    const int total = sh[BS / 32 - 1];
    for (int i = b0; i < b1; ++i) { const int v = in[i]; out[i] = run; run += v; }
    return total;
}

// Value of row i's entry in column j (rows are sorted by column; 0 if absent).
__device__ __forceinline__ double klu_value(const KluArgs& a, int i, int j) {
    int lo = a.r_start[i], hi = lo + a.r_len[i];
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a.pool_col[mid] < j) lo = mid + 1; else hi = mid;
    }
    return (lo < a.r_start[i] + a.r_len[i] && a.pool_col[lo] == j) ? a.pool_val[lo] : 0.0;
}

__device__ __forceinline__ unsigned long long klu_key(int cost, int j) {
    return ((unsigned long long)(unsigned)cost << 32) | (unsigned)j;
}

// One CTA.  Rows of the active part live in a pool (start, length, capacity per
// row; a row that outgrows its capacity moves to the pool's end).  Column lists
// are rebuilt from the rows each round.  Every loop ends: a round pivots at
// least the best candidate (Luby), and the round count is bounded.
template <int BS>
__global__ void __launch_bounds__(BS, 1) k_kernel_lu(KluArgs a) {
    __shared__ int sh_i[BS / 32 + 1];
    __shared__ long long sh_l[BS / 32];
    __shared__ int s_npiv, s_err, s_round, s_nL;
    __shared__ unsigned long long s_top;   // 64-bit: requests past an overflow must not wrap
    const int km = a.km;
    const int tid = threadIdx.x;
    for (int i = tid; i < km; i += BS) {
        const int p0 = a.row_ptr[i], len = a.row_ptr[i + 1] - p0;
        const int st = p0 + 4 * i;
        a.r_start[i] = st; a.r_len[i] = len; a.r_cap[i] = len + 4;
        for (int e = 0; e < len; ++e) {
            a.pool_col[st + e] = a.row_col[p0 + e];
            a.pool_val[st + e] = a.cval[a.row_src[p0 + e]];
        }
        a.col_piv[i] = -1; a.row_piv[i] = -1;
    }
    if (tid == 0) { s_npiv = 0; s_err = KLU_OK; s_round = 0; s_nL = 0; s_top = (unsigned long long)(a.row_ptr[km] + 4 * km); }
    __syncthreads();
    while (a.sparse) {
        const int na = km - s_npiv;
        long long nz = 0;
        for (int i = tid; i < km; i += BS) if (a.row_piv[i] < 0) nz += a.r_len[i];
        nz = klu_sum<BS>(nz, sh_l);
        if (na == 0) break;
        if ((double)nz > KLU_DENSE * (double)na * (double)na && na <= KLU_DENSE_CAP) break;
        if (s_round >= KLU_MAX_ROUNDS) {
            if (na > KLU_DENSE_CAP && tid == 0) s_err = KLU_ROUNDS;
            break;
        }
        // column lists of the active part
        for (int j = tid; j < km; j += BS) a.c_cur[j] = 0;
        __syncthreads();
        for (int i = tid; i < km; i += BS) {
            if (a.row_piv[i] >= 0) continue;
            const int st = a.r_start[i], len = a.r_len[i];
            for (int x = 0; x < len; ++x) atomicAdd(&a.c_cur[a.pool_col[st + x]], 1);
        }
        __syncthreads();
        const int tot = klu_scan<BS>(a.c_cur, a.c_ptr, km, sh_i);
        __syncthreads();
        if (tid == 0) a.c_ptr[km] = tot;
        for (int j = tid; j < km; j += BS) a.c_cur[j] = a.c_ptr[j];
        __syncthreads();
        for (int i = tid; i < km; i += BS) {
            if (a.row_piv[i] >= 0) continue;
            const int st = a.r_start[i], len = a.r_len[i];
            for (int x = 0; x < len; ++x) a.c_row[atomicAdd(&a.c_cur[a.pool_col[st + x]], 1)] = i;
        }
        __syncthreads();
        // candidates: per active column the admissible row of least Markowitz cost
        int cmin = INT_MAX;
        for (int j = tid; j < km; j += BS) {
            a.cand_cost[j] = INT_MAX;
            if (a.col_piv[j] >= 0) continue;
            const int q0 = a.c_ptr[j], q1 = a.c_ptr[j + 1], cnt = q1 - q0;
            double mx = 0.0;
            for (int q = q0; q < q1; ++q) mx = fmax(mx, fabs(klu_value(a, a.c_row[q], j)));
            if (!(mx > 1e-300)) { atomicExch(&s_err, KLU_SINGULAR); continue; }
            int best = INT_MAX, bi = -1;
            double bv = 0.0;
            for (int q = q0; q < q1; ++q) {
                const int i = a.c_row[q];
                const double v = klu_value(a, i, j);
                if (fabs(v) >= KLU_U * mx) {
                    const int cost = (a.r_len[i] - 1) * (cnt - 1);
                    if (cost < best || (cost == best && i < bi)) { best = cost; bi = i; bv = v; }
                }
            }
            if (bi < 0) { atomicExch(&s_err, KLU_SINGULAR); continue; }
            a.cand_row[j] = bi; a.cand_cost[j] = best; a.cand_val[j] = bv;
            cmin = min(cmin, best);
        }
        const int mc = klu_min<BS>(cmin, sh_i);
        if (s_err != KLU_OK) break;
        const int thr = (int)min((long long)INT_MAX - 1, max(2LL * mc, (long long)mc + 2));
        // independent set: a candidate is kept when no conflicting candidate has a smaller key
        for (int i = tid; i < km; i += BS) a.row_key[i] = ~0ull;
        __syncthreads();
        for (int j = tid; j < km; j += BS)
            if (a.col_piv[j] < 0 && a.cand_cost[j] <= thr) atomicMin(&a.row_key[a.cand_row[j]], klu_key(a.cand_cost[j], j));
        __syncthreads();
        for (int j = tid; j < km; j += BS) {
            int ok = 0;
            if (a.col_piv[j] < 0 && a.cand_cost[j] <= thr) {
                const unsigned long long key = klu_key(a.cand_cost[j], j);
                const int i = a.cand_row[j];
                ok = (a.row_key[i] == key);
                for (int q = a.c_ptr[j]; ok && q < a.c_ptr[j + 1]; ++q) {
                    const int r = a.c_row[q];
                    if (r != i && a.row_key[r] < key) ok = 0;
                }
                const int st = a.r_start[i], len = a.r_len[i];
                for (int x = 0; ok && x < len; ++x) {
                    const int c = a.pool_col[st + x];
                    if (c != j && a.col_piv[c] < 0 && a.cand_cost[c] <= thr && klu_key(a.cand_cost[c], c) < key) ok = 0;
                }
            }
            a.cand_ok[j] = (unsigned char)ok;
        }
        __syncthreads();
        for (int j = tid; j < km; j += BS) a.c_cur[j] = a.cand_ok[j];
        __syncthreads();
        const int nsel = klu_scan<BS>(a.c_cur, a.c_cur, km, sh_i);
        __syncthreads();
        const int base = s_npiv;
        for (int j = tid; j < km; j += BS) {
            if (!a.cand_ok[j]) continue;
            const int p = base + a.c_cur[j];
            const int i = a.cand_row[j];
            a.piv_row[p] = i; a.piv_col[p] = j;
            a.piv_uidx[p] = a.r_start[i]; a.piv_ulen[p] = a.r_len[i];
            a.col_piv[j] = p; a.row_piv[i] = p;
        }
        __syncthreads();
        if (nsel == 0) { if (tid == 0) s_err = KLU_STALL; break; }
        // elimination: the owner of each active row applies every pivot whose
        // column it meets.  Rows stay sorted by column: the pivot column's
        // entry is removed by a shift, the fill is counted by a two-pointer
        // pass, and the scaled pivot row is merged in place from the back.
        for (int r = tid; r < km; r += BS) {
            if (a.row_piv[r] >= 0) continue;
            int st = a.r_start[r], len = a.r_len[r];
            for (;;) {
                int e = -1;
                for (int x = 0; x < len; ++x)
                    if (a.col_piv[a.pool_col[st + x]] >= 0) { e = x; break; }
                if (e < 0) break;
                const int c = a.pool_col[st + e];
                const double arc = a.pool_val[st + e];
                const int p = a.col_piv[c];
                const double l = arc / a.cand_val[c];
                const int li = atomicAdd(&s_nL, 1);
                if (li < a.L_cap) { a.L_row[li] = r; a.L_piv[li] = p; a.L_val[li] = l; }
                else { atomicExch(&s_err, KLU_L_FULL); break; }
                for (int x = e; x + 1 < len; ++x) { a.pool_col[st + x] = a.pool_col[st + x + 1]; a.pool_val[st + x] = a.pool_val[st + x + 1]; }
                --len;
                const int u0 = a.piv_uidx[p], ul = a.piv_ulen[p];
                int fill = 0;
                for (int x = 0, y = 0; y < ul; ++y) {
                    const int cb = a.pool_col[u0 + y];
                    if (cb == c) continue;
                    while (x < len && a.pool_col[st + x] < cb) ++x;
                    if (x == len || a.pool_col[st + x] != cb) ++fill;
                }
                const int nlen = len + fill;
                if (nlen > a.r_cap[r]) {
                    const int ncap = max(2 * a.r_cap[r] + 4, nlen + 4);
                    if (*(volatile int*)&s_err != KLU_OK) break;   // the pool already overflowed
                    const unsigned long long ns64 = atomicAdd(&s_top, (unsigned long long)ncap);
                    if (ns64 + (unsigned long long)ncap > (unsigned long long)a.pool_cap) { atomicExch(&s_err, KLU_POOL_FULL); break; }
                    const int ns = (int)ns64;
                    for (int x = 0; x < len; ++x) { a.pool_col[ns + x] = a.pool_col[st + x]; a.pool_val[ns + x] = a.pool_val[st + x]; }
                    st = ns;
                    a.r_start[r] = ns; a.r_cap[r] = ncap;
                }
                int ra = len - 1, rb = ul - 1, w = nlen - 1;
                while (rb >= 0) {
                    const int cb = a.pool_col[u0 + rb];
                    if (cb == c) { --rb; continue; }
                    const int ca = ra >= 0 ? a.pool_col[st + ra] : -1;
                    if (ca > cb) {
                        a.pool_col[st + w] = ca; a.pool_val[st + w] = a.pool_val[st + ra]; --ra;
                    } else if (ca == cb) {
                        a.pool_col[st + w] = ca; a.pool_val[st + w] = a.pool_val[st + ra] - l * a.pool_val[u0 + rb]; --ra; --rb;
                    } else {
                        a.pool_col[st + w] = cb; a.pool_val[st + w] = -l * a.pool_val[u0 + rb]; --rb;
                    }
                    --w;
                }
                len = nlen;
            }
            a.r_len[r] = len;
        }
        __syncthreads();
        if (s_err != KLU_OK) break;
        if (tid == 0) { s_npiv += nsel; ++s_round; }
        __syncthreads();
    }
    __syncthreads();
    // dense block: the rows and columns still active, in index order
    for (int i = tid; i < km; i += BS) a.c_cur[i] = (a.row_piv[i] < 0) ? 1 : 0;
    __syncthreads();
    const int kd = klu_scan<BS>(a.c_cur, a.c_cur, km, sh_i);
    __syncthreads();
    for (int i = tid; i < km; i += BS) a.dense_row[i] = (a.row_piv[i] < 0) ? a.c_cur[i] : -1;
    __syncthreads();
    for (int j = tid; j < km; j += BS) a.c_cur[j] = (a.col_piv[j] < 0) ? 1 : 0;
    __syncthreads();
    const int kdc = klu_scan<BS>(a.c_cur, a.c_cur, km, sh_i);
    __syncthreads();
    for (int j = tid; j < km; j += BS) a.dense_col[j] = (a.col_piv[j] < 0) ? a.c_cur[j] : -1;
    if (tid == 0) {
        if (kd != kdc && s_err == KLU_OK) s_err = KLU_SINGULAR;
        a.out[0] = s_npiv; a.out[1] = min(s_nL, a.L_cap); a.out[2] = s_err; a.out[3] = s_round;
        a.out[4] = (int)min(s_top, (unsigned long long)a.pool_cap); a.out[5] = kd;
    }
}

// S[a + b kd] = active row a's entry in active column b.
__global__ void k_klu_dense_build(KluArgs a, int kd, double* S) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.km) return;
    const int r = a.dense_row[i];
    if (r < 0) return;
    const int st = a.r_start[i], len = a.r_len[i];
    for (int x = 0; x < len; ++x) {
        const int b = a.dense_col[a.pool_col[st + x]];
        if (b >= 0) S[(size_t)r + (size_t)b * kd] = a.pool_val[st + x];
    }
}

__global__ void k_klu_zero(double* p, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] = 0.0;
}

__global__ void k_klu_transpose(const double* in, int n, double* out) {
    __shared__ double t[32][33];
    const int x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 32 + threadIdx.y;
    if (x < n && y < n) t[threadIdx.y][threadIdx.x] = in[(size_t)x + (size_t)y * n];
    __syncthreads();
    const int x2 = blockIdx.y * 32 + threadIdx.x, y2 = blockIdx.x * 32 + threadIdx.y;
    if (x2 < n && y2 < n) out[(size_t)x2 + (size_t)y2 * n] = t[threadIdx.x][threadIdx.y];
}

// Coefficient gather: src < 0 -> 1.0; [0, nA) -> A's CSC values; then the
// kernel's L values; then its pool (U rows).
__global__ void k_sf_gather(const long long* src, long long n, const double* cval, long long nA, const double* lval,
                            long long nL, const double* pval, double* dst) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long x = src[i];
        double v;
        if (x < 0) v = 1.0;
        else if (x < nA) v = cval[x];
        else if (x < nA + nL) v = lval[x - nA];
        else v = pval[x - nA - nL];
        dst[i] = v;
    }
}

// ------------------------------------------------------------- host side
namespace {

struct ProgBuild {
    // flattened program
    std::vector<int> lvl_ptr{0}, lvl_kind, op_slot, op_ptr{0}, ent_slot;
    std::vector<long long> diag_src, ent_src;
    // ops of the current phase, in dependency order
    struct Op { int slot; long long diag; int e0, e1; };
    std::vector<Op> ops;
    std::vector<int> pe_slot;
    std::vector<long long> pe_src;
    std::vector<int> lev;   // per slot: level within the current phase (0: not in it)

    explicit ProgBuild(int k) : lev(k, 0) {}
    void begin() { ops.clear(); pe_slot.clear(); pe_src.clear(); }
    void add(int slot, int src_slot, long long src) { (void)slot; pe_slot.push_back(src_slot); pe_src.push_back(src); }
    // close an op whose entries were added since the previous close
    void close(int slot, long long diag, bool keep_empty) {
        const int e0 = ops.empty() ? 0 : ops.back().e1;
        const int e1 = (int)pe_slot.size();
        if (e1 == e0 && !keep_empty) return;
        ops.push_back({slot, diag, e0, e1});
    }
    void end_phase() {
        int maxl = 0;
        std::vector<int> lv(ops.size());
        for (size_t o = 0; o < ops.size(); ++o) {
            int l = 1;
            for (int e = ops[o].e0; e < ops[o].e1; ++e) l = std::max(l, lev[pe_slot[e]] + 1);
            lev[ops[o].slot] = l;
            lv[o] = l;
            maxl = std::max(maxl, l);
        }
        std::vector<int> cnt(maxl + 2, 0);
        for (int l : lv) cnt[l + 1]++;
        for (int l = 1; l <= maxl + 1; ++l) cnt[l] += cnt[l - 1];
        std::vector<int> order(ops.size());
        for (size_t o = 0; o < ops.size(); ++o) order[cnt[lv[o]]++] = (int)o;   // stable within a level
        size_t w = 0;
        for (int l = 1; l <= maxl; ++l) {
            while (w < order.size() && lv[order[w]] == l) {
                const Op& op = ops[order[w]];
                op_slot.push_back(op.slot);
                diag_src.push_back(op.diag);
                for (int e = op.e0; e < op.e1; ++e) { ent_slot.push_back(pe_slot[e]); ent_src.push_back(pe_src[e]); }
                op_ptr.push_back((int)ent_slot.size());
                ++w;
            }
            lvl_ptr.push_back((int)op_slot.size());
            lvl_kind.push_back(0);
        }
        for (const Op& op : ops) lev[op.slot] = 0;
        begin();
    }
    void dense_level(int kind) { lvl_ptr.push_back((int)op_slot.size()); lvl_kind.push_back(kind); }
    int nlev() const { return (int)lvl_kind.size(); }
};

template <typename T>
void upload(DBuf<T>& b, const std::vector<T>& v, cudaStream_t s) {
    b.ensure(s, std::max<size_t>(v.size(), 1));
    if (!v.empty()) CK(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
}
template <typename T>
std::vector<T> download(const T* p, size_t n, cudaStream_t s) {
    std::vector<T> v(n);
    if (n) CK(cudaMemcpyAsync(v.data(), p, n * sizeof(T), cudaMemcpyDeviceToHost, s));
    return v;
}

}  // namespace

// Singleton triangularisation of a k x k pattern (CSC kc_*, CSR kr_* with the
// entry index into the CSC in the CSR's order implied): column singletons of
// the active part are pivoted first (in queue order), then row singletons;
// the rows and columns left over form the kernel.  u1_e indexes the CSC entry
// of a column-singleton pivot, u3_e the CSR entry of a row-singleton pivot.
// Returns null, or why the pattern is structurally singular.
const char* triangularise(int k, const int* kc_ptr, const int* kc_row, const int* kr_ptr, const int* kr_col,
                          Triangular& T) {
    std::vector<int> ccnt(k), rcnt(k), q;
    T = Triangular{};
    T.rdone.assign(k, 0);
    T.cdone.assign(k, 0);
    std::vector<char>& rdone = T.rdone;
    std::vector<char>& cdone = T.cdone;
    for (int j = 0; j < k; ++j) { ccnt[j] = kc_ptr[j + 1] - kc_ptr[j]; if (!ccnt[j]) return "empty column in the structural block"; }
    for (int t = 0; t < k; ++t) { rcnt[t] = kr_ptr[t + 1] - kr_ptr[t]; if (!rcnt[t]) return "empty row in the structural block"; }
    for (int j = 0; j < k; ++j) if (ccnt[j] == 1) q.push_back(j);
    for (size_t h = 0; h < q.size(); ++h) {
        const int j = q[h];
        if (cdone[j] || ccnt[j] != 1) continue;
        int t = -1, ex = -1;
        for (int x = kc_ptr[j]; x < kc_ptr[j + 1]; ++x) if (!rdone[kc_row[x]]) { t = kc_row[x]; ex = x; break; }
        if (t < 0) return "structurally singular structural block";
        rdone[t] = 1; cdone[j] = 1;
        T.u1_t.push_back(t); T.u1_j.push_back(j); T.u1_e.push_back(ex);
        for (int y = kr_ptr[t]; y < kr_ptr[t + 1]; ++y) {
            const int c = kr_col[y];
            if (cdone[c]) continue;
            if (--ccnt[c] == 1) q.push_back(c);
            else if (ccnt[c] == 0) return "structurally singular structural block";
        }
    }
    q.clear();
    for (int t = 0; t < k; ++t) if (!rdone[t] && rcnt[t] == 1) q.push_back(t);
    for (size_t h = 0; h < q.size(); ++h) {
        const int t = q[h];
        if (rdone[t] || rcnt[t] != 1) continue;
        int j = -1, ey = -1;
        for (int y = kr_ptr[t]; y < kr_ptr[t + 1]; ++y) if (!cdone[kr_col[y]]) { j = kr_col[y]; ey = y; break; }
        if (j < 0) return "structurally singular structural block";
        rdone[t] = 1; cdone[j] = 1;
        T.u3_t.push_back(t); T.u3_j.push_back(j); T.u3_e.push_back(ey);
        for (int x = kc_ptr[j]; x < kc_ptr[j + 1]; ++x) {
            const int r = kc_row[x];
            if (rdone[r]) continue;
            if (--rcnt[r] == 1) q.push_back(r);
            else if (rcnt[r] == 0) return "structurally singular structural block";
        }
    }
    int kr = 0, kc = 0;
    for (int t = 0; t < k; ++t) kr += !rdone[t];
    for (int j = 0; j < k; ++j) kc += !cdone[j];
    if (kr != kc) return "structurally singular structural block";
    return nullptr;
}

SfInfo SparseLU::factor(const SfInput& in, const double* d_cval, cudaStream_t s, SfDev* out) {
    SfInfo info;
    const int k = in.k;
    auto fail = [&](const char* why) {
        info.singular = 1;
        snprintf(info.msg, sizeof(info.msg), "%s", why);
        return info;
    };
    if (!ev0) { CK(cudaEventCreate(&ev0)); CK(cudaEventCreate(&ev1)); }
    // ---- K by columns and by rows (entries carry their index in A's CSC)
    std::vector<int> kc_ptr(k + 1, 0), kc_row;
    std::vector<long long> kc_e;
    for (int j = 0; j < k; ++j) {
        const int v = in.s_var[j];
        for (int e = in.cptr[v]; e < in.cptr[v + 1]; ++e) {
            const int t = in.row_kidx[in.crow[e]];
            if (t >= 0 && in.cval[e] != 0.0) { kc_row.push_back(t); kc_e.push_back(e); }
        }
        kc_ptr[j + 1] = (int)kc_row.size();
    }
    const int nnzK = kc_ptr[k];
    std::vector<int> kr_ptr(k + 1, 0), kr_col(nnzK);
    std::vector<long long> kr_e(nnzK);
    for (int x = 0; x < nnzK; ++x) kr_ptr[kc_row[x] + 1]++;
    for (int t = 0; t < k; ++t) kr_ptr[t + 1] += kr_ptr[t];
    {
        std::vector<int> cur(kr_ptr.begin(), kr_ptr.end() - 1);
        for (int j = 0; j < k; ++j)
            for (int x = kc_ptr[j]; x < kc_ptr[j + 1]; ++x) { const int p = cur[kc_row[x]]++; kr_col[p] = j; kr_e[p] = kc_e[x]; }
    }
    // ---- triangularisation
    Triangular tri;
    if (const char* why = triangularise(k, kc_ptr.data(), kc_row.data(), kr_ptr.data(), kr_col.data(), tri))
        return fail(why);
    const std::vector<int>&u1_t = tri.u1_t, &u1_j = tri.u1_j, &u1_e = tri.u1_e;
    const std::vector<int>&u3_t = tri.u3_t, &u3_j = tri.u3_j, &u3_e = tri.u3_e;
    const std::vector<char>&rdone = tri.rdone, &cdone = tri.cdone;
    std::vector<int> krow, kcol, loc_row(k, -1), loc_col(k, -1);
    for (int t = 0; t < k; ++t) if (!rdone[t]) { loc_row[t] = (int)krow.size(); krow.push_back(t); }
    for (int j = 0; j < k; ++j) if (!cdone[j]) { loc_col[j] = (int)kcol.size(); kcol.push_back(j); }
    const int km = (int)krow.size();
    info.km = km;
    // ---- kernel LU on the device
    int ks = 0, kd = 0, nL = 0, pool_top = 0, Lcap = 1;
    std::vector<int> piv_row, piv_col, piv_uidx, piv_ulen, L_row, L_piv, pool_col, dense_row, dense_col;
    CK(cudaEventRecord(ev0, s));
    if (km > 0) {
        std::vector<int> rp(km + 1, 0), rc;
        std::vector<long long> rs;
        for (int a = 0; a < km; ++a) {
            const int t = krow[a];
            for (int y = kr_ptr[t]; y < kr_ptr[t + 1]; ++y)
                if (loc_col[kr_col[y]] >= 0) { rc.push_back(loc_col[kr_col[y]]); rs.push_back(kr_e[y]); }
            rp[a + 1] = (int)rc.size();
        }
        const int nnzM = rp[km];
        // work area: a first guess from the kernel's size, doubled (and kept
        // for the next factorisation) whenever the fill outgrows it
        long long want = std::max(4LL * (nnzM + 4LL * km) + 65536, pool_hint);
        upload(k_row_ptr, rp, s); upload(k_row_col, rc, s); upload(k_row_src, rs, s);
        k_r_start.ensure(s, km); k_r_len.ensure(s, km); k_r_cap.ensure(s, km);
        k_c_ptr.ensure(s, km + 1); k_c_cur.ensure(s, km);
        k_cand_row.ensure(s, km); k_cand_cost.ensure(s, km); k_cand_val.ensure(s, km); k_cand_ok.ensure(s, km);
        k_row_key.ensure(s, km); k_col_piv.ensure(s, km); k_row_piv.ensure(s, km);
        k_piv_row.ensure(s, km); k_piv_col.ensure(s, km); k_piv_uidx.ensure(s, km); k_piv_ulen.ensure(s, km);
        k_dense_row.ensure(s, km); k_dense_col.ensure(s, km); k_out.ensure(s, 8);
        int o[8] = {0};
        int sparse_rounds = 1;
        KluArgs A{};
        for (int attempt = 0; attempt < 6; ++attempt) {
            const int pool_cap = (int)std::min<long long>(want, INT_MAX / 2);
            Lcap = pool_cap;
            k_pool_col.ensure(s, pool_cap); k_pool_val.ensure(s, pool_cap); k_c_row.ensure(s, pool_cap);
            k_L_row.ensure(s, Lcap); k_L_piv.ensure(s, Lcap); k_L_val.ensure(s, Lcap);
            A = KluArgs{km, k_row_ptr.p, k_row_col.p, k_row_src.p, d_cval, pool_cap, k_pool_col.p, k_pool_val.p,
                      k_r_start.p, k_r_len.p, k_r_cap.p, k_c_ptr.p, k_c_cur.p, k_c_row.p,
                      k_cand_row.p, k_cand_cost.p, k_cand_val.p, k_cand_ok.p, k_row_key.p, k_col_piv.p, k_row_piv.p,
                      k_piv_row.p, k_piv_col.p, k_piv_uidx.p, k_piv_ulen.p, k_L_row.p, k_L_piv.p, k_L_val.p, Lcap,
                      k_dense_row.p, k_dense_col.p, k_out.p, sparse_rounds};
            k_kernel_lu<KLU_BS><<<1, KLU_BS, 0, s>>>(A);
            count_launch(1);
            CK(cudaGetLastError());
            CK(cudaMemcpyAsync(o, k_out.p, sizeof(int) * 6, cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            if ((o[2] == KLU_POOL_FULL || o[2] == KLU_L_FULL) && want < INT_MAX / 2) {
                want *= 2;
                pool_hint = want;
                continue;
            }
            if (o[2] == KLU_ROUNDS && sparse_rounds && km <= KLU_DENSE_FALLBACK) {
                sparse_rounds = 0;         // factorise the whole kernel as the dense block
                info.dense_fallback = 1;
                continue;
            }
            break;
        }
        if (o[2] != KLU_OK) {
            char m2[160];
            snprintf(m2, sizeof(m2), "kernel factorisation failed (code %d, kernel %d, round %d)", o[2], km, o[3]);
            return fail(m2);
        }
        ks = o[0]; nL = o[1]; info.rounds = o[3]; pool_top = o[4]; kd = o[5];
        piv_row = download(k_piv_row.p, ks, s); piv_col = download(k_piv_col.p, ks, s);
        piv_uidx = download(k_piv_uidx.p, ks, s); piv_ulen = download(k_piv_ulen.p, ks, s);
        L_row = download(k_L_row.p, nL, s); L_piv = download(k_L_piv.p, nL, s);
        pool_col = download(k_pool_col.p, pool_top, s);
        dense_row = download(k_dense_row.p, km, s); dense_col = download(k_dense_col.p, km, s);
        if (kd > 0) {
            const size_t kk = (size_t)kd * kd;
            g_S.ensure(s, kk); g_Sinv.ensure(s, kk); g_SinvT.ensure(s, kk);
            g_Pan.ensure(s, (size_t)kd * 16); g_Wk.ensure(s, (size_t)kd * 16); g_Winv.ensure(s, 16 * 16);
            g_rowpiv.ensure(s, kd); g_pivrows.ensure(s, kd); g_err.ensure(s, 1);
            k_klu_zero<<<592, 256, 0, s>>>(g_S.p, kk);
            k_klu_dense_build<<<(km + 255) / 256, 256, 0, s>>>(A, kd, g_S.p);
            count_launch(2);
            CK(cudaGetLastError());
            FactorBufs F{g_S.p, g_Pan.p, g_Wk.p, g_rowpiv.p, g_pivrows.p, g_Winv.p, g_err.p, nullptr, nullptr};
            CK(gj_inverse(F, kd, g_Sinv.p, s));
            dim3 g((kd + 31) / 32, (kd + 31) / 32), b(32, 32);
            k_klu_transpose<<<g, b, 0, s>>>(g_Sinv.p, kd, g_SinvT.p);
            count_launch(1);
            CK(cudaGetLastError());
            int ferr = 0;
            CK(cudaMemcpyAsync(&ferr, g_err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            if (ferr) return fail("singular dense block in the kernel factorisation");
        }
    } else {
        CK(cudaStreamSynchronize(s));
    }
    CK(cudaEventRecord(ev1, s));
    info.ks = ks; info.kd = kd;
    // ---- slots
    const int c1 = (int)u1_t.size(), c3 = (int)u3_t.size();
    const int d0 = c1 + ks;
    if (c1 + ks + kd + c3 != k) return fail("inconsistent factor size");
    std::vector<int> pos_row(k, -1), pos_col(k, -1), slot_t(k), slot_j(k);
    for (int i = 0; i < c1; ++i) { pos_row[u1_t[i]] = i; pos_col[u1_j[i]] = i; }
    for (int p = 0; p < ks; ++p) { pos_row[krow[piv_row[p]]] = c1 + p; pos_col[kcol[piv_col[p]]] = c1 + p; }
    for (int a = 0; a < km; ++a) {
        if (dense_row[a] >= 0) pos_row[krow[a]] = d0 + dense_row[a];
        if (dense_col[a] >= 0) pos_col[kcol[a]] = d0 + dense_col[a];
    }
    for (int i = 0; i < c3; ++i) { pos_row[u3_t[i]] = k - 1 - i; pos_col[u3_j[i]] = k - 1 - i; }
    for (int t = 0; t < k; ++t) { if (pos_row[t] < 0) return fail("inconsistent factor rows"); slot_t[pos_row[t]] = t; }
    for (int j = 0; j < k; ++j) { if (pos_col[j] < 0) return fail("inconsistent factor columns"); slot_j[pos_col[j]] = j; }
    std::vector<int> slot_row(k), slot_kcol(k), slot_pos(k);
    for (int x = 0; x < k; ++x) { slot_row[x] = in.rp_row[slot_t[x]]; slot_kcol[x] = slot_j[x]; slot_pos[x] = in.s_pos[slot_j[x]]; }
    // kernel L by target row and by pivot; U rows and U columns
    const long long nA = in.nnzA;
    const long long srcL = nA, srcP = nA + Lcap;
    std::vector<int> Lr_ptr(km + 1, 0), Lr_idx(nL), Lp_ptr(ks + 1, 0), Lp_idx(nL);
    for (int x = 0; x < nL; ++x) { Lr_ptr[L_row[x] + 1]++; Lp_ptr[L_piv[x] + 1]++; }
    for (int a = 0; a < km; ++a) Lr_ptr[a + 1] += Lr_ptr[a];
    for (int p = 0; p < ks; ++p) Lp_ptr[p + 1] += Lp_ptr[p];
    {
        std::vector<int> idx(nL);
        for (int x = 0; x < nL; ++x) idx[x] = x;
        std::sort(idx.begin(), idx.end(), [&](int u, int v) { return L_piv[u] != L_piv[v] ? L_piv[u] < L_piv[v] : L_row[u] < L_row[v]; });
        std::vector<int> cr(Lr_ptr.begin(), Lr_ptr.end() - 1), cp(Lp_ptr.begin(), Lp_ptr.end() - 1);
        for (int x : idx) { Lr_idx[cr[L_row[x]]++] = x; Lp_idx[cp[L_piv[x]]++] = x; }
    }
    info.lnnz = nL;
    std::vector<int> piv_diag(ks, -1);
    std::vector<std::vector<std::pair<int, int>>> ucol(km);   // kernel column -> (pivot, pool index)
    long long unnz = 0;
    for (int p = 0; p < ks; ++p)
        for (int y = 0; y < piv_ulen[p]; ++y) {
            const int idx = piv_uidx[p] + y;
            const int b = pool_col[idx];
            if (b == piv_col[p]) piv_diag[p] = idx;
            else ucol[b].push_back({p, idx});
            ++unnz;
        }
    info.unnz = (int)unnz;
    for (int p = 0; p < ks; ++p) if (piv_diag[p] < 0) return fail("kernel pivot without its entry");
    auto is_u3col = [&](int j) { return pos_col[j] >= d0 + kd; };
    auto is_u1row = [&](int t) { return pos_row[t] < c1; };
    // ---- FTRAN program
    ProgBuild F(k);
    for (int i = 0; i < c3; ++i) {                         // U3, peel order
        const int t = u3_t[i], j = u3_j[i];
        for (int y = kr_ptr[t]; y < kr_ptr[t + 1]; ++y) if (kr_col[y] != j) F.add(0, pos_col[kr_col[y]], kr_e[y]);
        F.close(k - 1 - i, kr_e[u3_e[i]], true);
    }
    F.end_phase();
    auto kernel_row_op = [&](ProgBuild& P, int a, int slot) {   // Z terms, then L terms
        const int t = krow[a];
        for (int y = kr_ptr[t]; y < kr_ptr[t + 1]; ++y) if (is_u3col(kr_col[y])) P.add(0, pos_col[kr_col[y]], kr_e[y]);
        for (int x = Lr_ptr[a]; x < Lr_ptr[a + 1]; ++x) { const int li = Lr_idx[x]; P.add(0, c1 + L_piv[li], srcL + li); }
        P.close(slot, -1, false);
    };
    for (int p = 0; p < ks; ++p) kernel_row_op(F, piv_row[p], c1 + p);
    {
        std::vector<int> drows(kd, -1);
        for (int a = 0; a < km; ++a) if (dense_row[a] >= 0) drows[dense_row[a]] = a;
        for (int x = 0; x < kd; ++x) kernel_row_op(F, drows[x], d0 + x);
    }
    F.end_phase();
    if (kd > 0) F.dense_level(1);
    for (int p = ks - 1; p >= 0; --p) {                    // kernel U, backwards
        for (int y = 0; y < piv_ulen[p]; ++y) {
            const int idx = piv_uidx[p] + y;
            if (idx != piv_diag[p]) F.add(0, pos_col[kcol[pool_col[idx]]], srcP + idx);
        }
        F.close(c1 + p, srcP + piv_diag[p], true);
    }
    F.end_phase();
    for (int i = c1 - 1; i >= 0; --i) {                    // U1, backwards
        const int t = u1_t[i], j = u1_j[i];
        for (int y = kr_ptr[t]; y < kr_ptr[t + 1]; ++y) if (kr_col[y] != j) F.add(0, pos_col[kr_col[y]], kr_e[y]);
        F.close(i, kc_e[u1_e[i]], true);
    }
    F.end_phase();
    // ---- BTRAN program
    ProgBuild B(k);
    for (int i = 0; i < c1; ++i) {                         // U1^T, forwards
        const int t = u1_t[i], j = u1_j[i];
        for (int x = kc_ptr[j]; x < kc_ptr[j + 1]; ++x) if (kc_row[x] != t) B.add(0, pos_row[kc_row[x]], kc_e[x]);
        B.close(i, kc_e[u1_e[i]], true);
    }
    B.end_phase();
    auto kernel_col_op = [&](ProgBuild& P, int b, int slot, long long diag) {   // X^T terms, then U^T terms
        const int j = kcol[b];
        for (int x = kc_ptr[j]; x < kc_ptr[j + 1]; ++x) if (is_u1row(kc_row[x])) P.add(0, pos_row[kc_row[x]], kc_e[x]);
        for (const auto& pu : ucol[b]) P.add(0, c1 + pu.first, srcP + pu.second);
        P.close(slot, diag, diag >= 0);
    };
    for (int p = 0; p < ks; ++p) kernel_col_op(B, piv_col[p], c1 + p, srcP + piv_diag[p]);
    {
        std::vector<int> dcols(kd, -1);
        for (int b = 0; b < km; ++b) if (dense_col[b] >= 0) dcols[dense_col[b]] = b;
        for (int x = 0; x < kd; ++x) kernel_col_op(B, dcols[x], d0 + x, -1);
    }
    B.end_phase();
    if (kd > 0) B.dense_level(2);
    for (int p = ks - 1; p >= 0; --p) {                    // kernel L^T, backwards
        for (int x = Lp_ptr[p]; x < Lp_ptr[p + 1]; ++x) { const int li = Lp_idx[x]; B.add(0, pos_row[krow[L_row[li]]], srcL + li); }
        B.close(c1 + p, -1, false);
    }
    B.end_phase();
    for (int i = c3 - 1; i >= 0; --i) {                    // U3^T, in slot order
        const int t = u3_t[i], j = u3_j[i];
        for (int x = kc_ptr[j]; x < kc_ptr[j + 1]; ++x) if (kc_row[x] != t) B.add(0, pos_row[kc_row[x]], kc_e[x]);
        B.close(k - 1 - i, kr_e[u3_e[i]], true);
    }
    B.end_phase();
    // ---- upload and gather the coefficients
    upload(p_slot_row, slot_row, s); upload(p_slot_kcol, slot_kcol, s); upload(p_slot_pos, slot_pos, s);
    ProgBuild* PB[2] = {&F, &B};
    SfProg* PO[2] = {&out->ft, &out->bt};
    for (int w = 0; w < 2; ++w) {
        ProgBuild& P = *PB[w];
        upload(p_lvl_ptr[w], P.lvl_ptr, s); upload(p_lvl_kind[w], P.lvl_kind, s);
        upload(p_op_slot[w], P.op_slot, s); upload(p_op_ptr[w], P.op_ptr, s); upload(p_ent_slot[w], P.ent_slot, s);
        upload(p_diag_src[w], P.diag_src, s); upload(p_ent_src[w], P.ent_src, s);
        p_op_diag[w].ensure(s, std::max<size_t>(P.diag_src.size(), 1));
        p_ent_coef[w].ensure(s, std::max<size_t>(P.ent_src.size(), 1));
        const double* lv = km > 0 ? k_L_val.p : d_cval;
        const double* pv = km > 0 ? k_pool_val.p : d_cval;
        if (!P.diag_src.empty())
            k_sf_gather<<<148, 256, 0, s>>>(p_diag_src[w].p, (long long)P.diag_src.size(), d_cval, nA, lv, Lcap, pv, p_op_diag[w].p);
        if (!P.ent_src.empty())
            k_sf_gather<<<296, 256, 0, s>>>(p_ent_src[w].p, (long long)P.ent_src.size(), d_cval, nA, lv, Lcap, pv, p_ent_coef[w].p);
        count_launch(2);
        CK(cudaGetLastError());
        SfProg& G = *PO[w];
        G.nlev = P.nlev();
        G.lvl_ptr = p_lvl_ptr[w].p; G.lvl_kind = p_lvl_kind[w].p; G.op_slot = p_op_slot[w].p;
        G.op_ptr = p_op_ptr[w].p; G.op_diag = p_op_diag[w].p; G.ent_slot = p_ent_slot[w].p; G.ent_coef = p_ent_coef[w].p;
    }
    info.lev_ft = F.nlev(); info.lev_bt = B.nlev();
    info.ent_ft = (long long)F.ent_src.size(); info.ent_bt = (long long)B.ent_src.size();
    info.op_ft = (long long)F.op_slot.size(); info.op_bt = (long long)B.op_slot.size();
    out->on = 1; out->k = k; out->d0 = d0; out->kd = kd;
    out->smem = k <= SF_SMEM_SLOTS ? 1 : 0;
    out->Sinv = kd > 0 ? g_Sinv.p : nullptr; out->SinvT = kd > 0 ? g_SinvT.p : nullptr;
    out->slot_row = p_slot_row.p; out->slot_kcol = p_slot_kcol.p; out->slot_pos = p_slot_pos.p;
    p_gvec.ensure(s, out->smem ? 1 : (size_t)MAX_FTRAN_RHS * k);
    p_gtmp.ensure(s, (size_t)MAX_FTRAN_RHS * std::max(kd, 1));
    out->gvec = p_gvec.p; out->gtmp = p_gtmp.p;
    CK(cudaStreamSynchronize(s));
    CK(cudaEventElapsedTime(&info.kernel_ms, ev0, ev1));
    return info;
}

}  // namespace ds

// Singleton triangularisation of a k x k sparse pattern (CSC col_ptr/row_idx),
// for host-side tests: row_order and col_order list the rows and columns in
// pivot order (column singletons, then the kernel's rows / columns in index
// order, then the row singletons in reverse peel order), so that the permuted
// matrix is block upper triangular around the kernel.  *n_col1 / *n_kernel
// receive the counts.  DS_ERR_NUMERIC if the pattern is structurally singular.
extern "C" int ds_sparse_triangularise(int k, const int* col_ptr, const int* row_idx, int* row_order, int* col_order,
                                       int* n_col1, int* n_kernel) {
    if (k <= 0 || !col_ptr || !row_idx || !row_order || !col_order || !n_col1 || !n_kernel) return DS_ERR_ARG;
    if (col_ptr[0] != 0) return DS_ERR_ARG;
    for (int j = 0; j < k; ++j)
        if (col_ptr[j + 1] < col_ptr[j]) return DS_ERR_ARG;
    const int nnz = col_ptr[k];
    std::vector<int> rp(k + 1, 0), rc(nnz);
    for (int x = 0; x < nnz; ++x) {
        if (row_idx[x] < 0 || row_idx[x] >= k) return DS_ERR_ARG;
        rp[row_idx[x] + 1]++;
    }
    for (int t = 0; t < k; ++t) rp[t + 1] += rp[t];
    {
        std::vector<int> cur(rp.begin(), rp.end() - 1);
        for (int j = 0; j < k; ++j)
            for (int x = col_ptr[j]; x < col_ptr[j + 1]; ++x) rc[cur[row_idx[x]]++] = j;
    }
    ds::Triangular T;
    if (ds::triangularise(k, col_ptr, row_idx, rp.data(), rc.data(), T)) return DS_ERR_NUMERIC;
    int w = 0;
    for (size_t i = 0; i < T.u1_t.size(); ++i) { row_order[w] = T.u1_t[i]; col_order[w] = T.u1_j[i]; ++w; }
    const int c1 = w;
    int wr = w, wc = w;
    for (int t = 0; t < k; ++t) if (!T.rdone[t]) row_order[wr++] = t;
    for (int j = 0; j < k; ++j) if (!T.cdone[j]) col_order[wc++] = j;
    for (int i = (int)T.u3_t.size() - 1; i >= 0; --i) { row_order[wr++] = T.u3_t[i]; col_order[wc++] = T.u3_j[i]; }
    *n_col1 = c1;
    *n_kernel = wr - c1 - (int)T.u3_t.size();
    return DS_OK;
}
