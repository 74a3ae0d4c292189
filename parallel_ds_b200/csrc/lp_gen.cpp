// Seeded synthetic LP generator: min c^T x, A x <= b, x >= 0.
//
// A has N(0,1) entries (Bernoulli(density) per entry, a fixed count per column,
// or a block-angular pattern), x0 ~ U[0,1]^n, b = A x0 + U[0.1,1]^m and
// c ~ U[0,1]^n, so every instance is feasible and bounded and the slack basis
// is dual feasible.  The random stream is counter based (SplitMix64 finaliser
// over (seed, stream, index)), so any entry can be drawn independently and the
// output does not depend on thread count.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>

#include "../../include/ds_api.h"

namespace {

enum : uint64_t { S_STRUCT = 1, S_VAL = 2, S_X0 = 3, S_B = 4, S_C = 5, S_DIM = 6 };

inline uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
inline uint64_t stream_key(uint64_t seed, uint64_t stream) {
    return mix64(seed * 0x9E3779B97F4A7C15ull + stream * 0xD1B54A32D192ED03ull + 1ull);
}
inline uint64_t draw(uint64_t key, uint64_t i) { return mix64(key + (i + 1ull) * 0x9E3779B97F4A7C15ull); }
inline double u01(uint64_t h) { return (double)(h >> 11) * 0x1.0p-53; }
inline double normal(uint64_t key, uint64_t i) {
    const double u1 = ((double)(draw(key, 2 * i) >> 11) + 1.0) * 0x1.0p-53;  // (0,1]
    const double u2 = u01(draw(key, 2 * i + 1));
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586476925 * u2);
}
inline uint64_t threshold(double p) {
    if (p >= 1.0) return ~0ull;
    if (p <= 0.0) return 0ull;
    return (uint64_t)std::ldexp((long double)p, 64);
}

struct Triplets { std::vector<int> rptr, col; std::vector<double> val; };

// Bernoulli pattern over a row range [r0, r1) x column range [c0, c1), global
// entry index i*n + j so every entry has one fixed draw.
void density_rows(uint64_t seed, int n, int r0, int r1, int c0, int c1, double p,
                  std::vector<std::vector<int>>& cols, std::vector<std::vector<double>>& vals) {
    const uint64_t ks = stream_key(seed, S_STRUCT), kv = stream_key(seed, S_VAL);
    const uint64_t thr = threshold(p);
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = r0; i < r1; ++i) {
        for (int j = c0; j < c1; ++j) {
            const uint64_t e = (uint64_t)i * (uint64_t)n + (uint64_t)j;
            if (draw(ks, e) < thr) {
                cols[i].push_back(j);
                vals[i].push_back(normal(kv, e));
            }
        }
    }
}

}  // namespace

extern "C" int ds_gen_batch_m(unsigned long long seed, int i, int m_lo, int m_hi) {
    if (m_hi < m_lo) return m_lo;
    const uint64_t k = stream_key(seed + (unsigned long long)i, S_DIM);
    return m_lo + (int)(draw(k, 0) % (uint64_t)(m_hi - m_lo + 1));
}

extern "C" long long ds_gen_lp(const ds_gen_spec* sp, int* row_ptr, int* col_idx, double* val,
                               double* b, double* c, long long capacity) {
    if (!sp || sp->m <= 0 || sp->n <= 0) return DS_ERR_ARG;
    const int m = sp->m, n = sp->n;
    const uint64_t seed = sp->seed;
    std::vector<std::vector<int>> cols(m);
    std::vector<std::vector<double>> vals(m);

    if (sp->kind == DS_GEN_DENSITY) {
        density_rows(seed, n, 0, m, 0, n, sp->density, cols, vals);
    } else if (sp->kind == DS_GEN_PER_COL) {
        const int k = sp->per_col;
        if (k <= 0 || k > m) return DS_ERR_ARG;
        const uint64_t ks = stream_key(seed, S_STRUCT), kv = stream_key(seed, S_VAL);
        std::vector<int> rows_of(n * (size_t)k);
#pragma omp parallel for schedule(static)
        for (int j = 0; j < n; ++j) {
            int* r = &rows_of[(size_t)j * k];
            int got = 0;
            for (uint64_t t = 0; got < k; ++t) {
                const int cand = (int)(draw(ks, (uint64_t)j * 4096ull + t) % (uint64_t)m);
                bool dup = false;
                for (int u = 0; u < got; ++u) dup |= (r[u] == cand);
                if (!dup) r[got++] = cand;
            }
        }
        for (int j = 0; j < n; ++j)
            for (int s = 0; s < k; ++s) {
                const int i = rows_of[(size_t)j * k + s];
                cols[i].push_back(j);
                vals[i].push_back(normal(kv, (uint64_t)j * k + s));
            }
    } else if (sp->kind == DS_GEN_BLOCK) {
        const int B = sp->blocks, mb = sp->block_m, nb = sp->block_n, L = sp->link_rows;
        if (B <= 0 || (long long)B * mb + L != m || (long long)B * nb != n) return DS_ERR_ARG;
        for (int blk = 0; blk < B; ++blk)
            density_rows(seed, n, blk * mb, (blk + 1) * mb, blk * nb, (blk + 1) * nb,
                         sp->block_density, cols, vals);
        density_rows(seed, n, B * mb, m, 0, n, sp->link_density, cols, vals);
    } else {
        return DS_ERR_ARG;
    }

    long long nnz = 0;
    for (int i = 0; i < m; ++i) nnz += (long long)cols[i].size();
    if (!val || !row_ptr || !col_idx || capacity < nnz) return nnz;

    // rows come out column-sorted: per-row generation walks j ascending; the
    // per-column kind is sorted here.
    long long pos = 0;
    row_ptr[0] = 0;
    for (int i = 0; i < m; ++i) {
        std::vector<int> ord(cols[i].size());
        for (size_t t = 0; t < ord.size(); ++t) ord[t] = (int)t;
        std::sort(ord.begin(), ord.end(), [&](int a, int b2) { return cols[i][a] < cols[i][b2]; });
        for (int t : ord) { col_idx[pos] = cols[i][t]; val[pos] = vals[i][t]; ++pos; }
        row_ptr[i + 1] = (int)pos;
    }

    const uint64_t kx = stream_key(seed, S_X0), kb = stream_key(seed, S_B), kc = stream_key(seed, S_C);
    std::vector<double> x0(n);
    for (int j = 0; j < n; ++j) x0[j] = u01(draw(kx, j));
    if (b) {
        for (int i = 0; i < m; ++i) {
            double s = 0.0;
            for (int e = row_ptr[i]; e < row_ptr[i + 1]; ++e) s += val[e] * x0[col_idx[e]];
            b[i] = s + (0.1 + 0.9 * u01(draw(kb, i)));
        }
    }
    if (c)
        for (int j = 0; j < n; ++j) c[j] = u01(draw(kc, j));
    return nnz;
}
