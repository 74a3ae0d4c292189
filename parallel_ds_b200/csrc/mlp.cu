// Learned leaving-row scorer: MLP 12 -> 64 -> 64 -> 1 on the 5th-generation
// tensor cores (tcgen05, BF16 operands, FP32 accumulation in tensor memory).
// No counterpart in the reference.
//
// Forward (one CTA = 128 rows, 4 warps; warp w owns TMEM lanes 32w..32w+31):
//   X (128 x 16 bf16, 12 features zero-padded) --tcgen05.mma--> TMEM cols 0..63
//   + b1, ReLU -> H1 (bf16, shared memory) --4 x tcgen05.mma--> TMEM cols 64..127
//   + b2, ReLU -> H2;  logit = b3 + H2 . w3 (CUDA cores; N = 1 is below the MMA size)
// Backward (per 128-row tile): dH1 = dH2 W2, dW2^T = H1^T dH2 and dW1^T = X^T dH1
// on tcgen05 (M = 128 by zero-padding the 64- and 16-row operands), bias and w3
// gradients on CUDA cores; tile partials are reduced in tile order, then Adam.
//
// Shared-memory operands use the canonical K-major no-swizzle layout: 8x16-byte
// core matrices; for a (rows x 16) K block, element (r, k) sits at
//   (r / 8) * 256 + ((k % 16) / 8) * 128 + (r % 8) * 16 + (k % 8) * 2
// bytes, i.e. LBO = 128 (next 8 K elements), SBO = 256 (next 8 rows).
// Every wait on the MMA-completion mbarrier is bounded; on timeout the kernel
// sets the model's error flag (the host reports DS_ERR_DEVICE_WAIT), marks its
// scores unusable (CHUZR then falls back to DSE), frees its TMEM and returns.
#include <cuda_bf16.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <utility>
#include <vector>

#include "../../include/ds_api.h"
#include "engine.cuh"
#include "kernels.cuh"
#include "mlp.cuh"

namespace ds {

// ------------------------------------------------------------ tcgen05 helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t kmajor_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((128u >> 4) & 0x3FFFu) << 16;   // LBO: next 8 K elements
    d |= (uint64_t)((256u >> 4) & 0x3FFFu) << 32;   // SBO: next 8 rows
    d |= 1ull << 46;                                 // descriptor version for sm_100
    return d;                                        // base offset 0, SWIZZLE_NONE
}

// kind::f16 instruction descriptor: D = F32, A = B = BF16, both K-major.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void umma_commit(uint64_t* mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(smem_u32(mbar)) : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(mbar)), "r"(count));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait for mbarrier phase `parity`; returns false on timeout.
// test_polls > 0 (set by ds_model_set_wait_limit for failure-path tests)
// replaces the bound by that many non-blocking polls; when they run out, the
// wait still drains (bounded) until the MMAs have finished, because they keep
// writing their TMEM columns, which are then read and freed.
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, int test_polls) {
    const uint32_t addr = smem_u32(mbar);
    if (test_polls > 0) {
        for (int it = 0; it < test_polls; ++it) {
            uint32_t done;
            asm volatile("{\n\t.reg .pred P1;\n\t"
                         "mbarrier.test_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                         "selp.b32 %0, 1, 0, P1;\n\t}\n"
                         : "=r"(done) : "r"(addr), "r"(parity) : "memory");
            if (done) return true;
        }
        for (long it = 0; it < (1L << 26); ++it) {
            uint32_t done;
            asm volatile("{\n\t.reg .pred P1;\n\t"
                         "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                         "selp.b32 %0, 1, 0, P1;\n\t}\n"
                         : "=r"(done) : "r"(addr), "r"(parity) : "memory");
            if (done) break;
        }
        return false;
    }
    for (long it = 0; it < (1L << 26); ++it) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred P1;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                     "selp.b32 %0, 1, 0, P1;\n\t}\n"
                     : "=r"(done) : "r"(addr), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" :: "r"(smem_u32(dst_smem)), "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(ncols));
}

// 32 lanes x 64 consecutive 32-bit columns -> 64 registers per thread.
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, float* v) {
    uint32_t r[64];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x64.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,"
        "%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47,"
        "%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%64];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]),
          "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]),
          "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]),
          "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]),
          "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 64; ++i) v[i] = __uint_as_float(r[i]);
}

// byte offset of element (r, k) in a K-major operand of K-blocks of 16
__device__ __forceinline__ uint32_t kofs(int r, int k, uint32_t kblock_bytes) {
    return (uint32_t)(k >> 4) * kblock_bytes + (uint32_t)(r >> 3) * 256u + (uint32_t)((k & 15) >> 3) * 128u +
           (uint32_t)(r & 7) * 16u + (uint32_t)(k & 7) * 2u;
}
__device__ __forceinline__ void st_bf16(unsigned char* base, uint32_t off, float v) {
    *reinterpret_cast<__nv_bfloat16*>(base + off) = __float2bfloat16_rn(v);
}
// Eight consecutive K elements of one row are one 16-byte core-matrix row.
__device__ __forceinline__ void st_bf16x8(unsigned char* base, uint32_t off, const float* v) {
    uint4 u;
    __nv_bfloat162 p0 = __floats2bfloat162_rn(v[0], v[1]), p1 = __floats2bfloat162_rn(v[2], v[3]);
    __nv_bfloat162 p2 = __floats2bfloat162_rn(v[4], v[5]), p3 = __floats2bfloat162_rn(v[6], v[7]);
    u.x = *reinterpret_cast<uint32_t*>(&p0); u.y = *reinterpret_cast<uint32_t*>(&p1);
    u.z = *reinterpret_cast<uint32_t*>(&p2); u.w = *reinterpret_cast<uint32_t*>(&p3);
    *reinterpret_cast<uint4*>(base + off) = u;
}

// --------------------------------------------------------------- parameters
// fp32 master layout (DS_MLP_NPARAMS floats): W1[64][12], b1[64], W2[64][64], b2[64], w3[64], b3.
// The bf16 copies the MMAs read: W1 padded to [64][16] (zero columns 12..15) and W2
// [64][64], so that every row is a whole number of 16-byte core-matrix rows.
constexpr int NF = DS_NUM_FEATURES;
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + 64 * NF, OFF_W2 = OFF_B1 + 64, OFF_B2 = OFF_W2 + 64 * 64,
              OFF_W3 = OFF_B2 + 64, OFF_B3 = OFF_W3 + 64, NPARAMS = OFF_B3 + 1;
static_assert(NPARAMS == DS_MLP_NPARAMS, "parameter count");
static_assert(NF <= 16, "features fit one K block");

__device__ __forceinline__ float clampf(double v, double lo, double hi) { return (float)fmin(fmax(v, lo), hi); }
// log10 of v clamped to [lo, hi] (lo >= -30), in single precision.
__device__ __forceinline__ float lg10f(double v, float lo, float hi) {
    const float a = (float)fmin(fmax(v, 1e-30), 1e30);
    return fminf(fmaxf(log10f(a), lo), hi);
}

// Iteration number the pricing of this launch belongs to.
__device__ __forceinline__ int pricing_iteration(const Ctl* c) { return c->iteration + (c->top_done ? 0 : 1); }

// Features of basis position i for the current iteration (the order listed in
// ds_api.h).  Returns false when the row is not a leaving-row candidate (not
// primal infeasible, or a zero DSE weight), exactly the rows k_chuzr skips.
__device__ bool row_features(const Dev& D, int i, int it, float* f) {
    const int j = D.basis[i];
    const double be = D.beta[i];
    const double x = D.x[j];
    const unsigned char t = D.type[j];
    const double l = D.lb[j], u = D.ub[j];
    const float pg = D.pd_gap[j], pdu = D.pd_dual[j];
    const int ec = D.enter_count[j], ea = D.entered_at[j];
    const Ctl* c = D.ctl;
    const double bp = c->beta_p, dl = c->delta;
    const int ninf = c->ninfeas;
    double dt = 0.0;
    const bool inf = var_infeas(t, x, l, u, &dt) && fabs(dt) > 1e-8;
    const double w = inf ? (dt * dt) / be : 0.0;
    const double wl = (bp > 0.0) ? (dl * dl) / bp : 0.0;   // last pick's weight
    // The logarithms run in single precision (the features are rounded to
    // bf16 for the tensor cores); arguments are floored at 1e-30, below every
    // clamp, so that underflow to zero in the conversion changes nothing.
    f[0] = (j >= D.n) ? 1.f : 0.f;
    f[1] = lg10f(fabs(dt), -12.f, 4.f) * 0.25f;
    f[2] = lg10f(be, -12.f, 12.f) * 0.25f;
    f[3] = lg10f(w, -24.f, 12.f) * 0.25f;
    f[4] = (wl > 0.0 && w > 0.0) ? lg10f(w / wl, -12.f, 12.f) * 0.25f : 0.f;
    f[5] = fminf(fmaxf(asinhf(1000.f * pg) * 0.125f, -2.f), 2.f);
    f[6] = fminf(fmaxf(asinhf(1000.f * pdu) * 0.125f, -2.f), 2.f);
    f[7] = (float)ninf / (float)D.m;
    f[8] = clampf((double)it / D.m, 0, 10) / 5.f;
    f[9] = (float)min(ec, 20) / 5.f;
    f[10] = clampf((double)(it - ea) / D.m, 0, 5);
    const double ax = fabs(x);
    const float lx = ax < 1e30 ? log10f(1.f + (float)ax) : (float)log10(1.0 + ax);
    f[11] = x < 0.0 ? -lx : lx;
    for (int k = NF; k < 16; ++k) f[k] = 0.f;
    return inf && w > 0.0;
}

// Append a candidate row's features to the trace on sampled iterations.
__device__ void trace_row(const Dev& D, int i, int it, const float* f) {
    const int slot = atomicAdd(&D.ctl->ftr_n, 1);
    if (slot >= D.ftr_cap) return;
    for (int k = 0; k < NF; ++k) D.ftr_feat[(size_t)slot * NF + k] = f[k];
    D.ftr_meta[3 * (size_t)slot] = it;
    D.ftr_meta[3 * (size_t)slot + 1] = i;
    D.ftr_meta[3 * (size_t)slot + 2] = D.basis[i];
}

__device__ __forceinline__ bool trace_now(const Dev& D, int it) {
    return D.ftr_every > 0 && (it % D.ftr_every) == 0;
}

// ------------------------------------------------------------------ forward
// mode 0: rows of X (M x NF fp32, row major) -> logits (+ H1, H2 post-ReLU
// activations, M x 64 fp32, for the backward pass).  mode 1: rows are the
// basis positions of the solver state in D; writes D.score (logit, or -inf for
// rows that cannot leave) and the feature trace.
struct FwdArgs {
    const float* X; int M;
    const __nv_bfloat16* W1b; const __nv_bfloat16* W2b; const float* P;
    float* logits; float* H1; float* H2;
    int* err;
};

constexpr uint32_t KB_A = 128 * 16 * 2;   // bytes of a 128-row, 16-wide K block
constexpr uint32_t KB_B = 64 * 16 * 2;    // bytes of a 64-row, 16-wide K block

__global__ void __launch_bounds__(128) k_mlp_fwd(FwdArgs a, Dev D, int mode) {
    __shared__ __align__(1024) unsigned char sA1[KB_A];          // X tile, 128 x 16
    __shared__ __align__(1024) unsigned char sB1[KB_B];          // W1, 64 x 16
    __shared__ __align__(1024) unsigned char sA2[4 * KB_A];      // H1 tile, 128 x 64
    __shared__ __align__(1024) unsigned char sB2[4 * KB_B];      // W2, 64 x 64
    __shared__ uint64_t mbar;
    __shared__ uint32_t tmem_base;
    __shared__ int bad;
    __shared__ float sP[3 * 64 + 1];                             // b1, b2, w3, b3
    const int tid = threadIdx.x, warp = tid >> 5;
    const int row = blockIdx.x * 128 + tid;
    const bool live = row < a.M;
    // Prologue that reads nothing the previous kernel writes (the weights are
    // fixed during a solve): under programmatic dependent launch it overlaps
    // the tail of that kernel.  The weights go straight into the K-major
    // core-matrix layout with 16-byte loads.
    if (mode == 1) asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if (tid == 0) { mbar_init(&mbar, 1); bad = 0; }
    if (warp == 0) tmem_alloc(&tmem_base, 128);
    *reinterpret_cast<uint4*>(sB1 + kofs(tid >> 1, 8 * (tid & 1), KB_B)) = reinterpret_cast<const uint4*>(a.W1b)[tid];
#pragma unroll
    for (int c = tid; c < 512; c += 128)
        *reinterpret_cast<uint4*>(sB2 + kofs(c >> 3, 8 * (c & 7), KB_B)) = reinterpret_cast<const uint4*>(a.W2b)[c];
    for (int e = tid; e < 3 * 64 + 1; e += 128)   // w3 and b3 are adjacent (OFF_W3 + 64 == OFF_B3)
        sP[e] = e < 64 ? a.P[OFF_B1 + e] : e < 128 ? a.P[OFF_B2 + e - 64] : a.P[OFF_W3 + e - 128];
    int it = 0;
    if (mode == 1) {
        asm volatile("griddepcontrol.wait;" ::: "memory");
        const Ctl* c = D.ctl;
        it = pricing_iteration(c);
        // block-uniform: no scores when halted, in phase 1, or while DSE prices
        // the first iterations; the TMEM columns are freed before returning
        if (__ldcg(&c->halt) || c->phase != 2 || it < D.learn_start) {
            tc_before_sync();
            __syncthreads();
            tc_after_sync();
            if (warp == 0) tmem_dealloc(tmem_base, 128);
            return;
        }
    }
    float f[16];
    bool cand = false;
    if (live) {
        if (mode == 0) {
            for (int k = 0; k < NF; ++k) f[k] = a.X[(size_t)row * NF + k];
            for (int k = NF; k < 16; ++k) f[k] = 0.f;
        } else {
            cand = row_features(D, row, it, f);
            if (cand && trace_now(D, it)) trace_row(D, row, it, f);
        }
    } else {
        for (int k = 0; k < 16; ++k) f[k] = 0.f;
    }
    st_bf16x8(sA1, kofs(tid, 0, KB_A), f);
    st_bf16x8(sA1, kofs(tid, 8, KB_A), f + 8);
    fence_async_smem();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tm = tmem_base;
    const uint32_t lane_base = (uint32_t)(32 * warp) << 16;
    if (tid == 0) {
        umma_bf16(tm, kmajor_desc(smem_u32(sA1)), kmajor_desc(smem_u32(sB1)), idesc_bf16(128, 64), 0u);
        umma_commit(&mbar);
    }
    if (!mbar_wait(&mbar, 0, a.err ? a.err[1] : 0)) bad = 1;
    tc_after_sync();
    float h[64];
    tmem_ld64(tm + lane_base, h);
#pragma unroll
    for (int k = 0; k < 64; ++k) h[k] = fmaxf(h[k] + sP[k], 0.f);
#pragma unroll
    for (int c8 = 0; c8 < 8; ++c8) st_bf16x8(sA2, kofs(tid, 8 * c8, KB_A), h + 8 * c8);
    if (live && a.H1) for (int k = 0; k < 64; ++k) a.H1[(size_t)row * 64 + k] = h[k];
    fence_async_smem();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    if (tid == 0) {
        for (int s = 0; s < 4; ++s)
            umma_bf16(tm + 64, kmajor_desc(smem_u32(sA2) + s * KB_A), kmajor_desc(smem_u32(sB2) + s * KB_B),
                      idesc_bf16(128, 64), s > 0 ? 1u : 0u);
        umma_commit(&mbar);
    }
    if (!mbar_wait(&mbar, 1, a.err ? a.err[1] : 0)) bad = 1;
    tc_after_sync();
    tmem_ld64(tm + lane_base + 64, h);
    float logit = sP[192];
    for (int k = 0; k < 64; ++k) {
        h[k] = fmaxf(h[k] + sP[64 + k], 0.f);
        logit += h[k] * sP[128 + k];
    }
    if (live && a.H2) for (int k = 0; k < 64; ++k) a.H2[(size_t)row * 64 + k] = h[k];
    if (live) {
        if (mode == 0) a.logits[row] = logit;
        else D.score[row] = (cand && !bad) ? logit : -INFINITY;
    }
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    if (warp == 0) tmem_dealloc(tm, 128);
    if (tid == 0 && bad && a.err) atomicExch(a.err, 1);
}

// Feature trace without a network (plain DSE solves that produce training data).
__global__ void __launch_bounds__(128) k_features(Dev D) {
    pdl_enter();
    const Ctl* c = D.ctl;
    if (*(volatile const int*)&c->halt || c->phase != 2) return;
    const int it = pricing_iteration(c);
    if (!trace_now(D, it)) return;
    const int row = blockIdx.x * 128 + threadIdx.x;
    if (row >= D.m) return;
    float f[16];
    if (row_features(D, row, it, f)) trace_row(D, row, it, f);
}

// ----------------------------------------------------------------- backward
// Binary cross-entropy with logits, mean over the M rows of the batch.
struct BwdArgs {
    const float* X; const float* y; const float* H1; const float* H2; const float* logits; int M;
    const float* P; const __nv_bfloat16* W2b;
    float* part;          // per tile: gradient partials in the parameter layout + loss
    int* err;
};
constexpr int PART = NPARAMS + 1;

constexpr size_t BW_H1T = 0;                        // [H1^T ; 0]  128 x 128 (K = tile rows)
constexpr size_t BW_XT = BW_H1T + 8 * KB_A;         // [X^T ; 0]   128 x 128
constexpr size_t BW_DH2T = BW_XT + 8 * KB_A;        // dH2 as B:    64 x 128 (N = unit, K = rows)
constexpr size_t BW_DH1T = BW_DH2T + 8 * KB_B;      // dH1 as B:    64 x 128
constexpr size_t BW_DH2 = BW_DH1T + 8 * KB_B;       // dH2 as A:   128 x 64  (K = unit)
constexpr size_t BW_W2T = BW_DH2 + 4 * KB_A;        // W2^T as B:   64 x 64  (N = input, K = output)
constexpr size_t BW_F = BW_W2T + 4 * KB_B;          // fp32 128 x 65 staging for column sums
constexpr size_t BWD_SMEM = BW_F + 128 * 65 * 4;

__global__ void __launch_bounds__(128) k_mlp_bwd(BwdArgs a) {
    extern __shared__ __align__(1024) unsigned char dyn[];
    unsigned char* sH1t = dyn + BW_H1T;
    unsigned char* sXt = dyn + BW_XT;
    unsigned char* sdH2t = dyn + BW_DH2T;
    unsigned char* sdH1t = dyn + BW_DH1T;
    unsigned char* sdH2 = dyn + BW_DH2;
    unsigned char* sW2t = dyn + BW_W2T;
    float* sF = reinterpret_cast<float*>(dyn + BW_F);
    __shared__ uint64_t mbar;
    __shared__ uint32_t tmem_base;
    __shared__ float sg3[128], sloss[128];
    __shared__ int bad;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int row = blockIdx.x * 128 + tid;
    const bool live = row < a.M;
    float* out = a.part + (size_t)blockIdx.x * PART;
    if (tid == 0) { mbar_init(&mbar, 1); bad = 0; }
    if (warp == 0) tmem_alloc(&tmem_base, 256);
    float g3 = 0.f, loss = 0.f;
    if (live) {
        const float z = a.logits[row], yy = a.y[row];
        const float sg = 1.f / (1.f + expf(-z));
        g3 = (sg - yy) / (float)a.M;
        loss = (fmaxf(z, 0.f) - z * yy + log1pf(expf(-fabsf(z)))) / (float)a.M;
    }
    sg3[tid] = g3;
    sloss[tid] = loss;
    // dH2 = dlogit * w3 through ReLU 2; operands of the three products
    for (int k = 0; k < 64; ++k) {
        const float hv = live ? a.H2[(size_t)row * 64 + k] : 0.f;
        const float d2 = (hv > 0.f) ? g3 * a.P[OFF_W3 + k] : 0.f;
        sF[tid * 65 + k] = d2;
        st_bf16(sdH2t, kofs(k, tid, KB_B), d2);
        st_bf16(sdH2, kofs(tid, k, KB_A), d2);
        st_bf16(sH1t, kofs(k, tid, KB_A), live ? a.H1[(size_t)row * 64 + k] : 0.f);
        st_bf16(sH1t, kofs(64 + k, tid, KB_A), 0.f);
    }
    for (int k = 0; k < 128; ++k)
        st_bf16(sXt, kofs(k, tid, KB_A), (k < NF && live) ? a.X[(size_t)row * NF + k] : 0.f);
    for (int e = tid; e < 64 * 64; e += 128) {
        const int o = e >> 6, i = e & 63;     // W2[o][i] -> B(n = i, k = o)
        *reinterpret_cast<__nv_bfloat16*>(sW2t + kofs(i, o, KB_B)) = a.W2b[o * 64 + i];
    }
    fence_async_smem();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tm = tmem_base;
    const uint32_t lane_base = (uint32_t)(32 * warp) << 16;
    // TMEM columns: 0..63 dH1 (128 x 64); 64..127 [dW2^T; 0]; 128..191 [dW1^T; 0]
    if (tid == 0) {
        for (int s = 0; s < 4; ++s)
            umma_bf16(tm, kmajor_desc(smem_u32(sdH2) + s * KB_A), kmajor_desc(smem_u32(sW2t) + s * KB_B),
                      idesc_bf16(128, 64), s > 0 ? 1u : 0u);
        for (int s = 0; s < 8; ++s)
            umma_bf16(tm + 64, kmajor_desc(smem_u32(sH1t) + s * KB_A), kmajor_desc(smem_u32(sdH2t) + s * KB_B),
                      idesc_bf16(128, 64), s > 0 ? 1u : 0u);
        umma_commit(&mbar);
    }
    // while the tensor cores run: db2 (threads 0..63) and dw3 (64..127), rows in order
    if (tid < 64) {
        float s = 0.f;
        for (int r = 0; r < 128; ++r) s += sF[r * 65 + tid];
        out[OFF_B2 + tid] = s;
    } else {
        const int k = tid - 64;
        float s = 0.f;
        for (int r = 0; r < 128; ++r) {
            const int gr = blockIdx.x * 128 + r;
            if (gr < a.M) s += sg3[r] * a.H2[(size_t)gr * 64 + k];
        }
        out[OFF_W3 + k] = s;
    }
    if (tid == 0) {
        float s = 0.f, l = 0.f;
        for (int r = 0; r < 128; ++r) { s += sg3[r]; l += sloss[r]; }
        out[OFF_B3] = s;
        out[NPARAMS] = l;
    }
    if (!mbar_wait(&mbar, 0, a.err ? a.err[1] : 0)) bad = 1;
    tc_after_sync();
    __syncthreads();                     // sF reads above are done
    float v[64];
    tmem_ld64(tm + lane_base, v);        // dH1 of this thread's row
    for (int k = 0; k < 64; ++k) {
        const bool on = live && a.H1[(size_t)row * 64 + k] > 0.f;   // through ReLU 1
        const float d1 = on ? v[k] : 0.f;
        sF[tid * 65 + k] = d1;
        st_bf16(sdH1t, kofs(k, tid, KB_B), d1);
    }
    fence_async_smem();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    if (tid == 0) {
        for (int s = 0; s < 8; ++s)
            umma_bf16(tm + 128, kmajor_desc(smem_u32(sXt) + s * KB_A), kmajor_desc(smem_u32(sdH1t) + s * KB_B),
                      idesc_bf16(128, 64), s > 0 ? 1u : 0u);
        umma_commit(&mbar);
    }
    if (tid < 64) {
        float s = 0.f;
        for (int r = 0; r < 128; ++r) s += sF[r * 65 + tid];
        out[OFF_B1 + tid] = s;
    }
    if (!mbar_wait(&mbar, 1, a.err ? a.err[1] : 0)) bad = 1;
    tc_after_sync();
    // dW2[o][i] = dW2^T[i][o]: rows i = 0..63 sit in TMEM lanes 0..63 (warps 0, 1)
    if (warp < 2) {
        tmem_ld64(tm + lane_base + 64, v);
        for (int o = 0; o < 64; ++o) out[OFF_W2 + o * 64 + tid] = v[o];
    }
    // dW1[o][f] = dW1^T[f][o]: rows f < NF sit in lanes 0..NF-1 (warp 0)
    if (warp == 0) {
        tmem_ld64(tm + lane_base + 128, v);
        if (lane < NF) for (int o = 0; o < 64; ++o) out[OFF_W1 + o * NF + lane] = v[o];
    }
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    if (warp == 0) tmem_dealloc(tm, 256);
    if (tid == 0 && bad && a.err) atomicExch(a.err, 1);
}

// Sum the tile partials in tile order -> gradient and loss.
__global__ void k_mlp_reduce(const float* part, int ntiles, float* grad, float* loss) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > NPARAMS) return;
    float s = 0.f;
    for (int t = 0; t < ntiles; ++t) s += part[(size_t)t * PART + p];
    if (p < NPARAMS) grad[p] = s;
    else *loss = s;
}

// Adam (Kingma & Ba 2015) on the fp32 master parameters; refreshes the bf16
// copies the tensor cores read.
__global__ void k_mlp_adam(float* P, float* m1, float* m2, const float* g, float lr, float b1, float b2,
                           float eps, int step, __nv_bfloat16* W1b, __nv_bfloat16* W2b) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= NPARAMS) return;
    const float gg = g[p];
    const float a1 = b1 * m1[p] + (1.f - b1) * gg;
    const float a2 = b2 * m2[p] + (1.f - b2) * gg * gg;
    m1[p] = a1;
    m2[p] = a2;
    const float mh = a1 / (1.f - powf(b1, (float)step));
    const float vh = a2 / (1.f - powf(b2, (float)step));
    const float v = P[p] - lr * mh / (sqrtf(vh) + eps);
    P[p] = v;
    if (p < OFF_B1) W1b[(p / NF) * 16 + p % NF] = __float2bfloat16_rn(v);
    else if (p >= OFF_W2 && p < OFF_B2) W2b[p - OFF_W2] = __float2bfloat16_rn(v);
}

__global__ void k_mlp_to_bf16(const float* P, __nv_bfloat16* W1b, __nv_bfloat16* W2b) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < 64 * 16) W1b[p] = __float2bfloat16_rn((p % 16) < NF ? P[OFF_W1 + (p / 16) * NF + p % 16] : 0.f);
    if (p < 64 * 64) W2b[p] = __float2bfloat16_rn(P[OFF_W2 + p]);
}

// Gather a training batch by row index from the resident training set.
__global__ void k_gather_rows(const float* X, const float* y, const int* idx, int M, float* Xb, float* yb) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= M) return;
    const int s = idx[r];
    for (int k = 0; k < NF; ++k) Xb[(size_t)r * NF + k] = X[(size_t)s * NF + k];
    yb[r] = y[s];
}

// ------------------------------------------------------------------ model
struct MlpModel {
    int device = 0;
    cudaStream_t stream = nullptr;
    float* P = nullptr; float* m1 = nullptr; float* m2 = nullptr; float* g = nullptr; float* loss = nullptr;
    __nv_bfloat16* W1b = nullptr; __nv_bfloat16* W2b = nullptr;
    int* err = nullptr;
    int step = 0;
    // batch scratch
    float* X = nullptr; float* y = nullptr; float* H1 = nullptr; float* H2 = nullptr; float* z = nullptr;
    float* part = nullptr; size_t cap = 0;
    // resident training set
    float* Xall = nullptr; float* yall = nullptr; int* idx = nullptr; size_t cap_all = 0;

    void free_batch() {
        for (void* p : {(void*)X, (void*)y, (void*)H1, (void*)H2, (void*)z, (void*)part}) if (p) cudaFree(p);
        X = y = H1 = H2 = z = part = nullptr;
        cap = 0;
    }
    void free_all_rows() {
        for (void* p : {(void*)Xall, (void*)yall, (void*)idx}) if (p) cudaFree(p);
        Xall = yall = nullptr; idx = nullptr;
        cap_all = 0;
    }
    ~MlpModel() {
        cudaSetDevice(device);
        free_batch();
        free_all_rows();
        for (void* p : {(void*)P, (void*)m1, (void*)m2, (void*)g, (void*)loss, (void*)W1b, (void*)W2b, (void*)err})
            if (p) cudaFree(p);
        if (stream) cudaStreamDestroy(stream);
    }
    bool ensure(size_t rows) {
        if (rows <= cap) return true;
        free_batch();
        const size_t tiles = (rows + 127) / 128;
        bool ok = cudaMalloc(&X, rows * NF * sizeof(float)) == cudaSuccess;
        ok = ok && cudaMalloc(&y, rows * sizeof(float)) == cudaSuccess;
        ok = ok && cudaMalloc(&H1, rows * 64 * sizeof(float)) == cudaSuccess;
        ok = ok && cudaMalloc(&H2, rows * 64 * sizeof(float)) == cudaSuccess;
        ok = ok && cudaMalloc(&z, rows * sizeof(float)) == cudaSuccess;
        ok = ok && cudaMalloc(&part, tiles * PART * sizeof(float)) == cudaSuccess;
        if (!ok) { free_batch(); return false; }
        cap = rows;
        return true;
    }
    bool ensure_all(size_t rows) {
        if (rows <= cap_all) return true;
        free_all_rows();
        bool ok = cudaMalloc(&Xall, rows * NF * sizeof(float)) == cudaSuccess;
        ok = ok && cudaMalloc(&yall, rows * sizeof(float)) == cudaSuccess;
        ok = ok && cudaMalloc(&idx, rows * sizeof(int)) == cudaSuccess;
        if (!ok) { free_all_rows(); return false; }
        cap_all = rows;
        return true;
    }
};

static cudaError_t forward(MlpModel* md, const float* dX, int M, float* dz, float* dH1, float* dH2) {
    FwdArgs a{dX, M, md->W1b, md->W2b, md->P, dz, dH1, dH2, md->err};
    Dev D{};
    k_mlp_fwd<<<(M + 127) / 128, 128, 0, md->stream>>>(a, D, 0);
    count_launch(1);
    return cudaGetLastError();
}

static cudaError_t backward(MlpModel* md, const float* dX, const float* dy, int M) {
    BwdArgs b{dX, dy, md->H1, md->H2, md->z, M, md->P, md->W2b, md->part, md->err};
    const int tiles = (M + 127) / 128;
    k_mlp_bwd<<<tiles, 128, BWD_SMEM, md->stream>>>(b);
    k_mlp_reduce<<<(NPARAMS + 1 + 255) / 256, 256, 0, md->stream>>>(md->part, tiles, md->g, md->loss);
    count_launch(2);
    return cudaGetLastError();
}

static cudaError_t init_mlp_attributes() {
    static std::once_flag once;
    static cudaError_t result = cudaSuccess;
    std::call_once(once, [] {
        result = cudaFuncSetAttribute(k_mlp_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)BWD_SMEM);
    });
    return result;
}

bool score_step_active(const Dev& D) { return D.learned || D.ftr_every > 0; }

cudaError_t launch_score(const Dev& D, cudaStream_t s) {
    const int grid = (D.m + 127) / 128;
    if (D.learned) {
        FwdArgs a{nullptr, D.m, (const __nv_bfloat16*)D.mlp_w1, (const __nv_bfloat16*)D.mlp_w2, D.mlp_p,
                  nullptr, nullptr, nullptr, D.mlp_err};
        cudaError_t e = launch_pdl(k_mlp_fwd, dim3(grid), dim3(128), 0, s, a, D, 1);
        if (e != cudaSuccess) return e;
    } else if (D.ftr_every > 0) {
        cudaError_t e = launch_pdl(k_features, dim3(grid), dim3(128), 0, s, D);
        if (e != cudaSuccess) return e;
    } else {
        return cudaSuccess;
    }
    count_launch(1);
    return cudaGetLastError();
}

void model_pointers(const MlpModel* md, const void** w1, const void** w2, const float** p, int** err) {
    *w1 = md->W1b; *w2 = md->W2b; *p = md->P; *err = md->err;
}
int model_device(const MlpModel* md) { return md->device; }

}  // namespace ds

using ds::MlpModel;

struct ds_model { MlpModel* md; };

MlpModel* ds_model_impl(ds_model* m) { return m->md; }

extern "C" {

int ds_model_create(int device, ds_model** out) {
    if (!out) return DS_ERR_ARG;
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) return DS_ERR_CUDA;
    if (ds::init_mlp_attributes() != cudaSuccess) return DS_ERR_CUDA;
    auto* md = new MlpModel();
    md->device = device;
    bool ok = cudaStreamCreateWithFlags(&md->stream, cudaStreamNonBlocking) == cudaSuccess;
    ok = ok && cudaMalloc(&md->P, ds::NPARAMS * sizeof(float)) == cudaSuccess;
    ok = ok && cudaMalloc(&md->m1, ds::NPARAMS * sizeof(float)) == cudaSuccess;
    ok = ok && cudaMalloc(&md->m2, ds::NPARAMS * sizeof(float)) == cudaSuccess;
    ok = ok && cudaMalloc(&md->g, ds::NPARAMS * sizeof(float)) == cudaSuccess;
    ok = ok && cudaMalloc(&md->loss, sizeof(float)) == cudaSuccess;
    ok = ok && cudaMalloc(&md->W1b, 64 * 16 * sizeof(__nv_bfloat16)) == cudaSuccess;
    ok = ok && cudaMalloc(&md->W2b, 64 * 64 * sizeof(__nv_bfloat16)) == cudaSuccess;
    ok = ok && cudaMalloc(&md->err, 2 * sizeof(int)) == cudaSuccess;   // [0] timeout flag, [1] test poll bound
    ok = ok && cudaMemsetAsync(md->P, 0, ds::NPARAMS * sizeof(float), md->stream) == cudaSuccess;
    ok = ok && cudaMemsetAsync(md->m1, 0, ds::NPARAMS * sizeof(float), md->stream) == cudaSuccess;
    ok = ok && cudaMemsetAsync(md->m2, 0, ds::NPARAMS * sizeof(float), md->stream) == cudaSuccess;
    ok = ok && cudaMemsetAsync(md->err, 0, 2 * sizeof(int), md->stream) == cudaSuccess;
    ok = ok && cudaMemsetAsync(md->W1b, 0, 64 * 16 * sizeof(__nv_bfloat16), md->stream) == cudaSuccess;
    ok = ok && cudaMemsetAsync(md->W2b, 0, 64 * 64 * sizeof(__nv_bfloat16), md->stream) == cudaSuccess;
    ok = ok && cudaStreamSynchronize(md->stream) == cudaSuccess;
    if (!ok) { delete md; return DS_ERR_CUDA; }
    *out = new ds_model{md};
    return DS_OK;
}

int ds_model_destroy(ds_model* m) {
    if (!m) return DS_ERR_ARG;
    delete m->md;
    delete m;
    return DS_OK;
}

int ds_model_set_wait_limit(ds_model* m, int polls) {
    if (!m || polls < 0) return DS_ERR_ARG;
    MlpModel* md = m->md;
    if (cudaSetDevice(md->device) != cudaSuccess) return DS_ERR_CUDA;
    const int v[2] = {0, polls};
    if (cudaMemcpyAsync(md->err, v, sizeof(v), cudaMemcpyHostToDevice, md->stream) != cudaSuccess) return DS_ERR_CUDA;
    return cudaStreamSynchronize(md->stream) == cudaSuccess ? DS_OK : DS_ERR_CUDA;
}

static int check_err(MlpModel* md) {
    int e = 0;
    if (cudaMemcpyAsync(&e, md->err, sizeof(int), cudaMemcpyDeviceToHost, md->stream) != cudaSuccess) return DS_ERR_CUDA;
    if (cudaStreamSynchronize(md->stream) != cudaSuccess) return DS_ERR_CUDA;
    return e ? DS_ERR_DEVICE_WAIT : DS_OK;
}

int ds_model_set_params(ds_model* m, const float* params, int count) {
    if (!m || !params || count != DS_MLP_NPARAMS) return DS_ERR_ARG;
    MlpModel* md = m->md;
    if (cudaSetDevice(md->device) != cudaSuccess) return DS_ERR_CUDA;
    if (cudaMemcpyAsync(md->P, params, sizeof(float) * count, cudaMemcpyHostToDevice, md->stream) != cudaSuccess)
        return DS_ERR_CUDA;
    cudaMemsetAsync(md->m1, 0, sizeof(float) * count, md->stream);
    cudaMemsetAsync(md->m2, 0, sizeof(float) * count, md->stream);
    md->step = 0;
    ds::k_mlp_to_bf16<<<(64 * 64 + 255) / 256, 256, 0, md->stream>>>(md->P, md->W1b, md->W2b);
    ds::count_launch(1);
    if (cudaGetLastError() != cudaSuccess) return DS_ERR_CUDA;
    return cudaStreamSynchronize(md->stream) == cudaSuccess ? DS_OK : DS_ERR_CUDA;
}

int ds_model_get_params(const ds_model* m, float* params, int count) {
    if (!m || !params || count != DS_MLP_NPARAMS) return DS_ERR_ARG;
    MlpModel* md = m->md;
    if (cudaSetDevice(md->device) != cudaSuccess) return DS_ERR_CUDA;
    if (cudaMemcpyAsync(params, md->P, sizeof(float) * count, cudaMemcpyDeviceToHost, md->stream) != cudaSuccess)
        return DS_ERR_CUDA;
    return cudaStreamSynchronize(md->stream) == cudaSuccess ? DS_OK : DS_ERR_CUDA;
}

int ds_model_forward(ds_model* m, const float* X, int rows, float* logits, float* H1, float* H2) {
    if (!m || !X || rows <= 0 || !logits) return DS_ERR_ARG;
    MlpModel* md = m->md;
    if (cudaSetDevice(md->device) != cudaSuccess) return DS_ERR_CUDA;
    if (!md->ensure(rows)) return DS_ERR_CUDA;
    if (cudaMemcpyAsync(md->X, X, sizeof(float) * ds::NF * rows, cudaMemcpyHostToDevice, md->stream) != cudaSuccess)
        return DS_ERR_CUDA;
    if (ds::forward(md, md->X, rows, md->z, md->H1, md->H2) != cudaSuccess) return DS_ERR_CUDA;
    cudaMemcpyAsync(logits, md->z, sizeof(float) * rows, cudaMemcpyDeviceToHost, md->stream);
    if (H1) cudaMemcpyAsync(H1, md->H1, sizeof(float) * 64 * rows, cudaMemcpyDeviceToHost, md->stream);
    if (H2) cudaMemcpyAsync(H2, md->H2, sizeof(float) * 64 * rows, cudaMemcpyDeviceToHost, md->stream);
    return check_err(md);
}

int ds_model_gradients(ds_model* m, const float* X, const float* y, int rows, float* grads, float* loss) {
    if (!m || !X || !y || rows <= 0 || !grads) return DS_ERR_ARG;
    MlpModel* md = m->md;
    if (cudaSetDevice(md->device) != cudaSuccess) return DS_ERR_CUDA;
    if (!md->ensure(rows)) return DS_ERR_CUDA;
    cudaMemcpyAsync(md->X, X, sizeof(float) * ds::NF * rows, cudaMemcpyHostToDevice, md->stream);
    cudaMemcpyAsync(md->y, y, sizeof(float) * rows, cudaMemcpyHostToDevice, md->stream);
    if (ds::forward(md, md->X, rows, md->z, md->H1, md->H2) != cudaSuccess) return DS_ERR_CUDA;
    if (ds::backward(md, md->X, md->y, rows) != cudaSuccess) return DS_ERR_CUDA;
    cudaMemcpyAsync(grads, md->g, sizeof(float) * ds::NPARAMS, cudaMemcpyDeviceToHost, md->stream);
    if (loss) cudaMemcpyAsync(loss, md->loss, sizeof(float), cudaMemcpyDeviceToHost, md->stream);
    return check_err(md);
}

int ds_model_train(ds_model* m, const float* X, const float* y, int rows, int epochs, int batch, float lr,
                   unsigned long long seed, float* mean_loss) {
    if (!m || !X || !y || rows <= 0 || epochs <= 0 || batch <= 0 || batch % 128 || batch > rows) return DS_ERR_ARG;
    MlpModel* md = m->md;
    if (cudaSetDevice(md->device) != cudaSuccess) return DS_ERR_CUDA;
    if (!md->ensure_all(rows) || !md->ensure(batch)) return DS_ERR_CUDA;
    cudaMemcpyAsync(md->Xall, X, sizeof(float) * ds::NF * rows, cudaMemcpyHostToDevice, md->stream);
    cudaMemcpyAsync(md->yall, y, sizeof(float) * rows, cudaMemcpyHostToDevice, md->stream);
    std::vector<int> perm(rows);
    uint64_t st = seed * 0x9E3779B97F4A7C15ull + 1;
    double lsum = 0.0;
    int nb = 0;
    for (int ep = 0; ep < epochs; ++ep) {
        for (int i = 0; i < rows; ++i) perm[i] = i;
        for (int i = rows - 1; i > 0; --i) {     // Fisher-Yates with a 64-bit LCG
            st = st * 6364136223846793005ull + 1442695040888963407ull;
            const int j = (int)((st >> 33) % (uint64_t)(i + 1));
            std::swap(perm[i], perm[j]);
        }
        if (cudaMemcpyAsync(md->idx, perm.data(), sizeof(int) * rows, cudaMemcpyHostToDevice, md->stream) != cudaSuccess)
            return DS_ERR_CUDA;
        std::vector<float> losses;
        for (int b0 = 0; b0 + batch <= rows; b0 += batch) {
            ds::k_gather_rows<<<(batch + 255) / 256, 256, 0, md->stream>>>(md->Xall, md->yall, md->idx + b0, batch,
                                                                         md->X, md->y);
            if (ds::forward(md, md->X, batch, md->z, md->H1, md->H2) != cudaSuccess) return DS_ERR_CUDA;
            if (ds::backward(md, md->X, md->y, batch) != cudaSuccess) return DS_ERR_CUDA;
            md->step += 1;
            ds::k_mlp_adam<<<(ds::NPARAMS + 255) / 256, 256, 0, md->stream>>>(md->P, md->m1, md->m2, md->g, lr, 0.9f,
                                                                             0.999f, 1e-8f, md->step, md->W1b, md->W2b);
            ds::count_launch(2);
            if (cudaGetLastError() != cudaSuccess) return DS_ERR_CUDA;
            if (ep == epochs - 1) {
                float l = 0.f;
                cudaMemcpyAsync(&l, md->loss, sizeof(float), cudaMemcpyDeviceToHost, md->stream);
                if (cudaStreamSynchronize(md->stream) != cudaSuccess) return DS_ERR_CUDA;
                losses.push_back(l);
            }
        }
        // the permutation buffer is reused by the next epoch's upload
        if (cudaStreamSynchronize(md->stream) != cudaSuccess) return DS_ERR_CUDA;
        if (ep == epochs - 1) for (float l : losses) { lsum += l; ++nb; }
    }
    if (mean_loss) *mean_loss = nb ? (float)(lsum / nb) : 0.f;
    return check_err(md);
}

}  // extern "C"
