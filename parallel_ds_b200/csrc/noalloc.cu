// CHUZC ratio test that allocates no device memory.
//
// Some callers of this library cannot call cudaMalloc: code that runs while a
// host framework owns every byte of device memory through its own pool (a
// stray cudaMalloc breaks its accounting and can fail under its memory cap),
// and code on a latency-critical path where cudaMalloc / cudaFree would stall
// the device.  ds_kernel_ratio_test_noalloc runs the same ratio-test kernel as
// ds_kernel_ratio_test on device arrays the caller already owns, and keeps its
// own scratch (candidate thetas and flags, per-block counts, the control block)
// in the file-scope array below, which every GPU that loads the library holds
// until the process exits.  The call copies its result to the host and
// synchronises its stream, so it is not for host functions queued on a stream
// (they may make no CUDA calls).  The device address of the array is looked up
// once per device and kept; a device reset (cudaDeviceReset) makes it stale, so
// the entry point is not for processes that reset the device.
#include <cstring>
#include <mutex>

#include "../../include/ds_api.h"
#include "engine.cuh"
#include "kernels.cuh"

namespace {

using namespace ds;

constexpr int kMaxSlots = DS_NOALLOC_MAX_SLOTS;
constexpr int kBlocks = (kMaxSlots + 255) / 256;
constexpr size_t align256(size_t b) { return (b + 255) & ~size_t(255); }
constexpr size_t kOffCtl = 0;
constexpr size_t kOffTheta = align256(sizeof(Ctl));
constexpr size_t kOffRed = kOffTheta + align256(sizeof(double) * kMaxSlots);
constexpr size_t kOffRedi = kOffRed + align256(sizeof(double) * 2 * (kBlocks + 8));
constexpr size_t kOffCand = kOffRedi + align256(sizeof(int) * 2 * (kBlocks + 8));
constexpr size_t kScratchBytes = kOffCand + align256(kMaxSlots);

// Shared by every call on a device; holds the last call's contents.
static __device__ __align__(256) unsigned char g_rt_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char* g_scratch_ptr[kMaxDevices] = {};   // device address of g_rt_scratch per device

// Device address of the scratch array on the current device (set up once per
// device, with that device current).
int scratch_for_current_device(unsigned char** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return DS_ERR_CUDA;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_rt_scratch) != cudaSuccess || !p) return DS_ERR_CUDA;
        g_scratch_ptr[dev] = (unsigned char*)p;
    }
    *out = g_scratch_ptr[dev];
    return DS_OK;
}

}  // namespace

extern "C" int ds_kernel_ratio_test_noalloc(int n, int N, const int* nonbasis, const double* alpha,
                                            double delta, int is_lower, const double* x, const double* d,
                                            const double* lb, const double* ub, const unsigned char* type,
                                            int* q, int* q_idx, double* theta, double* delta_out,
                                            int* num_candidates, void* stream) {
    if (n <= 0 || N < n || !nonbasis || !alpha || !x || !d || !lb || !ub || !type || !q || !q_idx ||
        !theta || !delta_out || !num_candidates)
        return DS_ERR_ARG;
    if (n > kMaxSlots) return DS_ERR_CAPACITY;   // more nonbasic slots than the scratch holds
    unsigned char* base = nullptr;
    int rc = scratch_for_current_device(&base);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;

    // the control block starts from zero every call: tickets, counters, results
    Ctl h;
    std::memset(&h, 0, sizeof(h));
    h.phase = 2; h.ybt_n = -1; h.prev_q = -1; h.max_iter = 1 << 30; h.R = 100; h.top_done = 1;
    h.delta = delta; h.is_lower = is_lower ? 1 : 0;
    Ctl* dctl = (Ctl*)(base + kOffCtl);
    if (cudaMemcpyAsync(dctl, &h, sizeof(Ctl), cudaMemcpyHostToDevice, s) != cudaSuccess) return DS_ERR_CUDA;

    Dev D{};
    D.n = n; D.N = N; D.m = N - n;
    D.nonbasis = const_cast<int*>(nonbasis);
    D.alpha = const_cast<double*>(alpha);
    D.x = const_cast<double*>(x); D.d = const_cast<double*>(d);
    D.lb = lb; D.ub = ub; D.type = type;
    D.theta_arr = (double*)(base + kOffTheta);
    D.red = (double*)(base + kOffRed);
    D.redi = (int*)(base + kOffRedi);
    D.cand = base + kOffCand;
    D.ctl = dctl;
    if (launch_pivot_row_mode(D, 2, s) != cudaSuccess) return DS_ERR_CUDA;
    if (cudaMemcpyAsync(&h, dctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s) != cudaSuccess) return DS_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return DS_ERR_CUDA;
    *num_candidates = h.ncand;
    if (h.event == EV_UNBOUNDED || h.event == EV_ERROR || h.ncand == 0) {
        *q = -1; *q_idx = -1; *theta = 0.0;
        *delta_out = (is_lower ? -1.0 : 1.0) * (delta < 0 ? -delta : delta);
        return DS_OK;
    }
    *q = h.q; *q_idx = h.q_idx; *theta = h.theta; *delta_out = h.delta_bfrt;
    return DS_OK;
}
