// Host-side helpers shared by the engine's translation units: the error type
// that carries a ds status code, the CUDA call check, and stream-ordered device
// buffers.
#pragma once
#include <algorithm>
#include <stdexcept>
#include <string>

#include <cuda_runtime.h>

#include "../../include/ds_api.h"

namespace ds {

struct CudaError : std::runtime_error {
    int code;
    CudaError(const std::string& s, int c) : std::runtime_error(s), code(c) {}
};

#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            throw CudaError(std::string(#call) + ": " + cudaGetErrorString(e_), DS_ERR_CUDA); \
    } while (0)

template <typename T>
struct DBuf {
    // Stream-ordered device buffer.  A reallocation frees the old block in the
    // owning stream's order (work already queued there that reads it finishes
    // first) without the device-wide synchronisation of cudaFree, so solver
    // handles growing their buffers do not stall one another; growth is
    // geometric, so a solve whose factor grows reallocates a few times only.
    T* p = nullptr;
    size_t n = 0;
    cudaStream_t s = nullptr;
    void alloc(cudaStream_t st, size_t count) {
        release();
        if (count == 0) count = 1;
        CK(cudaMallocAsync(&p, count * sizeof(T), st));
        n = count;
        s = st;
    }
    void ensure(cudaStream_t st, size_t count) { if (count > n) alloc(st, std::max(count, n + n / 2)); }
    void release() { if (p) cudaFreeAsync(p, s); p = nullptr; n = 0; }
    ~DBuf() { if (p) cudaFree(p); }      // handle teardown: its stream may already be gone
};

}  // namespace ds
