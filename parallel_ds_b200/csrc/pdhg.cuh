// First-order (PDHG) estimate of an optimal primal-dual pair (pdhg.cu).
#pragma once
#include <cuda_runtime.h>

namespace ds {

struct PdhgDev {
    int m, n, R;                                       // R: restart period
    const int* cptr; const int* crow; const double* cval;   // structural CSC
    const int* rptr; const int* rcol; const double* rval;   // structural CSR
    const double* c;                                   // n costs (unperturbed)
    const double* lo; const double* hi;                // n column bounds (+-inf where absent)
    const double* L; const double* U;                  // m row activity bounds
    const double* tau; const double* sigma;            // n, m step sizes
    double* x; double* xbar; double* xsum;             // n
    double* y; double* ysum;                           // m
};

cudaError_t launch_pdhg_init(const PdhgDev& P, cudaStream_t s);
cudaError_t launch_pdhg_period(const PdhgDev& P, cudaStream_t s);
// After the last period: x <- its running average (the pending restart).
cudaError_t launch_pdhg_finish(const PdhgDev& P, cudaStream_t s);
cudaError_t launch_pdhg_evidence(const PdhgDev& P, float* gap, float* dual, cudaStream_t s);

// One-cluster PDHG (16 CTAs, the LP's slices in shared memory): geometry from the
// host CSC/CSR pointers (CL == 0 when the LP does not fit), and the launch of
// `periods` restart periods followed by the pending restart of x; returns false
// without launching when the cluster cannot be placed.
struct PdhgClusterGeom {
    int CL, nc, nr, nzc_cap, nzr_cap;
    size_t smem;
};
PdhgClusterGeom pdhg_cluster_geometry(int m, int n, const int* cptr, const int* rptr);
bool launch_pdhg_cluster(const PdhgDev& P, const PdhgClusterGeom& G, int periods, cudaStream_t s);

}  // namespace ds
