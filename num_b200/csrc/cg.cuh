// cg.cuh -- device-resident CG state and the per-matrix CG workspace.
#pragma once

#include <map>

#include "csr.cuh"

namespace nm {

// Scalars of one CG solve, resident in device memory.  The host writes the
// inputs before a solve and reads the outputs after it; in between every
// scalar step (alpha, beta, the stopping test) runs on the device, in the last
// CTA of the reduction that produces its input.
struct CgState {
    // inputs
    const double* b;
    double* x;
    double tol;
    int32_t max_iter;
    int32_t guard;  // 1: reject |p.Ap| < 1e-300 (cg_solve_distributed)
    // scalars
    double bnorm, rr, pAp, alpha, beta, final_res;
    int32_t iter, done, converged, iters, status;
    unsigned int counter;  // arrival counter of the last-CTA reductions
    unsigned int bar_count, bar_gen;  // grid barrier of the persistent solve
};

// Status codes written to CgState::status.
constexpr int kCgOk = 0;
constexpr int kCgBreakdown = 1;
constexpr int kCgDeviceError = 2;

struct CgWorkspace {
    int64_t n = 0;
    bool coop = false;  // the persistent cooperative solve fits this matrix's SpMV grid
    bool coop_formed = false;  // ... in its two-barrier form (p formed inside the SpMV)
    double* r = nullptr;
    double* p = nullptr;
    double* p2 = nullptr;  // second p buffer of the two-barrier persistent solve
    double* Ap = nullptr;
    double* partials = nullptr;
    int partials_cap = 0;
    CgState* st = nullptr;
    void* dmem = nullptr;       // one device allocation holding r, p, p2, Ap, partials, st
    CgState* h_in = nullptr;    // pinned staging of the inputs (a slot of a shared slab)
    CgState* h_out = nullptr;   // pinned landing of the outputs (idem)
    int grid_spmv = 0, grid_vec = 0;
    unsigned int* err = nullptr;  // device error word (not owned)
    cudaStream_t cap_stream = nullptr;
    std::map<int, cudaGraphExec_t> graphs;  // iterations per graph -> exec
    ~CgWorkspace();
};

// Grid of the grid-stride vector kernels for n elements.
int vec_grid(int64_t n);

// Last-CTA grid reduction: every CTA passes K partial sums (valid in thread 0;
// `red` has one entry per warp of the CTA);
// returns true on thread 0 of the CTA that arrives last, with the grid totals
// summed in a fixed order (so results are bit-reproducible for a fixed grid).
// The counter is reset for the next launch.  Call from all threads.
template <int K>
__device__ __forceinline__ bool grid_reduce_last(const double (&part)[K], double* partials,
                                                 unsigned int* counter, double (&tot)[K],
                                                 double* red) {
    __shared__ bool am_last;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) partials[size_t(k) * gridDim.x + blockIdx.x] = part[k];
        __threadfence();
        const unsigned int prev = atomicAdd(counter, 1u);
        am_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (!am_last) return false;
    __threadfence();
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double s = 0.0;
        for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x)
            s += __ldcg(partials + size_t(k) * gridDim.x + i);
        tot[k] = block_sum(s, red);
    }
    if (threadIdx.x == 0) *counter = 0u;
    return threadIdx.x == 0;
}

}  // namespace nm
