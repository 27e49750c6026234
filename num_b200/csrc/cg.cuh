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
    bool graph_formed = false;  // the graph path's SpMV forms p (two kernels per iteration)
    int grid_spmv_f = 0;        // ... on this grid
    unsigned int* err = nullptr;  // device error word (not owned)
    cudaStream_t cap_stream = nullptr;
    std::map<int, cudaGraphExec_t> graphs;  // iterations per graph -> exec
    // the resident solve (cg_resident.cu), when the matrix qualifies
    bool resident = false;
    int32_t last_path = -1;  // path of the last solve (nm_cg_last_path)
    int res_tiles = 0, res_grid = 0, res_width = 0;
    size_t res_smem = 0;
    void* res_mem = nullptr;      // per-CTA row / window ranges and the sum slots
    int4* res_cta = nullptr;
    double* res_slots = nullptr;
    // the cluster solve (cg_cluster.cu), when the matrix qualifies
    bool cluster = false;
    int cl_rows_per_thread = 0, cl_width = 0, cl_class = 0, cl_halo = 0, cl_pmax = 0;
    bool cl_f32v = false;  // A's values held as floats (each a float exactly)
    size_t cl_smem = 0;
    void* cl_mem = nullptr;  // renumbered columns and the halo store lists
    uint16_t* cl_lcol = nullptr;
    int32_t* cl_push_off = nullptr;
    uint32_t* cl_push_ent = nullptr;
    ~CgWorkspace();
};

// The cluster solve: systems whose row blocks are whole 256-row tiles and
// whose rows fit the cluster's shared memory -- when every value is a float
// exactly, at most 65,536 rows of at most 5 nonzeros or 49,152 of 7 or 8;
// otherwise about 57,000 rows of at most 5 or 40,960 of 7 or 8 -- on one
// cluster of 16 CTAs when the device can schedule it.  NM_OK with
// ws->cluster false when it cannot.
int plan_cluster(const nm_csr* A, CgWorkspace* ws);
// One cluster solve on `s` after cg_init_kernel (ws->r, ws->p hold r0 = p0).
int launch_cluster(const nm_csr* A, CgWorkspace* ws, cudaStream_t s);

// The resident solve: systems of at most kResidentMaxRows rows whose row
// blocks are whole 256-row tiles, at most kResidentMaxTiles tiles per CTA,
// their rows of A and the window of the direction they multiply in at most
// kResidentMaxSmem bytes of shared memory per CTA.
constexpr int64_t kResidentMaxRows = 262144;
constexpr int kResidentMaxTiles = 8;
constexpr size_t kResidentMaxSmem = 200 * 1024;
// Decides whether A's solve can run resident and, if so, sets up ws (host
// work once per workspace).  NM_OK with ws->resident false when it cannot.
int plan_resident(const nm_csr* A, CgWorkspace* ws);
// One resident solve on `s` after cg_init_kernel (ws->r, ws->p hold r0 = p0).
int launch_resident(const nm_csr* A, CgWorkspace* ws, cudaStream_t s);

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

// Sum over the first 8 warps (256 threads) of the CTA: a shuffle tree per warp,
// then the warp sums added in warp order from 0.0 -- the order block_sum gives
// a 256-thread CTA.  Valid in thread 0; every thread of the CTA calls it.
__device__ __forceinline__ double block_sum8(double v, double* scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_sum(v);
    if (lane == 0 && warp < kWarps) scratch[warp] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int w = 0; w < kWarps; ++w) s += scratch[w];
    }
    __syncthreads();
    return s;
}

// The fixed order of every CG dot product.  Products are first summed per
// unit -- a row block for p.Ap (thread rows one per thread, a shuffle tree per
// warp, the eight warp sums in warp order), a 256-row tile for r.r and the
// initial norms (the same tree over the tile's 256 elements) -- and the unit
// sums are then added here: thread t < 256 adds part[t], part[t + 256], ...
// from 0.0 and block_sum8 combines the 256 sums.  The partition alone fixes
// the order, not the grid, so the CUDA-graph path, the persistent solve and
// the resident solve give the same bits.  Valid in thread 0; every thread of
// the CTA (blockDim >= 256) calls it.
__device__ __forceinline__ double reduce256(const double* part, int64_t count, double* scratch) {
    double s = 0.0;
    const int t = threadIdx.x;
    if (t < kThreads) {
        int64_t i = t;
        for (; i + 3 * kThreads < count; i += 4 * kThreads) {
            const double a = __ldcg(part + i), b = __ldcg(part + i + kThreads),
                         c = __ldcg(part + i + 2 * kThreads), d = __ldcg(part + i + 3 * kThreads);
            s += a;
            s += b;
            s += c;
            s += d;
        }
        for (; i < count; i += kThreads) s += __ldcg(part + i);
    }
    return block_sum8(s, scratch);
}

// Grid barrier on (count, gen) for `expected` arriving CTAs (0: the whole
// grid, every CTA resident); returns false when the wait gave up (after
// limit_ns, which only the failure-detection test kernels lower) or a CTA has
// marked the solve failed (*status == kCgDeviceError) -- read once, by
// thread 0, so every thread of the CTA gets the same answer.
__device__ __forceinline__ bool grid_barrier(unsigned int* count, unsigned int* gen,
                                             unsigned int* err, const int32_t* status,
                                             bool* flag, unsigned int expected = 0,
                                             uint64_t limit_ns = kWaitLimitNs) {
    if (expected == 0) expected = gridDim.x;
    __syncthreads();
    if (threadIdx.x == 0) {
        bool ok = true;
        // Arrival is an acq_rel add on count (a release sequence: the last
        // arriver acquires every CTA's writes); it resets count and releases
        // gen, on which the others spin with acquire loads.
        unsigned int g0, prev;
        asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(g0) : "l"(gen) : "memory");
        asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;"
                     : "=r"(prev) : "l"(count) : "memory");
        if (prev == expected - 1) {
            asm volatile("st.relaxed.gpu.global.u32 [%0], 0;" ::"l"(count) : "memory");
            asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(gen) : "memory");
        } else {
            const uint64_t t0 = global_timer_ns();
            for (uint32_t it = 0;; ++it) {
                unsigned int g;
                asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(g) : "l"(gen) : "memory");
                if (g != g0) break;
                if ((it & 255u) == 0 && (global_timer_ns() - t0 > limit_ns || it > (1u << 30))) {
                    atomicOr(err, kErrWaitTimeout);
                    ok = false;
                    break;
                }
            }
        }
        *flag = ok && __ldcg(status) != kCgDeviceError;
    }
    __syncthreads();
    return *flag;
}

}  // namespace nm
