// solver.cu -- batched, mixed-precision, continuously batched PCG engine.
//
// No counterpart in the reference (its CG solves one system at a time, in
// FP64, without a preconditioner, src/cg_solver.hpp:133-196).  Design:
//
// * Arena.  Every admitted system lives in one device arena: row-indexed
//   vectors (b, x, r64 in FP64; p, Ap, r, z, d, Jacobi inverse diagonal in the
//   inner precision T) and nonzero-indexed CSR arrays (column indices stored
//   as arena rows, FP64 values for the outer residual, inner-precision values
//   for the inner iterations).  The active systems therefore form one
//   block-diagonal matrix, and the pipelined SpMV kernel of spmv.cuh runs over
//   a list of the active systems' row blocks.  Admission takes first-fit
//   ranges of rows and nonzeros and fails (NM_ERR_NOMEM) when the arena is
//   full: admission by free device memory.
//
// * Lockstep iterations.  Every inner iteration advances all active systems
//   with per-system scalars:  SpMV + per-warp partials of p.Ap  ->  per-system
//   alpha  ->  d += alpha p, r -= alpha Ap, z = M^-1 r, partials of r.z and
//   r.r  ->  per-system beta and inner stopping test  ->  p = z + beta p.
//   Systems that stop are gated out of the SpMV and skipped by the vector
//   kernels; all grids are persistent, list lengths are read from device
//   memory.
//
// * Mixed precision with iterative refinement.  The inner Jacobi-PCG runs in
//   T = float (values float or bf16, FP32 accumulation) on the scaled
//   residual system A d = r64 / |r64|; an outer step (x += d |r64|,
//   r64 = b - A x with FP64 values, fused into the FP64 SpMV's epilogue,
//   |r64| / |b|) runs between chunks for systems whose inner solve stopped,
//   until |b - A x| / |b| < tol.  From the second outer step on, the inner
//   solve continues the previous Krylov direction instead of restarting
//   ("reliable update": the true residual replaces the recurred one, p = z +
//   gamma p), so refinement costs few extra iterations.  With T = double the
//   same machinery is a plain FP64 PCG (the inner test is the final one).
//
// * Continuous batching.  nm_solver_step runs the pending outer steps, then a
//   chunk of inner iterations, then reads every system's state; the host
//   admits new systems and retires finished ones between steps.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "cg.cuh"
#include "spmv.cuh"

namespace nm {

enum SysPhase : int32_t { kSysFree = 0, kSysOuter = 1, kSysInner = 2, kSysDone = 3 };

struct SysState {
    // set at admission
    int32_t row0, n, max_iter, max_outer;
    double tol, bnorm, inner_rtol, stop_frac, cont_window;
    // dynamic
    int32_t phase, it_total, it_inner, outer;
    int32_t converged, pad_;
    double rnorm, rr0, rr, alpha, beta, final_res;
    double rzp[2];      // r.z of the current inner iteration, alternating by iteration parity
    double rnorm_prev;  // scale of the previous inner solve
    double rz_keep;     // r.z of the last completed iteration of the previous inner solve
    double gamma;       // p = z + gamma p at an inner start (0: fresh start)
    unsigned int tile_arrivals;  // large systems: tile CTAs of bs_update done this iteration
    unsigned int pad2_;
};

struct SysRef {
    int32_t slot, blk0, blk1, tile0, tile1, pad_[3];
};

// Counts of the device-side work lists (bsys: the large systems of the inner
// list, whose scalars one CTA per system reduces).
struct ListHdr {
    int32_t iblk, itile, isys, oblk, otile, osys, bsys, pad_;
};

// Control words of a step's device-side loop: the iterations done so far in
// this step, systems still iterating after the loop body's last iteration,
// and the step's iteration cap.  The body is kLoopUnroll iterations (an even
// number, so the r.z parity of each iteration is fixed in the body).
struct StepCtl {
    unsigned int iter, live, cap, pad_;
    // the persistent step (bs_persist): its grid barrier, the systems still
    // iterating after each iteration (alternating by iteration parity), and
    // its failure flag
    unsigned int bar_count, bar_gen, live2[2];
    int32_t status, pad2_[3];
};


constexpr int kTileRows = 4096;  // rows per vector-kernel tile (within one system)

// A system is "large" when re-reducing its block sums in every tile CTA would
// cost more than a couple of loads per thread: its alpha and beta are then
// reduced once -- alpha by one CTA (bs_alpha), beta by the last of its tile
// CTAs in bs_update -- and the tile kernels read them.  Tiles of a large system carry w = 1.  The choice depends only on the
// system's own size, so a system takes the same path alone and in any mix.
constexpr int kLargeBlocks = 512;
constexpr int kLargeTiles = 256;

__device__ __forceinline__ int32_t sys_phase(const SysState* sys, int32_t slot) {
    return __ldcg(&sys[slot].phase);
}

// ---- SpMV epilogues / gates ---------------------------------------------------

// Ap = A p; per row block, the sum of p.Ap over its rows goes to part[b] (the
// block's consumer warps' sums, added in warp order by the producer warp).
template <typename T>
struct InnerEpi {
    static constexpr bool kBlockSums = true;
    T* __restrict__ Ap;
    const T* __restrict__ p;
    double* __restrict__ part;
    T acc;
    __device__ __forceinline__ void operator()(int32_t row, T v) {
        Ap[row] = v;
        acc += __ldg(p + row) * v;
    }
    __device__ __forceinline__ double take() {
        const double a = double(acc);
        acc = T(0);
        return a;
    }
    __device__ __forceinline__ void finish_block(int64_t b, const BlockDesc&, double sum) {
        part[b] = sum;
    }
};

struct OuterEpi {  // r64 = b - A x; per row block, the sum of r64.r64 -> part[b]
    static constexpr bool kBlockSums = true;
    double* __restrict__ r64;
    const double* __restrict__ b;
    double* __restrict__ part;
    double acc;
    __device__ __forceinline__ void operator()(int32_t row, double v) {
        const double r = __ldg(b + row) - v;
        r64[row] = r;
        acc = fma(r, r, acc);
    }
    __device__ __forceinline__ double take() {
        const double a = acc;
        acc = 0.0;
        return a;
    }
    __device__ __forceinline__ void finish_block(int64_t bb, const BlockDesc&, double sum) {
        part[bb] = sum;
    }
};

struct PhaseGate {  // only blocks of systems in the given phase
    const SysState* sys;
    int32_t phase;
    __device__ __forceinline__ bool operator()(const BlockDesc& d) const {
        return sys_phase(sys, d.aux.y) == phase;
    }
};

constexpr int kSolverTile = 2048;
constexpr int kSolverStages = 2;

template <typename V, typename T>
__global__ void __launch_bounds__(kCtaThreads)
    bs_spmv_inner(CsrView<V> M, const T* __restrict__ p, T* __restrict__ Ap, const SysState* sys,
                  double* part, unsigned int* err) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    auto& sm = *reinterpret_cast<SpmvSmem<V, T, T, kSolverTile, kSolverStages>*>(smem_raw);
    InnerEpi<T> epi{Ap, p, part, T(0)};
    spmv_pipeline<V, T, T, kSolverTile, kSolverStages>(M, p, sm, epi, err,
                                                       PhaseGate{sys, kSysInner});
}

__global__ void __launch_bounds__(kCtaThreads)
    bs_spmv_outer(CsrView<double> M, const double* __restrict__ x, const double* __restrict__ b,
                  double* __restrict__ r64, const SysState* sys, double* part, unsigned int* err) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    auto& sm =
        *reinterpret_cast<SpmvSmem<double, double, double, kSolverTile, kSolverStages>*>(smem_raw);
    OuterEpi epi{r64, b, part, 0.0};
    spmv_pipeline<double, double, double, kSolverTile, kSolverStages>(M, x, sm, epi, err,
                                                                      PhaseGate{sys, kSysOuter});
}

// ---- fixed-order reductions ---------------------------------------------------------

// CTA-wide sums of two values in a fixed order (shuffle tree per warp, warps
// in order), returned to every thread.  scratch: one entry per warp plus one
// for the result (which no warp slot overlaps, so back-to-back calls need no
// third barrier).
__device__ __forceinline__ double2 block_sum2_all(double a, double b, double2* scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = static_cast<int>(blockDim.x) >> 5;
    a = warp_sum(a);
    b = warp_sum(b);
    if (lane == 0) scratch[warp] = make_double2(a, b);
    __syncthreads();
    if (threadIdx.x == 0) {
        double2 t = make_double2(0.0, 0.0);
        for (int w = 0; w < nw; ++w) {
            t.x += scratch[w].x;
            t.y += scratch[w].y;
        }
        scratch[nw] = t;
    }
    __syncthreads();
    return scratch[nw];
}

// Sums of the pairs part[lo..hi) (as double2: .x and .y summed separately), or
// of single values when PAIRS is false (.y = 0), returned to every thread.
// Thread t owns the entries lo + t + k*blockDim (k = 0, 1, ...) and adds them
// into 8 accumulators by k % 8, combined as ((0+1)+(2+3))+((4+5)+(6+7)); then
// the CTA sum above.  The grouping depends only on the offset from lo, so a
// system's sums are the same bits wherever its entries sit and in every CTA
// that computes them.
template <bool PAIRS>
__device__ __forceinline__ double2 ordered_sum_all(const double* part, int64_t lo, int64_t hi,
                                                   double2* scratch) {
    double ax[8] = {0, 0, 0, 0, 0, 0, 0, 0}, ay[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const int64_t bs = blockDim.x;
    auto ld = [&](int64_t i) -> double2 {
        if (PAIRS) return __ldcg(reinterpret_cast<const double2*>(part) + i);
        return make_double2(__ldcg(part + i), 0.0);
    };
    int64_t i = lo + threadIdx.x;
    for (; i + 7 * bs < hi; i += 8 * bs) {
        double2 v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = ld(i + k * bs);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            ax[k] += v[k].x;
            ay[k] += v[k].y;
        }
    }
#pragma unroll
    for (int k = 0; k < 7; ++k) {  // the tail: fewer than 8 strides remain
        const int64_t j = i + k * bs;
        if (j < hi) {
            const double2 v = ld(j);
            ax[k] += v.x;
            ay[k] += v.y;
        }
    }
    const double sx = ((ax[0] + ax[1]) + (ax[2] + ax[3])) + ((ax[4] + ax[5]) + (ax[6] + ax[7]));
    const double sy = ((ay[0] + ay[1]) + (ay[2] + ay[3])) + ((ay[4] + ay[5]) + (ay[6] + ay[7]));
    return block_sum2_all(sx, sy, scratch);
}

// The per-system sums of the inner iteration (alpha's p.Ap, beta's r.z and
// r.r) in one order for every path: ordered_sum_all as a CTA of 256 threads
// computes it.  Threads 256 and up (the producer warp of a persistent CTA)
// add nothing; every thread of the CTA calls it and gets the result.
// scratch: kWarps + 1 entries.
template <bool PAIRS>
__device__ __forceinline__ double2 ordered_sum256(const double* part, int64_t lo, int64_t hi,
                                                  double2* scratch) {
    double ax[8] = {0, 0, 0, 0, 0, 0, 0, 0}, ay[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    constexpr int64_t bs = kThreads;
    auto ld = [&](int64_t i) -> double2 {
        if (PAIRS) return __ldcg(reinterpret_cast<const double2*>(part) + i);
        return make_double2(__ldcg(part + i), 0.0);
    };
    if (threadIdx.x < kThreads) {
        int64_t i = lo + threadIdx.x;
        for (; i + 7 * bs < hi; i += 8 * bs) {
            double2 v[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) v[k] = ld(i + k * bs);
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                ax[k] += v[k].x;
                ay[k] += v[k].y;
            }
        }
#pragma unroll
        for (int k = 0; k < 7; ++k) {
            const int64_t j = i + k * bs;
            if (j < hi) {
                const double2 v = ld(j);
                ax[k] += v.x;
                ay[k] += v.y;
            }
        }
    }
    double sx = ((ax[0] + ax[1]) + (ax[2] + ax[3])) + ((ax[4] + ax[5]) + (ax[6] + ax[7]));
    double sy = ((ay[0] + ay[1]) + (ay[2] + ay[3])) + ((ay[4] + ay[5]) + (ay[6] + ay[7]));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    sx = warp_sum(sx);
    sy = warp_sum(sy);
    if (lane == 0 && warp < kWarps) scratch[warp] = make_double2(sx, sy);
    __syncthreads();
    if (threadIdx.x == 0) {
        double2 t = make_double2(0.0, 0.0);
        for (int w = 0; w < kWarps; ++w) {
            t.x += scratch[w].x;
            t.y += scratch[w].y;
        }
        scratch[kWarps] = t;
    }
    __syncthreads();
    const double2 out = scratch[kWarps];
    __syncthreads();  // scratch is free for the next call
    return out;
}

// ordered_sum256 computed by a CTA of 1024 threads, the same bits: thread
// t + 256 g (g < 4) forms accumulators 2g and 2g + 1 of ordered_sum256's
// thread t -- the entries lo + t + 256 (8 m + k) in increasing m, as there --
// so the loads go out in one round instead of one round per 8 entries; the
// accumulators then meet in shared memory (acc: 8 x 256 entries) and thread
// t < 256 combines its eight in ordered_sum256's tree, then its warp and
// warp order.  Every thread calls it and gets the result.
template <bool PAIRS>
__device__ __forceinline__ double2 ordered_sum256_wide(const double* part, int64_t lo,
                                                       int64_t hi, double2 (*acc)[kThreads],
                                                       double2* scratch) {
    const int t = threadIdx.x & (kThreads - 1), g = threadIdx.x / kThreads;
    auto ld = [&](int64_t i) -> double2 {
        if (PAIRS) return __ldcg(reinterpret_cast<const double2*>(part) + i);
        return make_double2(__ldcg(part + i), 0.0);
    };
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int k = 2 * g + h;
        double ax = 0.0, ay = 0.0;
        // accumulator k's entries in increasing m, eight loads at a time
        constexpr int64_t kStride = 8 * int64_t(kThreads);
        for (int64_t e = lo + t + int64_t(kThreads) * k; e < hi; e += 8 * kStride) {
            double2 v[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int64_t j = e + q * kStride;
                v[q] = j < hi ? ld(j) : make_double2(0.0, 0.0);
            }
#pragma unroll
            for (int q = 0; q < 8; ++q)
                if (e + q * kStride < hi) {
                    ax += v[q].x;
                    ay += v[q].y;
                }
        }
        acc[k][t] = make_double2(ax, ay);
    }
    __syncthreads();
    double sx = 0.0, sy = 0.0;
    if (threadIdx.x < kThreads) {
        double a[8], b[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            a[k] = acc[k][t].x;
            b[k] = acc[k][t].y;
        }
        sx = ((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7]));
        sy = ((b[0] + b[1]) + (b[2] + b[3])) + ((b[4] + b[5]) + (b[6] + b[7]));
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    sx = warp_sum(sx);
    sy = warp_sum(sy);
    if (lane == 0 && warp < kWarps) scratch[warp] = make_double2(sx, sy);
    __syncthreads();
    if (threadIdx.x == 0) {
        double2 tt = make_double2(0.0, 0.0);
        for (int w = 0; w < kWarps; ++w) {
            tt.x += scratch[w].x;
            tt.y += scratch[w].y;
        }
        scratch[kWarps] = tt;
    }
    __syncthreads();
    const double2 out = scratch[kWarps];
    __syncthreads();  // scratch and acc are free for the next call
    return out;
}

// ---- per-system scalar steps (one CTA per system of the outer list) ----------------

enum ScalarKind { kOuterNorm = 2, kStart = 3 };

constexpr int kScalarThreads = 1024;

template <int KIND>
__global__ void __launch_bounds__(kScalarThreads)
    bs_scalar(const SysRef* list, const int32_t* count, SysState* sys, const double* part_blk,
              const double* part_tile) {
    __shared__ double2 red[kScalarThreads / 32 + 1];
    const int32_t n = __ldcg(count);
    for (int32_t i = blockIdx.x; i < n; i += gridDim.x) {
        const SysRef ref = list[i];
        SysState& S = sys[ref.slot];
        const int32_t ph = __ldcg(&S.phase);
        if (ph != kSysOuter) continue;  // uniform over the CTA
        if (KIND == kOuterNorm) {
            const double rr = ordered_sum_all<false>(part_blk, ref.blk0, ref.blk1, red).x;
            if (threadIdx.x == 0) {
                const double rnorm = sqrt(rr);
                const double res = rnorm / S.bnorm;
                S.rnorm_prev = S.rnorm;
                S.rnorm = rnorm;
                S.final_res = res;
                if (res < S.tol) {
                    S.phase = kSysDone;
                    S.converged = 1;
                } else if (S.outer >= S.max_outer || S.it_total >= S.max_iter) {
                    S.phase = kSysDone;
                    S.converged = 0;
                } else {
                    S.outer += 1;  // stays kSysOuter until the inner start below
                }
            }
        } else {  // kStart
            const double2 t = ordered_sum_all<true>(part_tile, ref.tile0, ref.tile1, red);
            if (threadIdx.x == 0) {
                // Reliable update: after the first inner solve the Krylov
                // direction is kept -- the true residual replaces the recurred
                // one and the CG step continues with p = z + gamma p, gamma =
                // beta of unscaled CG times the scale change (s_new / s_old):
                // (s_new / s_old) (r.z)_new / (r.z)_last.  Only while the
                // recurrence still tracks the true residual (the new |b - Ax|
                // within a factor cont_window, 2 by default, of the inner
                // solve's estimate rnorm_prev |r|);
                // when it does not (low-precision values, ill conditioning)
                // the inner solve restarts from p = z.
                const double est = S.rnorm_prev * sqrt(S.rr);
                const bool cont = S.outer >= 2 && S.rz_keep > 0.0 && S.rnorm_prev > 0.0 &&
                                  t.x > 0.0 && est > 0.0 && S.rnorm <= S.cont_window * est &&
                                  S.rnorm * S.cont_window >= est;
                S.gamma = cont ? (S.rnorm / S.rnorm_prev) * (t.x / S.rz_keep) : 0.0;
                S.rzp[0] = t.x;
                S.rzp[1] = t.x;
                S.rr0 = t.y > 0.0 ? t.y : 1.0;
                S.rr = t.y;
                S.it_inner = 0;
                S.phase = kSysInner;
            }
        }
        __syncthreads();  // red is reused by the next system
    }
}

// Large systems, inner iteration: alpha = r.z / p.Ap from the block sums
// (after the SpMV), and the stopping test and beta from the tile sums (after
// the update), one CTA per system; the same formulas as the tile kernels use
// for small systems.
// (1024-thread CTAs forming the sums every path forms, ordered_sum256.)
constexpr int kWideThreads = 4 * kThreads;

__global__ void __launch_bounds__(kWideThreads)
    bs_alpha(const SysRef* list, const int32_t* count, SysState* sys, const double* part_blk,
             int par) {
    __shared__ double2 red[kWarps + 1];
    __shared__ double2 acc[8][kThreads];
    const int32_t n = __ldcg(count);
    for (int32_t i = blockIdx.x; i < n; i += gridDim.x) {
        const SysRef ref = list[i];
        SysState& S = sys[ref.slot];
        if (__ldcg(&S.phase) != kSysInner) continue;  // uniform over the CTA
        const double pAp = ordered_sum256_wide<false>(part_blk, ref.blk0, ref.blk1, acc, red).x;
        if (threadIdx.x == 0) S.alpha = pAp != 0.0 ? __ldcg(&S.rzp[par]) / pAp : 0.0;
    }
}

// ---- per-row vector steps over tiles {row0, row1, slot} ----------------------------
//
// A tile is up to kTileRows consecutive rows of one system; tiles start on
// multiples of 4 rows (systems start on multiples of 4 and tiles are
// kTileRows apart).  Thread t handles the vectors of VN = 16 / sizeof(T)
// rows starting at row0 + VN*(t + k*blockDim).  A vector may reach past the
// system's last row into its own padding rows (each system owns at least one
// row beyond its end, rounded up to 4): those lanes are loaded but neither
// stored nor counted.

template <typename T>
struct Vec16;
template <>
struct Vec16<float> {
    using type = float4;
    static constexpr int N = 4;
};
template <>
struct Vec16<double> {
    using type = double2;
    static constexpr int N = 2;
};

template <typename T>
__device__ __forceinline__ void vload(const T* p, int64_t row, T (&v)[Vec16<T>::N]) {
    using VT = typename Vec16<T>::type;
    const VT q = *reinterpret_cast<const VT*>(p + row);
    memcpy(v, &q, sizeof q);
}

template <typename T>
__device__ __forceinline__ void vstore(T* p, int64_t row, const T (&v)[Vec16<T>::N], int valid) {
    using VT = typename Vec16<T>::type;
    constexpr int N = Vec16<T>::N;
    if (valid >= N) {
        VT q;
        memcpy(&q, v, sizeof q);
        *reinterpret_cast<VT*>(p + row) = q;
    } else {
#pragma unroll
        for (int e = 0; e < N; ++e)
            if (e < valid) p[row + e] = v[e];
    }
}

// x += d * rnorm (the inner solution solves A d = r64 / rnorm), before the outer SpMV.
template <typename T>
__global__ void __launch_bounds__(kThreads)
    bs_xupdate(const int4* tiles, const int32_t* count, const SysState* sys,
               const T* __restrict__ d, double* __restrict__ x) {
    const int32_t n = __ldcg(count);
    for (int32_t i = blockIdx.x; i < n; i += gridDim.x) {
        const int4 tl = tiles[i];
        if (sys_phase(sys, tl.z) != kSysOuter) continue;
        const double s = __ldcg(&sys[tl.z].rnorm);
        if (__ldcg(&sys[tl.z].outer) == 0) continue;  // first outer step: d is not a correction
        for (int32_t r = tl.x + threadIdx.x; r < tl.y; r += blockDim.x)
            x[r] = fma(double(d[r]), s, x[r]);
    }
}

// Start an inner solve: r = r64 / rnorm, z = M^-1 r, d = 0; partials (r.z,
// r.r).  p is set by bs_pstart once r.z is known.
template <typename T>
__global__ void __launch_bounds__(kThreads)
    bs_inner_start(const int4* tiles, const int32_t* count, const SysState* sys,
                   const double* __restrict__ r64, const T* __restrict__ dinv, T* __restrict__ r,
                   T* __restrict__ z, T* __restrict__ d, double* part) {
    __shared__ double2 red[kWarps + 1];
    const int32_t n = __ldcg(count);
    for (int32_t i = blockIdx.x; i < n; i += gridDim.x) {
        const int4 tl = tiles[i];
        T rz = T(0), rr = T(0);
        if (sys_phase(sys, tl.z) == kSysOuter) {
            const double rn = __ldcg(&sys[tl.z].rnorm);
            const double sc = rn > 0.0 ? 1.0 / rn : 1.0;
            for (int32_t row = tl.x + threadIdx.x; row < tl.y; row += blockDim.x) {
                const T ri = T(r64[row] * sc);
                const T zi = dinv[row] * ri;
                r[row] = ri;
                z[row] = zi;
                d[row] = T(0);
                rz += ri * zi;
                rr += ri * ri;
            }
        }
        const double2 t = block_sum2_all(double(rz), double(rr), red);
        if (threadIdx.x == 0) reinterpret_cast<double2*>(part)[i] = t;
    }
}

// Inner start, second half: p = z (fresh start) or p = z + gamma p (continued
// Krylov direction), for the systems the start just moved to the inner phase.
template <typename T>
__global__ void __launch_bounds__(kThreads)
    bs_pstart(const int4* tiles, const int32_t* count, const SysState* sys,
              const T* __restrict__ z, T* __restrict__ p) {
    const int32_t n = __ldcg(count);
    for (int32_t i = blockIdx.x; i < n; i += gridDim.x) {
        const int4 tl = tiles[i];
        if (sys_phase(sys, tl.z) != kSysInner) continue;
        const double g = __ldcg(&sys[tl.z].gamma);
        if (g == 0.0) {
            for (int32_t row = tl.x + threadIdx.x; row < tl.y; row += blockDim.x) p[row] = z[row];
        } else {
            const T gt = T(g);
            for (int32_t row = tl.x + threadIdx.x; row < tl.y; row += blockDim.x)
                p[row] = fma(gt, p[row], z[row]);
        }
    }
}

__host__ __device__ constexpr int kVecIters(int vn) { return kTileRows / (vn * kThreads); }

// Loads of the vector steps.  COH: the data may have been written earlier in
// the same launch (the persistent step), so it is read through L2
// (ld.global.cg), never from a possibly stale L1 line.
template <typename T, bool COH>
__device__ __forceinline__ void vload_c(const T* p, int64_t row, T (&v)[Vec16<T>::N]) {
    using VT = typename Vec16<T>::type;
    VT q;
    if constexpr (COH)
        q = __ldcg(reinterpret_cast<const VT*>(p + row));
    else
        q = *reinterpret_cast<const VT*>(p + row);
    memcpy(v, &q, sizeof q);
}

// Sums of two values over the first 8 warps (256 threads) in warp order, to
// every thread: block_sum2_all as a 256-thread CTA forms it.
__device__ __forceinline__ double2 block_sum2_8(double a, double b, double2* scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    a = warp_sum(a);
    b = warp_sum(b);
    if (lane == 0 && warp < kWarps) scratch[warp] = make_double2(a, b);
    __syncthreads();
    if (threadIdx.x == 0) {
        double2 t = make_double2(0.0, 0.0);
        for (int w = 0; w < kWarps; ++w) {
            t.x += scratch[w].x;
            t.y += scratch[w].y;
        }
        scratch[kWarps] = t;
    }
    __syncthreads();
    const double2 out = scratch[kWarps];
    __syncthreads();
    return out;
}

// Inner iteration, step 2 (after the SpMV), for tile i: alpha = r.z / p.Ap
// from the system's block sums (every CTA of the system sums them, in the same
// order), d += alpha p, r -= alpha Ap, z = M^-1 r, and the tile's (r.z, r.r)
// -> part.  The system's first tile counts the iteration.  No atomics: step 3
// reduces the tile sums.  Threads 0..255 of the CTA carry the tile; every
// thread calls it.  SELF: a large system's alpha is reduced here too, in the
// same order bs_alpha uses, instead of read from bs_alpha.
template <typename T, bool COH, bool SELF>
__device__ __forceinline__ void update_tile(int32_t i, const int4 tl, SysState* sys,
                                            const int2* sblk, const int2* stile,
                                            const double* part_blk, const T* __restrict__ p,
                                            const T* __restrict__ Ap, const T* __restrict__ dinv,
                                            T* __restrict__ r, T* __restrict__ z,
                                            T* __restrict__ d, double* part_tile, int par,
                                            double2* red) {
    constexpr int VN = Vec16<T>::N;
    constexpr int IT = kVecIters(VN);
    const int32_t slot = tl.z;
    const bool mine = threadIdx.x < kThreads;
    T rz = T(0), rr = T(0);
    if (sys_phase(sys, slot) == kSysInner) {  // phase is not written in this step
        double alpha_d;
        if (tl.w && !SELF) {  // large system: bs_alpha reduced it
            alpha_d = __ldcg(&sys[slot].alpha);
        } else {  // every CTA of the system sums its block sums in the same order
            const int2 br = __ldg(sblk + slot);
            const double pAp = ordered_sum256<false>(part_blk, br.x, br.y, red).x;
            const double rz_old = __ldcg(&sys[slot].rzp[par]);
            alpha_d = pAp != 0.0 ? rz_old / pAp : 0.0;
        }
        const T alpha = T(alpha_d);
        // vectors of each operand per thread in flight at a time (within 64
        // registers): two for FP32, one for FP64 -- and one in the persistent
        // step, whose CTAs also hold the SpMV pipeline's registers
        constexpr int KB = (sizeof(T) == 4 && !COH) ? (IT < 2 ? IT : 2) : 1;
#pragma unroll
        for (int k0 = 0; k0 < IT; k0 += KB) {
            T pv[KB][VN], av[KB][VN], rv[KB][VN], dv[KB][VN], mv[KB][VN];
#pragma unroll
            for (int k = 0; k < KB; ++k) {
                const int64_t row = tl.x + int64_t(VN) * (threadIdx.x + (k0 + k) * kThreads);
                if (mine && row < tl.y) {
                    vload_c<T, COH>(p, row, pv[k]);
                    vload_c<T, COH>(Ap, row, av[k]);
                    vload_c<T, COH>(r, row, rv[k]);
                    vload_c<T, COH>(d, row, dv[k]);
                    vload_c<T, false>(dinv, row, mv[k]);
                }
            }
#pragma unroll
            for (int k = 0; k < KB; ++k) {
                const int64_t row = tl.x + int64_t(VN) * (threadIdx.x + (k0 + k) * kThreads);
                if (mine && row < tl.y) {
                    const int valid = int(min(int64_t(VN), int64_t(tl.y) - row));
                    T zo[VN];
#pragma unroll
                    for (int e = 0; e < VN; ++e) {
                        dv[k][e] = fma(alpha, pv[k][e], dv[k][e]);
                        rv[k][e] = fma(-alpha, av[k][e], rv[k][e]);
                        zo[e] = mv[k][e] * rv[k][e];
                        if (e < valid) {
                            rz = fma(rv[k][e], zo[e], rz);
                            rr = fma(rv[k][e], rv[k][e], rr);
                        }
                    }
                    vstore(d, row, dv[k], valid);
                    vstore(r, row, rv[k], valid);
                    vstore(z, row, zo, valid);
                }
            }
        }
        if (threadIdx.x == 0 && i == __ldg(stile + slot).x) {
            sys[slot].it_inner += 1;
            sys[slot].it_total += 1;
        }
    }
    const double2 t = block_sum2_8(double(rz), double(rr), red);
    if (threadIdx.x == 0) reinterpret_cast<double2*>(part_tile)[i] = t;
}

template <typename T>
__global__ void __launch_bounds__(kThreads, 4)
    bs_update(const int4* tiles, const int32_t* count, SysState* sys, const int2* sblk,
              const int2* stile, const double* part_blk, const T* __restrict__ p,
              const T* __restrict__ Ap, const T* __restrict__ dinv, T* __restrict__ r,
              T* __restrict__ z, T* __restrict__ d, double* part_tile, int par, StepCtl* ctl) {
    __shared__ double2 red[kWarps + 1];
    __shared__ bool last;
    const int32_t i = blockIdx.x;
    if (i >= __ldcg(count)) return;
    const int4 tl = tiles[i];
    update_tile<T, false, false>(i, tl, sys, sblk, stile, part_blk, p, Ap, dinv, r, z, d,
                                 part_tile, par, red);
    if (!tl.w) return;  // a small system: its tile CTAs decide in step 3
    // A large system's stopping test and beta, by the last of its tile CTAs
    // to finish (its tile sums in ordered_sum256's order, as the persistent
    // step forms them), so the iteration needs no kernel of its own for them.
    SysState& S = sys[tl.z];
    const int2 tr = __ldg(stile + tl.z);
    if (threadIdx.x == 0) {
        __threadfence();  // this CTA's tile sum (and iteration count) before its arrival
        last = atomicAdd(&S.tile_arrivals, 1u) == unsigned(tr.y - tr.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (threadIdx.x == 0) S.tile_arrivals = 0u;
    if (__ldcg(&S.phase) != kSysInner) return;  // uniform over the CTA
    const double2 t = ordered_sum256<true>(part_tile, tr.x, tr.y, red);
    if (threadIdx.x == 0) {
        const double inner_rel = sqrt(t.y / __ldcg(&S.rr0));
        const double est = __ldcg(&S.rnorm) * sqrt(t.y) / __ldcg(&S.bnorm);
        const bool stop = !(inner_rel > __ldcg(&S.inner_rtol)) ||
                          !(est >= __ldcg(&S.stop_frac) * __ldcg(&S.tol)) ||
                          __ldcg(&S.it_total) >= __ldcg(&S.max_iter);
        const double rz_old = __ldcg(&S.rzp[par]);
        S.rr = t.y;
        if (stop) {
            S.rz_keep = rz_old;
            S.phase = kSysOuter;
        } else {
            S.beta = t.x / rz_old;
            S.rzp[par ^ 1] = t.x;
            if (ctl) atomicAdd(&ctl->live, 1u);
        }
    }
}

// Inner iteration, step 3, for tile i: (r.z, r.r) of the system from its tile
// sums (every CTA, same order); the inner stopping test; p = z + beta p with
// beta = r.z / previous r.z.  r.z alternates between rzp[par] (read) and
// rzp[par ^ 1] (written by the system's first tile), so no CTA reads a value
// another CTA of this step writes; the phase change of a stopping system is
// the one write others may see early, and they then skip exactly as the test
// would make them.  A continuing system's first tile counts it in *live.
// SELF: a large system is decided here too, in bs_update's order.
template <typename T, bool COH, bool SELF>
__device__ __forceinline__ void pupdate_tile(int32_t i, const int4 tl, SysState* sys,
                                             const int2* stile, const double* part_tile,
                                             const T* __restrict__ z, T* __restrict__ p, int par,
                                             unsigned int* live, double2* red, int32_t* sh) {
    constexpr int VN = Vec16<T>::N;
    constexpr int IT = kVecIters(VN);
    const int32_t slot = tl.z;
    if (threadIdx.x == 0) *sh = sys_phase(sys, slot);
    __syncthreads();
    const int32_t phase = *sh;
    __syncthreads();  // *sh is free for the next tile
    if (phase != kSysInner) return;  // uniform over the CTA
    double beta_d;
    if (tl.w && !SELF) {  // large system: bs_update ran the test and set beta (phase above)
        beta_d = __ldcg(&sys[slot].beta);
    } else {  // reduce the tile sums and decide, as every CTA of the system does
        const int2 tr = __ldg(stile + slot);
        const double2 t = ordered_sum256<true>(part_tile, tr.x, tr.y, red);  // (r.z, r.r)
        const SysState& S = sys[slot];
        const double rr0 = __ldcg(&S.rr0), rnorm = __ldcg(&S.rnorm), bnorm = __ldcg(&S.bnorm);
        const double inner_rel = sqrt(t.y / rr0);
        const double est = rnorm * sqrt(t.y) / bnorm;  // estimated |b - Ax| / |b|
        const bool stop = !(inner_rel > __ldcg(&S.inner_rtol)) ||
                          !(est >= __ldcg(&S.stop_frac) * __ldcg(&S.tol)) ||
                          __ldcg(&S.it_total) >= __ldcg(&S.max_iter);
        const bool first = i == tr.x;
        const double rz_old = __ldcg(&S.rzp[par]);
        if (stop) {  // stop the inner solve; refine next step
            if (first && threadIdx.x == 0) {
                sys[slot].rr = t.y;
                sys[slot].rz_keep = rz_old;
                sys[slot].phase = kSysOuter;
            }
            return;
        }
        beta_d = t.x / rz_old;
        if (first && threadIdx.x == 0) {
            sys[slot].rr = t.y;
            sys[slot].beta = beta_d;
            sys[slot].rzp[par ^ 1] = t.x;
            if (live) atomicAdd(live, 1u);
        }
    }
    if (threadIdx.x >= kThreads) return;
    const T beta = T(beta_d);
    // four vectors of each operand per thread in flight at a time (two in the
    // persistent step)
    constexpr int KB = COH ? (IT < 2 ? IT : 2) : (IT < 4 ? IT : 4);
#pragma unroll
    for (int k0 = 0; k0 < IT; k0 += KB) {
        T zv[KB][VN], pv[KB][VN];
#pragma unroll
        for (int k = 0; k < KB; ++k) {
            const int64_t row = tl.x + int64_t(VN) * (threadIdx.x + (k0 + k) * kThreads);
            if (row < tl.y) {
                vload_c<T, COH>(z, row, zv[k]);
                vload_c<T, COH>(p, row, pv[k]);
            }
        }
#pragma unroll
        for (int k = 0; k < KB; ++k) {
            const int64_t row = tl.x + int64_t(VN) * (threadIdx.x + (k0 + k) * kThreads);
            if (row < tl.y) {
                const int valid = int(min(int64_t(VN), int64_t(tl.y) - row));
#pragma unroll
                for (int e = 0; e < VN; ++e) pv[k][e] = fma(beta, pv[k][e], zv[k][e]);
                vstore(p, row, pv[k], valid);
            }
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kThreads, 4)
    bs_pupdate(const int4* tiles, const int32_t* count, SysState* sys, const int2* stile,
               const double* part_tile, const T* __restrict__ z, T* __restrict__ p, int par,
               StepCtl* ctl) {
    __shared__ double2 red[kWarps + 1];
    __shared__ int32_t sh;
    const int32_t i = blockIdx.x;
    if (i >= __ldcg(count)) return;
    pupdate_tile<T, false, false>(i, tiles[i], sys, stile, part_tile, z, p, par,
                                  ctl ? &ctl->live : nullptr, red, &sh);
}

// ---- the persistent step: the whole iteration loop in one cooperative launch ----------
//
// Every CTA of a co-resident grid runs the step's iterations itself: the SpMV
// pipeline over the inner block list (PhaseGate, InnerEpi), then the update of
// the tiles blockIdx.x, + gridDim.x, ..., then their p update, with a bounded
// grid barrier after each phase -- the three phases the graph path launches as
// kernels, with the same per-block / per-tile sums and the same per-system
// reductions (ordered_sum256, also for large systems, whose alpha / beta the
// graph path reduces in bs_alpha / bs_update in the same order), so the two
// paths give the same bits.  Data written inside the launch is read through
// L2.  After the third barrier every CTA reads how many systems go on (counted
// by their first tiles into live2[parity]); the loop ends when none does or at
// the step's cap.  A wait that gives up sets the error word and ctl->status,
// and every CTA leaves at its next barrier.

__device__ __forceinline__ void fence_proxy_async_global() {
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

template <typename T>
struct InnerEpiCoherent {  // InnerEpi reading p through L2
    static constexpr bool kBlockSums = true;
    T* __restrict__ Ap;
    const T* __restrict__ p;
    double* __restrict__ part;
    T acc;
    __device__ __forceinline__ void operator()(int32_t row, T v) {
        Ap[row] = v;
        acc += __ldcg(p + row) * v;
    }
    __device__ __forceinline__ double take() {
        const double a = double(acc);
        acc = T(0);
        return a;
    }
    __device__ __forceinline__ void finish_block(int64_t b, const BlockDesc&, double sum) {
        part[b] = sum;
    }
};

template <typename V, typename T>
__global__ void __launch_bounds__(kCtaThreads, 2)
    bs_persist(CsrView<V> M, T* p, T* Ap, const T* dinv, T* r, T* z, T* d, SysState* sys,
               const int4* tiles, const int32_t* tile_count, const int2* sblk, const int2* stile,
               double* part_blk, double* part_tile, StepCtl* ctl, unsigned int* err) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    auto& sm = *reinterpret_cast<SpmvSmem<V, T, T, kSolverTile, kSolverStages>*>(smem_raw);
    __shared__ double2 red[kWarps + 1];
    __shared__ int32_t sh;
    __shared__ bool flag;
    const int t = threadIdx.x;
    const unsigned int cap = __ldcg(&ctl->cap);
    M.coherent_x = 1;
    unsigned int it = 0;
    bool failed = false;
    while (it < cap) {
        const int par = int(it & 1u);
        fence_proxy_async_global();  // p written by the previous iteration, then read by TMA
        InnerEpiCoherent<T> epi{Ap, p, part_blk, T(0)};
        const bool ok = spmv_pipeline<V, T, T, kSolverTile, kSolverStages>(
            M, p, sm, epi, err, PhaseGate{sys, kSysInner});
        __syncthreads();
        if (t == 0) {  // the ring's barriers are initialised again by the next SpMV
#pragma unroll
            for (int q = 0; q < kSolverStages; ++q) {
                asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(&sm.full[q]))
                             : "memory");
                asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(&sm.empty[q]))
                             : "memory");
            }
        }
        if (!ok) atomicExch(&ctl->status, kCgDeviceError);
        if (!grid_barrier(&ctl->bar_count, &ctl->bar_gen, err, &ctl->status, &flag)) {
            failed = true;
            break;
        }
        if (blockIdx.x == 0 && t == 0) ctl->live2[par ^ 1] = 0u;  // read before the last barrier
        const int32_t ntile = __ldcg(tile_count);
        for (int32_t i = blockIdx.x; i < ntile; i += gridDim.x)
            update_tile<T, true, true>(i, tiles[i], sys, sblk, stile, part_blk, p, Ap, dinv, r, z,
                                       d, part_tile, par, red);
        if (!grid_barrier(&ctl->bar_count, &ctl->bar_gen, err, &ctl->status, &flag)) {
            failed = true;
            break;
        }
        for (int32_t i = blockIdx.x; i < ntile; i += gridDim.x)
            pupdate_tile<T, true, true>(i, tiles[i], sys, stile, part_tile, z, p, par,
                                        &ctl->live2[par], red, &sh);
        if (!grid_barrier(&ctl->bar_count, &ctl->bar_gen, err, &ctl->status, &flag)) {
            failed = true;
            break;
        }
        ++it;
        if (__ldcg(&ctl->live2[par]) == 0u) break;  // the same value in every CTA
    }
    if (failed && t == 0) atomicExch(&ctl->status, kCgDeviceError);
    if (blockIdx.x == 0 && t == 0) ctl->iter = it;
}

constexpr int kLoopUnroll = 8;  // iterations per body of a step's loop

// Last kernel of a step loop's body: count its iterations, and keep looping
// while some system still iterates and the cap is not reached.
__global__ void bs_control(StepCtl* ctl, cudaGraphConditionalHandle loop) {
    const unsigned int it = ctl->iter + unsigned(kLoopUnroll);
    const unsigned int live = ctl->live;
    ctl->iter = it;
    ctl->live = 0u;
    cudaGraphSetConditional(loop, (live > 0u && it < ctl->cap) ? 1u : 0u);
}

// Marks the listed slots free (nm_solver_take_batch).
__global__ void bs_free_slots(const int32_t* slots, int32_t count, SysState* sys) {
    for (int32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x)
        sys[slots[k]].phase = kSysFree;
}

// ---- host side --------------------------------------------------------------------

// First-fit range allocator over [0, cap).
struct RangeAlloc {
    std::vector<std::pair<int64_t, int64_t>> free_;  // (start, len), sorted by start
    int64_t cap = 0, used = 0;
    void init(int64_t c) {
        cap = c;
        used = 0;
        free_.assign(1, {0, c});
    }
    int64_t alloc(int64_t len) {
        for (size_t i = 0; i < free_.size(); ++i) {
            if (free_[i].second >= len) {
                const int64_t s = free_[i].first;
                free_[i].first += len;
                free_[i].second -= len;
                if (free_[i].second == 0) free_.erase(free_.begin() + long(i));
                used += len;
                return s;
            }
        }
        return -1;
    }
    void release(int64_t s, int64_t len) {
        auto it = std::lower_bound(free_.begin(), free_.end(), std::make_pair(s, int64_t(0)));
        it = free_.insert(it, {s, len});
        used -= len;
        // merge with the right, then the left neighbour
        if (it + 1 != free_.end() && it->first + it->second == (it + 1)->first) {
            it->second += (it + 1)->second;
            free_.erase(it + 1);
        }
        if (it != free_.begin() && (it - 1)->first + (it - 1)->second == it->first) {
            (it - 1)->second += it->second;
            free_.erase(it);
        }
    }
    int64_t largest() const {
        int64_t m = 0;
        for (auto& f : free_) m = std::max(m, f.second);
        return m;
    }
};

struct HostSys {
    SysState init{};  // state at admission (nm_solver_resolve starts from it)
    bool used = false;
    int64_t row0 = 0, nrows_alloc = 0, z0 = 0, nnz_alloc = 0;
    int32_t n = 0;
    int32_t phase = kSysFree;
    std::vector<BlockDesc> blocks;  // arena-global
    std::vector<int4> tiles;
};

}  // namespace nm

struct nm_solver {
    int device = 0;
    int inner = NM_F32;  // inner value precision: NM_F64 (plain PCG), NM_F32 or NM_BF16
    int precond = 1;
    double inner_rtol = 1e-3;
    int max_outer = 30;
    double cont_window = 2.0;
    int64_t cap_rows = 0, cap_nnz = 0;
    int32_t cap_sys = 0;
    nm::RangeAlloc rows, nnz;
    std::vector<nm::HostSys> sys;
    // arena (device)
    int32_t* rp = nullptr;     // [cap_rows + 16]
    int32_t* col = nullptr;    // [cap_nnz + 16]
    double* v64 = nullptr;     // [cap_nnz + 16]
    void* vin = nullptr;       // inner values [cap_nnz + 16] (float / bf16 / unused for FP64)
    double *b = nullptr, *x = nullptr, *r64 = nullptr;  // [cap_rows + 16]
    void *p = nullptr, *Ap = nullptr, *r = nullptr, *z = nullptr, *d = nullptr, *dinv = nullptr;
    nm::SysState* st = nullptr;     // [cap_sys]
    nm::SysState* h_st = nullptr;   // pinned copy
    // lists (device) and their pinned staging
    nm::ListHdr* hdr = nullptr;
    nm::ListHdr* h_hdr = nullptr;
    nm::BlockDesc *iblk = nullptr, *oblk = nullptr;
    int4 *itile = nullptr, *otile = nullptr;
    nm::SysRef *isys = nullptr, *osys = nullptr, *bsys = nullptr;
    int64_t cap_blk = 0, cap_tile = 0;
    double *part_blk = nullptr, *part_tile = nullptr;
    int2 *sblk = nullptr, *stile = nullptr;                // per slot ranges in the inner lists
    int2 *h_sblk = nullptr, *h_stile = nullptr;
    nm::BlockDesc* h_blk = nullptr;  // pinned staging (iblk then oblk)
    int4* h_tile = nullptr;
    nm::SysRef* h_ref = nullptr;
    bool lists_dirty = true;
    // CUDA graph of one chunk of inner iterations; valid while the lists (and
    // so every kernel argument) are unchanged
    cudaGraphExec_t chunk_exec = nullptr;
    bool chunk_valid = false;
    // nm_solver_take_batch: pinned landing of the solutions, slot lists
    double* take_stage = nullptr;
    size_t take_cap = 0;
    int32_t *d_slots = nullptr, *h_slots = nullptr;
    nm::StepCtl* ctl = nullptr;    // device control words of the step loop
    nm::StepCtl* h_ctl = nullptr;  // pinned: the cap going in, the counts coming back
    int grid_spmv_inner = 0, grid_spmv_outer = 0, grid_vec = 0, grid_scalar = 0;
    int grid_persist = 0;     // co-resident grid of bs_persist (0: not available)
    int64_t lists_gen = 0;   // bumped when the work-list arrays are reallocated
    int64_t graph_gen = -1;  // lists_gen the step graph was built against
    int graph_tiles = 0;     // tile grid of the step graph
    bool graph_big = false;  // the step graph includes bs_alpha
    // pinned staging of admission uploads: a bump allocator, reset once the
    // stream has caught up (after each step's synchronisation)
    unsigned char* stage = nullptr;
    size_t stage_cap = 0, stage_used = 0;
    unsigned int* err = nullptr;
    cudaStream_t stream = nullptr;  // the iterations
    cudaStream_t up = nullptr;      // admission uploads (overlap a running step)
    cudaEvent_t up_ev = nullptr;    // orders the uploads before the next kernels
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;  // device time of the running step
    bool in_step = false;           // between nm_solver_step_begin and _end
    bool step_loops = false;        // the running step launched the iteration loop
    nm_solver_counters ctr{};
    ~nm_solver();
};

nm_solver::~nm_solver() {
    cudaFree(rp); cudaFree(col); cudaFree(v64); cudaFree(vin);
    cudaFree(b); cudaFree(x); cudaFree(r64);
    cudaFree(p); cudaFree(Ap); cudaFree(r); cudaFree(z); cudaFree(d); cudaFree(dinv);
    cudaFree(st); cudaFreeHost(h_st);
    cudaFree(hdr); cudaFreeHost(h_hdr);
    cudaFree(iblk); cudaFree(oblk); cudaFree(itile); cudaFree(otile); cudaFree(isys); cudaFree(osys); cudaFree(bsys);
    cudaFree(part_blk); cudaFree(part_tile);
    cudaFree(sblk); cudaFree(stile);
    cudaFreeHost(h_sblk); cudaFreeHost(h_stile);
    cudaFreeHost(h_blk); cudaFreeHost(h_tile); cudaFreeHost(h_ref); cudaFreeHost(stage);
    if (chunk_exec) cudaGraphExecDestroy(chunk_exec);
    cudaFree(ctl);
    cudaFreeHost(h_ctl);
    cudaFreeHost(take_stage);
    cudaFree(d_slots);
    cudaFreeHost(h_slots);
    if (up_ev) cudaEventDestroy(up_ev);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (up) cudaStreamDestroy(up);
    if (stream) cudaStreamDestroy(stream);
}

namespace nm {
namespace {

size_t inner_bytes(int inner) { return inner == NM_F64 ? 8 : 4; }
size_t inner_val_bytes(int inner) { return inner == NM_F64 ? 8 : (inner == NM_F32 ? 4 : 2); }

int grow_lists(nm_solver* S, int64_t need_blk, int64_t need_tile) {
    if (need_blk > S->cap_blk || need_tile > S->cap_tile) S->lists_gen += 1;
    if (need_blk > S->cap_blk) {
        const int64_t c = std::max<int64_t>(need_blk, 2 * S->cap_blk);
        cudaFree(S->iblk); cudaFree(S->oblk); cudaFree(S->part_blk); cudaFreeHost(S->h_blk);
        S->iblk = S->oblk = nullptr; S->part_blk = nullptr; S->h_blk = nullptr;
        NM_CUDA_TRY(cudaMalloc(&S->iblk, sizeof(BlockDesc) * size_t(c)));
        NM_CUDA_TRY(cudaMalloc(&S->oblk, sizeof(BlockDesc) * size_t(c)));
        NM_CUDA_TRY(cudaMalloc(&S->part_blk, sizeof(double) * size_t(c)));
        NM_CUDA_TRY(cudaMallocHost(&S->h_blk, sizeof(BlockDesc) * size_t(c) * 2));
        S->cap_blk = c;
    }
    if (need_tile > S->cap_tile) {
        const int64_t c = std::max<int64_t>(need_tile, 2 * S->cap_tile);
        cudaFree(S->itile); cudaFree(S->otile); cudaFree(S->part_tile); cudaFreeHost(S->h_tile);
        S->itile = S->otile = nullptr; S->part_tile = nullptr; S->h_tile = nullptr;
        NM_CUDA_TRY(cudaMalloc(&S->itile, sizeof(int4) * size_t(c)));
        NM_CUDA_TRY(cudaMalloc(&S->otile, sizeof(int4) * size_t(c)));
        NM_CUDA_TRY(cudaMalloc(&S->part_tile, sizeof(double) * size_t(c) * 2));
        NM_CUDA_TRY(cudaMallocHost(&S->h_tile, sizeof(int4) * size_t(c) * 2));
        S->cap_tile = c;
    }
    return NM_OK;
}

// Rebuild the inner list (systems in an inner or outer phase) and the outer
// list (systems with a pending outer step) and upload them.
int upload_lists(nm_solver* S) {
    int64_t nb_i = 0, nt_i = 0, nb_o = 0, nt_o = 0;
    for (auto& h : S->sys) {
        if (!h.used) continue;
        if (h.phase == kSysInner || h.phase == kSysOuter) {
            nb_i += int64_t(h.blocks.size());
            nt_i += int64_t(h.tiles.size());
        }
        if (h.phase == kSysOuter) {
            nb_o += int64_t(h.blocks.size());
            nt_o += int64_t(h.tiles.size());
        }
    }
    int st = grow_lists(S, std::max<int64_t>(1, std::max(nb_i, nb_o)),
                        std::max<int64_t>(1, std::max(nt_i, nt_o)));
    if (st != NM_OK) return st;
    BlockDesc* bi = S->h_blk;
    BlockDesc* bo = S->h_blk + S->cap_blk;
    int4* ti = S->h_tile;
    int4* to = S->h_tile + S->cap_tile;
    SysRef* ri = S->h_ref;
    SysRef* ro = S->h_ref + S->cap_sys;
    SysRef* rb = S->h_ref + 2 * int64_t(S->cap_sys);
    int32_t cb_i = 0, ct_i = 0, cs_i = 0, cb_o = 0, ct_o = 0, cs_o = 0, cs_b = 0;
    for (int32_t slot = 0; slot < S->cap_sys; ++slot) {
        HostSys& h = S->sys[slot];
        if (!h.used || (h.phase != kSysInner && h.phase != kSysOuter)) continue;
        SysRef a{slot, cb_i, cb_i + int32_t(h.blocks.size()), ct_i,
                 ct_i + int32_t(h.tiles.size()), {0, 0, 0}};
        std::memcpy(bi + cb_i, h.blocks.data(), sizeof(BlockDesc) * h.blocks.size());
        std::memcpy(ti + ct_i, h.tiles.data(), sizeof(int4) * h.tiles.size());
        S->h_sblk[slot] = make_int2(a.blk0, a.blk1);
        S->h_stile[slot] = make_int2(a.tile0, a.tile1);
        cb_i = a.blk1;
        ct_i = a.tile1;
        ri[cs_i++] = a;
        if (!h.tiles.empty() && h.tiles[0].w) rb[cs_b++] = a;
        if (h.phase == kSysOuter) {
            SysRef o{slot, cb_o, cb_o + int32_t(h.blocks.size()), ct_o,
                     ct_o + int32_t(h.tiles.size()), {0, 0, 0}};
            std::memcpy(bo + cb_o, h.blocks.data(), sizeof(BlockDesc) * h.blocks.size());
            std::memcpy(to + ct_o, h.tiles.data(), sizeof(int4) * h.tiles.size());
            cb_o = o.blk1;
            ct_o = o.tile1;
            ro[cs_o++] = o;
        }
    }
    cudaStream_t s = S->stream;
    *S->h_hdr = ListHdr{cb_i, ct_i, cs_i, cb_o, ct_o, cs_o, cs_b, 0};
    NM_CUDA_TRY(cudaMemcpyAsync(S->hdr, S->h_hdr, sizeof(ListHdr), cudaMemcpyHostToDevice, s));
    if (cb_i) NM_CUDA_TRY(cudaMemcpyAsync(S->iblk, bi, sizeof(BlockDesc) * cb_i, cudaMemcpyHostToDevice, s));
    if (cb_o) NM_CUDA_TRY(cudaMemcpyAsync(S->oblk, bo, sizeof(BlockDesc) * cb_o, cudaMemcpyHostToDevice, s));
    if (ct_i) NM_CUDA_TRY(cudaMemcpyAsync(S->itile, ti, sizeof(int4) * ct_i, cudaMemcpyHostToDevice, s));
    if (ct_o) NM_CUDA_TRY(cudaMemcpyAsync(S->otile, to, sizeof(int4) * ct_o, cudaMemcpyHostToDevice, s));
    if (cs_i) NM_CUDA_TRY(cudaMemcpyAsync(S->isys, ri, sizeof(SysRef) * cs_i, cudaMemcpyHostToDevice, s));
    if (cs_o) NM_CUDA_TRY(cudaMemcpyAsync(S->osys, ro, sizeof(SysRef) * cs_o, cudaMemcpyHostToDevice, s));
    if (cs_b) NM_CUDA_TRY(cudaMemcpyAsync(S->bsys, rb, sizeof(SysRef) * cs_b, cudaMemcpyHostToDevice, s));
    NM_CUDA_TRY(cudaMemcpyAsync(S->sblk, S->h_sblk, sizeof(int2) * size_t(S->cap_sys),
                                cudaMemcpyHostToDevice, s));
    NM_CUDA_TRY(cudaMemcpyAsync(S->stile, S->h_stile, sizeof(int2) * size_t(S->cap_sys),
                                cudaMemcpyHostToDevice, s));
    S->lists_dirty = false;
    return NM_OK;
}

// `bytes` of pinned staging for an asynchronous upload on S->up.  When the
// staging buffer is full the upload stream is drained first (its earlier
// uploads are then complete) and the buffer reused or grown.
int stage_alloc(nm_solver* S, size_t bytes, void** out) {
    bytes = (bytes + 255) & ~size_t(255);
    if (S->stage_used + bytes > S->stage_cap) {
        NM_CUDA_TRY(cudaStreamSynchronize(S->up));
        S->stage_used = 0;
        if (bytes > S->stage_cap) {
            cudaFreeHost(S->stage);
            S->stage = nullptr;
            const size_t cap = std::max<size_t>(bytes, std::max<size_t>(64u << 20, 2 * S->stage_cap));
            NM_CUDA_TRY(cudaMallocHost(&S->stage, cap));
            S->stage_cap = cap;
        }
    }
    *out = S->stage + S->stage_used;
    S->stage_used += bytes;
    return NM_OK;
}

template <typename V>
CsrView<V> arena_view(const nm_solver* S, const void* values, const BlockDesc* list,
                      const int32_t* count) {
    CsrView<V> M;
    M.row_ptr = S->rp;
    M.col_idx = S->col;
    M.values = static_cast<const V*>(values);
    M.desc = list;
    M.nblk = 0;
    M.nrows = int32_t(S->cap_rows);
    M.short_max = kDefaultShortMax;
    M.stage_x = 1;
    M.nblk_dev = count;
    return M;
}

// One CTA per tile: the tile count rounded up to a power of two.
int tile_bucket(int64_t tiles) {
    int64_t b = 1;
    while (b < tiles) b <<= 1;
    return int(std::min<int64_t>(b, INT32_MAX));
}

// Grid of a persistent kernel over `count` items (at least one CTA).
int fit_grid(int cap, int64_t count) {
    return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(cap, count)));
}

// One iteration of every live system (the body of a step's loop).
template <typename V, typename T>
int launch_inner_body(nm_solver* S, cudaGraphConditionalHandle loop) {
    cudaStream_t s = S->stream;
    const ListHdr* H = S->hdr;
    const ListHdr& h = *S->h_hdr;
    // Grids that do not follow every change of the lists (their lengths are
    // read on the device): the persistent SpMV and scalar grids are fixed,
    // the one-CTA-per-tile grid is the tile count rounded up to a power of
    // two (CTAs past the count return at once), so the step graph is rebuilt
    // only when the tile count crosses a power of two.
    const int g_spmv = S->grid_spmv_inner;
    const int g_vec = tile_bucket(h.itile);
    const int g_big = h.bsys > 0 ? S->grid_scalar : 0;
    const CsrView<V> M = arena_view<V>(S, S->vin ? S->vin : S->v64, S->iblk, &H->iblk);
    constexpr size_t smem = spmv_smem_bytes<V, T, T, kSolverTile, kSolverStages>();
    T* p = static_cast<T*>(S->p);
    T* Ap = static_cast<T*>(S->Ap);
    T* r = static_cast<T*>(S->r);
    T* z = static_cast<T*>(S->z);
    T* d = static_cast<T*>(S->d);
    const T* dinv = static_cast<const T*>(S->dinv);
    for (int it = 0; it < kLoopUnroll; ++it) {
        const int par = it & 1;
        // the last iteration of the body counts the systems that go on
        StepCtl* ctl = it == kLoopUnroll - 1 ? S->ctl : nullptr;
        bs_spmv_inner<V, T><<<g_spmv, kCtaThreads, smem, s>>>(M, p, Ap, S->st, S->part_blk,
                                                              S->err);
        if (g_big) bs_alpha<<<g_big, kWideThreads, 0, s>>>(S->bsys, &H->bsys, S->st,
                                                           S->part_blk, par);
        bs_update<T><<<g_vec, kThreads, 0, s>>>(S->itile, &H->itile, S->st, S->sblk, S->stile,
                                                S->part_blk, p, Ap, dinv, r, z, d, S->part_tile,
                                                par, ctl);
        bs_pupdate<T><<<g_vec, kThreads, 0, s>>>(S->itile, &H->itile, S->st, S->stile,
                                                 S->part_tile, z, p, par, ctl);
    }
    bs_control<<<1, 1, 0, s>>>(S->ctl, loop);
    NM_CHECK_LAUNCH();
    return NM_OK;
}

template <typename T>
int launch_outer(nm_solver* S) {
    cudaStream_t s = S->stream;
    const ListHdr* H = S->hdr;
    const ListHdr& h = *S->h_hdr;
    const int g_spmv = fit_grid(S->grid_spmv_outer, h.oblk);
    const int g_vec = fit_grid(INT32_MAX, h.otile);  // one CTA per tile
    const int g_sys = fit_grid(S->grid_scalar, h.osys);
    const CsrView<double> M = arena_view<double>(S, S->v64, S->oblk, &H->oblk);
    constexpr size_t smem = spmv_smem_bytes<double, double, double, kSolverTile, kSolverStages>();
    bs_xupdate<T><<<g_vec, kThreads, 0, s>>>(S->otile, &H->otile, S->st,
                                             static_cast<const T*>(S->d), S->x);
    bs_spmv_outer<<<g_spmv, kCtaThreads, smem, s>>>(M, S->x, S->b, S->r64, S->st, S->part_blk,
                                                    S->err);
    bs_scalar<kOuterNorm><<<g_sys, kScalarThreads, 0, s>>>(S->osys, &H->osys, S->st,
                                                           S->part_blk, S->part_tile);
    bs_inner_start<T><<<g_vec, kThreads, 0, s>>>(
        S->otile, &H->otile, S->st, S->r64, static_cast<const T*>(S->dinv),
        static_cast<T*>(S->r), static_cast<T*>(S->z), static_cast<T*>(S->d), S->part_tile);
    bs_scalar<kStart><<<g_sys, kScalarThreads, 0, s>>>(S->osys, &H->osys, S->st, S->part_blk,
                                                       S->part_tile);
    bs_pstart<T><<<g_vec, kThreads, 0, s>>>(S->otile, &H->otile, S->st,
                                            static_cast<const T*>(S->z), static_cast<T*>(S->p));
    NM_CHECK_LAUNCH();
    return NM_OK;
}

template <typename V, typename T>
int prepare_solver_kernels(nm_solver* S) {
    int occ = 0;
    // Load every kernel of a chunk now (lazy module loading), not during capture.
    cudaFuncAttributes fa;
    NM_CUDA_TRY(cudaFuncGetAttributes(&fa, bs_update<T>));
    NM_CUDA_TRY(cudaFuncGetAttributes(&fa, bs_pupdate<T>));
    NM_CUDA_TRY(cudaFuncGetAttributes(&fa, bs_pstart<T>));
    NM_CUDA_TRY(cudaFuncGetAttributes(&fa, bs_alpha));
    NM_CUDA_TRY(cudaFuncGetAttributes(&fa, bs_control));
    NM_CUDA_TRY(cudaFuncGetAttributes(&fa, bs_free_slots));
    int st = prepare_kernel(reinterpret_cast<const void*>(bs_spmv_inner<V, T>), kCtaThreads,
                            spmv_smem_bytes<V, T, T, kSolverTile, kSolverStages>(), &occ);
    if (st != NM_OK) return st;
    S->grid_spmv_inner = sm_count() * occ;
    st = prepare_kernel(reinterpret_cast<const void*>(bs_spmv_outer), kCtaThreads,
                        spmv_smem_bytes<double, double, double, kSolverTile, kSolverStages>(),
                        &occ);
    if (st != NM_OK) return st;
    S->grid_spmv_outer = sm_count() * occ;
    S->grid_vec = sm_count() * 4;
    S->grid_scalar = sm_count() * 2;
    int dev = 0, coop = 0;
    NM_CUDA_TRY(cudaGetDevice(&dev));
    NM_CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    S->grid_persist = 0;
    if (coop) {
        st = prepare_kernel(reinterpret_cast<const void*>(bs_persist<V, T>), kCtaThreads,
                            spmv_smem_bytes<V, T, T, kSolverTile, kSolverStages>(), &occ);
        if (st != NM_OK) return st;
        S->grid_persist = sm_count() * occ;
    }
    return NM_OK;
}

// The step loop as one cooperative launch (bs_persist).
template <typename V, typename T>
int launch_persist(nm_solver* S) {
    const ListHdr* H = S->hdr;
    CsrView<V> M = arena_view<V>(S, S->vin ? S->vin : S->v64, S->iblk, &H->iblk);
    T* p = static_cast<T*>(S->p);
    T* Ap = static_cast<T*>(S->Ap);
    const T* dinv = static_cast<const T*>(S->dinv);
    T* r = static_cast<T*>(S->r);
    T* z = static_cast<T*>(S->z);
    T* d = static_cast<T*>(S->d);
    SysState* sys = S->st;
    const int4* tiles = S->itile;
    const int32_t* tcount = &H->itile;
    const int2* sblk = S->sblk;
    const int2* stile = S->stile;
    double* pb = S->part_blk;
    double* pt = S->part_tile;
    StepCtl* ctl = S->ctl;
    unsigned int* err = S->err;
    void* args[] = {&M,    &p,     &Ap,    &dinv, &r,  &z,  &d,   &sys,
                    &tiles, &tcount, &sblk, &stile, &pb, &pt, &ctl, &err};
    NM_CUDA_TRY(cudaLaunchCooperativeKernel(
        reinterpret_cast<const void*>(bs_persist<V, T>), dim3(S->grid_persist), dim3(kCtaThreads),
        args, spmv_smem_bytes<V, T, T, kSolverTile, kSolverStages>(), S->stream));
    return NM_OK;
}

// nm_solver_set_persistent.  Default: the CUDA-graph step (on the 128^3
// variable-coefficient system, FP32 + refinement: 22.6 solves/s against 17.5
// for the persistent step, whose three grid barriers and per-CTA alpha / beta
// reductions per iteration cost more than the graph's kernel boundaries).
std::atomic<int> g_engine_persistent{0};

// FP64 -> BF16 through FP32, round to nearest even, NaN kept quiet; written
// without branches so the loop vectorises.
void to_bf16(const double* v, size_t n, uint16_t* out) {
    for (size_t i = 0; i < n; ++i) {
        const float f = static_cast<float>(v[i]);
        uint32_t u;
        std::memcpy(&u, &f, 4);
        const uint32_t rounded = (u + 0x7fffu + ((u >> 16) & 1u)) >> 16;
        const uint32_t quiet = (u >> 16) | 0x40u;
        out[i] = static_cast<uint16_t>((u & 0x7fffffffu) > 0x7f800000u ? quiet : rounded);
    }
}

void to_f32(const double* v, size_t n, float* out) {
    for (size_t i = 0; i < n; ++i) out[i] = static_cast<float>(v[i]);
}

}  // namespace
}  // namespace nm

using nm::fail;

extern "C" int nm_solver_create(int64_t max_rows, int64_t max_nnz, int32_t max_systems,
                                const nm_solver_opts* opts, nm_solver** out) {
    using namespace nm;
    clear_error();
    if (!out) return fail(NM_ERR_INVALID, "nm_solver_create: out is NULL");
    *out = nullptr;
    if (max_rows <= 0 || max_nnz <= 0 || max_systems <= 0)
        return fail(NM_ERR_INVALID, "nm_solver_create: capacities must be positive");
    if (max_rows > INT32_MAX - 4096 || max_nnz > INT32_MAX - 4096)
        return fail(NM_ERR_INVALID, "nm_solver_create: capacities exceed the int32 index range");
    auto S = std::make_unique<nm_solver>();
    if (opts) {
        S->inner = opts->inner;
        S->precond = opts->precond;
        if (opts->inner_rtol > 0) S->inner_rtol = opts->inner_rtol;
        if (opts->max_outer > 0) S->max_outer = opts->max_outer;
        if (opts->cont_window > 0) S->cont_window = opts->cont_window;
    }
    if (S->inner != NM_F64 && S->inner != NM_F32 && S->inner != NM_BF16)
        return fail(NM_ERR_TYPE, "nm_solver_create: unknown inner precision %d", S->inner);
    NM_CUDA_TRY(cudaGetDevice(&S->device));
    S->cap_rows = max_rows;
    S->cap_nnz = max_nnz;
    S->cap_sys = max_systems;
    S->rows.init(max_rows);
    S->nnz.init(max_nnz);
    S->sys.resize(size_t(max_systems));
    const size_t R = size_t(max_rows) + 16, Z = size_t(max_nnz) + 16;
    const size_t tb = inner_bytes(S->inner);
    NM_CUDA_TRY(cudaMalloc(&S->rp, sizeof(int32_t) * R));
    NM_CUDA_TRY(cudaMemset(S->rp, 0, sizeof(int32_t) * R));
    NM_CUDA_TRY(cudaMalloc(&S->col, sizeof(int32_t) * Z));
    NM_CUDA_TRY(cudaMemset(S->col, 0, sizeof(int32_t) * Z));
    NM_CUDA_TRY(cudaMalloc(&S->v64, sizeof(double) * Z));
    if (S->inner != NM_F64) NM_CUDA_TRY(cudaMalloc(&S->vin, inner_val_bytes(S->inner) * Z));
    NM_CUDA_TRY(cudaMalloc(&S->b, sizeof(double) * R));
    NM_CUDA_TRY(cudaMalloc(&S->x, sizeof(double) * R));
    NM_CUDA_TRY(cudaMalloc(&S->r64, sizeof(double) * R));
    for (void** v : {&S->p, &S->Ap, &S->r, &S->z, &S->d, &S->dinv}) {
        NM_CUDA_TRY(cudaMalloc(v, tb * R));
        NM_CUDA_TRY(cudaMemset(*v, 0, tb * R));
    }
    NM_CUDA_TRY(cudaMalloc(&S->st, sizeof(SysState) * size_t(max_systems)));
    NM_CUDA_TRY(cudaMemset(S->st, 0, sizeof(SysState) * size_t(max_systems)));
    NM_CUDA_TRY(cudaMallocHost(&S->h_st, sizeof(SysState) * size_t(max_systems)));
    NM_CUDA_TRY(cudaMalloc(&S->hdr, sizeof(ListHdr)));
    NM_CUDA_TRY(cudaMallocHost(&S->h_hdr, sizeof(ListHdr)));
    NM_CUDA_TRY(cudaMalloc(&S->isys, sizeof(SysRef) * size_t(max_systems)));
    NM_CUDA_TRY(cudaMalloc(&S->osys, sizeof(SysRef) * size_t(max_systems)));
    NM_CUDA_TRY(cudaMalloc(&S->bsys, sizeof(SysRef) * size_t(max_systems)));
    NM_CUDA_TRY(cudaMalloc(&S->ctl, sizeof(StepCtl)));
    NM_CUDA_TRY(cudaMalloc(&S->d_slots, sizeof(int32_t) * size_t(max_systems)));
    NM_CUDA_TRY(cudaMallocHost(&S->h_slots, sizeof(int32_t) * size_t(max_systems)));
    NM_CUDA_TRY(cudaMallocHost(&S->h_ctl, sizeof(StepCtl) * 2));
    NM_CUDA_TRY(cudaMallocHost(&S->h_ref, sizeof(SysRef) * size_t(max_systems) * 3));
    for (int2** r : {&S->sblk, &S->stile}) {
        NM_CUDA_TRY(cudaMalloc(r, sizeof(int2) * size_t(max_systems)));
        NM_CUDA_TRY(cudaMemset(*r, 0, sizeof(int2) * size_t(max_systems)));
    }
    NM_CUDA_TRY(cudaMallocHost(&S->h_sblk, sizeof(int2) * size_t(max_systems)));
    NM_CUDA_TRY(cudaMallocHost(&S->h_stile, sizeof(int2) * size_t(max_systems)));
    // Lists sized for a full arena of typical systems (they still grow if a
    // workload needs more): one descriptor per kSolverTile/2 nonzeros or per
    // 128 rows, two per system; one tile per kTileRows rows, two per system.
    const int64_t blk0 = std::max(max_nnz / (kSolverTile / 2), max_rows / 128) + 2 * max_systems;
    const int64_t tile0 = max_rows / kTileRows + 2 * int64_t(max_systems);
    int st = grow_lists(S.get(), blk0, tile0);
    if (st != NM_OK) return st;
    // Pinned staging of admissions, allocated once (grows only for a single
    // system larger than it).
    S->stage_cap = size_t(256) << 20;
    NM_CUDA_TRY(cudaMallocHost(&S->stage, S->stage_cap));
    NM_CUDA_TRY(cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking));
    NM_CUDA_TRY(cudaStreamCreateWithFlags(&S->up, cudaStreamNonBlocking));
    NM_CUDA_TRY(cudaEventCreateWithFlags(&S->up_ev, cudaEventDisableTiming));
    NM_CUDA_TRY(cudaEventCreate(&S->ev0));
    NM_CUDA_TRY(cudaEventCreate(&S->ev1));
    S->err = device_error_word();
    if (!S->err) return fail(NM_ERR_CUDA, "nm_solver_create: cannot map the device error word");
    switch (S->inner) {
        case NM_F64: st = prepare_solver_kernels<double, double>(S.get()); break;
        case NM_F32: st = prepare_solver_kernels<float, float>(S.get()); break;
        default: st = prepare_solver_kernels<__nv_bfloat16, float>(S.get()); break;
    }
    if (st != NM_OK) return st;
    *out = S.release();
    return NM_OK;
}

extern "C" int nm_solver_set_persistent(int32_t enable) {
    nm::clear_error();
    if (enable != 0 && enable != 1)
        return fail(NM_ERR_INVALID, "nm_solver_set_persistent: 0 or 1");
    nm::g_engine_persistent.store(enable);
    return NM_OK;
}

extern "C" int nm_solver_destroy(nm_solver* S) {
    nm::clear_error();
    if (S) {
        cudaStreamSynchronize(S->stream);
        cudaStreamSynchronize(S->up);
    }
    delete S;
    return NM_OK;
}

namespace nm {
namespace {

// Runs f(begin, end) over [0, n) on up to hardware_concurrency threads, in
// chunks of at least `grain` items.
template <class F>
void parallel_for(int64_t n, int64_t grain, const F& f) {
    const int64_t hw = std::max(1u, std::thread::hardware_concurrency());
    const int64_t nt = std::max<int64_t>(1, std::min<int64_t>(hw, n / std::max<int64_t>(1, grain)));
    if (nt <= 1) {
        if (n > 0) f(int64_t(0), n);
        return;
    }
    std::vector<std::thread> th;
    th.reserve(size_t(nt));
    for (int64_t t = 0; t < nt; ++t)
        th.emplace_back([&f, n, nt, t] { f(n * t / nt, n * (t + 1) / nt); });
    for (auto& x : th) x.join();
}

// One admission: inputs, the ranges it was given, its pinned staging.
struct AdmitJob {
    const int32_t* row_ptr;
    const int32_t* col_idx;
    const double* values;
    int32_t n;
    const double* b;
    const double* x0;
    double tol;
    int32_t max_iter;
    // assigned
    int32_t slot = -1;
    int64_t r0 = 0, nrows_alloc = 0, z0 = 0, nnz_alloc = 0;
    unsigned char* stage = nullptr;
    int bad_col = -1;     // an invalid column index found by the preparation
    bool bad_rp = false;  // row_ptr decreases somewhere
    std::vector<BlockDesc> blocks;
    std::vector<int4> tiles;
};

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// Staging layout of a job: row_ptr, col_idx, FP64 values, inner values, b,
// x0, inverse diagonal, SysState.
void stage_sizes(const nm_solver* S, const AdmitJob& J, size_t sz[8]) {
    const size_t n = size_t(J.n), nz = size_t(J.row_ptr[J.n]);
    sz[0] = align256(sizeof(int32_t) * (n + 1));
    sz[1] = align256(sizeof(int32_t) * nz);
    sz[2] = align256(sizeof(double) * nz);
    sz[3] = align256(S->inner != NM_F64 ? inner_val_bytes(S->inner) * nz : 0);
    sz[4] = align256(sizeof(double) * n);
    sz[5] = align256(J.x0 ? sizeof(double) * n : 0);
    sz[6] = align256(inner_bytes(S->inner) * n);
    sz[7] = align256(sizeof(SysState));
}

size_t stage_total(const nm_solver* S, const AdmitJob& J) {
    size_t sz[8];
    stage_sizes(S, J, sz);
    size_t t = 0;
    for (size_t q : sz) t += q;
    return t;
}

// Cheap checks before any allocation.
int job_check(const AdmitJob& J) {
    if (!J.row_ptr || !J.b) return fail(NM_ERR_INVALID, "nm_solver_admit: NULL argument");
    if (J.n <= 0) return fail(NM_ERR_INVALID, "nm_solver_admit: non-positive dimensions");
    if (J.row_ptr[0] != 0) return fail(NM_ERR_INVALID, "nm_solver_admit: row_ptr[0] must be 0");
    if (J.row_ptr[J.n] < 0) return fail(NM_ERR_INVALID, "nm_solver_admit: row_ptr decreases");
    if (J.row_ptr[J.n] > 0 && (!J.col_idx || !J.values))
        return fail(NM_ERR_INVALID, "nm_solver_admit: NULL array");
    return NM_OK;
}

// Slot and arena ranges; NM_ERR_NOMEM when they do not fit.
int job_alloc(nm_solver* S, AdmitJob& J) {
    int32_t slot = -1;
    for (int32_t k = 0; k < S->cap_sys; ++k)
        if (!S->sys[k].used) {
            slot = k;
            break;
        }
    if (slot < 0) return fail(NM_ERR_NOMEM, "nm_solver_admit: all %d system slots are in use", S->cap_sys);
    const int32_t nz = J.row_ptr[J.n];
    // One spare row for the closing row_ptr entry; nonzero ranges padded to 8.
    const int64_t nrows_alloc = ((int64_t(J.n) + 1 + 3) / 4) * 4;
    const int64_t nnz_alloc = ((int64_t(nz) + 7) / 8) * 8 + 8;
    const int64_t r0 = S->rows.alloc(nrows_alloc);
    if (r0 < 0) return fail(NM_ERR_NOMEM, "nm_solver_admit: no room for %d rows", J.n);
    const int64_t z0 = S->nnz.alloc(nnz_alloc);
    if (z0 < 0) {
        S->rows.release(r0, nrows_alloc);
        return fail(NM_ERR_NOMEM, "nm_solver_admit: no room for %d nonzeros", nz);
    }
    S->sys[slot].used = true;  // reserved; filled in by job_commit
    J.slot = slot;
    J.r0 = r0;
    J.nrows_alloc = nrows_alloc;
    J.z0 = z0;
    J.nnz_alloc = nnz_alloc;
    return NM_OK;
}

void job_release(nm_solver* S, AdmitJob& J) {
    if (J.slot < 0) return;
    S->rows.release(J.r0, J.nrows_alloc);
    S->nnz.release(J.z0, J.nnz_alloc);
    S->sys[J.slot] = HostSys{};
    J.slot = -1;
}

// Host preparation of one job into its staging; touches nothing shared, so
// jobs run concurrently.  `inner_threads`: parallelise this job's rows.
void job_prep(const nm_solver* S, AdmitJob& J, bool inner_threads) {
    size_t sz[8];
    stage_sizes(S, J, sz);
    unsigned char* q = J.stage;
    int32_t* grp = reinterpret_cast<int32_t*>(q); q += sz[0];
    int32_t* gci = reinterpret_cast<int32_t*>(q); q += sz[1];
    double* v64s = reinterpret_cast<double*>(q); q += sz[2];
    void* vins = q; q += sz[3];
    double* bs = reinterpret_cast<double*>(q); q += sz[4];
    double* x0s = reinterpret_cast<double*>(q); q += sz[5];
    void* dinvs = q; q += sz[6];
    SysState* ss = reinterpret_cast<SysState*>(q);
    const int32_t n = J.n;
    const int32_t* rp = J.row_ptr;
    const int32_t* ci = J.col_idx;
    const double* val = J.values;
    const int32_t r0 = int32_t(J.r0), z0 = int32_t(J.z0);
    const bool dbl = inner_bytes(S->inner) == 8;
    const int precond = S->precond;
    const int inner = S->inner;
    for (int32_t i = 0; i < n; ++i)
        if (rp[i + 1] < rp[i]) {
            J.bad_rp = true;
            return;
        }
    std::mutex mu;
    auto rows = [&](int64_t i0, int64_t i1) {
        int badc = -1;
        for (int64_t i = i0; i < i1; ++i) {
            grp[i] = z0 + rp[i];
            double dg = 0.0;
            for (int32_t j = rp[i]; j < rp[i + 1]; ++j) {
                const int32_t c = ci[j];
                if ((c < 0 || c >= n) && badc < 0) badc = c;
                gci[j] = r0 + c;
                if (c == i) dg += val[j];
            }
            const double di = (precond && dg != 0.0) ? 1.0 / dg : 1.0;
            if (dbl) static_cast<double*>(dinvs)[i] = di;
            else static_cast<float*>(dinvs)[i] = float(di);
            bs[i] = J.b[i];
            if (J.x0) x0s[i] = J.x0[i];
        }
        if (i1 > i0) {
            const size_t z0c = size_t(rp[i0]), nzc = size_t(rp[i1] - rp[i0]);
            std::memcpy(v64s + z0c, val + z0c, sizeof(double) * nzc);
            if (inner == NM_F32) to_f32(val + z0c, nzc, static_cast<float*>(vins) + z0c);
            if (inner == NM_BF16) to_bf16(val + z0c, nzc, static_cast<uint16_t*>(vins) + z0c);
        }
        std::lock_guard<std::mutex> g(mu);
        if (badc >= 0 && J.bad_col < 0) J.bad_col = badc;
    };
    if (inner_threads) parallel_for(n, 65536, rows);
    else rows(0, n);
    grp[n] = z0 + rp[n];
    if (J.bad_col >= 0) return;
    // |b|^2 in row order (the same bits however the rows were prepared)
    double bb = 0.0;
    for (int32_t i = 0; i < n; ++i) bb += J.b[i] * J.b[i];
    // row blocks (default partition), arena-global descriptors and x windows
    std::vector<int32_t> blk;
    build_row_blocks(rp, n, kSolverTile, kDefaultMaxRows, kDefaultShortMax, blk, nullptr);
    const int64_t nb = int64_t(blk.size()) - 1;
    J.blocks.assign(size_t(nb), BlockDesc{});
    const int32_t cap_rows = int32_t(S->cap_rows);
    const int32_t slot = J.slot;
    auto blocks = [&](int64_t k0, int64_t k1) {
        std::vector<int32_t> scratch;
        for (int64_t k = k0; k < k1; ++k) {
            BlockDesc& dsc = J.blocks[size_t(k)];
            const int32_t lz0 = rp[blk[k]], lz1 = rp[blk[k + 1]];
            int32_t nlong = 0;
            for (int32_t rr = blk[k]; rr < blk[k + 1]; ++rr)
                nlong += (rp[rr + 1] - rp[rr]) > kDefaultShortMax;
            dsc.rz = make_int4(r0 + blk[k], r0 + blk[k + 1], z0 + lz0, z0 + lz1);
            dsc.aux = make_int4(nlong, slot, 0, 0);
            if (lz1 - lz0 > kSolverTile) {
                dsc.xs = make_int4(-1, INT_MAX, INT_MAX, INT_MAX);
                dsc.xl = make_int4(0, 0, 0, 0);
            } else {
                block_xwindows(gci, lz0, lz1, cap_rows, xwin_capacity(kSolverTile), scratch,
                               &dsc.xs, &dsc.xl);
            }
        }
    };
    if (inner_threads) parallel_for(nb, 64, blocks);
    else blocks(0, nb);
    J.tiles.clear();
    const int32_t ntile = (n + kTileRows - 1) / kTileRows;
    const int32_t large = (nb > kLargeBlocks || ntile > kLargeTiles) ? 1 : 0;
    for (int32_t t0 = 0; t0 < n; t0 += kTileRows)
        J.tiles.push_back(make_int4(r0 + t0, r0 + std::min(n, t0 + kTileRows), slot, large));
    std::memset(ss, 0, sizeof(SysState));
    ss->row0 = r0;
    ss->n = n;
    ss->max_iter = J.max_iter;
    ss->max_outer = S->max_outer;
    ss->tol = J.tol;
    ss->bnorm = bb > 0.0 ? std::sqrt(bb) : 1.0;
    ss->inner_rtol = S->inner == NM_F64 ? 0.0 : S->inner_rtol;
    ss->stop_frac = S->inner == NM_F64 ? 1.0 : 0.5;
    ss->cont_window = S->cont_window;
    ss->phase = kSysOuter;
}

// Asynchronous uploads of a prepared job and its host record.
int job_commit(nm_solver* S, AdmitJob& J) {
    size_t sz[8];
    stage_sizes(S, J, sz);
    unsigned char* q = J.stage;
    unsigned char* ptr[8];
    for (int k = 0; k < 8; ++k) {
        ptr[k] = q;
        q += sz[k];
    }
    const size_t n = size_t(J.n), nz = size_t(J.row_ptr[J.n]);
    const size_t tb = inner_bytes(S->inner), vb = inner_val_bytes(S->inner);
    cudaStream_t s = S->up;
    const int64_t r0 = J.r0, z0 = J.z0;
    NM_CUDA_TRY(cudaMemcpyAsync(S->rp + r0, ptr[0], sizeof(int32_t) * (n + 1), cudaMemcpyHostToDevice, s));
    if (nz) {
        NM_CUDA_TRY(cudaMemcpyAsync(S->col + z0, ptr[1], sizeof(int32_t) * nz, cudaMemcpyHostToDevice, s));
        NM_CUDA_TRY(cudaMemcpyAsync(S->v64 + z0, ptr[2], sizeof(double) * nz, cudaMemcpyHostToDevice, s));
        if (S->inner != NM_F64)
            NM_CUDA_TRY(cudaMemcpyAsync(static_cast<unsigned char*>(S->vin) + vb * size_t(z0), ptr[3],
                                        vb * nz, cudaMemcpyHostToDevice, s));
    }
    NM_CUDA_TRY(cudaMemcpyAsync(S->b + r0, ptr[4], sizeof(double) * n, cudaMemcpyHostToDevice, s));
    if (J.x0) {
        NM_CUDA_TRY(cudaMemcpyAsync(S->x + r0, ptr[5], sizeof(double) * n, cudaMemcpyHostToDevice, s));
    } else {
        NM_CUDA_TRY(cudaMemsetAsync(S->x + r0, 0, sizeof(double) * n, s));
    }
    NM_CUDA_TRY(cudaMemsetAsync(static_cast<unsigned char*>(S->d) + tb * size_t(r0), 0, tb * n, s));
    NM_CUDA_TRY(cudaMemcpyAsync(static_cast<unsigned char*>(S->dinv) + tb * size_t(r0), ptr[6], tb * n,
                                cudaMemcpyHostToDevice, s));
    const SysState* ss = reinterpret_cast<const SysState*>(ptr[7]);
    S->h_st[J.slot] = *ss;
    NM_CUDA_TRY(cudaMemcpyAsync(S->st + J.slot, ss, sizeof(SysState), cudaMemcpyHostToDevice, s));
    HostSys& h = S->sys[J.slot];
    h.used = true;
    h.row0 = J.r0;
    h.nrows_alloc = J.nrows_alloc;
    h.z0 = J.z0;
    h.nnz_alloc = J.nnz_alloc;
    h.n = J.n;
    h.phase = kSysOuter;
    h.blocks = std::move(J.blocks);
    h.tiles = std::move(J.tiles);
    h.init = *ss;
    S->lists_dirty = true;
    return NM_OK;
}

// Admits jobs[0..count) in order, preparing them in parallel; stops at the
// first one that does not fit.  *admitted = jobs admitted.
int admit_jobs(nm_solver* S, AdmitJob* jobs, int32_t count, int32_t* admitted) {
    *admitted = 0;
    int32_t done = 0;
    // Sub-batches of at most half the staging buffer, so they fit it without
    // growing it.
    const size_t kBatchStage = std::max<size_t>(S->stage_cap / 2, size_t(1) << 20);
    while (done < count) {
        int32_t k = done;
        size_t bytes = 0;
        int st = NM_OK;
        for (; k < count; ++k) {
            st = job_check(jobs[k]);
            if (st != NM_OK) break;
            const size_t tb = stage_total(S, jobs[k]);
            if (k > done && bytes + tb > kBatchStage) break;
            st = job_alloc(S, jobs[k]);
            if (st != NM_OK) break;
            bytes += tb;
        }
        const int32_t end = k;
        if (end == done) return st;  // the first job of this sub-batch was refused
        unsigned char* base = nullptr;
        int sst = stage_alloc(S, bytes, reinterpret_cast<void**>(&base));
        if (sst != NM_OK) {
            for (int32_t j = done; j < end; ++j) job_release(S, jobs[j]);
            return sst;
        }
        for (int32_t j = done; j < end; ++j) {
            jobs[j].stage = base;
            base += stage_total(S, jobs[j]);
        }
        const auto tp = std::chrono::steady_clock::now();
        // large systems one at a time, each over all host threads; the rest
        // in parallel, one thread per system
        constexpr int32_t kLargeRows = 65536;
        std::vector<int32_t> small;
        for (int32_t j = done; j < end; ++j) {
            if (jobs[j].n >= kLargeRows || end - done == 1) job_prep(S, jobs[j], true);
            else small.push_back(j);
        }
        parallel_for(int64_t(small.size()), 1, [&](int64_t a, int64_t b) {
            for (int64_t j = a; j < b; ++j) job_prep(S, jobs[small[size_t(j)]], false);
        });
        const auto tc = std::chrono::steady_clock::now();
        S->ctr.s_admit_prep += std::chrono::duration<double>(tc - tp).count();
        for (int32_t j = done; j < end; ++j) {
            if (jobs[j].bad_col >= 0 || jobs[j].bad_rp) {
                const AdmitJob& b = jobs[j];
                const int c = b.bad_col;
                const bool rp_bad = b.bad_rp;
                const int32_t bn = b.n;
                for (int32_t q = j; q < end; ++q) job_release(S, jobs[q]);
                if (rp_bad) return fail(NM_ERR_INVALID, "nm_solver_admit: row_ptr decreases");
                return fail(NM_ERR_INVALID, "nm_solver_admit: column %d outside [0, %d)", c, bn);
            }
            const int cst = job_commit(S, jobs[j]);
            if (cst != NM_OK) return cst;
            ++*admitted;
        }
        S->ctr.s_admit_commit +=
            std::chrono::duration<double>(std::chrono::steady_clock::now() - tc).count();
        done = end;
        if (st != NM_OK) return st;  // stopped early (no room or an invalid system)
    }
    return NM_OK;
}

}  // namespace
}  // namespace nm

extern "C" int nm_solver_admit(nm_solver* S, const int32_t* row_ptr, const int32_t* col_idx,
                               const double* values, int32_t n, const double* b, const double* x0,
                               double tol, int32_t max_iter, int32_t* slot_out) {
    using namespace nm;
    clear_error();
    if (!S || !slot_out) return fail(NM_ERR_INVALID, "nm_solver_admit: NULL argument");
    AdmitJob J{row_ptr, col_idx, values, n, b, x0, tol, max_iter};
    int32_t admitted = 0;
    const int st = admit_jobs(S, &J, 1, &admitted);
    if (st != NM_OK) return st;
    *slot_out = J.slot;
    return NM_OK;
}

extern "C" int nm_solver_admit_batch(nm_solver* S, int32_t count, const int32_t* const* row_ptr,
                                     const int32_t* const* col_idx, const double* const* values,
                                     const int32_t* n, const double* const* b, double tol,
                                     int32_t max_iter, int32_t* slots, int32_t* admitted) {
    using namespace nm;
    clear_error();
    if (!S || count < 0 || !slots || !admitted || (count > 0 && (!row_ptr || !n || !b)))
        return fail(NM_ERR_INVALID, "nm_solver_admit_batch: NULL argument");
    std::vector<AdmitJob> jobs;
    jobs.reserve(size_t(count));
    for (int32_t k = 0; k < count; ++k)
        jobs.push_back(AdmitJob{row_ptr[k], col_idx ? col_idx[k] : nullptr,
                                values ? values[k] : nullptr, n[k], b[k], nullptr, tol, max_iter});
    const int st = admit_jobs(S, jobs.data(), count, admitted);
    for (int32_t k = 0; k < *admitted; ++k) slots[k] = jobs[k].slot;
    if (st == NM_ERR_NOMEM) {
        clear_error();
        return NM_OK;  // the rest did not fit now; *admitted tells how many did
    }
    return st;
}

extern "C" int nm_solver_step_begin(nm_solver* S, int32_t iters) {
    using namespace nm;
    using clk = std::chrono::steady_clock;
    clear_error();
    if (!S) return fail(NM_ERR_INVALID, "nm_solver_step_begin: NULL solver");
    if (S->in_step) return fail(NM_ERR_INVALID, "nm_solver_step_begin: a step is running");
    if (iters < 0) return fail(NM_ERR_INVALID, "nm_solver_step_begin: iters must be >= 0");
    iters = (iters + kLoopUnroll - 1) / kLoopUnroll * kLoopUnroll;  // whole loop bodies
    int st = NM_OK;
    auto t0 = clk::now();
    auto lap = [&t0](double& acc) {
        const auto t = clk::now();
        acc += std::chrono::duration<double>(t - t0).count();
        t0 = t;
    };
    // admissions' uploads land before anything reads the new systems
    NM_CUDA_TRY(cudaEventRecord(S->up_ev, S->up));
    NM_CUDA_TRY(cudaStreamWaitEvent(S->stream, S->up_ev, 0));
    if (S->lists_dirty) {
        st = upload_lists(S);
        if (st != NM_OK) return st;
        S->ctr.list_uploads += 1;
    }
    lap(S->ctr.s_lists);
    S->in_step = true;
    NM_CUDA_TRY(cudaEventRecord(S->ev0, S->stream));
    const ListHdr& H = *S->h_hdr;
    if (H.isys == 0) {
        NM_CUDA_TRY(cudaEventRecord(S->ev1, S->stream));
        return NM_OK;
    }
    S->ctr.steps += 1;
    if (H.osys > 0) {
        st = S->inner == NM_F64 ? launch_outer<double>(S) : launch_outer<float>(S);
        if (st != NM_OK) return st;
        S->ctr.outer_launches += 1;
    }
    lap(S->ctr.s_outer);
    if (iters > 0 && S->grid_persist > 0 && g_engine_persistent.load()) {
        // the whole loop in one cooperative launch
        *S->h_ctl = StepCtl{};
        S->h_ctl->cap = unsigned(iters);
        NM_CUDA_TRY(cudaMemcpyAsync(S->ctl, S->h_ctl, sizeof(StepCtl), cudaMemcpyHostToDevice,
                                    S->stream));
        switch (S->inner) {
            case NM_F64: st = launch_persist<double, double>(S); break;
            case NM_F32: st = launch_persist<float, float>(S); break;
            default: st = launch_persist<__nv_bfloat16, float>(S); break;
        }
        if (st != NM_OK) return st;
        S->step_loops = true;
    } else if (iters > 0) {
        const bool big = S->h_hdr->bsys > 0;
        const int tiles = tile_bucket(S->h_hdr->itile);
        if (!S->chunk_valid || S->graph_big != big || S->graph_tiles != tiles ||
            S->graph_gen != S->lists_gen) {
            S->ctr.graph_captures += 1;
            // The step graph: a WHILE node whose body is one iteration of every
            // live system, ended on the device by bs_control.  Rebuilt when the
            // work lists change; the executable graph is updated in place when
            // the driver accepts it.
            cudaGraph_t g = nullptr;
            NM_CUDA_TRY(cudaGraphCreate(&g, 0));
            cudaGraphConditionalHandle loop;
            cudaError_t ec = cudaGraphConditionalHandleCreate(&loop, g, 1, cudaGraphCondAssignDefault);
            cudaGraphNodeParams cp = {};
            cudaGraphNode_t node = nullptr;
            if (ec == cudaSuccess) {
                cp.type = cudaGraphNodeTypeConditional;
                cp.conditional.handle = loop;
                cp.conditional.type = cudaGraphCondTypeWhile;
                cp.conditional.size = 1;
                ec = cudaGraphAddNode(&node, g, nullptr, 0, &cp);
            }
            if (ec == cudaSuccess)
                ec = cudaStreamBeginCaptureToGraph(S->stream, cp.conditional.phGraph_out[0], nullptr,
                                                   nullptr, 0, cudaStreamCaptureModeThreadLocal);
            if (ec != cudaSuccess) {
                cudaGraphDestroy(g);
                return fail(NM_ERR_CUDA, "solver step graph: %s", cudaGetErrorString(ec));
            }
            switch (S->inner) {
                case NM_F64: st = launch_inner_body<double, double>(S, loop); break;
                case NM_F32: st = launch_inner_body<float, float>(S, loop); break;
                default: st = launch_inner_body<__nv_bfloat16, float>(S, loop); break;
            }
            cudaGraph_t body = nullptr;
            ec = cudaStreamEndCapture(S->stream, &body);
            if (st != NM_OK) {
                cudaGraphDestroy(g);
                return st;
            }
            if (ec != cudaSuccess) {
                cudaGraphDestroy(g);
                return fail(NM_ERR_CUDA, "solver step capture failed: %s", cudaGetErrorString(ec));
            }
            bool updated = false;
            if (S->chunk_exec) {
                cudaGraphExecUpdateResultInfo info;
                updated = cudaGraphExecUpdate(S->chunk_exec, g, &info) == cudaSuccess;
                cudaGetLastError();  // an update refusal is not an error
            }
            if (!updated) {
                S->ctr.graph_instantiations += 1;
                if (S->chunk_exec) cudaGraphExecDestroy(S->chunk_exec);
                S->chunk_exec = nullptr;
                const cudaError_t ei = cudaGraphInstantiate(&S->chunk_exec, g, 0);
                if (ei != cudaSuccess) {
                    cudaGraphDestroy(g);
                    return fail(NM_ERR_CUDA, "solver chunk instantiate failed: %s",
                                cudaGetErrorString(ei));
                }
            }
            cudaGraphDestroy(g);
            S->chunk_valid = true;
            S->graph_big = big;
            S->graph_tiles = tiles;
            S->graph_gen = S->lists_gen;
        }
        lap(S->ctr.s_capture);
        *S->h_ctl = StepCtl{};
        S->h_ctl->cap = unsigned(iters);
        NM_CUDA_TRY(cudaMemcpyAsync(S->ctl, S->h_ctl, sizeof(StepCtl), cudaMemcpyHostToDevice,
                                    S->stream));
        NM_CUDA_TRY(cudaGraphLaunch(S->chunk_exec, S->stream));
        S->step_loops = true;
    }
    NM_CUDA_TRY(cudaEventRecord(S->ev1, S->stream));
    return NM_OK;
}

extern "C" int nm_solver_step_end(nm_solver* S, int32_t* n_done) {
    using namespace nm;
    using clk = std::chrono::steady_clock;
    clear_error();
    if (!S) return fail(NM_ERR_INVALID, "nm_solver_step_end: NULL solver");
    if (!S->in_step) return fail(NM_ERR_INVALID, "nm_solver_step_end: no step is running");
    S->in_step = false;
    auto t0 = clk::now();
    // uploads of systems admitted during the step land before the state read-back
    NM_CUDA_TRY(cudaEventRecord(S->up_ev, S->up));
    NM_CUDA_TRY(cudaStreamWaitEvent(S->stream, S->up_ev, 0));
    NM_CUDA_TRY(cudaMemcpyAsync(S->h_st, S->st, sizeof(SysState) * size_t(S->cap_sys),
                                cudaMemcpyDeviceToHost, S->stream));
    if (S->step_loops)
        NM_CUDA_TRY(cudaMemcpyAsync(S->h_ctl + 1, S->ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost,
                                    S->stream));
    NM_CUDA_TRY(cudaStreamSynchronize(S->stream));
    if (S->step_loops) {
        S->ctr.inner_iterations += S->h_ctl[1].iter;
        S->ctr.last_step_iters = S->h_ctl[1].iter;
        S->step_loops = false;
    } else {
        S->ctr.last_step_iters = 0;
    }
    S->stage_used = 0;  // every staged upload has landed
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, S->ev0, S->ev1) == cudaSuccess) {
        S->ctr.last_step_ms = ms;
        S->ctr.s_device += ms * 1e-3;
    }
    S->ctr.s_run += std::chrono::duration<double>(clk::now() - t0).count();
    t0 = clk::now();
    int st = nm_check_device_errors();
    if (st != NM_OK) return st;
    int32_t done = 0;
    for (int32_t k = 0; k < S->cap_sys; ++k) {
        HostSys& h = S->sys[k];
        if (!h.used) continue;
        const int32_t ph = S->h_st[k].phase;
        if (ph != h.phase) {
            // membership of the outer list changes with every phase change
            S->lists_dirty = true;
            if (ph == kSysDone) ++done;
            h.phase = ph;
        }
    }
    if (n_done) *n_done = done;
    S->ctr.s_scan += std::chrono::duration<double>(clk::now() - t0).count();
    return NM_OK;
}

extern "C" int nm_solver_step(nm_solver* S, int32_t iters, int32_t* n_done) {
    const int st = nm_solver_step_begin(S, iters);
    if (st != NM_OK) {
        if (S && S->in_step) {  // end the step without hiding the first error
            const std::string msg = nm_last_error();
            nm_solver_step_end(S, nullptr);
            return fail(st, "%s", msg.c_str());
        }
        return st;
    }
    return nm_solver_step_end(S, n_done);
}

extern "C" int nm_solver_counters_get(const nm_solver* S, nm_solver_counters* out) {
    nm::clear_error();
    if (!S || !out) return fail(NM_ERR_INVALID, "nm_solver_counters_get: NULL argument");
    *out = S->ctr;
    return NM_OK;
}

extern "C" int nm_solver_status(const nm_solver* S, int32_t slot, int32_t* phase,
                                nm_cg_result* res, int32_t* outer) {
    using namespace nm;
    clear_error();
    if (!S || slot < 0 || slot >= S->cap_sys || !S->sys[slot].used)
        return fail(NM_ERR_INVALID, "nm_solver_status: no system in slot %d", slot);
    const SysState& ss = S->h_st[slot];
    if (phase) *phase = S->sys[slot].phase;
    if (res) {
        res->iters = ss.it_total;
        res->final_res = ss.final_res;
        res->converged = ss.converged;
    }
    if (outer) *outer = ss.outer;
    return NM_OK;
}

extern "C" int nm_solver_take(nm_solver* S, int32_t slot, double* x_host) {
    using namespace nm;
    clear_error();
    if (!S || slot < 0 || slot >= S->cap_sys || !S->sys[slot].used)
        return fail(NM_ERR_INVALID, "nm_solver_take: no system in slot %d", slot);
    if (S->in_step) return fail(NM_ERR_INVALID, "nm_solver_take: a step is running");
    HostSys& h = S->sys[slot];
    if (x_host)
        NM_CUDA_TRY(cudaMemcpyAsync(x_host, S->x + h.row0, sizeof(double) * size_t(h.n),
                                    cudaMemcpyDeviceToHost, S->stream));
    NM_CUDA_TRY(cudaStreamSynchronize(S->stream));
    S->rows.release(h.row0, h.nrows_alloc);
    S->nnz.release(h.z0, h.nnz_alloc);
    const bool was_active = h.phase == kSysInner || h.phase == kSysOuter;
    h = HostSys{};
    S->h_st[slot].phase = kSysFree;
    NM_CUDA_TRY(cudaMemcpyAsync(&S->st[slot].phase, &S->h_st[slot].phase, sizeof(int32_t),
                                cudaMemcpyHostToDevice, S->stream));
    NM_CUDA_TRY(cudaStreamSynchronize(S->stream));
    if (was_active) S->lists_dirty = true;
    return NM_OK;
}

extern "C" int nm_solver_resolve(nm_solver* S, int32_t slot, const double* b_host,
                                 const double* x0_host) {
    using namespace nm;
    clear_error();
    if (!S || slot < 0 || slot >= S->cap_sys || !S->sys[slot].used)
        return fail(NM_ERR_INVALID, "nm_solver_resolve: no system in slot %d", slot);
    if (S->in_step) return fail(NM_ERR_INVALID, "nm_solver_resolve: a step is running");
    HostSys& h = S->sys[slot];
    SysState ss = h.init;
    const size_t n = size_t(h.n);
    NM_CUDA_TRY(cudaStreamSynchronize(S->up));
    if (b_host) {
        double bb = 0.0;
        for (size_t i = 0; i < n; ++i) bb += b_host[i] * b_host[i];
        ss.bnorm = bb > 0.0 ? std::sqrt(bb) : 1.0;
        h.init.bnorm = ss.bnorm;
        NM_CUDA_TRY(cudaMemcpyAsync(S->b + h.row0, b_host, sizeof(double) * n,
                                    cudaMemcpyHostToDevice, S->stream));
    }
    if (x0_host) {
        NM_CUDA_TRY(cudaMemcpyAsync(S->x + h.row0, x0_host, sizeof(double) * n,
                                    cudaMemcpyHostToDevice, S->stream));
    } else {
        NM_CUDA_TRY(cudaMemsetAsync(S->x + h.row0, 0, sizeof(double) * n, S->stream));
    }
    const size_t tb = inner_bytes(S->inner);
    NM_CUDA_TRY(cudaMemsetAsync(static_cast<unsigned char*>(S->d) + tb * size_t(h.row0), 0, tb * n,
                                S->stream));
    S->h_st[slot] = ss;
    NM_CUDA_TRY(cudaMemcpyAsync(S->st + slot, &S->h_st[slot], sizeof(SysState),
                                cudaMemcpyHostToDevice, S->stream));
    NM_CUDA_TRY(cudaStreamSynchronize(S->stream));  // the host copies may go away
    if (h.phase != kSysOuter) S->lists_dirty = true;
    h.phase = kSysOuter;
    return NM_OK;
}

extern "C" int nm_solver_solution(nm_solver* S, int32_t slot, double* x_host) {
    using namespace nm;
    clear_error();
    if (!S || !x_host || slot < 0 || slot >= S->cap_sys || !S->sys[slot].used)
        return fail(NM_ERR_INVALID, "nm_solver_solution: no system in slot %d", slot);
    if (S->in_step) return fail(NM_ERR_INVALID, "nm_solver_solution: a step is running");
    const HostSys& h = S->sys[slot];
    NM_CUDA_TRY(cudaMemcpyAsync(x_host, S->x + h.row0, sizeof(double) * size_t(h.n),
                                cudaMemcpyDeviceToHost, S->stream));
    NM_CUDA_TRY(cudaStreamSynchronize(S->stream));
    return NM_OK;
}

extern "C" int nm_solver_stream(const nm_solver* S, void** stream) {
    nm::clear_error();
    if (!S || !stream) return fail(NM_ERR_INVALID, "nm_solver_stream: NULL argument");
    *stream = S->stream;
    return NM_OK;
}

extern "C" int nm_solver_take_batch(nm_solver* S, int32_t count, const int32_t* slots,
                                    double* const* x_host) {
    using namespace nm;
    clear_error();
    if (!S || count < 0 || (count > 0 && !slots))
        return fail(NM_ERR_INVALID, "nm_solver_take_batch: NULL argument");
    if (S->in_step) return fail(NM_ERR_INVALID, "nm_solver_take_batch: a step is running");
    if (count > S->cap_sys) return fail(NM_ERR_INVALID, "nm_solver_take_batch: too many slots");
    if (count == 0) return NM_OK;
    size_t rows = 0;
    std::vector<char> seen(size_t(S->cap_sys), 0);
    for (int32_t k = 0; k < count; ++k) {
        const int32_t sl = slots[k];
        if (sl < 0 || sl >= S->cap_sys || !S->sys[sl].used)
            return fail(NM_ERR_INVALID, "nm_solver_take_batch: no system in slot %d", sl);
        if (seen[size_t(sl)]) return fail(NM_ERR_INVALID, "nm_solver_take_batch: slot %d twice", sl);
        seen[size_t(sl)] = 1;
        rows += size_t(S->sys[sl].n);
    }
    if (x_host && rows > S->take_cap) {
        const size_t cap = std::max(rows, 2 * S->take_cap);
        cudaFreeHost(S->take_stage);
        S->take_stage = nullptr;
        S->take_cap = 0;
        NM_CUDA_TRY(cudaMallocHost(&S->take_stage, sizeof(double) * cap));
        S->take_cap = cap;
    }
    cudaStream_t s = S->stream;
    size_t off = 0;
    if (x_host) {
        for (int32_t k = 0; k < count; ++k) {
            const HostSys& h = S->sys[slots[k]];
            NM_CUDA_TRY(cudaMemcpyAsync(S->take_stage + off, S->x + h.row0, sizeof(double) * size_t(h.n),
                                        cudaMemcpyDeviceToHost, s));
            off += size_t(h.n);
        }
    }
    std::memcpy(S->h_slots, slots, sizeof(int32_t) * size_t(count));
    NM_CUDA_TRY(cudaMemcpyAsync(S->d_slots, S->h_slots, sizeof(int32_t) * size_t(count),
                                cudaMemcpyHostToDevice, s));
    bs_free_slots<<<(count + 255) / 256, 256, 0, s>>>(S->d_slots, count, S->st);
    NM_CHECK_LAUNCH();
    NM_CUDA_TRY(cudaStreamSynchronize(s));
    off = 0;
    for (int32_t k = 0; k < count; ++k) {
        HostSys& h = S->sys[slots[k]];
        if (x_host && x_host[k]) std::memcpy(x_host[k], S->take_stage + off, sizeof(double) * size_t(h.n));
        off += size_t(h.n);
        S->rows.release(h.row0, h.nrows_alloc);
        S->nnz.release(h.z0, h.nnz_alloc);
        if (h.phase == kSysInner || h.phase == kSysOuter) S->lists_dirty = true;
        h = HostSys{};
        S->h_st[slots[k]].phase = kSysFree;
    }
    return NM_OK;
}

extern "C" int nm_solver_info(const nm_solver* S, int64_t* free_rows, int64_t* free_nnz,
                              int32_t* active, int32_t* free_slots) {
    using namespace nm;
    clear_error();
    if (!S) return fail(NM_ERR_INVALID, "nm_solver_info: NULL solver");
    if (free_rows) *free_rows = S->rows.largest();
    if (free_nnz) *free_nnz = S->nnz.largest();
    int32_t a = 0, f = 0;
    for (auto& h : S->sys) {
        if (!h.used) ++f;
        else if (h.phase == kSysInner || h.phase == kSysOuter) ++a;
    }
    if (active) *active = a;
    if (free_slots) *free_slots = f;
    return NM_OK;
}
