// common.cuh -- shared definitions of the num_b200 CUDA library (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>
#include <stdarg.h>
#include <stdio.h>

#include "../../include/num_b200.h"

namespace nm {

// One CTA of every SpMV-family kernel has this many threads; the row-block
// partition never puts more rows than this into one block.
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

// Records a formatted message as the calling thread's last error and returns
// the status, so call sites read `return fail(NM_ERR_INVALID, "...")`.
int fail(int status, const char* fmt, ...);
void clear_error();

// Number of SMs of the current device (cached per device).
int sm_count();

// Device-visible error word of the current device (mapped pinned host memory,
// zero until a kernel reports a failed bounded wait).  Kernels OR codes into
// it; nm_check_device_errors() reads and clears it on the host.
unsigned int* device_error_word();

// Opts kernel `fn` into `smem` bytes of dynamic shared memory and the
// maximum shared-memory carveout on the current device (once per device) and
// returns how many CTAs of `threads` threads fit on one SM.
int prepare_kernel(const void* fn, int threads, size_t smem, int* ctas_per_sm);

// Device error codes.
constexpr unsigned int kErrWaitTimeout = 1u;  // a bounded mbarrier wait gave up

}  // namespace nm

#define NM_CUDA_TRY(call)                                                     \
    do {                                                                      \
        cudaError_t e_ = (call);                                              \
        if (e_ != cudaSuccess)                                                \
            return ::nm::fail(NM_ERR_CUDA, "%s failed: %s", #call,            \
                              cudaGetErrorString(e_));                        \
    } while (0)

#define NM_CHECK_LAUNCH()                                                     \
    do {                                                                      \
        cudaError_t e_ = cudaGetLastError();                                  \
        if (e_ != cudaSuccess)                                                \
            return ::nm::fail(NM_ERR_CUDA, "kernel launch failed: %s",        \
                              cudaGetErrorString(e_));                        \
    } while (0)

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------
namespace nm {

// Matrix data is streamed once per SpMV: load it with the evict-first cache
// policy (ld.global.cs) so it does not push the gathered vector out of L2.
__device__ __forceinline__ int4 ld_stream(const int4* p) { return __ldcs(p); }
__device__ __forceinline__ double2 ld_stream(const double2* p) { return __ldcs(p); }
__device__ __forceinline__ float4 ld_stream(const float4* p) { return __ldcs(p); }
__device__ __forceinline__ uint2 ld_stream(const uint2* p) { return __ldcs(p); }

// Four consecutive matrix values starting at a 4-aligned index, widened to the
// accumulation type.
template <typename V, typename A>
struct Load4;

template <>
struct Load4<double, double> {
    __device__ __forceinline__ static void run(const double* v, int64_t j, double out[4]) {
        double2 a = ld_stream(reinterpret_cast<const double2*>(v + j));
        double2 b = ld_stream(reinterpret_cast<const double2*>(v + j + 2));
        out[0] = a.x; out[1] = a.y; out[2] = b.x; out[3] = b.y;
    }
};

template <>
struct Load4<float, float> {
    __device__ __forceinline__ static void run(const float* v, int64_t j, float out[4]) {
        float4 a = ld_stream(reinterpret_cast<const float4*>(v + j));
        out[0] = a.x; out[1] = a.y; out[2] = a.z; out[3] = a.w;
    }
};

template <>
struct Load4<__nv_bfloat16, float> {
    __device__ __forceinline__ static void run(const __nv_bfloat16* v, int64_t j, float out[4]) {
        uint2 a = ld_stream(reinterpret_cast<const uint2*>(v + j));
        __nv_bfloat162 lo = *reinterpret_cast<__nv_bfloat162*>(&a.x);
        __nv_bfloat162 hi = *reinterpret_cast<__nv_bfloat162*>(&a.y);
        float2 l = __bfloat1622float2(lo), h = __bfloat1622float2(hi);
        out[0] = l.x; out[1] = l.y; out[2] = h.x; out[3] = h.y;
    }
};

template <typename V, typename A>
__device__ __forceinline__ A widen(V v) { return static_cast<A>(v); }
template <>
__device__ __forceinline__ float widen<__nv_bfloat16, float>(__nv_bfloat16 v) {
    return __bfloat162float(v);
}

// Unfused multiply and add, so serial sums reproduce the CPU order bit for bit
// (nvcc would otherwise contract a*b + c into one FMA).
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }

// ---- TMA bulk copies and mbarriers (inline PTX, sm_90+ / sm_100a) ----------

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this thread's generic-proxy shared-memory accesses before later
// async-proxy (TMA) accesses to the same shared memory.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Arrive on the barrier and add `bytes` to the transaction count it waits for.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// One-dimensional TMA bulk copy global -> shared; completion is signalled on
// `bar` as `bytes` transaction bytes.  src, dst 16-byte aligned, bytes % 16 == 0.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_timer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Wait for phase `parity` of `bar` to complete, giving up after ~2 s of
// wall time (and after a fixed number of polls) so that no fault can turn
// into a hang.  Returns false when it gave up.  `limit_ns` is lowered only by
// the failure-detection test kernels (nm_test_wait_timeout).
constexpr uint64_t kWaitLimitNs = 2000000000ull;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity,
                                                  uint64_t limit_ns = kWaitLimitNs) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_timer_ns();
    for (uint32_t it = 0; it < (1u << 30); ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 255u) == 0 && global_timer_ns() - t0 > limit_ns) return false;
    }
    return false;
}

// Plain arrival (no transaction bytes) on an mbarrier.
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Deterministic CTA-wide sum: fixed shuffle tree per warp, then thread 0 adds
// the warp totals in warp order.  Result is valid in thread 0 only.
// `scratch` needs one entry per warp of the CTA.  Contains __syncthreads();
// call from all threads.
template <typename T>
__device__ __forceinline__ T block_sum(T v, T* scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_sum(v);
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    T s = T(0);
    if (threadIdx.x == 0) {
        const int nw = static_cast<int>(blockDim.x) >> 5;
        for (int w = 0; w < nw; ++w) s += scratch[w];
    }
    __syncthreads();
    return s;
}

}  // namespace nm
