// waits.cu -- failure-detection hook: a bounded device wait that runs out.
//
// Every spin-wait of this library's kernels (the TMA pipelines' mbarrier waits
// and the persistent CG's grid barriers) gives up after a time limit, sets the
// device error word and lets its kernel return, so a lost arrival can never
// hang the GPU.  nm_test_wait_timeout runs those same wait routines
// (mbar_wait_bounded, grid_barrier) in a kernel whose wait cannot complete --
// one arrival fewer than the barrier expects, nothing else pending -- with a
// short limit, so a test can check that the wait ends, the kernel returns,
// the host reads the error, and the context stays usable.  No counterpart in
// the reference (its kernels have no bounded waits).
#include <algorithm>

#include "cg.cuh"

namespace nm {
namespace {

constexpr int kMaxProbeCtas = 64;

struct WaitProbe {
    unsigned int count, gen;      // grid barrier words
    int32_t status;               // stays kCgOk
    int32_t pad;
    unsigned long long waited_ns[kMaxProbeCtas];
    int32_t gave_up[kMaxProbeCtas];
};

// One CTA: an mbarrier initialised for two arrivals receives one, then the
// CTA's thread 0 waits for the phase to complete.
__global__ void wait_probe_mbar_kernel(uint64_t limit_ns, unsigned int* err, WaitProbe* out) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 2);
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        mbar_arrive(&bar);  // the second arrival never comes
        const uint64_t t0 = global_timer_ns();
        const bool ok = mbar_wait_bounded(&bar, 0, limit_ns);
        out->waited_ns[blockIdx.x] = global_timer_ns() - t0;
        out->gave_up[blockIdx.x] = ok ? 0 : 1;
        if (!ok) atomicOr(err, kErrWaitTimeout);
    }
}

// A co-resident grid meets a grid barrier that expects one CTA more than the
// grid has; every CTA gives up after limit_ns.
__global__ void wait_probe_grid_kernel(uint64_t limit_ns, unsigned int* err, WaitProbe* out) {
    __shared__ bool flag;
    const uint64_t t0 = global_timer_ns();
    const bool ok = grid_barrier(&out->count, &out->gen, err, &out->status, &flag,
                                 gridDim.x + 1, limit_ns);
    if (threadIdx.x == 0) {
        out->waited_ns[blockIdx.x] = global_timer_ns() - t0;
        out->gave_up[blockIdx.x] = ok ? 0 : 1;
    }
}

}  // namespace
}  // namespace nm

extern "C" int nm_test_wait_timeout(int32_t kind, int32_t ctas, double limit_ms, double* waited_ms,
                                    void* stream) {
    using namespace nm;
    clear_error();
    if (kind != 0 && kind != 1) return fail(NM_ERR_INVALID, "nm_test_wait_timeout: kind 0 or 1");
    if (kind == 0) ctas = 1;
    if (ctas < 1 || ctas > kMaxProbeCtas)
        return fail(NM_ERR_INVALID, "nm_test_wait_timeout: ctas in [1, %d]", kMaxProbeCtas);
    if (!(limit_ms > 0.0 && limit_ms <= 2000.0))
        return fail(NM_ERR_INVALID, "nm_test_wait_timeout: limit_ms in (0, 2000]");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned int* err = device_error_word();
    if (!err) return fail(NM_ERR_CUDA, "nm_test_wait_timeout: no device error word");
    WaitProbe* d = nullptr;
    NM_CUDA_TRY(cudaMalloc(&d, sizeof(WaitProbe)));
    WaitProbe h;
    cudaError_t e = cudaMemsetAsync(d, 0, sizeof(WaitProbe), s);
    const uint64_t limit_ns = static_cast<uint64_t>(limit_ms * 1e6);
    if (e == cudaSuccess) {
        if (kind == 0) {
            wait_probe_mbar_kernel<<<1, 32, 0, s>>>(limit_ns, err, d);
            e = cudaGetLastError();
        } else {
            // a cooperative launch guarantees every CTA is resident, so the
            // barrier's only missing arrival is the one it was told to expect
            uint64_t lim = limit_ns;
            void* args[] = {&lim, &err, &d};
            e = cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(wait_probe_grid_kernel),
                                            dim3(ctas), dim3(32), args, 0, s);
        }
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d, sizeof(WaitProbe), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(d);
    if (e != cudaSuccess)
        return fail(NM_ERR_CUDA, "nm_test_wait_timeout: %s", cudaGetErrorString(e));
    int gave_up = 0;
    unsigned long long most = 0;
    for (int i = 0; i < ctas; ++i) {
        gave_up += h.gave_up[i];
        most = std::max(most, h.waited_ns[i]);
    }
    if (waited_ms) *waited_ms = double(most) * 1e-6;
    if (gave_up == 0) return NM_OK;  // the wait completed: not what the probe sets up
    return fail(NM_ERR_RUNTIME,
                "nm_test_wait_timeout: %d of %d waits gave up after %.3f ms as set up; the "
                "device error word is set",
                gave_up, ctas, double(most) * 1e-6);
}
