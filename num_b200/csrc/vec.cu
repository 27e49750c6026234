// vec.cu -- vector ops of the CG solver (src/vec_ops.hpp), one kernel each,
// plus the deterministic dot product.
#include <mutex>
#include <unordered_map>

#include "cg.cuh"

namespace nm {

int vec_grid(int64_t n) {
    const int64_t want = (n + kThreads - 1) / kThreads;
    const int64_t cap = int64_t(sm_count()) * 8;
    return static_cast<int>(std::max<int64_t>(1, std::min(want, cap)));
}

// Element-wise kernels: operands may alias (z == x or z == y), as in the
// reference where CG calls vec_axpy(alpha, p, x, x).
__global__ void axpy_kernel(int64_t n, double a, const double* x, const double* y, double* z) {
    for (int64_t i = int64_t(blockIdx.x) * kThreads + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * kThreads)
        z[i] = fma(a, x[i], y[i]);
}

__global__ void axpy2_kernel(int64_t n, double a, const double* x, double b, const double* y,
                             double* z) {
    for (int64_t i = int64_t(blockIdx.x) * kThreads + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * kThreads)
        z[i] = fma(b, y[i], a * x[i]);
}

__global__ void fill_kernel(int64_t n, double v, double* x) {
    for (int64_t i = int64_t(blockIdx.x) * kThreads + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * kThreads)
        x[i] = v;
}

__global__ void scale_kernel(int64_t n, double a, double* x) {
    for (int64_t i = int64_t(blockIdx.x) * kThreads + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * kThreads)
        x[i] *= a;
}

__global__ void __launch_bounds__(kThreads)
    dot_kernel(int64_t n, const double* __restrict__ x, const double* __restrict__ y,
               double* partials, unsigned int* counter, double* result) {
    __shared__ double red[kWarps];
    double s = 0.0;
    for (int64_t i = int64_t(blockIdx.x) * kThreads + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * kThreads)
        s = fma(x[i], y[i], s);
    double part[1] = {block_sum(s, red)};
    double tot[1];
    if (grid_reduce_last<1>(part, partials, counter, tot, red)) *result = tot[0];
}

namespace {

// Scratch of nm_dot: CTA partials, the arrival counter, the result and its
// pinned host landing.  One per (device, stream), created on first use.
struct DotScratch {
    double* partials = nullptr;
    unsigned int* counter = nullptr;
    double* result = nullptr;
    double* h_result = nullptr;
};

std::mutex g_dot_mu;
std::unordered_map<uint64_t, DotScratch> g_dot;

int dot_scratch(cudaStream_t s, DotScratch** out) {
    int dev = 0;
    NM_CUDA_TRY(cudaGetDevice(&dev));
    const uint64_t key = (uint64_t(uint32_t(dev)) << 48) ^ reinterpret_cast<uint64_t>(s);
    std::lock_guard<std::mutex> g(g_dot_mu);
    auto it = g_dot.find(key);
    if (it != g_dot.end()) {
        *out = &it->second;
        return NM_OK;
    }
    DotScratch d;
    const int cap = sm_count() * 8;
    NM_CUDA_TRY(cudaMalloc(&d.partials, sizeof(double) * cap));
    NM_CUDA_TRY(cudaMalloc(&d.counter, sizeof(unsigned int)));
    NM_CUDA_TRY(cudaMemset(d.counter, 0, sizeof(unsigned int)));
    NM_CUDA_TRY(cudaMalloc(&d.result, sizeof(double)));
    NM_CUDA_TRY(cudaMallocHost(&d.h_result, sizeof(double)));
    *out = &(g_dot[key] = d);
    return NM_OK;
}

}  // namespace

void release_dot_scratch() {
    std::lock_guard<std::mutex> g(g_dot_mu);
    for (auto& kv : g_dot) {
        cudaFree(kv.second.partials);
        cudaFree(kv.second.counter);
        cudaFree(kv.second.result);
        cudaFreeHost(kv.second.h_result);
    }
    g_dot.clear();
}

}  // namespace nm

using nm::fail;

#define NM_VEC_PRELUDE(name)                                                   \
    nm::clear_error();                                                         \
    if (n < 0) return fail(NM_ERR_INVALID, name ": n must be >= 0");           \
    if (n == 0) return NM_OK;                                                  \
    cudaStream_t s = static_cast<cudaStream_t>(stream);                        \
    const int grid = nm::vec_grid(n)

extern "C" int nm_axpy(int64_t n, double alpha, const double* x, const double* y, double* z,
                       void* stream) {
    NM_VEC_PRELUDE("nm_axpy");
    if (!x || !y || !z) return fail(NM_ERR_INVALID, "nm_axpy: NULL vector");
    nm::axpy_kernel<<<grid, nm::kThreads, 0, s>>>(n, alpha, x, y, z);
    NM_CHECK_LAUNCH();
    return NM_OK;
}

extern "C" int nm_axpy2(int64_t n, double alpha, const double* x, double beta, const double* y,
                        double* z, void* stream) {
    NM_VEC_PRELUDE("nm_axpy2");
    if (!x || !y || !z) return fail(NM_ERR_INVALID, "nm_axpy2: NULL vector");
    nm::axpy2_kernel<<<grid, nm::kThreads, 0, s>>>(n, alpha, x, beta, y, z);
    NM_CHECK_LAUNCH();
    return NM_OK;
}

extern "C" int nm_dot(int64_t n, const double* x, const double* y, double* result, void* stream) {
    nm::clear_error();
    if (!result) return fail(NM_ERR_INVALID, "nm_dot: NULL result");
    if (n < 0) return fail(NM_ERR_INVALID, "nm_dot: n must be >= 0");
    if (n == 0) {
        *result = 0.0;
        return NM_OK;
    }
    if (!x || !y) return fail(NM_ERR_INVALID, "nm_dot: NULL vector");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    nm::DotScratch* d = nullptr;
    int st = nm::dot_scratch(s, &d);
    if (st != NM_OK) return st;
    const int grid = nm::vec_grid(n);
    nm::dot_kernel<<<grid, nm::kThreads, 0, s>>>(n, x, y, d->partials, d->counter, d->result);
    NM_CHECK_LAUNCH();
    NM_CUDA_TRY(cudaMemcpyAsync(d->h_result, d->result, sizeof(double), cudaMemcpyDeviceToHost, s));
    NM_CUDA_TRY(cudaStreamSynchronize(s));
    *result = *d->h_result;
    return NM_OK;
}

extern "C" int nm_norm2(int64_t n, const double* x, double* result, void* stream) {
    int st = nm_dot(n, x, x, result, stream);
    if (st == NM_OK) *result = std::sqrt(*result);
    return st;
}

extern "C" int nm_copy(int64_t n, const double* src, double* dst, void* stream) {
    nm::clear_error();
    if (n < 0) return fail(NM_ERR_INVALID, "nm_copy: n must be >= 0");
    if (n == 0) return NM_OK;
    if (!src || !dst) return fail(NM_ERR_INVALID, "nm_copy: NULL vector");
    NM_CUDA_TRY(cudaMemcpyAsync(dst, src, sizeof(double) * size_t(n), cudaMemcpyDeviceToDevice,
                                static_cast<cudaStream_t>(stream)));
    return NM_OK;
}

extern "C" int nm_fill(int64_t n, double value, double* x, void* stream) {
    NM_VEC_PRELUDE("nm_fill");
    if (!x) return fail(NM_ERR_INVALID, "nm_fill: NULL vector");
    nm::fill_kernel<<<grid, nm::kThreads, 0, s>>>(n, value, x);
    NM_CHECK_LAUNCH();
    return NM_OK;
}

extern "C" int nm_scale(int64_t n, double alpha, double* x, void* stream) {
    NM_VEC_PRELUDE("nm_scale");
    if (!x) return fail(NM_ERR_INVALID, "nm_scale: NULL vector");
    nm::scale_kernel<<<grid, nm::kThreads, 0, s>>>(n, alpha, x);
    NM_CHECK_LAUNCH();
    return NM_OK;
}
