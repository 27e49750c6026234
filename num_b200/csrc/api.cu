// api.cu -- error reporting, device context, host-only helpers.
#include <map>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "csr.cuh"

namespace nm {

namespace {
thread_local std::string g_last_error;
std::mutex g_sm_mu;
std::unordered_map<int, int> g_sm_count;
}  // namespace

int fail(int status, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return status;
}

void clear_error() { g_last_error.clear(); }

int sm_count() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 1;
    std::lock_guard<std::mutex> g(g_sm_mu);
    auto it = g_sm_count.find(dev);
    if (it != g_sm_count.end()) return it->second;
    int n = 1;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1)
        n = 1;
    g_sm_count[dev] = n;
    return n;
}

void release_dot_scratch();  // vec.cu

namespace {
std::mutex g_kern_mu;
std::map<std::pair<const void*, int>, int> g_kern_occ;  // (kernel, device) -> CTAs per SM
}  // namespace

int prepare_kernel(const void* fn, int threads, size_t smem, int* ctas_per_sm) {
    int dev = 0;
    NM_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> g(g_kern_mu);
    auto key = std::make_pair(fn, dev);
    auto it = g_kern_occ.find(key);
    if (it != g_kern_occ.end()) {
        *ctas_per_sm = it->second;
        return NM_OK;
    }
    if (smem > 48 * 1024)
        NM_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem)));
    NM_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     cudaSharedmemCarveoutMaxShared));
    int occ = 0;
    NM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, threads, smem));
    if (occ < 1) return fail(NM_ERR_CUDA, "kernel does not fit on an SM (%zu B shared)", smem);
    g_kern_occ[key] = occ;
    *ctas_per_sm = occ;
    return NM_OK;
}

namespace {
std::mutex g_err_mu;
std::unordered_map<int, std::pair<unsigned int*, unsigned int*>> g_err;  // dev -> (host, device)
}  // namespace

unsigned int* device_error_word() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    std::lock_guard<std::mutex> g(g_err_mu);
    auto it = g_err.find(dev);
    if (it != g_err.end()) return it->second.second;
    unsigned int* h = nullptr;
    unsigned int* d = nullptr;
    if (cudaHostAlloc(reinterpret_cast<void**>(&h), sizeof(unsigned int), cudaHostAllocMapped) !=
        cudaSuccess)
        return nullptr;
    *h = 0u;
    if (cudaHostGetDevicePointer(reinterpret_cast<void**>(&d), h, 0) != cudaSuccess) {
        cudaFreeHost(h);
        return nullptr;
    }
    g_err[dev] = {h, d};
    return d;
}

}  // namespace nm

using nm::fail;

extern "C" const char* nm_last_error(void) { return nm::g_last_error.c_str(); }

extern "C" const char* nm_version(void) { return "num_b200 0.1.0 (sm_100a)"; }

extern "C" int nm_init(int device_id, int32_t* rank, int32_t* size) {
    nm::clear_error();
    int n = 0;
    NM_CUDA_TRY(cudaGetDeviceCount(&n));
    if (device_id < 0 || device_id >= n)
        return fail(NM_ERR_INVALID, "init: device_id %d outside [0, %d)", device_id, n);
    NM_CUDA_TRY(cudaSetDevice(device_id));
    NM_CUDA_TRY(cudaFree(nullptr));  // create the context now
    if (rank) *rank = 0;
    if (size) *size = 1;
    return NM_OK;
}

extern "C" int nm_check_device_errors(void) {
    nm::clear_error();
    int dev = 0;
    NM_CUDA_TRY(cudaGetDevice(&dev));
    unsigned int code = 0;
    {
        std::lock_guard<std::mutex> g(nm::g_err_mu);
        auto it = nm::g_err.find(dev);
        if (it == nm::g_err.end()) return NM_OK;
        code = *reinterpret_cast<volatile unsigned int*>(it->second.first);
        *reinterpret_cast<volatile unsigned int*>(it->second.first) = 0u;
    }
    if (code & nm::kErrWaitTimeout)
        return fail(NM_ERR_RUNTIME,
                    "a kernel gave up a bounded wait (for TMA copies or a grid barrier); results are invalid");
    if (code) return fail(NM_ERR_RUNTIME, "device error code 0x%x", code);
    return NM_OK;
}

extern "C" int nm_finalize(void) {
    nm::clear_error();
    nm::release_dot_scratch();
    return NM_OK;
}

// Host-only: the row-block partition nm_csr_create would build for `row_ptr`
// under tuning `t` (NULL = defaults).  Needs no GPU.
extern "C" int nm_row_blocks_host(const int32_t* row_ptr, int32_t nrows, const nm_tuning* t,
                                  int32_t* blk, int32_t cap, int8_t* bins, int32_t* nblk) {
    nm::clear_error();
    if (!row_ptr || !blk || !nblk || nrows < 0)
        return fail(NM_ERR_INVALID, "nm_row_blocks_host: bad argument");
    nm_tuning tt = t ? *t : nm_tuning{0, 0, 0, 0, 0, 0};
    if (tt.tile <= 0) tt.tile = nm::kDefaultTile;
    if (tt.max_rows <= 0) tt.max_rows = nm::kDefaultMaxRows;
    if (tt.short_max <= 0) tt.short_max = nm::kDefaultShortMax;
    std::vector<int32_t> b;
    std::vector<int8_t> bn;
    const int nb = nm::build_row_blocks(row_ptr, nrows, tt.tile, tt.max_rows, tt.short_max, b,
                                        bins ? &bn : nullptr);
    if (nb + 1 > cap) return fail(NM_ERR_INVALID, "nm_row_blocks_host: cap %d < %d", cap, nb + 1);
    std::copy(b.begin(), b.end(), blk);
    if (bins && !bn.empty()) std::copy(bn.begin(), bn.end(), bins);
    *nblk = nb;
    return NM_OK;
}
