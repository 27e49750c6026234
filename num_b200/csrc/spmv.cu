// spmv.cu -- plain SpMV and multi-RHS SpMV kernels and their launchers.
#include "spmv.cuh"

#include <algorithm>
#include <atomic>
#include <new>
#include <vector>

namespace nm {

template <typename V, typename X, typename A, int TILE, int STAGES>
__global__ void __launch_bounds__(kCtaThreads)
    spmv_kernel(const CsrView<V> M, const X* __restrict__ x, X* __restrict__ y,
                unsigned int* err) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    auto& sm = *reinterpret_cast<SpmvSmem<V, X, A, TILE, STAGES>*>(smem_raw);
    StoreEpi<X, A> epi{y};
    spmv_pipeline<V, X, A, TILE, STAGES>(M, x, sm, epi, err);
}

// ---------------------------------------------------------------------------
// Scattered-column SpMV: matrices whose row blocks mostly have no x windows
// (nm_csr::warp_gather).  One warp per group of 32 consecutive rows, groups
// strided over the resident warps.  The group's nonzeros stream through in
// chunks of 32 * kGatherU, the next chunk's columns and values loaded while
// this chunk's x gathers are in flight and the next group's row bounds one
// group ahead; each lane parks its products v * x[col] in the warp's chunk
// buffer, then lane l adds the products of row r0 + l that fall in the chunk.
// Every row is summed serially in CSR order (bit-identical to the reference's
// serial row loop, src/spmv_kernel.hpp:90-97), rows up to kWarpGatherMaxRow
// nonzeros.  No TMA ring and no CTA barrier: the x gathers set the rate
// (power-law rows, 2 M rows / 32 M nonzeros: 200 us against 238 us for the
// row-block pipeline).
constexpr int kGatherThreads = 128;
constexpr int kGatherU = 6;
constexpr int kGatherRows = 32;

template <typename V>
__device__ __forceinline__ V ld_value_cs(const V* p) {
    if constexpr (std::is_same_v<V, __nv_bfloat16>)
        return __ushort_as_bfloat16(__ldcs(reinterpret_cast<const unsigned short*>(p)));
    else
        return __ldcs(p);
}

template <typename V, typename X, typename A>
__global__ void __launch_bounds__(kGatherThreads)
    spmv_gather_kernel(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                       const V* __restrict__ vals, const X* __restrict__ x, X* __restrict__ y,
                       int32_t nrows) {
    constexpr int kChunk = 32 * kGatherU;
    __shared__ A prod[kGatherThreads / 32][kChunk];
    const int lane = threadIdx.x & 31;
    A* pw = prod[threadIdx.x >> 5];
    const int64_t ngroups = (int64_t(nrows) + kGatherRows - 1) / kGatherRows;
    const int64_t nw = int64_t(gridDim.x) * (kGatherThreads / 32);
    int64_t g = (int64_t(blockIdx.x) * kGatherThreads + threadIdx.x) >> 5;  // same for the warp
    auto bounds = [&](int64_t gg, int32_t& s0, int32_t& s1) {
        s0 = 0;
        s1 = 0;
        const int64_t r = gg * kGatherRows + lane;
        if (gg < ngroups && r < nrows) {
            s0 = __ldg(rp + r);
            s1 = __ldg(rp + r + 1);
        }
    };
    int32_t nrs, nre;
    bounds(g, nrs, nre);
    for (; g < ngroups; g += nw) {
        const int32_t r0 = static_cast<int32_t>(g * kGatherRows);
        const int nr = nrows - r0 < kGatherRows ? nrows - r0 : kGatherRows;
        const int32_t rs = nrs, re = nre;
        bounds(g + nw, nrs, nre);
        const int32_t z0 = __shfl_sync(0xffffffffu, rs, 0);
        const int32_t z1 = __shfl_sync(0xffffffffu, re, nr - 1);
        A acc = A(0);
        int32_t c[kGatherU];
        V v[kGatherU];
#pragma unroll
        for (int u = 0; u < kGatherU; ++u) {
            const int32_t j = z0 + u * 32 + lane;
            c[u] = j < z1 ? __ldcs(ci + j) : 0;
            v[u] = j < z1 ? ld_value_cs(vals + j) : V(0.0f);
        }
        for (int32_t c0 = z0; c0 < z1; c0 += kChunk) {
            X xv[kGatherU];
            V vv[kGatherU];
#pragma unroll
            for (int u = 0; u < kGatherU; ++u) {
                xv[u] = __ldcg(x + c[u]);
                vv[u] = v[u];
            }
#pragma unroll
            for (int u = 0; u < kGatherU; ++u) {
                const int32_t j = c0 + kChunk + u * 32 + lane;
                c[u] = j < z1 ? __ldcs(ci + j) : 0;
                v[u] = j < z1 ? ld_value_cs(vals + j) : V(0.0f);
            }
#pragma unroll
            for (int u = 0; u < kGatherU; ++u)
                pw[u * 32 + lane] = mul_rn(widen<V, A>(vv[u]), static_cast<A>(xv[u]));
            __syncwarp();
            const int32_t a = rs > c0 ? rs : c0;
            const int32_t b = re < c0 + kChunk ? re : c0 + kChunk;
            for (int32_t j = a; j < b; ++j) acc = add_rn(acc, pw[j - c0]);
            __syncwarp();
        }
        if (lane < nr) y[r0 + lane] = static_cast<X>(acc);
    }
}

template <typename V, typename X, typename A>
static int launch_gather(const nm_csr* Am, const X* x, X* y, cudaStream_t s) {
    static std::atomic<int> occ_cache{0};  // resident CTAs per SM (same on every device here)
    int occ = occ_cache.load(std::memory_order_relaxed);
    if (occ == 0) {
        NM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &occ, spmv_gather_kernel<V, X, A>, kGatherThreads, 0));
        occ = occ > 0 ? occ : 1;
        occ_cache.store(occ, std::memory_order_relaxed);
    }
    const int64_t groups = (int64_t(Am->nrows) + kGatherRows - 1) / kGatherRows;
    const int64_t need = (groups + kGatherThreads / 32 - 1) / (kGatherThreads / 32);
    const int grid = static_cast<int>(std::min<int64_t>(need, int64_t(sm_count()) * occ));
    spmv_gather_kernel<V, X, A><<<grid, kGatherThreads, 0, s>>>(
        Am->d_row_ptr, Am->d_col_idx, static_cast<const V*>(Am->d_values), x, y, Am->nrows);
    NM_CHECK_LAUNCH();
    return NM_OK;
}

// ---------------------------------------------------------------------------
// Sliced gather kernel: the same serial CSR-order row sums, from the
// length-sorted sliced copy (nm_csr::d_sell_*).  One warp per slice of 32
// sorted rows, slices strided over the resident warps; lane l owns the
// slice's row l and adds its products in its own register, reading entry k of
// all 32 rows with one coalesced load per array (the slice is column-major)
// and gathering x[col] through L2, kSellU entries ahead.  The 32 rows of a
// slice have nearly the same length (sorted within kSellWindow rows), so no
// lane waits long for the others, and no product goes through shared memory
// -- the x gathers are left as the only scattered traffic.  Slice metadata is
// fetched one slice ahead.
constexpr int kSellThreads = 128;
constexpr int kSellU = 8;

template <typename V, typename X, typename A>
__global__ void __launch_bounds__(kSellThreads)
    spmv_sell_kernel(const int64_t* __restrict__ sp, const int32_t* __restrict__ srow,
                     const int32_t* __restrict__ slen, const int32_t* __restrict__ col,
                     const V* __restrict__ val, const X* __restrict__ x, X* __restrict__ y,
                     int32_t nslices, int32_t nrows) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = int64_t(gridDim.x) * (kSellThreads / 32);
    int64_t s = (int64_t(blockIdx.x) * kSellThreads + threadIdx.x) >> 5;  // same for the warp
    auto meta = [&](int64_t ss, int64_t& b, int64_t& e, int32_t& r, int32_t& len) {
        b = e = 0;
        r = -1;
        len = 0;
        if (ss < nslices) {
            b = __ldg(sp + ss);
            e = __ldg(sp + ss + 1);
            const int64_t i = ss * 32 + lane;
            if (i < nrows) {
                r = __ldg(srow + i);
                len = __ldg(slen + i);
            }
        }
    };
    int64_t nb, ne;
    int32_t nr, nl;
    meta(s, nb, ne, nr, nl);
    for (; s < nslices; s += nw) {
        const int64_t base = nb;
        const int32_t width = static_cast<int32_t>((ne - nb) >> 5);
        const int32_t r = nr, len = nl;
        meta(s + nw, nb, ne, nr, nl);
        const int32_t* __restrict__ cp = col + base + lane;
        const V* __restrict__ vp = val + base + lane;
        A acc = A(0);
        int32_t k = 0;
        for (; k + kSellU <= width; k += kSellU) {
            int32_t c[kSellU];
            V v[kSellU];
            X xv[kSellU];
#pragma unroll
            for (int u = 0; u < kSellU; ++u) {
                c[u] = __ldcs(cp + int64_t(k + u) * 32);
                v[u] = ld_value_cs(vp + int64_t(k + u) * 32);
            }
#pragma unroll
            for (int u = 0; u < kSellU; ++u) xv[u] = k + u < len ? __ldcg(x + c[u]) : X(0);
#pragma unroll
            for (int u = 0; u < kSellU; ++u)
                if (k + u < len) acc = add_rn(acc, mul_rn(widen<V, A>(v[u]), static_cast<A>(xv[u])));
        }
        for (; k < width; ++k) {
            if (k < len) {
                const int32_t c = __ldcs(cp + int64_t(k) * 32);
                const V v = ld_value_cs(vp + int64_t(k) * 32);
                acc = add_rn(acc, mul_rn(widen<V, A>(v), static_cast<A>(__ldcg(x + c))));
            }
        }
        if (r >= 0) y[r] = static_cast<X>(acc);
    }
}

// Fills the sliced copy from the device CSR: one warp per slice, lane l
// copies the row of sorted position 32 s + l and zero-pads it to the slice
// width.
template <typename V>
__global__ void sell_fill_kernel(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                 const V* __restrict__ vals, const int64_t* __restrict__ sp,
                                 const int32_t* __restrict__ srow, const int32_t* __restrict__ slen,
                                 int32_t* __restrict__ col, V* __restrict__ val, int32_t nslices,
                                 int32_t nrows) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = int64_t(gridDim.x) * (blockDim.x / 32);
    for (int64_t s = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; s < nslices; s += nw) {
        const int64_t base = sp[s];
        const int32_t width = static_cast<int32_t>((sp[s + 1] - base) >> 5);
        const int64_t i = s * 32 + lane;
        int32_t z0 = 0, len = 0;
        if (i < nrows) {
            z0 = rp[srow[i]];
            len = slen[i];
        }
        for (int32_t k = 0; k < width; ++k) {
            const int64_t dst = base + int64_t(k) * 32 + lane;
            col[dst] = k < len ? ci[z0 + k] : 0;
            val[dst] = k < len ? vals[z0 + k] : V(0.0f);
        }
    }
}

template <typename V>
static int fill_sell(nm_csr* A, int64_t total) {
    NM_CUDA_TRY(cudaMalloc(&A->d_sell_col, sizeof(int32_t) * size_t(total)));
    NM_CUDA_TRY(cudaMalloc(&A->d_sell_val, sizeof(V) * size_t(total)));
    const int64_t blocks = std::min<int64_t>((int64_t(A->sell_slices) + 7) / 8, 65535);
    sell_fill_kernel<V><<<static_cast<int>(std::max<int64_t>(1, blocks)), 256>>>(
        A->d_row_ptr, A->d_col_idx, static_cast<const V*>(A->d_values), A->d_sell_ptr,
        A->d_sell_row, A->d_sell_len, A->d_sell_col, static_cast<V*>(A->d_sell_val),
        A->sell_slices, A->nrows);
    NM_CHECK_LAUNCH();
    NM_CUDA_TRY(cudaDeviceSynchronize());
    return NM_OK;
}

template <typename V, typename X, typename A>
static int launch_sell(const nm_csr* Am, const X* x, X* y, cudaStream_t s) {
    static std::atomic<int> occ_cache{0};  // resident CTAs per SM (same on every device here)
    int occ = occ_cache.load(std::memory_order_relaxed);
    if (occ == 0) {
        NM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &occ, spmv_sell_kernel<V, X, A>, kSellThreads, 0));
        occ = occ > 0 ? occ : 1;
        occ_cache.store(occ, std::memory_order_relaxed);
    }
    const int64_t need = (int64_t(Am->sell_slices) + kSellThreads / 32 - 1) / (kSellThreads / 32);
    const int grid = static_cast<int>(
        std::max<int64_t>(1, std::min<int64_t>(need, int64_t(sm_count()) * occ)));
    spmv_sell_kernel<V, X, A><<<grid, kSellThreads, 0, s>>>(
        Am->d_sell_ptr, Am->d_sell_row, Am->d_sell_len, Am->d_sell_col,
        static_cast<const V*>(Am->d_sell_val), x, y, Am->sell_slices, Am->nrows);
    NM_CHECK_LAUNCH();
    return NM_OK;
}

int build_sell(nm_csr* A) {
    A->sell_tried = true;
    const int32_t n = A->nrows;
    const int32_t* rp = A->h_row_ptr.data();
    std::vector<int32_t> perm(n), lens(n);
    for (int32_t w0 = 0; w0 < n; w0 += kSellWindow) {
        const int32_t w1 = std::min(n, w0 + kSellWindow);
        for (int32_t i = w0; i < w1; ++i) perm[i] = i;
        std::stable_sort(perm.begin() + w0, perm.begin() + w1, [&](int32_t a, int32_t b) {
            return rp[a + 1] - rp[a] > rp[b + 1] - rp[b];
        });
    }
    for (int32_t i = 0; i < n; ++i) lens[i] = rp[perm[i] + 1] - rp[perm[i]];
    const int32_t ns = (n + 31) / 32;
    std::vector<int64_t> sp(size_t(ns) + 1, 0);
    for (int32_t s = 0; s < ns; ++s) {
        int32_t w = 0;
        for (int32_t i = s * 32; i < std::min(n, s * 32 + 32); ++i) w = std::max(w, lens[i]);
        sp[s + 1] = sp[s] + 32 * int64_t(w);
    }
    const int64_t total = sp[ns];
    // too much padding (a few very long rows among short ones): keep the
    // per-group gather kernel
    if (total > 2 * int64_t(A->nnz) + 32 * int64_t(kSellWindow)) return NM_OK;
    A->sell_slices = ns;
    NM_CUDA_TRY(cudaMalloc(&A->d_sell_ptr, sizeof(int64_t) * sp.size()));
    NM_CUDA_TRY(cudaMalloc(&A->d_sell_row, sizeof(int32_t) * size_t(n)));
    NM_CUDA_TRY(cudaMalloc(&A->d_sell_len, sizeof(int32_t) * size_t(n)));
    NM_CUDA_TRY(cudaMemcpy(A->d_sell_ptr, sp.data(), sizeof(int64_t) * sp.size(),
                           cudaMemcpyHostToDevice));
    NM_CUDA_TRY(cudaMemcpy(A->d_sell_row, perm.data(), sizeof(int32_t) * size_t(n),
                           cudaMemcpyHostToDevice));
    NM_CUDA_TRY(cudaMemcpy(A->d_sell_len, lens.data(), sizeof(int32_t) * size_t(n),
                           cudaMemcpyHostToDevice));
    int st = NM_OK;
    switch (A->dtype) {
        case NM_F64: st = fill_sell<double>(A, total); break;
        case NM_F32: st = fill_sell<float>(A, total); break;
        default: st = fill_sell<__nv_bfloat16>(A, total); break;
    }
    if (st != NM_OK) return st;
    A->sell_ready = true;
    return NM_OK;
}

// nb >= 0: only the row blocks [b0, b0 + nb) (their rows of y are written,
// no others).
template <typename V, typename X, typename A, int TILE, int STAGES>
static int launch_tile(const nm_csr* Am, const X* x, X* y, cudaStream_t s, int32_t b0,
                       int32_t nb) {
    CsrView<V> M = Am->view<V>();
    if (nb >= 0) {
        M.desc += b0;
        M.nblk = nb;
    }
    M.stage_x = (reinterpret_cast<uintptr_t>(x) % 16) == 0;
    constexpr size_t smem = spmv_smem_bytes<V, X, A, TILE, STAGES>();
    auto* fn = spmv_kernel<V, X, A, TILE, STAGES>;
    int occ = 0;
    int st = prepare_kernel(reinterpret_cast<const void*>(fn), kCtaThreads, smem, &occ);
    if (st != NM_OK) return st;
    unsigned int* err = device_error_word();
    if (!err) return fail(NM_ERR_CUDA, "spmv: cannot map the device error word");
    const int grid = std::max(1, std::min(spmv_grid(Am, occ), M.nblk));
    fn<<<grid, kCtaThreads, smem, s>>>(M, x, y, err);
    NM_CHECK_LAUNCH();
    return NM_OK;
}

// y[rows[i]] = (A x)[i]: a matrix of some rows of a longer one, each row's
// result written to its place in the longer y (the interior / boundary rows of
// a distributed slice).
struct MapStoreEpi {
    static constexpr bool kBlockSums = false;
    double* __restrict__ y;
    const int32_t* __restrict__ rows;
    __device__ __forceinline__ void operator()(int32_t row, double v) { y[__ldg(rows + row)] = v; }
    __device__ __forceinline__ double take() { return 0.0; }
    __device__ __forceinline__ void finish_block(int64_t, const BlockDesc&, double) {}
};

template <int TILE, int STAGES>
__global__ void __launch_bounds__(kCtaThreads)
    spmv_rows_kernel(const CsrView<double> M, const double* __restrict__ x, double* y,
                     const int32_t* rows, unsigned int* err) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    auto& sm = *reinterpret_cast<SpmvSmem<double, double, double, TILE, STAGES>*>(smem_raw);
    MapStoreEpi epi{y, rows};
    spmv_pipeline<double, double, double, TILE, STAGES>(M, x, sm, epi, err);
}

template <int TILE, int STAGES>
static int launch_rows_tile(const nm_csr* Am, const double* x, double* y, const int32_t* rows,
                            cudaStream_t s) {
    CsrView<double> M = Am->view<double>();
    M.stage_x = (reinterpret_cast<uintptr_t>(x) % 16) == 0;
    constexpr size_t smem = spmv_smem_bytes<double, double, double, TILE, STAGES>();
    auto* fn = spmv_rows_kernel<TILE, STAGES>;
    int occ = 0;
    int st = prepare_kernel(reinterpret_cast<const void*>(fn), kCtaThreads, smem, &occ);
    if (st != NM_OK) return st;
    unsigned int* err = device_error_word();
    if (!err) return fail(NM_ERR_CUDA, "spmv: cannot map the device error word");
    fn<<<spmv_grid(Am, occ), kCtaThreads, smem, s>>>(M, x, y, rows, err);
    NM_CHECK_LAUNCH();
    return NM_OK;
}

template <int TILE>
static int launch_rows_stages(const nm_csr* Am, const double* x, double* y, const int32_t* rows,
                              cudaStream_t s) {
    if (Am->tune.stages == 4) return launch_rows_tile<TILE, 4>(Am, x, y, rows, s);
    if (Am->tune.stages == 3) return launch_rows_tile<TILE, 3>(Am, x, y, rows, s);
    return launch_rows_tile<TILE, 2>(Am, x, y, rows, s);
}

int launch_spmv_rows(const nm_csr* A, const double* x, double* y, const int32_t* rows,
                     cudaStream_t s) {
    if (A->dtype != NM_F64) return fail(NM_ERR_TYPE, "spmv_rows: float64 matrices only");
    switch (A->tune.tile) {
        case 1024: return launch_rows_stages<1024>(A, x, y, rows, s);
        case 4096: return launch_rows_stages<4096>(A, x, y, rows, s);
        default: return launch_rows_stages<2048>(A, x, y, rows, s);
    }
}

template <typename V, typename X, typename A, int TILE>
static int launch_stages(const nm_csr* Am, const X* x, X* y, cudaStream_t s, int32_t b0,
                         int32_t nb) {
    if (Am->tune.stages == 4) return launch_tile<V, X, A, TILE, 4>(Am, x, y, s, b0, nb);
    if (Am->tune.stages == 3) return launch_tile<V, X, A, TILE, 3>(Am, x, y, s, b0, nb);
    return launch_tile<V, X, A, TILE, 2>(Am, x, y, s, b0, nb);
}

// nb >= 0: the row blocks [b0, b0 + nb) of the row-block kernel only.
template <typename V, typename X, typename A>
static int launch_typed(const nm_csr* Am, const X* x, X* y, cudaStream_t s, int32_t b0 = 0,
                        int32_t nb = -1) {
    if (Am->warp_gather) {
        if (nb >= 0) return fail(NM_ERR_RUNTIME, "spmv: block range on the gather kernel");
        return Am->tune.kernel == NM_KERNEL_SLICED && Am->sell_ready
                   ? launch_sell<V, X, A>(Am, x, y, s)
                   : launch_gather<V, X, A>(Am, x, y, s);
    }
    switch (Am->tune.tile) {
        case 1024: return launch_stages<V, X, A, 1024>(Am, x, y, s, b0, nb);
        case 2048: return launch_stages<V, X, A, 2048>(Am, x, y, s, b0, nb);
        case 4096: return launch_stages<V, X, A, 4096>(Am, x, y, s, b0, nb);
        default: return fail(NM_ERR_INVALID, "spmv: unsupported tile %d", Am->tune.tile);
    }
}

template <typename V, typename X, typename A, int TILE>
static size_t smem_stages(int stages) {
    switch (stages) {
        case 2: return spmv_smem_bytes<V, X, A, TILE, 2>();
        case 3: return spmv_smem_bytes<V, X, A, TILE, 3>();
        case 4: return spmv_smem_bytes<V, X, A, TILE, 4>();
        default: return 0;
    }
}

template <typename V, typename X, typename A>
static size_t smem_tile(int tile, int stages) {
    switch (tile) {
        case 1024: return smem_stages<V, X, A, 1024>(stages);
        case 2048: return smem_stages<V, X, A, 2048>(stages);
        case 4096: return smem_stages<V, X, A, 4096>(stages);
        default: return 0;
    }
}

size_t spmv_smem_for(int dtype, int tile, int stages) {
    switch (dtype) {
        case NM_F64: return smem_tile<double, double, double>(tile, stages);
        case NM_F32: return smem_tile<float, float, float>(tile, stages);
        case NM_BF16: return smem_tile<__nv_bfloat16, float, float>(tile, stages);
        default: return 0;
    }
}

// nb >= 0: the row blocks [b0, b0 + nb) only (row-block kernel).
static int launch_spmv_range(const nm_csr* A, const void* x, void* y, int32_t b0, int32_t nb,
                             cudaStream_t s) {
    switch (A->dtype) {
        case NM_F64:
            return launch_typed<double, double, double>(A, static_cast<const double*>(x),
                                                        static_cast<double*>(y), s, b0, nb);
        case NM_F32:
            return launch_typed<float, float, float>(A, static_cast<const float*>(x),
                                                     static_cast<float*>(y), s, b0, nb);
        case NM_BF16:
            return launch_typed<__nv_bfloat16, float, float>(A, static_cast<const float*>(x),
                                                             static_cast<float*>(y), s, b0, nb);
        default: return fail(NM_ERR_TYPE, "spmv: unknown dtype %d", A->dtype);
    }
}

int launch_spmv(const nm_csr* A, const void* x, void* y, cudaStream_t s) {
    return launch_spmv_range(A, x, y, 0, -1, s);
}

// ---------------------------------------------------------------------------
// Multi-RHS SpMV  Y(nrows,k) = A * X(ncols,k), row-major.
//
// A group of TPR = 2^tpr_log2 consecutive lanes owns one row; lane g of the
// group owns the columns g*VEC + m*TPR*VEC (m < CH) of the current column
// pass, VEC = 2 with 16-byte loads when k is even, CH sized to k at launch.  Each (row, column) sum
// runs serially in CSR order with unfused multiply/add, i.e. exactly the
// reference's per-(i,b) loop (src/batch_spmv_kernel.hpp:95-102).  The
// matrix entries of a row are read once per column pass and broadcast to the
// group; X rows are read as contiguous segments (coalesced).
// ---------------------------------------------------------------------------
constexpr int kBatchChunks = 4;  // most column chunks per lane in one pass
constexpr int kBatchNz = 4;      // nonzeros whose X rows are loaded together

template <int VEC, int CH>
__global__ void __launch_bounds__(kThreads)
    batch_spmv_kernel(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                      const double* __restrict__ vals, int32_t nrows, int32_t k, int tpr_log2,
                      const double* __restrict__ X, double* __restrict__ Y) {
    const int tpr = 1 << tpr_log2;
    const int64_t gtid = int64_t(blockIdx.x) * kThreads + threadIdx.x;
    const int64_t row = gtid >> tpr_log2;
    const int g = static_cast<int>(gtid & (tpr - 1));
    if (row >= nrows) return;
    const int32_t s0 = rp[row], s1 = rp[row + 1];
    const int pass_cols = tpr * VEC * CH;
    for (int c0 = 0; c0 < k; c0 += pass_cols) {
        double acc[CH][VEC];
#pragma unroll
        for (int m = 0; m < CH; ++m)
#pragma unroll
            for (int e = 0; e < VEC; ++e) acc[m][e] = 0.0;
        // kBatchNz nonzeros at a time: their columns and values first, then
        // all their X row segments in flight together, then the products
        // added in CSR order
        for (int32_t j0 = s0; j0 < s1; j0 += kBatchNz) {
            int64_t xr[kBatchNz];
            double v[kBatchNz];
#pragma unroll
            for (int q = 0; q < kBatchNz; ++q) {
                const bool in = j0 + q < s1;
                xr[q] = in ? int64_t(__ldg(ci + j0 + q)) * k : 0;
                v[q] = in ? __ldg(vals + j0 + q) : 0.0;
            }
            double xv[kBatchNz][CH][VEC];
#pragma unroll
            for (int q = 0; q < kBatchNz; ++q)
#pragma unroll
                for (int m = 0; m < CH; ++m) {
                    const int c = c0 + (m * tpr + g) * VEC;
                    if (j0 + q < s1 && c < k) {
                        if (VEC == 2) {
                            const double2 t = __ldg(reinterpret_cast<const double2*>(X + xr[q] + c));
                            xv[q][m][0] = t.x;
                            xv[q][m][VEC - 1] = t.y;
                        } else {
                            xv[q][m][0] = __ldg(X + xr[q] + c);
                        }
                    }
                }
#pragma unroll
            for (int q = 0; q < kBatchNz; ++q)
                if (j0 + q < s1) {
#pragma unroll
                    for (int m = 0; m < CH; ++m)
#pragma unroll
                        for (int e = 0; e < VEC; ++e)
                            acc[m][e] = add_rn(acc[m][e], mul_rn(v[q], xv[q][m][e]));
                }
        }
#pragma unroll
        for (int m = 0; m < CH; ++m) {
            const int c = c0 + (m * tpr + g) * VEC;
            if (c < k) {
                if (VEC == 2) {
                    *reinterpret_cast<double2*>(Y + row * k + c) =
                        make_double2(acc[m][0], acc[m][VEC - 1]);
                } else {
                    Y[row * k + c] = acc[m][0];
                }
            }
        }
    }
}

// One warp per row (k wide enough for the row's columns to span the warp),
// rows strided by the number of resident warps.  The warp reads a row's first
// 32 columns and values in one coalesced access, one row ahead, and its
// row_ptr entries two rows ahead, so the row's X loads are the only memory
// latency on its critical path; later 32-nonzero windows of longer rows are
// read when reached.  Columns and values reach the lanes by shuffles; each
// (row, column) sum is still serial in CSR order.  CTAs of 4 warps: the
// kernel needs ~96 registers, and small CTAs keep 5 of them (20 warps) on an
// SM where 256-thread CTAs fit only 2 (100^3 Laplacian, k = 128: 659 us
// against 802 us, and 788 us for the one-pass kernel above).
constexpr int kBatchWarpThreads = 128;

template <int VEC, int CH>
__global__ void __launch_bounds__(kBatchWarpThreads)
    batch_spmv_warp_kernel(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                           const double* __restrict__ vals, int32_t nrows, int32_t k,
                           const double* __restrict__ X, double* __restrict__ Y) {
    constexpr unsigned kFull = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    // Rows strided over all resident warps: the whole GPU sweeps the rows in
    // order, so the X rows a band of rows shares (the +-1, +-L and +-L^2
    // neighbours of a stencil) are read close together in time and stay in
    // L2 between their uses.  (A contiguous row range per CTA, for L1 reuse of
    // the +-1 neighbours, measured 1,025 us against 663 us on the 100^3
    // Laplacian with k = 128: the CTAs' separate sweeps overflow L2.)
    const int64_t r_end = nrows;
    const int64_t nw = int64_t(gridDim.x) * (kBatchWarpThreads / 32);
    int64_t row = (int64_t(blockIdx.x) * kBatchWarpThreads + threadIdx.x) >> 5;  // same for the warp
    if (row >= r_end) return;
    int32_t s0 = __ldg(rp + row), s1 = __ldg(rp + row + 1);
    int32_t c_nx = 0;
    double v_nx = 0.0;
    if (s0 + lane < s1) {
        c_nx = __ldg(ci + s0 + lane);
        v_nx = __ldg(vals + s0 + lane);
    }
    int32_t t0 = 0, t1 = 0;  // row_ptr entries of the next row
    if (row + nw < r_end) {
        t0 = __ldg(rp + row + nw);
        t1 = __ldg(rp + row + nw + 1);
    }
    const int pass_cols = 32 * VEC * CH;
    for (; row < r_end; row += nw) {
        const int32_t r_s0 = s0, r_s1 = s1;
        const int32_t c_first = c_nx;
        const double v_first = v_nx;
        // the next row's first window and the row_ptr entries of the one after
        s0 = t0;
        s1 = t1;
        c_nx = 0;
        v_nx = 0.0;
        if (s0 + lane < s1) {
            c_nx = __ldg(ci + s0 + lane);
            v_nx = __ldg(vals + s0 + lane);
        }
        if (row + 2 * nw < r_end) {
            t0 = __ldg(rp + row + 2 * nw);
            t1 = __ldg(rp + row + 2 * nw + 1);
        }
        for (int c0 = 0; c0 < k; c0 += pass_cols) {
            double acc[CH][VEC];
#pragma unroll
            for (int m = 0; m < CH; ++m)
#pragma unroll
                for (int e = 0; e < VEC; ++e) acc[m][e] = 0.0;
            for (int32_t w0 = r_s0; w0 < r_s1; w0 += 32) {
                int32_t cw = c_first;
                double vw = v_first;
                if (w0 != r_s0) {
                    cw = 0;
                    vw = 0.0;
                    if (w0 + lane < r_s1) {
                        cw = __ldg(ci + w0 + lane);
                        vw = __ldg(vals + w0 + lane);
                    }
                }
                const int wn = r_s1 - w0 < 32 ? r_s1 - w0 : 32;
                for (int j0 = 0; j0 < wn; j0 += kBatchNz) {
                    int64_t xr[kBatchNz];
                    double v[kBatchNz];
#pragma unroll
                    for (int q = 0; q < kBatchNz; ++q) {
                        const int jj = j0 + q;
                        const int32_t c = __shfl_sync(kFull, cw, jj & 31);
                        const double vv = __shfl_sync(kFull, vw, jj & 31);
                        xr[q] = jj < wn ? int64_t(c) * k : 0;
                        v[q] = jj < wn ? vv : 0.0;
                    }
                    double xv[kBatchNz][CH][VEC];
#pragma unroll
                    for (int q = 0; q < kBatchNz; ++q)
#pragma unroll
                        for (int m = 0; m < CH; ++m) {
                            const int c = c0 + (m * 32 + lane) * VEC;
                            if (j0 + q < wn && c < k) {
                                if (VEC == 2) {
                                    const double2 t =
                                        __ldg(reinterpret_cast<const double2*>(X + xr[q] + c));
                                    xv[q][m][0] = t.x;
                                    xv[q][m][VEC - 1] = t.y;
                                } else {
                                    xv[q][m][0] = __ldg(X + xr[q] + c);
                                }
                            }
                        }
#pragma unroll
                    for (int q = 0; q < kBatchNz; ++q)
                        if (j0 + q < wn) {
#pragma unroll
                            for (int m = 0; m < CH; ++m)
#pragma unroll
                                for (int e = 0; e < VEC; ++e)
                                    acc[m][e] = add_rn(acc[m][e], mul_rn(v[q], xv[q][m][e]));
                        }
                }
            }
#pragma unroll
            for (int m = 0; m < CH; ++m) {
                const int c = c0 + (m * 32 + lane) * VEC;
                if (c < k) {
                    if (VEC == 2) {
                        *reinterpret_cast<double2*>(Y + row * k + c) =
                            make_double2(acc[m][0], acc[m][VEC - 1]);
                    } else {
                        Y[row * k + c] = acc[m][0];
                    }
                }
            }
        }
    }
}

template <int VEC, int CH>
static int launch_batch_warp_t(const nm_csr* A, const double* X, double* Y, int32_t k,
                               cudaStream_t s) {
    static std::atomic<int> occ_cache{0};  // resident CTAs per SM (same on every device here)
    int occ = occ_cache.load(std::memory_order_relaxed);
    if (occ == 0) {
        NM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &occ, batch_spmv_warp_kernel<VEC, CH>, kBatchWarpThreads, 0));
        occ = occ > 0 ? occ : 1;
        occ_cache.store(occ, std::memory_order_relaxed);
    }
    constexpr int warps = kBatchWarpThreads / 32;
    const int64_t need = (int64_t(A->nrows) + warps - 1) / warps;
    const int grid = static_cast<int>(std::min<int64_t>(need, int64_t(sm_count()) * occ));
    batch_spmv_warp_kernel<VEC, CH><<<grid, kBatchWarpThreads, 0, s>>>(
        A->d_row_ptr, A->d_col_idx, static_cast<const double*>(A->d_values), A->nrows, k, X, Y);
    return NM_OK;
}

template <int VEC>
static int launch_batch_warp_v(const nm_csr* A, const double* X, double* Y, int32_t k, int ch,
                               cudaStream_t s) {
    if (ch >= 4) return launch_batch_warp_t<VEC, 4>(A, X, Y, k, s);
    if (ch >= 2) return launch_batch_warp_t<VEC, 2>(A, X, Y, k, s);
    return launch_batch_warp_t<VEC, 1>(A, X, Y, k, s);
}

template <int VEC, int CH>
static void launch_batch_t(const nm_csr* A, const double* X, double* Y, int32_t k, int tpr_log2,
                           int grid, cudaStream_t s) {
    batch_spmv_kernel<VEC, CH><<<grid, kThreads, 0, s>>>(
        A->d_row_ptr, A->d_col_idx, static_cast<const double*>(A->d_values), A->nrows, k,
        tpr_log2, X, Y);
}

template <int VEC>
static void launch_batch_v(const nm_csr* A, const double* X, double* Y, int32_t k, int tpr_log2,
                           int ch, int grid, cudaStream_t s) {
    if (ch >= 4) launch_batch_t<VEC, 4>(A, X, Y, k, tpr_log2, grid, s);
    else if (ch == 2 || ch == 3) launch_batch_t<VEC, 2>(A, X, Y, k, tpr_log2, grid, s);
    else launch_batch_t<VEC, 1>(A, X, Y, k, tpr_log2, grid, s);
}

static int launch_batch(const nm_csr* A, const double* X, double* Y, int32_t k, cudaStream_t s) {
    const bool vec2 = (k % 2 == 0) && (reinterpret_cast<uintptr_t>(X) % 16 == 0) &&
                      (reinterpret_cast<uintptr_t>(Y) % 16 == 0);
    const int vec = vec2 ? 2 : 1;
    const int groups = (k + vec - 1) / vec;  // lane-columns needed for one pass
    int tpr_log2 = 0;
    while ((1 << tpr_log2) < groups && tpr_log2 < 5) ++tpr_log2;
    // column chunks per lane: enough for k in one pass, at most kBatchChunks
    const int ch = std::min(kBatchChunks, (groups + (1 << tpr_log2) - 1) >> tpr_log2);
    const int64_t threads = int64_t(A->nrows) << tpr_log2;
    const int64_t grid = (threads + kThreads - 1) / kThreads;
    if (grid > INT32_MAX) return fail(NM_ERR_INVALID, "batch_spmv: problem too large");
    if (tpr_log2 == 5) {  // a warp per row: the prefetching kernel
        const int st = vec2 ? launch_batch_warp_v<2>(A, X, Y, k, ch, s)
                            : launch_batch_warp_v<1>(A, X, Y, k, ch, s);
        if (st != NM_OK) return st;
        NM_CHECK_LAUNCH();
        return NM_OK;
    }
    if (vec2) launch_batch_v<2>(A, X, Y, k, tpr_log2, ch, static_cast<int>(grid), s);
    else launch_batch_v<1>(A, X, Y, k, tpr_log2, ch, static_cast<int>(grid), s);
    NM_CHECK_LAUNCH();
    return NM_OK;
}

// ---------------------------------------------------------------------------
// y = A x with x and y in host memory (nm_spmv_host).
//
// x goes in as pieces on one stream and y comes out as chunks on another; the
// row blocks run in chunks on the caller's stream, each after the x pieces up
// to the last one its nonzeros read (found once per partition from the host
// copy of the column indices), and each chunk's rows of y leave while the
// next chunks compute.  A banded matrix's chunk waits for about one piece
// beyond its own rows, so the copy-out runs beside the copy-in and the call
// takes about one direction's transfer time instead of both.  The
// warp-gather kernels (scattered columns: every chunk would wait for all of
// x) and vectors of under two pieces run as one copy in, one SpMV, one copy
// out.
// ---------------------------------------------------------------------------

HostSpmv::~HostSpmv() {
    for (cudaEvent_t e : x_ready) cudaEventDestroy(e);
    for (cudaEvent_t e : y_ready) cudaEventDestroy(e);
    if (begin) cudaEventDestroy(begin);
    if (done) cudaEventDestroy(done);
    if (in) cudaStreamDestroy(in);
    if (out) cudaStreamDestroy(out);
    if (dx) cudaFree(dx);
    if (dy) cudaFree(dy);
}

namespace {

constexpr int64_t kHostPieceBytes = int64_t(2) << 20;  // x piece / y chunk size aimed at
constexpr int kHostMaxPieces = 16;
// A chunk also waits for the x elements up to this far past its largest
// column (the staged x windows end on multiples of 4 elements).
constexpr int64_t kHostXMargin = 8;

int host_vec_bytes(int dtype) { return dtype == NM_F64 ? 8 : 4; }

int host_pieces(int64_t n, int esz) {
    return int(std::max<int64_t>(1, std::min<int64_t>(kHostMaxPieces, n * esz / kHostPieceBytes)));
}

int grow_events(std::vector<cudaEvent_t>& ev, size_t n) {
    while (ev.size() < n) {
        cudaEvent_t e = nullptr;
        NM_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        ev.push_back(e);
    }
    return NM_OK;
}

// The split of x into pieces and of the row blocks into chunks (no chunks:
// one copy in, one SpMV, one copy out).
int plan_host_spmv(const nm_csr* A, HostSpmv* h) {
    const int esz = host_vec_bytes(A->dtype);
    h->xcut.clear();
    h->blk.clear();
    h->row.clear();
    h->need.clear();
    const int P = host_pieces(A->ncols, esz);
    const int C = std::min(host_pieces(A->nrows, esz), std::max(1, A->nblk));
    if (A->warp_gather || P < 2 || C < 2) return NM_OK;
    if (A->h_row_ptr.size() != size_t(A->nrows) + 1 || A->h_col_idx.size() < size_t(A->nnz))
        return NM_OK;  // no host copy of the pattern to find each chunk's columns
    for (int p = 0; p < P; ++p) {
        const int64_t c = (int64_t(A->ncols) * p / P) & ~int64_t(63);
        if (h->xcut.empty() || c > h->xcut.back()) h->xcut.push_back(c);
    }
    h->xcut.push_back(A->ncols);
    std::vector<int32_t> bh(size_t(A->nblk) + 1);
    NM_CUDA_TRY(cudaMemcpy(bh.data(), A->d_blk, sizeof(int32_t) * bh.size(),
                           cudaMemcpyDeviceToHost));
    h->blk.push_back(0);
    h->row.push_back(0);
    for (int c = 1; c < C; ++c) {
        const int64_t target = int64_t(A->nrows) * c / C;
        const int32_t b = int32_t(std::lower_bound(bh.begin(), bh.end(), target) - bh.begin());
        if (b <= h->blk.back() || b >= A->nblk) continue;
        h->blk.push_back(b);
        h->row.push_back(bh[b]);
    }
    h->blk.push_back(A->nblk);
    h->row.push_back(A->nrows);
    const int32_t* rp = A->h_row_ptr.data();
    const int32_t* ci = A->h_col_idx.data();
    for (size_t c = 0; c + 1 < h->blk.size(); ++c) {
        int32_t mx = -1;
        for (int32_t z = rp[h->row[c]]; z < rp[h->row[c + 1]]; ++z) mx = std::max(mx, ci[z]);
        int32_t need = -1;
        if (mx >= 0) {
            const int64_t last = std::min<int64_t>(int64_t(mx) + kHostXMargin, A->ncols - 1);
            need = int32_t(std::upper_bound(h->xcut.begin(), h->xcut.end(), last) -
                           h->xcut.begin()) - 1;
        }
        h->need.push_back(need);
    }
    int st = grow_events(h->x_ready, h->xcut.size() - 1);
    if (st == NM_OK) st = grow_events(h->y_ready, h->blk.size() - 1);
    return st;
}

int spmv_host(const nm_csr* A, const void* x, void* y, cudaStream_t s) {
    HostSpmv* h = nullptr;
    {
        std::lock_guard<std::mutex> g(A->host_mutex);
        if (!A->host_spmv) A->host_spmv.reset(new (std::nothrow) HostSpmv());
        h = A->host_spmv.get();
    }
    if (!h) return fail(NM_ERR_NOMEM, "spmv_host: out of host memory");
    std::lock_guard<std::mutex> g(h->mu);
    if (A->nrows == 0) return NM_OK;
    const int esz = host_vec_bytes(A->dtype);
    const size_t xb = size_t(A->ncols) * esz, yb = size_t(A->nrows) * esz;
    if (!h->dx && cudaMalloc(&h->dx, std::max<size_t>(xb, 16)) != cudaSuccess) {
        cudaGetLastError();
        h->dx = nullptr;
        return fail(NM_ERR_NOMEM, "spmv_host: cannot allocate the device x (%zu bytes)", xb);
    }
    if (!h->dy && cudaMalloc(&h->dy, yb) != cudaSuccess) {
        cudaGetLastError();
        h->dy = nullptr;
        return fail(NM_ERR_NOMEM, "spmv_host: cannot allocate the device y (%zu bytes)", yb);
    }
    if (!h->in) NM_CUDA_TRY(cudaStreamCreateWithFlags(&h->in, cudaStreamNonBlocking));
    if (!h->out) NM_CUDA_TRY(cudaStreamCreateWithFlags(&h->out, cudaStreamNonBlocking));
    if (!h->begin) NM_CUDA_TRY(cudaEventCreateWithFlags(&h->begin, cudaEventDisableTiming));
    if (!h->done) NM_CUDA_TRY(cudaEventCreateWithFlags(&h->done, cudaEventDisableTiming));
    if (h->gen != A->layout_gen) {
        const int st = plan_host_spmv(A, h);
        if (st != NM_OK) return st;
        h->gen = A->layout_gen;
    }
    int st = NM_OK;
    auto cu = [&](cudaError_t e, const char* what) {
        if (st == NM_OK && e != cudaSuccess)
            st = fail(NM_ERR_CUDA, "spmv_host: %s failed: %s", what, cudaGetErrorString(e));
    };
    char* dx = static_cast<char*>(h->dx);
    char* dy = static_cast<char*>(h->dy);
    if (h->blk.empty()) {
        if (xb) cu(cudaMemcpyAsync(dx, x, xb, cudaMemcpyHostToDevice, s), "copy of x");
        if (st == NM_OK) st = launch_spmv(A, dx, dy, s);
        if (st == NM_OK) cu(cudaMemcpyAsync(y, dy, yb, cudaMemcpyDeviceToHost, s), "copy of y");
        const cudaError_t e = cudaStreamSynchronize(s);
        cu(e, "stream synchronize");
        return st;
    }
    // Both copy streams start after the work already queued on s.
    cu(cudaEventRecord(h->begin, s), "event record");
    cu(cudaStreamWaitEvent(h->in, h->begin, 0), "stream wait");
    cu(cudaStreamWaitEvent(h->out, h->begin, 0), "stream wait");
    const char* xh = static_cast<const char*>(x);
    char* yh = static_cast<char*>(y);
    for (size_t p = 0; st == NM_OK && p + 1 < h->xcut.size(); ++p) {
        const int64_t a = h->xcut[p], b = h->xcut[p + 1];
        cu(cudaMemcpyAsync(dx + a * esz, xh + a * esz, size_t(b - a) * esz,
                           cudaMemcpyHostToDevice, h->in), "copy of x");
        cu(cudaEventRecord(h->x_ready[p], h->in), "event record");
    }
    int32_t waited = -1;  // the x pieces 0..waited are known to be in for s
    for (size_t c = 0; st == NM_OK && c + 1 < h->blk.size(); ++c) {
        if (h->need[c] > waited) {
            cu(cudaStreamWaitEvent(s, h->x_ready[h->need[c]], 0), "stream wait");
            waited = h->need[c];
        }
        if (st != NM_OK) break;
        st = launch_spmv_range(A, dx, dy, h->blk[c], h->blk[c + 1] - h->blk[c], s);
        if (st != NM_OK) break;
        cu(cudaEventRecord(h->y_ready[c], s), "event record");
        cu(cudaStreamWaitEvent(h->out, h->y_ready[c], 0), "stream wait");
        const int64_t r0 = h->row[c], r1 = h->row[c + 1];
        if (r1 > r0)
            cu(cudaMemcpyAsync(yh + r0 * esz, dy + r0 * esz, size_t(r1 - r0) * esz,
                               cudaMemcpyDeviceToHost, h->out), "copy of y");
    }
    cu(cudaEventRecord(h->done, h->out), "event record");
    cu(cudaStreamWaitEvent(s, h->done, 0), "stream wait");
    // Everything this call queued has finished before it returns, also after
    // a failure (the host buffers are the caller's again).
    const cudaError_t e1 = cudaStreamSynchronize(h->in);
    const cudaError_t e2 = cudaStreamSynchronize(h->out);
    const cudaError_t e3 = cudaStreamSynchronize(s);
    cu(e1, "stream synchronize");
    cu(e2, "stream synchronize");
    cu(e3, "stream synchronize");
    return st;
}

}  // namespace

}  // namespace nm

using nm::fail;

extern "C" int nm_spmv_host(const nm_csr* A, const void* x, void* y, void* stream) {
    nm::clear_error();
    if (!A) return fail(NM_ERR_INVALID, "nm_spmv_host: NULL matrix");
    if ((!x && A->ncols > 0) || (!y && A->nrows > 0))
        return fail(NM_ERR_INVALID, "nm_spmv_host: NULL argument");
    return nm::spmv_host(A, x, y, static_cast<cudaStream_t>(stream));
}

extern "C" int nm_spmv(const nm_csr* A, const void* x, void* y, void* stream) {
    nm::clear_error();
    if (!A || !x || !y) return fail(NM_ERR_INVALID, "nm_spmv: NULL argument");
    return nm::launch_spmv(A, x, y, static_cast<cudaStream_t>(stream));
}

extern "C" int nm_batch_spmv(const nm_csr* A, const double* X, double* Y, int32_t k,
                             void* stream) {
    nm::clear_error();
    if (!A || !X || !Y) return fail(NM_ERR_INVALID, "nm_batch_spmv: NULL argument");
    if (A->dtype != NM_F64) return fail(NM_ERR_TYPE, "batch_spmv: float64 matrices only");
    if (k < 0) return fail(NM_ERR_INVALID, "batch_spmv: k must be >= 0");
    if (k == 0) return NM_OK;  // launch_batch_spmv returns early for k == 0
    return nm::launch_batch(A, X, Y, k, static_cast<cudaStream_t>(stream));
}
