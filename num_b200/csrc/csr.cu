// csr.cu -- device CSR matrix: upload, validation, row-block partition.
//
// Replaces CrsMatrixHandle (src/crs_matrix.hpp:37-73) and the global
// rows-per-team pick of the reference custom kernel (src/spmv_kernel.hpp:102-109)
// with a per-row-block partition computed once at upload.
#include <algorithm>
#include <climits>
#include <cstring>
#include <string>
#include <thread>

#include "cg.cuh"
#include "csr.cuh"

namespace nm {

int build_row_blocks(const int32_t* rp, int32_t nrows, int tile, int max_rows, int short_max,
                     std::vector<int32_t>& blk, std::vector<int8_t>* bins) {
    blk.clear();
    blk.push_back(0);
    if (bins) bins->assign(static_cast<size_t>(nrows), 0);
    int32_t r = 0;
    while (r < nrows) {
        const int32_t len = rp[r + 1] - rp[r];
        if (len > tile) {
            if (bins) (*bins)[r] = 2;
            ++r;
        } else {
            const int32_t start = r;
            int64_t nz = 0;
            while (r < nrows && r - start < max_rows) {
                const int32_t l = rp[r + 1] - rp[r];
                if (nz + l > tile) break;
                if (bins) (*bins)[r] = static_cast<int8_t>(l <= short_max ? 0 : 1);
                nz += l;
                ++r;
            }
        }
        blk.push_back(r);
    }
    return static_cast<int>(blk.size()) - 1;
}

void block_xwindows(const int32_t* ci, int32_t z0, int32_t z1, int32_t ncols, int xw,
                    std::vector<int32_t>& c, int4* xs, int4* xl) {
    *xs = make_int4(-1, INT_MAX, INT_MAX, INT_MAX);
    *xl = make_int4(0, 0, 0, 0);
    if (z1 <= z0) return;
    int32_t cmin = ci[z0], cmax = ci[z0];
    for (int32_t j = z0 + 1; j < z1; ++j) {
        cmin = std::min(cmin, ci[j]);
        cmax = std::max(cmax, ci[j]);
    }
    const int64_t span = int64_t(cmax) - cmin + 1;
    if (span <= 64 * int64_t(z1 - z0)) {
        // narrow range: mark the columns in a bitmap, read them back in order
        std::vector<uint64_t> bits(size_t((span + 63) / 64), 0);
        for (int32_t j = z0; j < z1; ++j) {
            const int64_t o = ci[j] - cmin;
            bits[size_t(o >> 6)] |= uint64_t(1) << (o & 63);
        }
        c.clear();
        for (size_t w = 0; w < bits.size(); ++w)
            for (uint64_t m = bits[w]; m; m &= m - 1)
                c.push_back(cmin + int32_t(w * 64 + size_t(__builtin_ctzll(m))));
    } else {
        c.assign(ci + z0, ci + z1);
        std::sort(c.begin(), c.end());
    }
    int32_t st[kXSeg], en[kXSeg];
    int nseg = 0;
    int32_t cs = c[0] & ~3, ce = (c[0] | 3) + 1;
    for (size_t k = 1; k < c.size(); ++k) {
        const int32_t a = c[k] & ~3, e = (c[k] | 3) + 1;
        if (a <= ce + kXGap) {
            ce = std::max(ce, e);
        } else {
            if (nseg == kXSeg) return;  // too many windows: gather from global
            st[nseg] = cs;
            en[nseg] = ce;
            ++nseg;
            cs = a;
            ce = e;
        }
    }
    if (nseg == kXSeg) return;
    st[nseg] = cs;
    en[nseg] = ce;
    ++nseg;
    int64_t total = 0;
    for (int k = 0; k < nseg; ++k) total += en[k] - st[k];
    if (total > xw || en[nseg - 1] > (ncols & ~3)) return;  // too wide, or would read past x
    int32_t sv[kXSeg] = {INT_MAX, INT_MAX, INT_MAX, INT_MAX}, lv[kXSeg] = {0, 0, 0, 0};
    for (int k = 0; k < nseg; ++k) {
        sv[k] = st[k];
        lv[k] = en[k] - st[k];
    }
    *xs = make_int4(sv[0], sv[1], sv[2], sv[3]);
    *xl = make_int4(lv[0], lv[1], lv[2], lv[3]);
}

namespace {

size_t dtype_size(int dtype) {
    switch (dtype) {
        case NM_F64: return 8;
        case NM_F32: return 4;
        case NM_BF16: return 2;
        default: return 0;
    }
}

int normalise_tuning(nm_tuning& t) {
    if (t.tile <= 0) t.tile = kDefaultTile;
    if (t.max_rows <= 0) t.max_rows = kDefaultMaxRows;
    if (t.short_max <= 0) t.short_max = kDefaultShortMax;
    if (t.grid_mult < 0) t.grid_mult = 0;
    if (t.stages <= 0) t.stages = kDefaultStages;
    if (t.kernel <= 0) t.kernel = NM_KERNEL_AUTO;
    if (t.kernel > NM_KERNEL_SLICED)
        return fail(NM_ERR_INVALID, "tuning: kernel must be 1 (auto), 2 (blocks), 3 (gather) or "
                    "4 (sliced) (got %d)", t.kernel);
    if (t.stages < 2 || t.stages > 4)
        return fail(NM_ERR_INVALID, "tuning: stages must be 2, 3 or 4 (got %d)", t.stages);
    if (t.tile != 1024 && t.tile != 2048 && t.tile != 4096)
        return fail(NM_ERR_INVALID, "tuning: tile must be 1024, 2048 or 4096 (got %d)", t.tile);
    if (t.max_rows > kThreads)
        return fail(NM_ERR_INVALID, "tuning: max_rows must be <= %d (got %d)", kThreads,
                    t.max_rows);
    return NM_OK;
}

// Checks row_ptr (starts at 0, non-decreasing) and column bounds on the host.
int validate_csr(const int32_t* rp, const int32_t* ci, int32_t nrows, int32_t ncols,
                 const char* who) {
    if (rp[0] != 0) return fail(NM_ERR_INVALID, "%s: row_ptr[0] must be 0 (got %d)", who, rp[0]);
    for (int32_t i = 0; i < nrows; ++i)
        if (rp[i + 1] < rp[i])
            return fail(NM_ERR_INVALID, "%s: row_ptr decreases at row %d", who, i);
    const int32_t nnz = rp[nrows];
    if (nnz > INT32_MAX - 16384)
        return fail(NM_ERR_INVALID, "%s: nnz %d exceeds the int32 offset range", who, nnz);
    for (int32_t j = 0; j < nnz; ++j)
        if (ci[j] < 0 || ci[j] >= ncols)
            return fail(NM_ERR_INVALID, "%s: column index %d at nonzero %d outside [0, %d)", who,
                        ci[j], j, ncols);
    return NM_OK;
}

int upload(nm_csr* A, const int32_t* rp, const int32_t* ci, const void* vals) {
    const size_t es = dtype_size(A->dtype);
    const int64_t nnz_pad = ((static_cast<int64_t>(A->nnz) + 7) & ~int64_t(7)) + 8;
    const size_t rp_len = size_t(A->nrows) + 1 + 8;
    NM_CUDA_TRY(cudaMalloc(&A->d_row_ptr, sizeof(int32_t) * rp_len));
    NM_CUDA_TRY(cudaMalloc(&A->d_col_idx, sizeof(int32_t) * size_t(nnz_pad)));
    NM_CUDA_TRY(cudaMalloc(&A->d_values, es * size_t(nnz_pad)));
    {
        std::vector<int32_t> rpp(rp, rp + A->nrows + 1);
        rpp.resize(rp_len, rp[A->nrows]);
        NM_CUDA_TRY(cudaMemcpy(A->d_row_ptr, rpp.data(), sizeof(int32_t) * rp_len,
                               cudaMemcpyHostToDevice));
    }
    NM_CUDA_TRY(cudaMemset(A->d_col_idx, 0, sizeof(int32_t) * size_t(nnz_pad)));
    NM_CUDA_TRY(cudaMemset(A->d_values, 0, es * size_t(nnz_pad)));
    if (A->nnz > 0) {
        NM_CUDA_TRY(cudaMemcpy(A->d_col_idx, ci, sizeof(int32_t) * size_t(A->nnz),
                               cudaMemcpyHostToDevice));
        NM_CUDA_TRY(cudaMemcpy(A->d_values, vals, es * size_t(A->nnz), cudaMemcpyHostToDevice));
    }
    return NM_OK;
}

}  // namespace

int rebuild_blocks(nm_csr* A) {
    ++A->layout_gen;
    std::vector<int32_t> blk;
    A->nblk = build_row_blocks(A->h_row_ptr.data(), A->nrows, A->tune.tile, A->tune.max_rows,
                               A->tune.short_max, blk, nullptr);
    std::vector<BlockDesc> desc(size_t(A->nblk));
    const int32_t* rp = A->h_row_ptr.data();
    const int32_t* ci = A->h_col_idx.data();
    const int tile = A->tune.tile;
    const int short_max = A->tune.short_max;
    const int32_t nb = A->nblk, ncols = A->ncols;
    auto fill = [&](int32_t b0, int32_t b1) {
        std::vector<int32_t> scratch;
        for (int32_t b = b0; b < b1; ++b) {
            BlockDesc& d = desc[b];
            const int32_t z0 = rp[blk[b]], z1 = rp[blk[b + 1]];
            d.rz = make_int4(blk[b], blk[b + 1], z0, z1);
            int32_t nlong = 0;
            for (int32_t r = blk[b]; r < blk[b + 1]; ++r) nlong += (rp[r + 1] - rp[r]) > short_max;
            d.aux = make_int4(nlong, 0, 0, 0);
            if (z1 - z0 > tile) {
                d.xs = make_int4(-1, INT_MAX, INT_MAX, INT_MAX);
                d.xl = make_int4(0, 0, 0, 0);
            } else {
                block_xwindows(ci, z0, z1, ncols, xwin_capacity(tile), scratch, &d.xs, &d.xl);
            }
        }
    };
    const int nthr = static_cast<int>(std::min<int64_t>(
        std::max(1u, std::thread::hardware_concurrency()), std::max<int64_t>(1, nb / 256)));
    if (nthr <= 1) {
        fill(0, nb);
    } else {
        std::vector<std::thread> th;
        for (int i = 0; i < nthr; ++i)
            th.emplace_back(fill, int32_t(int64_t(nb) * i / nthr), int32_t(int64_t(nb) * (i + 1) / nthr));
        for (auto& t : th) t.join();
    }
    {
        // Scattered columns (at least 3/4 of the nonzeros in blocks without x
        // windows) and no long row: the plain SpMV gathers warp by warp.
        int64_t gathered = 0;
        for (int32_t b = 0; b < nb; ++b)
            if (desc[b].xs.x < 0) gathered += desc[b].rz.w - desc[b].rz.z;
        int32_t max_row = 0;
        for (int32_t r = 0; r < A->nrows; ++r) max_row = std::max(max_row, rp[r + 1] - rp[r]);
        const bool scattered = A->nnz > 0 && 4 * gathered >= 3 * int64_t(A->nnz) &&
                               max_row <= kWarpGatherMaxRow;
        A->warp_gather = A->tune.kernel == NM_KERNEL_GATHER ||
                         A->tune.kernel == NM_KERNEL_SLICED ||
                         (A->tune.kernel == NM_KERNEL_AUTO && scattered);
    }
    if (A->tune.kernel == NM_KERNEL_SLICED && !A->sell_tried) {
        const int st = build_sell(A);
        if (st != NM_OK) return st;
    }
    if (A->d_blk) {
        cudaFree(A->d_blk);
        A->d_blk = nullptr;
    }
    if (A->d_desc) {
        cudaFree(A->d_desc);
        A->d_desc = nullptr;
    }
    NM_CUDA_TRY(cudaMalloc(&A->d_blk, sizeof(int32_t) * blk.size()));
    NM_CUDA_TRY(cudaMalloc(&A->d_desc, sizeof(BlockDesc) * desc.size()));
    NM_CUDA_TRY(cudaMemcpy(A->d_blk, blk.data(), sizeof(int32_t) * blk.size(),
                           cudaMemcpyHostToDevice));
    NM_CUDA_TRY(cudaMemcpy(A->d_desc, desc.data(), sizeof(BlockDesc) * desc.size(),
                           cudaMemcpyHostToDevice));
    return NM_OK;
}

namespace {

int finish_create(nm_csr* A, const int32_t* rp, const int32_t* ci, const void* vals,
                  nm_csr** out) {
    int st = upload(A, rp, ci, vals);
    if (st == NM_OK) {
        A->h_row_ptr.assign(rp, rp + A->nrows + 1);
        A->h_col_idx.assign(ci, ci + A->nnz);
        st = rebuild_blocks(A);
    }
    if (st != NM_OK) {
        delete A;
        return st;
    }
    *out = A;
    return NM_OK;
}

}  // namespace

void reset_cg(nm_csr* A) {
    std::lock_guard<std::mutex> lock(A->cg_mutex);
    A->cg.reset();
}

int spmv_grid(const nm_csr* A, int ctas_per_sm) {
    // Persistent grid: every CTA that fits (or grid_mult per SM when set).
    const int mult = A->tune.grid_mult > 0 ? A->tune.grid_mult : ctas_per_sm;
    const int64_t g = int64_t(sm_count()) * mult;
    return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(g, A->nblk)));
}

}  // namespace nm

nm_csr::~nm_csr() {
    cg.reset();
    host_spmv.reset();
    if (d_row_ptr) cudaFree(d_row_ptr);
    if (d_col_idx) cudaFree(d_col_idx);
    if (d_values) cudaFree(d_values);
    if (d_blk) cudaFree(d_blk);
    if (d_desc) cudaFree(d_desc);
    if (d_sell_ptr) cudaFree(d_sell_ptr);
    if (d_sell_row) cudaFree(d_sell_row);
    if (d_sell_len) cudaFree(d_sell_len);
    if (d_sell_col) cudaFree(d_sell_col);
    if (d_sell_val) cudaFree(d_sell_val);
}

using nm::fail;

extern "C" int nm_csr_create(const int32_t* row_ptr, const int32_t* col_idx, const void* values,
                             int dtype, int32_t nrows, int32_t ncols, nm_csr** out) {
    nm::clear_error();
    if (!out) return fail(NM_ERR_INVALID, "nm_csr_create: out is NULL");
    *out = nullptr;
    if (nrows <= 0 || ncols <= 0)
        return fail(NM_ERR_INVALID, "CrsMatrixHandle: non-positive dimensions");
    if (nm::dtype_size(dtype) == 0) return fail(NM_ERR_TYPE, "nm_csr_create: unknown dtype %d", dtype);
    if (!row_ptr || (row_ptr[nrows] > 0 && (!col_idx || !values)))
        return fail(NM_ERR_INVALID, "nm_csr_create: NULL array");
    int st = nm::validate_csr(row_ptr, col_idx, nrows, ncols, "nm_csr_create");
    if (st != NM_OK) return st;
    auto* A = new nm_csr();
    cudaGetDevice(&A->device);
    A->nrows = nrows;
    A->ncols = ncols;
    A->nnz = row_ptr[nrows];
    A->dtype = dtype;
    A->tune = nm_tuning{0, 0, 0, 0, 0, 0};
    nm::normalise_tuning(A->tune);
    return nm::finish_create(A, row_ptr, col_idx, values, out);
}

extern "C" int nm_csr_create_batched(int32_t count, const int32_t* nrows, const int32_t* ncols,
                                     const int32_t* row_ptr, const int32_t* col_idx,
                                     const void* values, int dtype, nm_csr** out) {
    nm::clear_error();
    if (!out) return fail(NM_ERR_INVALID, "nm_csr_create_batched: out is NULL");
    *out = nullptr;
    if (count <= 0) return fail(NM_ERR_INVALID, "nm_csr_create_batched: count must be > 0");
    const size_t es = nm::dtype_size(dtype);
    if (es == 0) return fail(NM_ERR_TYPE, "nm_csr_create_batched: unknown dtype %d", dtype);
    std::vector<int32_t> row_off(count + 1, 0), col_off(count + 1, 0);
    int64_t tot_rows = 0, tot_cols = 0, tot_nnz = 0, rp_pos = 0;
    for (int32_t m = 0; m < count; ++m) {
        if (nrows[m] <= 0 || ncols[m] <= 0)
            return fail(NM_ERR_INVALID, "nm_csr_create_batched: matrix %d has non-positive dims", m);
        const int32_t* rp = row_ptr + rp_pos;
        char who[64];
        snprintf(who, sizeof who, "nm_csr_create_batched[%d]", m);
        int st = nm::validate_csr(rp, col_idx + tot_nnz, nrows[m], ncols[m], who);
        if (st != NM_OK) return st;
        tot_nnz += rp[nrows[m]];
        rp_pos += nrows[m] + 1;
        tot_rows += nrows[m];
        tot_cols += ncols[m];
        if (tot_rows > INT32_MAX - 1 || tot_cols > INT32_MAX - 1 || tot_nnz > INT32_MAX - 16384)
            return fail(NM_ERR_INVALID, "nm_csr_create_batched: totals exceed the int32 range");
        row_off[m + 1] = static_cast<int32_t>(tot_rows);
        col_off[m + 1] = static_cast<int32_t>(tot_cols);
    }
    // Block-diagonal assembly: global row_ptr and column indices shifted by
    // each matrix's column offset.
    std::vector<int32_t> grp(static_cast<size_t>(tot_rows) + 1);
    std::vector<int32_t> gci(static_cast<size_t>(tot_nnz));
    grp[0] = 0;
    int64_t nz_base = 0;
    rp_pos = 0;
    for (int32_t m = 0; m < count; ++m) {
        const int32_t* rp = row_ptr + rp_pos;
        for (int32_t i = 0; i < nrows[m]; ++i)
            grp[row_off[m] + i + 1] = static_cast<int32_t>(nz_base + rp[i + 1]);
        const int32_t nzm = rp[nrows[m]];
        for (int32_t j = 0; j < nzm; ++j)
            gci[nz_base + j] = col_idx[nz_base + j] + col_off[m];
        nz_base += nzm;
        rp_pos += nrows[m] + 1;
    }
    auto* A = new nm_csr();
    cudaGetDevice(&A->device);
    A->nrows = static_cast<int32_t>(tot_rows);
    A->ncols = static_cast<int32_t>(tot_cols);
    A->nnz = static_cast<int32_t>(tot_nnz);
    A->dtype = dtype;
    A->tune = nm_tuning{0, 0, 0, 0, 0, 0};
    nm::normalise_tuning(A->tune);
    A->batch_row_off = row_off;
    A->batch_col_off = col_off;
    return nm::finish_create(A, grp.data(), gci.data(), values, out);
}

extern "C" int nm_csr_laplacian(int32_t dim, int32_t L, int dtype, nm_csr** out) {
    nm::clear_error();
    if (!out) return fail(NM_ERR_INVALID, "nm_csr_laplacian: out is NULL");
    *out = nullptr;
    if (dim != 2 && dim != 3)
        return fail(NM_ERR_INVALID, "nm_csr_laplacian: dim must be 2 or 3 (got %d)", dim);
    if (L <= 0) return fail(NM_ERR_INVALID, "CrsMatrixHandle: non-positive dimensions");
    const size_t es = nm::dtype_size(dtype);
    if (es == 0) return fail(NM_ERR_TYPE, "nm_csr_laplacian: unknown dtype %d", dtype);
    // L^dim rows and their nonzeros must fit the int32 offsets (checked in
    // 64 bits; L above 46,341 / 1,291 already overflows the rows).
    if ((dim == 2 && L > 46341) || (dim == 3 && L > 1291))
        return fail(NM_ERR_INVALID, "nm_csr_laplacian: L = %d exceeds the int32 row range", L);
    const int64_t n = dim == 2 ? int64_t(L) * L : int64_t(L) * L * L;
    const int64_t nnz = nm::stencil_nnz(dim, L);
    if (n > INT32_MAX || nnz > INT32_MAX - 16384)
        return fail(NM_ERR_INVALID,
                    "nm_csr_laplacian: L = %d gives %lld rows / %lld nonzeros, beyond the int32 "
                    "offset range", L, (long long)n, (long long)nnz);
    auto* A = new nm_csr();
    cudaGetDevice(&A->device);
    A->nrows = A->ncols = static_cast<int32_t>(n);
    A->nnz = static_cast<int32_t>(nnz);
    A->dtype = dtype;
    A->tune = nm_tuning{0, 0, 0, 0, 0, 0};
    nm::normalise_tuning(A->tune);
    auto build = [&]() -> int {
        // Same allocation and padding as an uploaded matrix.
        const int64_t nnz_pad = ((nnz + 7) & ~int64_t(7)) + 8;
        const int64_t rp_len = n + 1 + 8;
        NM_CUDA_TRY(cudaMalloc(&A->d_row_ptr, sizeof(int32_t) * size_t(rp_len)));
        NM_CUDA_TRY(cudaMalloc(&A->d_col_idx, sizeof(int32_t) * size_t(nnz_pad)));
        NM_CUDA_TRY(cudaMalloc(&A->d_values, es * size_t(nnz_pad)));
        NM_CUDA_TRY(cudaMemset(A->d_col_idx + nnz, 0, sizeof(int32_t) * size_t(nnz_pad - nnz)));
        NM_CUDA_TRY(cudaMemset(static_cast<char*>(A->d_values) + es * size_t(nnz), 0,
                               es * size_t(nnz_pad - nnz)));
        int st = nm::launch_laplacian(dim, L, dtype, A->d_row_ptr, rp_len, A->d_col_idx,
                                      A->d_values, nullptr);
        if (st != NM_OK) return st;
        // The row-block partition is built on the host from row_ptr and the
        // columns (as for an uploaded matrix): read them back once.
        A->h_row_ptr.resize(size_t(n) + 1);
        A->h_col_idx.resize(size_t(nnz));
        NM_CUDA_TRY(cudaMemcpy(A->h_row_ptr.data(), A->d_row_ptr, sizeof(int32_t) * size_t(n + 1),
                               cudaMemcpyDeviceToHost));
        NM_CUDA_TRY(cudaMemcpy(A->h_col_idx.data(), A->d_col_idx, sizeof(int32_t) * size_t(nnz),
                               cudaMemcpyDeviceToHost));
        return nm::rebuild_blocks(A);
    };
    const int st = build();
    if (st != NM_OK) {
        delete A;
        return st;
    }
    *out = A;
    return NM_OK;
}

extern "C" int nm_csr_export(const nm_csr* A, int32_t* row_ptr, int32_t* col_idx, void* values) {
    nm::clear_error();
    if (!A || !row_ptr || (A->nnz > 0 && (!col_idx || !values)))
        return fail(NM_ERR_INVALID, "nm_csr_export: NULL argument");
    NM_CUDA_TRY(cudaMemcpy(row_ptr, A->d_row_ptr, sizeof(int32_t) * (size_t(A->nrows) + 1),
                           cudaMemcpyDeviceToHost));
    if (A->nnz > 0) {
        NM_CUDA_TRY(cudaMemcpy(col_idx, A->d_col_idx, sizeof(int32_t) * size_t(A->nnz),
                               cudaMemcpyDeviceToHost));
        NM_CUDA_TRY(cudaMemcpy(values, A->d_values, nm::dtype_size(A->dtype) * size_t(A->nnz),
                               cudaMemcpyDeviceToHost));
    }
    return NM_OK;
}

extern "C" int nm_csr_destroy(nm_csr* A) {
    nm::clear_error();
    delete A;
    return NM_OK;
}

extern "C" int nm_csr_info(const nm_csr* A, int32_t* nrows, int32_t* ncols, int32_t* nnz,
                           int32_t* dtype, int32_t* nblocks) {
    nm::clear_error();
    if (!A) return fail(NM_ERR_INVALID, "nm_csr_info: NULL matrix");
    if (nrows) *nrows = A->nrows;
    if (ncols) *ncols = A->ncols;
    if (nnz) *nnz = A->nnz;
    if (dtype) *dtype = A->dtype;
    if (nblocks) *nblocks = A->nblk;
    return NM_OK;
}

extern "C" int nm_csr_set_tuning(nm_csr* A, const nm_tuning* t) {
    nm::clear_error();
    if (!A || !t) return fail(NM_ERR_INVALID, "nm_csr_set_tuning: NULL argument");
    nm_tuning nt = *t;
    if (nt.tile <= 0) nt.tile = A->tune.tile;
    if (nt.max_rows <= 0) nt.max_rows = A->tune.max_rows;
    if (nt.short_max <= 0) nt.short_max = A->tune.short_max;
    if (nt.grid_mult < 0) nt.grid_mult = A->tune.grid_mult;
    if (nt.stages <= 0) nt.stages = A->tune.stages;
    if (nt.kernel <= 0) nt.kernel = A->tune.kernel;
    int st = nm::normalise_tuning(nt);
    if (st != NM_OK) return st;
    {
        // Cached CG graphs hold the old partition; drop them.
        std::lock_guard<std::mutex> lock(A->cg_mutex);
        A->cg.reset();
    }
    A->tune = nt;
    return nm::rebuild_blocks(A);
}

extern "C" int nm_csr_spmv_kernel(const nm_csr* A, int32_t* kernel) {
    nm::clear_error();
    if (!A || !kernel) return fail(NM_ERR_INVALID, "nm_csr_spmv_kernel: NULL argument");
    *kernel = !A->warp_gather ? NM_KERNEL_BLOCKS
              : (A->tune.kernel == NM_KERNEL_SLICED && A->sell_ready ? NM_KERNEL_SLICED
                                                                      : NM_KERNEL_GATHER);
    return NM_OK;
}

extern "C" int nm_csr_get_tuning(const nm_csr* A, nm_tuning* t) {
    nm::clear_error();
    if (!A || !t) return fail(NM_ERR_INVALID, "nm_csr_get_tuning: NULL argument");
    *t = A->tune;
    return NM_OK;
}

extern "C" int nm_csr_row_blocks(const nm_csr* A, int32_t* blk, int32_t cap, int8_t* bins) {
    nm::clear_error();
    if (!A || !blk) return fail(NM_ERR_INVALID, "nm_csr_row_blocks: NULL argument");
    std::vector<int32_t> b;
    std::vector<int8_t> bn;
    nm::build_row_blocks(A->h_row_ptr.data(), A->nrows, A->tune.tile, A->tune.max_rows,
                         A->tune.short_max, b, bins ? &bn : nullptr);
    if (static_cast<int64_t>(b.size()) > cap)
        return fail(NM_ERR_INVALID, "nm_csr_row_blocks: cap %d < %zu", cap, b.size());
    // The host copy is what the device holds; read the device copy back to
    // report exactly what the kernels use.
    NM_CUDA_TRY(cudaMemcpy(blk, A->d_blk, sizeof(int32_t) * size_t(A->nblk + 1),
                           cudaMemcpyDeviceToHost));
    if (bins) std::memcpy(bins, bn.data(), bn.size());
    return NM_OK;
}
