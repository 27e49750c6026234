// dist.cu -- one rank's slice of a row-distributed matrix, its halo plan, and
// the halo pack / unpack kernels.
//
// Host planning restates distribute_csr (src/dist_spmv.hpp:27-100),
// build_ghost_map (src/halo_exchange.hpp:38-130) and build_send_indices
// (src/halo_exchange.hpp:154-191) for rank `rank` of `size` without a
// communicator: every rank is given the global CSR (as in the reference), so
// the lists another rank would have sent over MPI are computed locally from
// that rank's rows.  The resulting lists are the reference's, entry for entry:
//   * rows split evenly, the first n % size ranks get one extra row;
//   * ghost ids grouped per owner rank, ascending, owners in rank order,
//     offsets assigned in that order;
//   * send list for neighbour q = the ids q requests from this rank,
//     ascending, neighbours in rank order; packed as LOCAL indices.
#include <algorithm>
#include <string>
#include <unordered_map>
#include <vector>

#include "csr.cuh"

struct nm_dist {
    int32_t global_nrows = 0, global_ncols = 0;
    int32_t rank = 0, size = 1;
    int32_t row_start = 0, row_end = 0;
    int32_t n_ghost = 0, total_send = 0;
    std::vector<int32_t> send_rank, send_count, send_off, send_idx;  // local indices
    std::vector<int32_t> recv_rank, recv_count, recv_off, ghost_ids;  // global ids
    std::vector<int32_t> local_rp, local_ci;  // remapped local CSR (host copy)
    std::vector<double> local_vals;
    nm_csr* local = nullptr;
    int32_t* d_send_idx = nullptr;
    // Interior rows (every column owned) and boundary rows (some ghost
    // column) as separate matrices, with their local row numbers, so the
    // interior can be multiplied while the halo is exchanged.
    int32_t n_interior = 0, n_boundary = 0;
    nm_csr* interior = nullptr;   // columns in [0, local_n): reads x_local
    nm_csr* boundary = nullptr;   // columns in [0, local_n + n_ghost): reads x_ext
    int32_t* d_rows = nullptr;    // interior row numbers, then boundary row numbers
    ~nm_dist() {
        if (local) nm_csr_destroy(local);
        if (interior) nm_csr_destroy(interior);
        if (boundary) nm_csr_destroy(boundary);
        if (d_send_idx) cudaFree(d_send_idx);
        if (d_rows) cudaFree(d_rows);
    }
};

namespace nm {
namespace {

void row_range(int32_t n, int32_t size, int32_t r, int32_t* start, int32_t* end) {
    const int32_t base = n / size, extra = n % size;
    *start = r * base + std::min(r, extra);
    *end = *start + base + (r < extra ? 1 : 0);
}

// Owner of a global column; -1 if outside [0, n).  (The reference scans the
// gathered ranges; the even split makes the owner computable directly.)
int32_t owner_of(int32_t col, int32_t n, int32_t size) {
    if (col < 0 || col >= n) return -1;
    const int32_t base = n / size, extra = n % size;
    const int64_t big = int64_t(extra) * (base + 1);
    if (col < big) return static_cast<int32_t>(col / (base + 1));
    return static_cast<int32_t>(extra + (col - big) / base);
}

// Sorted unique off-range columns of rows [s, e) owned by rank `owner`.
std::vector<int32_t> requested(const int32_t* rp, const int32_t* ci, int32_t s, int32_t e,
                               int32_t owner_start, int32_t owner_end) {
    std::vector<int32_t> ids;
    for (int32_t i = s; i < e; ++i)
        for (int32_t j = rp[i]; j < rp[i + 1]; ++j)
            if (ci[j] >= owner_start && ci[j] < owner_end) ids.push_back(ci[j]);
    std::sort(ids.begin(), ids.end());
    ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
    return ids;
}

__global__ void halo_pack_kernel(int32_t total, const int32_t* __restrict__ idx,
                                 const double* __restrict__ x, double* __restrict__ buf) {
    for (int32_t i = blockIdx.x * kThreads + threadIdx.x; i < total; i += gridDim.x * kThreads)
        buf[i] = x[idx[i]];
}

__global__ void halo_unpack_kernel(int32_t n_ghost, int32_t local_n,
                                   const double* __restrict__ rbuf, double* __restrict__ x_ext) {
    for (int32_t i = blockIdx.x * kThreads + threadIdx.x; i < n_ghost; i += gridDim.x * kThreads)
        x_ext[local_n + i] = rbuf[i];
}

int small_grid(int64_t n) {
    return static_cast<int>(std::max<int64_t>(
        1, std::min<int64_t>((n + kThreads - 1) / kThreads, int64_t(sm_count()) * 4)));
}

}  // namespace

int cg_run(nm_csr* A, const double* b, double* x, double tol, int32_t max_iter, int guard,
           nm_cg_result* res, cudaStream_t s);

}  // namespace nm

using nm::fail;

static void copy_out(const std::vector<int32_t>& v, int32_t* dst) {
    if (dst && !v.empty()) std::copy(v.begin(), v.end(), dst);
}

static int dist_build(const int32_t* rp, const int32_t* ci, const double* vals, int32_t n,
                      int32_t ncols, int32_t rank, int32_t size, bool upload, nm_dist** out) {
    if (!out) return fail(NM_ERR_INVALID, "nm_dist_create: out is NULL");
    *out = nullptr;
    if (n <= 0 || ncols <= 0) return fail(NM_ERR_INVALID, "CrsMatrixHandle: non-positive dimensions");
    if (size <= 0 || rank < 0 || rank >= size)
        return fail(NM_ERR_INVALID, "nm_dist_create: rank %d outside [0, %d)", rank, size);
    if (!rp) return fail(NM_ERR_INVALID, "nm_dist_create: NULL row_ptr");
    if (rp[0] != 0) return fail(NM_ERR_INVALID, "nm_dist_create: row_ptr[0] must be 0");
    for (int32_t i = 0; i < n; ++i)
        if (rp[i + 1] < rp[i]) return fail(NM_ERR_INVALID, "nm_dist_create: row_ptr decreases");

    auto D = std::make_unique<nm_dist>();
    D->global_nrows = n;
    D->global_ncols = ncols;
    D->rank = rank;
    D->size = size;
    nm::row_range(n, size, rank, &D->row_start, &D->row_end);
    const int32_t s = D->row_start, e = D->row_end, ln = e - s;

    // Local slice with global columns (src/dist_spmv.hpp:45-55).
    const int32_t z0 = rp[s], z1 = rp[e];
    std::vector<int32_t> lr(ln + 1), lc(ci + z0, ci + z1);
    for (int32_t i = 0; i <= ln; ++i) lr[i] = rp[s + i] - z0;

    // Ghost lists per owner (src/halo_exchange.hpp:62-72, 108-129).
    std::vector<std::vector<int32_t>> want(size);
    for (int32_t col : lc) {
        if (col >= s && col < e) continue;
        const int32_t o = nm::owner_of(col, n, size);
        if (o < 0)
            return fail(NM_ERR_RUNTIME,
                        "build_ghost_map: column index %d is out of the global row range", col);
        want[o].push_back(col);
    }
    int32_t off = 0;
    std::unordered_map<int32_t, int32_t> ghost_pos;
    for (int32_t r = 0; r < size; ++r) {
        if (r == rank) continue;
        auto& w = want[r];
        if (!w.empty()) {
            std::sort(w.begin(), w.end());
            w.erase(std::unique(w.begin(), w.end()), w.end());
            D->recv_rank.push_back(r);
            D->recv_count.push_back(static_cast<int32_t>(w.size()));
            D->recv_off.push_back(off);
            for (size_t i = 0; i < w.size(); ++i) {
                ghost_pos[w[i]] = off + static_cast<int32_t>(i);
                D->ghost_ids.push_back(w[i]);
            }
            off += static_cast<int32_t>(w.size());
        }
        // What rank r requests from this rank (its recv list for us).
        int32_t rs, re;
        nm::row_range(n, size, r, &rs, &re);
        std::vector<int32_t> req = nm::requested(rp, ci, rs, re, s, e);
        if (!req.empty()) {
            D->send_rank.push_back(r);
            D->send_count.push_back(static_cast<int32_t>(req.size()));
            D->send_off.push_back(static_cast<int32_t>(D->send_idx.size()));
            for (int32_t gid : req) D->send_idx.push_back(gid - s);  // build_send_indices
        }
    }
    D->n_ghost = off;
    D->total_send = static_cast<int32_t>(D->send_idx.size());

    // Column remap global -> [own | ghost] (src/dist_spmv.hpp:62-81).
    for (auto& col : lc) {
        if (col >= s && col < e) {
            col -= s;
        } else {
            auto it = ghost_pos.find(col);
            if (it == ghost_pos.end())
                return fail(NM_ERR_RUNTIME, "distribute_csr: ghost column %d not found in ghost map",
                            col);
            col = ln + it->second;
        }
    }
    D->local_rp = std::move(lr);
    D->local_ci = std::move(lc);
    if (vals) D->local_vals.assign(vals + z0, vals + z1);
    else D->local_vals.assign(size_t(z1 - z0), 0.0);
    // Interior / boundary split of the local rows (the overlap the reference
    // describes as future work, src/halo_exchange.hpp:28-33).
    std::vector<int32_t> rows_ib;  // interior rows, then boundary rows
    {
        std::vector<int32_t> brows;
        for (int32_t r = 0; r < ln; ++r) {
            bool ghost = false;
            for (int32_t j = D->local_rp[r]; j < D->local_rp[r + 1]; ++j) ghost |= D->local_ci[j] >= ln;
            (ghost ? brows : rows_ib).push_back(r);
        }
        D->n_interior = static_cast<int32_t>(rows_ib.size());
        D->n_boundary = static_cast<int32_t>(brows.size());
        rows_ib.insert(rows_ib.end(), brows.begin(), brows.end());
    }
    if (!upload) {
        *out = D.release();
        return NM_OK;
    }
    if (ln > 0) {
        int st = nm_csr_create(D->local_rp.data(), D->local_ci.data(), D->local_vals.data(),
                               NM_F64, ln, ln + D->n_ghost, &D->local);
        if (st != NM_OK) return st;
    }
    if (ln > 0 && D->n_ghost > 0) {
        // the two row subsets as matrices of their own (rows in local order)
        auto subset = [&](int32_t first, int32_t count, int32_t ncols_sub, nm_csr** outm) {
            std::vector<int32_t> srp(1, 0), sci;
            std::vector<double> sv;
            for (int32_t k = first; k < first + count; ++k) {
                const int32_t r = rows_ib[k];
                for (int32_t j = D->local_rp[r]; j < D->local_rp[r + 1]; ++j) {
                    sci.push_back(D->local_ci[j]);
                    sv.push_back(D->local_vals[j]);
                }
                srp.push_back(static_cast<int32_t>(sci.size()));
            }
            return nm_csr_create(srp.data(), sci.data(), sv.data(), NM_F64, count, ncols_sub, outm);
        };
        if (D->n_interior > 0) {
            int st = subset(0, D->n_interior, ln, &D->interior);
            if (st != NM_OK) return st;
        }
        if (D->n_boundary > 0) {
            int st = subset(D->n_interior, D->n_boundary, ln + D->n_ghost, &D->boundary);
            if (st != NM_OK) return st;
        }
        NM_CUDA_TRY(cudaMalloc(&D->d_rows, sizeof(int32_t) * size_t(ln)));
        NM_CUDA_TRY(cudaMemcpy(D->d_rows, rows_ib.data(), sizeof(int32_t) * size_t(ln),
                               cudaMemcpyHostToDevice));
    }
    if (D->total_send > 0) {
        NM_CUDA_TRY(cudaMalloc(&D->d_send_idx, sizeof(int32_t) * size_t(D->total_send)));
        NM_CUDA_TRY(cudaMemcpy(D->d_send_idx, D->send_idx.data(),
                               sizeof(int32_t) * size_t(D->total_send), cudaMemcpyHostToDevice));
    }
    *out = D.release();
    return NM_OK;
}

extern "C" int nm_dist_create(const int32_t* rp, const int32_t* ci, const double* vals,
                              int32_t n, int32_t ncols, int32_t rank, int32_t size,
                              nm_dist** out) {
    nm::clear_error();
    return dist_build(rp, ci, vals, n, ncols, rank, size, true, out);
}

extern "C" int nm_dist_plan(const int32_t* rp, const int32_t* ci, const double* vals, int32_t n,
                            int32_t ncols, int32_t rank, int32_t size, nm_dist** out) {
    nm::clear_error();
    return dist_build(rp, ci, vals, n, ncols, rank, size, false, out);
}

extern "C" int nm_dist_local_host(const nm_dist* D, int32_t* local_nnz, int32_t* row_ptr,
                                  int32_t* col_idx, double* values) {
    nm::clear_error();
    if (!D) return fail(NM_ERR_INVALID, "nm_dist_local_host: NULL handle");
    if (local_nnz) *local_nnz = static_cast<int32_t>(D->local_ci.size());
    copy_out(D->local_rp, row_ptr);
    copy_out(D->local_ci, col_idx);
    if (values && !D->local_vals.empty())
        std::copy(D->local_vals.begin(), D->local_vals.end(), values);
    return NM_OK;
}

extern "C" int nm_dist_destroy(nm_dist* D) {
    nm::clear_error();
    delete D;
    return NM_OK;
}

extern "C" int nm_dist_info(const nm_dist* D, int32_t* global_nrows, int32_t* row_start,
                            int32_t* row_end, int32_t* n_ghost, int32_t* total_send,
                            int32_t* n_send_nbrs, int32_t* n_recv_nbrs) {
    nm::clear_error();
    if (!D) return fail(NM_ERR_INVALID, "nm_dist_info: NULL handle");
    if (global_nrows) *global_nrows = D->global_nrows;
    if (row_start) *row_start = D->row_start;
    if (row_end) *row_end = D->row_end;
    if (n_ghost) *n_ghost = D->n_ghost;
    if (total_send) *total_send = D->total_send;
    if (n_send_nbrs) *n_send_nbrs = static_cast<int32_t>(D->send_rank.size());
    if (n_recv_nbrs) *n_recv_nbrs = static_cast<int32_t>(D->recv_rank.size());
    return NM_OK;
}

extern "C" int nm_dist_send_plan(const nm_dist* D, int32_t* nbr_rank, int32_t* count,
                                 int32_t* offset, int32_t* send_idx) {
    nm::clear_error();
    if (!D) return fail(NM_ERR_INVALID, "nm_dist_send_plan: NULL handle");
    copy_out(D->send_rank, nbr_rank);
    copy_out(D->send_count, count);
    copy_out(D->send_off, offset);
    copy_out(D->send_idx, send_idx);
    return NM_OK;
}

extern "C" int nm_dist_recv_plan(const nm_dist* D, int32_t* nbr_rank, int32_t* count,
                                 int32_t* offset, int32_t* ghost_ids) {
    nm::clear_error();
    if (!D) return fail(NM_ERR_INVALID, "nm_dist_recv_plan: NULL handle");
    copy_out(D->recv_rank, nbr_rank);
    copy_out(D->recv_count, count);
    copy_out(D->recv_off, offset);
    copy_out(D->ghost_ids, ghost_ids);
    return NM_OK;
}

extern "C" int nm_dist_local(const nm_dist* D, const nm_csr** local) {
    nm::clear_error();
    if (!D || !local) return fail(NM_ERR_INVALID, "nm_dist_local: NULL argument");
    *local = D->local;
    return NM_OK;
}

extern "C" int nm_halo_pack(const nm_dist* D, const double* x_local, double* send_buf,
                            void* stream) {
    nm::clear_error();
    if (!D) return fail(NM_ERR_INVALID, "nm_halo_pack: NULL handle");
    if (D->total_send == 0) return NM_OK;
    if (!D->d_send_idx) return fail(NM_ERR_INVALID, "nm_halo_pack: host-only plan handle");
    if (!x_local || !send_buf) return fail(NM_ERR_INVALID, "nm_halo_pack: NULL buffer");
    nm::halo_pack_kernel<<<nm::small_grid(D->total_send), nm::kThreads, 0,
                           static_cast<cudaStream_t>(stream)>>>(D->total_send, D->d_send_idx,
                                                                x_local, send_buf);
    NM_CHECK_LAUNCH();
    return NM_OK;
}

extern "C" int nm_halo_unpack(const nm_dist* D, const double* recv_buf, double* x_ext,
                              void* stream) {
    nm::clear_error();
    if (!D) return fail(NM_ERR_INVALID, "nm_halo_unpack: NULL handle");
    if (D->n_ghost == 0) return NM_OK;  // halo_exchange returns early (halo_exchange.hpp:217)
    if (!recv_buf || !x_ext) return fail(NM_ERR_INVALID, "nm_halo_unpack: NULL buffer");
    nm::halo_unpack_kernel<<<nm::small_grid(D->n_ghost), nm::kThreads, 0,
                             static_cast<cudaStream_t>(stream)>>>(
        D->n_ghost, D->row_end - D->row_start, recv_buf, x_ext);
    NM_CHECK_LAUNCH();
    return NM_OK;
}

extern "C" int nm_dist_spmv_local(const nm_dist* D, const double* x_ext, double* y_local,
                                  void* stream) {
    nm::clear_error();
    if (!D) return fail(NM_ERR_INVALID, "nm_dist_spmv_local: NULL handle");
    if (D->row_end == D->row_start) return NM_OK;  // rank owns no rows
    if (!D->local) return fail(NM_ERR_INVALID, "nm_dist_spmv_local: host-only plan handle");
    if (!x_ext || !y_local) return fail(NM_ERR_INVALID, "nm_dist_spmv_local: NULL vector");
    return nm::launch_spmv(D->local, x_ext, y_local, static_cast<cudaStream_t>(stream));
}

extern "C" int nm_dist_row_split(const nm_dist* D, int32_t* n_interior, int32_t* n_boundary) {
    nm::clear_error();
    if (!D) return fail(NM_ERR_INVALID, "nm_dist_row_split: NULL handle");
    if (n_interior) *n_interior = D->n_interior;
    if (n_boundary) *n_boundary = D->n_boundary;
    return NM_OK;
}

extern "C" int nm_dist_spmv_interior(const nm_dist* D, const double* x_local, double* y_local,
                                     void* stream) {
    nm::clear_error();
    if (!D) return fail(NM_ERR_INVALID, "nm_dist_spmv_interior: NULL handle");
    if (D->row_end == D->row_start) return NM_OK;  // rank owns no rows
    if (!D->local) return fail(NM_ERR_INVALID, "nm_dist_spmv_interior: host-only plan handle");
    if (!x_local || !y_local) return fail(NM_ERR_INVALID, "nm_dist_spmv_interior: NULL vector");
    auto s = static_cast<cudaStream_t>(stream);
    if (D->n_ghost == 0) return nm::launch_spmv(D->local, x_local, y_local, s);  // all interior
    if (!D->interior) return NM_OK;
    return nm::launch_spmv_rows(D->interior, x_local, y_local, D->d_rows, s);
}

extern "C" int nm_dist_spmv_boundary(const nm_dist* D, const double* x_ext, double* y_local,
                                     void* stream) {
    nm::clear_error();
    if (!D) return fail(NM_ERR_INVALID, "nm_dist_spmv_boundary: NULL handle");
    if (D->row_end == D->row_start || D->n_ghost == 0 || !D->boundary) return NM_OK;
    if (!x_ext || !y_local) return fail(NM_ERR_INVALID, "nm_dist_spmv_boundary: NULL vector");
    return nm::launch_spmv_rows(D->boundary, x_ext, y_local, D->d_rows + D->n_interior,
                                static_cast<cudaStream_t>(stream));
}

extern "C" int nm_dist_cg_single(nm_dist* D, const double* b, double* x, double tol,
                                 int32_t max_iter, nm_cg_result* result, void* stream) {
    nm::clear_error();
    if (!D) return fail(NM_ERR_INVALID, "nm_dist_cg_single: NULL handle");
    if (D->size != 1 || D->n_ghost != 0)
        return fail(NM_ERR_INVALID,
                    "nm_dist_cg_single: handle spans %d ranks; use the per-rank building blocks",
                    D->size);
    return nm::cg_run(D->local, b, x, tol, max_iter, 1, result, static_cast<cudaStream_t>(stream));
}
