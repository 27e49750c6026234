// csr.cuh -- internal layout of a device CSR matrix.
//
// HBM layout (one cudaMalloc each, 256-byte aligned):
//   row_ptr  int32[nrows + 1 + 8]  pad = nnz
//   col_idx  int32[nnz_pad]        nnz_pad = round_up(nnz, 8) + 8, pad = column 0
//   values   V[nnz_pad]            pad = 0
//   blk      int32[nblk + 1]       row-block boundaries (see build_row_blocks)
//   desc     BlockDesc[nblk]       per block rows, nonzeros and x windows
// The padding lets the TMA bulk copies of a block start and end on 16-byte
// boundaries (nonzeros rounded to multiples of 8, row_ptr to multiples of 4),
// and lets a thread load 4 consecutive nonzeros with one 16-byte access,
// without leaving the allocation.
#pragma once

#include <memory>
#include <mutex>
#include <vector>

#include "common.cuh"

namespace nm {

struct CgWorkspace;  // cg.cu

// Row-block descriptor, one 64-byte record per block.
//   rz = {first row, end row, first nonzero, end nonzero}
//   xs = starts of the block's x windows (xs.x < 0: no windows; unused: INT_MAX)
//   xl = lengths of the x windows (0: unused)
// The x windows are up to kXSeg ranges of x, each starting and ending on a
// multiple of 4 elements, that together hold every column the block's
// nonzeros reference; the SpMV kernels stage them with the block's nonzeros.
constexpr int kXSeg = 4;
// Elements of x a block of a TILE-nonzero partition may stage.
__host__ __device__ constexpr int xwin_capacity(int tile) { return tile / 2 + 384; }
constexpr int kXGap = 16;  // gaps up to this many elements are bridged
struct BlockDesc {
    int4 rz;
    int4 xs;
    int4 xl;
    // {rows reduced by a warp (nnz > short_max), system slot, 0, 0}; in the
    // staged copy the SpMV producer sets z = 1 for a block its gate skips and
    // w = 1 when it staged the x windows
    int4 aux;
};

// Kernel-side view of a matrix.
template <typename V>
struct CsrView {
    const int32_t* __restrict__ row_ptr;
    const int32_t* __restrict__ col_idx;
    const V* __restrict__ values;
    const BlockDesc* __restrict__ desc;
    int32_t nblk;
    int32_t nrows;
    int32_t short_max;
    int32_t stage_x;  // 1: x windows are staged (x 16-byte aligned); 0: gather from global
    const int32_t* nblk_dev;  // when set, the block count is read from device memory
    // 1: x is written by other CTAs of the same kernel (a persistent solver),
    // so x values not staged by TMA are read through L2 (ld.global.cg), not
    // the non-coherent read-only path
    int32_t coherent_x = 0;
};

// Default row-block parameters.
constexpr int kDefaultTile = 2048;
constexpr int kDefaultMaxRows = kThreads;
constexpr int kDefaultShortMax = 32;
constexpr int kDefaultStages = 2;

// x windows of the multi-row block with nonzeros [z0, z1) (see BlockDesc);
// xw = largest total window length, ncols = length of x.
void block_xwindows(const int32_t* col_idx, int32_t z0, int32_t z1, int32_t ncols, int xw,
                    std::vector<int32_t>& scratch, int4* xs, int4* xl);

// Row-block partition rule, shared by the device library and restated by the
// CPU oracle (oracle.c, or_row_blocks).  Returns nblk; blk gets nblk+1 entries.
int build_row_blocks(const int32_t* row_ptr, int32_t nrows, int tile, int max_rows,
                     int short_max, std::vector<int32_t>& blk, std::vector<int8_t>* bins);

// State of nm_spmv_host (spmv.cu) on one handle, made on its first call: the
// device copies of x and y, a copy-in and a copy-out stream, and the split of
// x into pieces and of the row blocks into chunks, each chunk with the last x
// piece its nonzeros read.
struct HostSpmv {
    std::mutex mu;  // one call at a time on the handle
    void* dx = nullptr;
    void* dy = nullptr;
    cudaStream_t in = nullptr, out = nullptr;
    cudaEvent_t begin = nullptr, done = nullptr;
    std::vector<cudaEvent_t> x_ready;  // per x piece
    std::vector<cudaEvent_t> y_ready;  // per row chunk
    uint32_t gen = ~0u;                // nm_csr::layout_gen the split was made for
    std::vector<int64_t> xcut;         // x piece p: elements [xcut[p], xcut[p+1])
    std::vector<int32_t> blk;          // row chunk c: blocks [blk[c], blk[c+1])
    std::vector<int32_t> row;          // row chunk c: rows [row[c], row[c+1])
    std::vector<int32_t> need;         // row chunk c reads x pieces 0..need[c] (-1: none)
    ~HostSpmv();
};

}  // namespace nm

struct nm_csr {
    int32_t nrows = 0, ncols = 0, nnz = 0;
    int dtype = NM_F64;
    int device = 0;
    int32_t* d_row_ptr = nullptr;
    int32_t* d_col_idx = nullptr;
    void* d_values = nullptr;
    int32_t* d_blk = nullptr;
    nm::BlockDesc* d_desc = nullptr;
    int32_t nblk = 0;
    nm_tuning tune{};
    // Plain SpMV by the warp-gather kernel (spmv.cu): set by rebuild_blocks
    // from tune.kernel (AUTO: most nonzeros in blocks without x windows and no
    // row longer than kWarpGatherMaxRow).
    bool warp_gather = false;
    // The gather kernel's copy of the matrix (built the first time that kernel
    // is selected, kept until the handle is freed): rows sorted by length
    // (descending, stable) within windows of kSellWindow rows, cut into slices
    // of 32 sorted rows, each slice stored column-major -- entry k of the
    // slice's lane l at sell_ptr[s] + 32 k + l, zero-padded to the slice's
    // longest row -- with the original row and the length of every sorted
    // position.  A matrix whose padding would exceed its nonzeros keeps the
    // per-group gather kernel instead (sell_ready false).
    bool sell_tried = false, sell_ready = false;
    int32_t sell_slices = 0;
    int64_t* d_sell_ptr = nullptr;
    int32_t* d_sell_row = nullptr;
    int32_t* d_sell_len = nullptr;
    int32_t* d_sell_col = nullptr;
    void* d_sell_val = nullptr;
    std::vector<int32_t> h_row_ptr;  // kept to rebuild the partition on retuning
    std::vector<int32_t> h_col_idx;  // kept to rebuild the x windows on retuning
    // Many-matrix handles: per-matrix row / column offsets (count + 1 each).
    std::vector<int32_t> batch_row_off, batch_col_off;
    // Incremented by every rebuild of the row-block partition.
    uint32_t layout_gen = 0;
    std::mutex cg_mutex;
    std::unique_ptr<nm::CgWorkspace> cg;
    mutable std::mutex host_mutex;  // guards host_spmv's creation
    mutable std::unique_ptr<nm::HostSpmv> host_spmv;
    ~nm_csr();

    template <typename V>
    nm::CsrView<V> view() const {
        return nm::CsrView<V>{d_row_ptr, d_col_idx, static_cast<const V*>(d_values),
                              d_desc,    nblk,      nrows,
                              tune.short_max, 0, nullptr};
    }
};

namespace nm {
// Number of CTAs of a persistent SpMV-family grid for this matrix.
int spmv_grid(const nm_csr* A, int ctas_per_sm);
// Launches y = A*x on `stream` (dtype-dispatched).  Used by the API and CG.
int launch_spmv(const nm_csr* A, const void* x, void* y, cudaStream_t stream);
// FP64 row-block SpMV of a row-subset matrix: y[rows[i]] = (A x)[i].
int launch_spmv_rows(const nm_csr* A, const double* x, double* y, const int32_t* rows,
                     cudaStream_t stream);
// Dynamic shared memory of the SpMV kernel for (dtype, tile, stages); 0 if
// the combination does not exist.
size_t spmv_smem_for(int dtype, int tile, int stages);
// Rebuilds the row-block partition and descriptors of A under A->tune (and
// the choice of plain-SpMV kernel).
int rebuild_blocks(nm_csr* A);
// Longest row the warp-gather kernel takes (each row is summed by one lane).
constexpr int32_t kWarpGatherMaxRow = 4096;
// Rows sorted by length together in the gather kernel's sliced copy.
constexpr int32_t kSellWindow = 65536;
// Builds A's sliced copy for the gather kernel once (spmv.cu); NM_OK also
// when the layout would pad too much (A->sell_ready stays false).
int build_sell(nm_csr* A);
// Drops A's cached CG workspace (its graphs hold the current descriptors).
void reset_cg(nm_csr* A);
// Nonzeros of the Laplacian on an L^dim grid (dim 2: 5-point, dim 3: 7-point).
int64_t stencil_nnz(int dim, int32_t L);
// Writes that Laplacian's row_ptr (rp_len entries, those past the last row =
// nnz), col_idx and values (dtype) into device arrays on `stream` (gen.cu).
int launch_laplacian(int dim, int32_t L, int dtype, int32_t* rp, int64_t rp_len, int32_t* ci,
                     void* val, cudaStream_t stream);
}  // namespace nm
