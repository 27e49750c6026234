// gen.cu -- on-device assembly of the stencil test matrices.
//
// The 5-point 2-D and 7-point 3-D Dirichlet Laplacians of the reference's
// generator module (python/matrix_generators.py: make_laplacian_2d :16-37,
// make_laplacian_3d_fast :68-80 -- same rows, same ascending columns, same
// values 4 / -1 and 6 / -1) written straight into a CSR handle's device
// arrays.  Each row's offset is a closed-form count of the nonzeros before
// it, so one thread per row writes its row_ptr entry, its columns and its
// values with no scan, and the matrix never crosses PCIe on the way in.
// HBM-bound: 4 (n + 1) + (4 + value bytes) nnz written, nothing read.
#include "csr.cuh"

#include <algorithm>

namespace nm {

// Nonzeros in rows [0, i) of the Laplacian on an L^dim grid (x fastest):
// i diagonal entries, plus, for each of the 2*dim neighbour directions, the
// number of rows before i whose neighbour in that direction is on the grid.
// Requires i <= n = L^dim < 2^31.
__host__ __device__ inline int64_t stencil_before(int dim, uint32_t L, uint32_t n, uint32_t i) {
    const int64_t ii = i, nn = n, l = L;
    int64_t s = ii;
    s += ii - (i + L - 1) / L;  // x > 0: every row but x == 0 (rows 0, L, 2L, ...)
    s += ii - i / L;            // x < L-1: every row but x == L-1
    if (dim == 2) {
        s += ii > l ? ii - l : 0;   // y > 0: rows L ... n-1
        s += ii < nn - l ? ii : nn - l;  // y < L-1: rows 0 ... n-L-1
    } else {
        const uint32_t LL = L * L;
        const uint32_t pl = i / LL, r = i % LL;  // whole planes before row i, offset in its plane
        s += ii - (int64_t(pl) * l + (r < L ? r : L));                   // y > 0
        s += ii - (int64_t(pl) * l + (r > LL - L ? r - (LL - L) : 0));  // y < L-1
        s += ii > int64_t(LL) ? ii - LL : 0;                            // z > 0
        s += ii < nn - LL ? ii : nn - LL;                               // z < L-1
    }
    return s;
}

int64_t stencil_nnz(int dim, int32_t L) {
    const int64_t l = L;
    return dim == 2 ? 5 * l * l - 4 * l : 7 * l * l * l - 6 * l * l;
}

namespace {

// Rows in CTA-sized groups: each thread writes its row's row_ptr entry and
// stages the row's nonzeros in shared memory at their offset within the
// group; the CTA then writes the group's contiguous column / value range with
// consecutive threads on consecutive elements (full-sector stores), and CTA 0
// fills the row_ptr padding past row n - 1 with nnz.
constexpr int kGenRows = 256;
constexpr int kGenMaxNz = 7;  // nonzeros of a 7-point row

template <typename V>
__global__ void __launch_bounds__(kGenRows)
    laplacian_kernel(int dim, uint32_t L, uint32_t n, int64_t rp_len, int32_t* __restrict__ rp,
                     int32_t* __restrict__ ci, V* __restrict__ val, V diag, V off) {
    __shared__ int32_t s_ci[kGenRows * kGenMaxNz];
    __shared__ V s_v[kGenRows * kGenMaxNz];
    const uint32_t LL = L * L;
    const int64_t groups = (int64_t(n) + kGenRows - 1) / kGenRows;
    for (int64_t g = blockIdx.x; g < groups; g += gridDim.x) {
        const uint32_t r0 = uint32_t(g * kGenRows);
        const uint32_t r1 = n - r0 < uint32_t(kGenRows) ? n : r0 + kGenRows;
        const int64_t base = stencil_before(dim, L, n, r0);
        const uint32_t i = r0 + threadIdx.x;
        if (i < r1) {
            const int64_t j0 = stencil_before(dim, L, n, i);
            rp[i] = static_cast<int32_t>(j0);
            int k = static_cast<int>(j0 - base);
            const uint32_t x = i % L;
            const uint32_t y = dim == 2 ? i / L : (i / L) % L;
            const uint32_t z = dim == 2 ? 0 : i / LL;
            if (dim == 3 && z > 0) { s_ci[k] = int32_t(i - LL); s_v[k] = off; ++k; }
            if (y > 0) { s_ci[k] = int32_t(i - L); s_v[k] = off; ++k; }
            if (x > 0) { s_ci[k] = int32_t(i - 1); s_v[k] = off; ++k; }
            s_ci[k] = int32_t(i); s_v[k] = diag; ++k;
            if (x + 1 < L) { s_ci[k] = int32_t(i + 1); s_v[k] = off; ++k; }
            if (y + 1 < L) { s_ci[k] = int32_t(i + L); s_v[k] = off; ++k; }
            if (dim == 3 && z + 1 < L) { s_ci[k] = int32_t(i + LL); s_v[k] = off; }
        }
        __syncthreads();
        const int cnt = static_cast<int>(stencil_before(dim, L, n, r1) - base);
        for (int e = threadIdx.x; e < cnt; e += kGenRows) {
            ci[base + e] = s_ci[e];
            val[base + e] = s_v[e];
        }
        __syncthreads();
    }
    if (blockIdx.x == 0 && int64_t(n) + threadIdx.x < rp_len)
        rp[int64_t(n) + threadIdx.x] = static_cast<int32_t>(stencil_before(dim, L, n, n));
}

template <typename V>
int launch_t(int dim, int32_t L, int32_t n, int64_t rp_len, int32_t* rp, int32_t* ci, void* val,
             V diag, V off, cudaStream_t s) {
    if (rp_len < int64_t(n) + 1 || rp_len - n > kGenRows)
        return fail(NM_ERR_INVALID, "laplacian: row_ptr length %lld for %d rows", (long long)rp_len, n);
    const int64_t blocks =
        std::min<int64_t>((int64_t(n) + kGenRows - 1) / kGenRows, int64_t(sm_count()) * 8);
    laplacian_kernel<V><<<static_cast<int>(blocks), kGenRows, 0, s>>>(
        dim, uint32_t(L), uint32_t(n), rp_len, rp, ci, static_cast<V*>(val), diag, off);
    NM_CHECK_LAUNCH();
    return NM_OK;
}

}  // namespace

int launch_laplacian(int dim, int32_t L, int dtype, int32_t* rp, int64_t rp_len, int32_t* ci,
                     void* val, cudaStream_t s) {
    const int32_t n = dim == 2 ? L * L : L * L * L;
    const double d = dim == 2 ? 4.0 : 6.0;
    switch (dtype) {
        case NM_F64: return launch_t<double>(dim, L, n, rp_len, rp, ci, val, d, -1.0, s);
        case NM_F32:
            return launch_t<float>(dim, L, n, rp_len, rp, ci, val, float(d), -1.0f, s);
        case NM_BF16:
            return launch_t<__nv_bfloat16>(dim, L, n, rp_len, rp, ci, val,
                                           __float2bfloat16_rn(float(d)),
                                           __float2bfloat16_rn(-1.0f), s);
        default: return fail(NM_ERR_TYPE, "laplacian: unknown dtype %d", dtype);
    }
}

}  // namespace nm
