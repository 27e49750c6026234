// spmv.cuh -- device body of the row-block CSR SpMV, shared by the plain SpMV
// kernel and the fused CG kernels.
//
// One CTA (256 threads) processes one row block at a time:
//
//  * multi-row block (nnz <= TILE): the CTA streams the block's nonzeros
//    [row_ptr[r0], row_ptr[r1]) from a 4-aligned start with 16-byte loads of
//    col_idx and values (evict-first, read once), gathers x[col] through the
//    read-only path (x stays in L2), and writes each product v*x to shared
//    memory.  Then every row is reduced from shared memory: rows with
//    <= short_max nonzeros by one thread, serially in CSR order (bit-identical
//    to the reference's serial row loop, src/spmv_kernel.hpp:90-97), longer
//    rows by one warp each (strided partial sums + shuffle tree).
//  * single-row block (nnz > TILE): the whole CTA strides the row with the
//    same 16-byte loads and reduces with a deterministic CTA-wide sum.
//
// The epilogue functor receives (row, value) exactly once per row, on one
// thread; CG uses it to store Ap and to accumulate p.Ap on the fly.
#pragma once

#include "csr.cuh"

namespace nm {

template <typename A, int TILE>
struct SpmvSmem {
    A prod[TILE + 4];        // products of the block's nonzeros (aligned start)
    int32_t rp[kThreads + 1];  // row_ptr of the block
    int32_t long_rows[kThreads];
    int32_t warp_cnt[kWarps];
    A red[kWarps];
};

template <typename V, typename X, typename A, int TILE, class Epi>
__device__ __forceinline__ void spmv_block(const CsrView<V>& M, int32_t r0, int32_t r1,
                                           const X* __restrict__ x, SpmvSmem<A, TILE>& sm,
                                           Epi& epi) {
    const int t = threadIdx.x;
    const int lane = t & 31, warp = t >> 5;
    const int nr = r1 - r0;
    for (int i = t; i <= nr; i += kThreads) sm.rp[i] = M.row_ptr[r0 + i];
    __syncthreads();
    const int32_t z0 = sm.rp[0], z1 = sm.rp[nr];
    const int32_t a0 = z0 & ~3;

    if (z1 - z0 > TILE) {
        // ---- one long row, whole CTA ----
        A s = A(0);
        for (int32_t j = a0 + 4 * t; j < z1; j += 4 * kThreads) {
            const int4 c = ld_stream(reinterpret_cast<const int4*>(M.col_idx + j));
            A v[4];
            Load4<V, A>::run(M.values, j, v);
            const int32_t cc[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int32_t jj = j + q;
                if (jj >= z0 && jj < z1) s += v[q] * static_cast<A>(__ldg(x + cc[q]));
            }
        }
        s = block_sum(s, sm.red);
        if (t == 0) epi(r0, s);
        __syncthreads();
        return;
    }

    // ---- multi-row block: stage products ----
    for (int32_t j = a0 + 4 * t; j < z1; j += 4 * kThreads) {
        const int4 c = ld_stream(reinterpret_cast<const int4*>(M.col_idx + j));
        A v[4];
        Load4<V, A>::run(M.values, j, v);
        const int32_t cc[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int32_t jj = j + q;
            if (jj >= z0 && jj < z1)
                sm.prod[jj - a0] = mul_rn(v[q], static_cast<A>(__ldg(x + cc[q])));
        }
    }
    __syncthreads();

    // ---- thread-per-row reduction; flag the long rows ----
    bool is_long = false;
    if (t < nr) {
        const int32_t s0 = sm.rp[t], s1 = sm.rp[t + 1];
        if (s1 - s0 <= M.short_max) {
            A acc = A(0);
            for (int32_t j = s0; j < s1; ++j) acc = add_rn(acc, sm.prod[j - a0]);
            epi(r0 + t, acc);
        } else {
            is_long = true;
        }
    }
    // Deterministic list of long rows in row order (ballot + warp prefix).
    const unsigned m = __ballot_sync(0xffffffffu, is_long);
    if (lane == 0) sm.warp_cnt[warp] = __popc(m);
    __syncthreads();
    int base = 0, nl = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
        const int c = sm.warp_cnt[w];
        if (w < warp) base += c;
        nl += c;
    }
    if (is_long) sm.long_rows[base + __popc(m & ((1u << lane) - 1u))] = t;
    __syncthreads();

    // ---- warp-per-row reduction of the long rows ----
    for (int q = warp; q < nl; q += kWarps) {
        const int tt = sm.long_rows[q];
        const int32_t s0 = sm.rp[tt], s1 = sm.rp[tt + 1];
        A acc = A(0);
        for (int32_t j = s0 + lane; j < s1; j += 32) acc += sm.prod[j - a0];
        acc = warp_sum(acc);
        if (lane == 0) epi(r0 + tt, acc);
    }
    __syncthreads();  // shared memory is reused by the next block
}

// Epilogue: y[row] = value.
template <typename X, typename A>
struct StoreEpi {
    X* __restrict__ y;
    __device__ __forceinline__ void operator()(int32_t row, A v) { y[row] = static_cast<X>(v); }
};

}  // namespace nm
