// spmv.cuh -- device body of the row-block CSR SpMV, shared by the plain SpMV
// kernel and the fused CG kernel.
//
// Persistent CTAs (256 threads) walk the row blocks b = blockIdx.x + k*gridDim.x.
// Each block's col_idx, values and row_ptr slices are brought into shared
// memory by TMA bulk copies (cp.async.bulk, one elected thread), completion
// tracked by an mbarrier per stage; STAGES stages form a ring, so the copies
// of the next blocks are in flight while the current one is reduced:
//
//  * multi-row block (nnz <= TILE): every thread multiplies staged values
//    with x[col] (gathered through the read-only path; x stays in L2) and
//    writes the product back over its staged operand.  Rows with
//    <= short_max nonzeros are then summed by one thread each, serially in
//    CSR order (bit-identical to the reference's serial row loop,
//    src/spmv_kernel.hpp:90-97); longer rows by one warp each.
//  * single-row block (nnz > TILE): nothing is staged; the whole CTA strides
//    the row with 16-byte loads and reduces with a deterministic CTA-wide sum.
//
// The epilogue functor receives (row, value) exactly once per row, on one
// thread; CG uses it to store Ap and to accumulate p.Ap on the fly.
//
// Alignment (TMA bulk copies need 16-byte aligned addresses and sizes): the
// staged nonzero range is [z0 & ~7, (z1 + 7) & ~7) and the row_ptr range
// [r0 & ~3, (r1 + 4) & ~3); the device arrays are padded so these never leave
// the allocation (see upload in csr.cu).
#pragma once

#include "csr.cuh"

namespace nm {

template <typename V, int TILE>
struct alignas(16) SpmvStage {
    int32_t col[TILE + 16];
    V val[TILE + 16];
    int32_t rp[kThreads + 8];
};

template <typename V, typename A, int TILE, int STAGES>
struct SpmvSmem {
    SpmvStage<V, TILE> st[STAGES];
    uint64_t bar[STAGES];
    int32_t meta[STAGES][4];  // r0, r1, z0, z1 of the block in each stage
    int32_t long_rows[kThreads];
    int32_t warp_cnt[kWarps];
    A red[kWarps];
};

// Product storage: over the staged values when they are as wide as the
// accumulator, else over the staged column indices (bf16 values, float
// products).  Each slot is read by the thread that then overwrites it.
template <typename V, typename A, int TILE>
__device__ __forceinline__ A* prod_slots(SpmvStage<V, TILE>& st) {
    static_assert(sizeof(A) == sizeof(V) || sizeof(A) == sizeof(int32_t), "product slot");
    if constexpr (sizeof(A) == sizeof(V)) return reinterpret_cast<A*>(st.val);
    else return reinterpret_cast<A*>(st.col);
}

// Issued by one thread: stage the block described by d into stage s.
template <typename V, typename A, int TILE, int STAGES>
__device__ __forceinline__ void spmv_issue(const CsrView<V>& M, int4 d,
                                           SpmvSmem<V, A, TILE, STAGES>& sm, int s) {
    const int32_t r0 = d.x, r1 = d.y, z0 = d.z, z1 = d.w;
    sm.meta[s][0] = r0;
    sm.meta[s][1] = r1;
    sm.meta[s][2] = z0;
    sm.meta[s][3] = z1;
    if (z1 - z0 > TILE) {  // long row: read from global by the consumer
        mbar_arrive_expect_tx(&sm.bar[s], 0u);
        return;
    }
    const int32_t a0 = z0 & ~7, a1 = (z1 + 7) & ~7;
    const int32_t ra0 = r0 & ~3, ra1 = (r1 + 4) & ~3;
    const uint32_t ncol = static_cast<uint32_t>(a1 - a0);
    const uint32_t nrp = static_cast<uint32_t>(ra1 - ra0);
    const uint32_t bytes = ncol * uint32_t(sizeof(int32_t) + sizeof(V)) + nrp * 4u;
    SpmvStage<V, TILE>& st = sm.st[s];
    mbar_arrive_expect_tx(&sm.bar[s], bytes);
    if (ncol) {
        bulk_g2s(st.col, M.col_idx + a0, ncol * 4u, &sm.bar[s]);
        bulk_g2s(st.val, M.values + a0, ncol * uint32_t(sizeof(V)), &sm.bar[s]);
    }
    bulk_g2s(st.rp, M.row_ptr + ra0, nrp * 4u, &sm.bar[s]);
}

// One long row (nnz > TILE) straight from global memory, whole CTA.
template <typename V, typename X, typename A, int TILE, int STAGES, class Epi>
__device__ __forceinline__ void spmv_long_row(const CsrView<V>& M, int32_t r0, int32_t z0,
                                              int32_t z1, const X* __restrict__ x,
                                              SpmvSmem<V, A, TILE, STAGES>& sm, Epi& epi) {
    const int t = threadIdx.x;
    A s = A(0);
    for (int32_t j = (z0 & ~3) + 4 * t; j < z1; j += 4 * kThreads) {
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
}

// A staged multi-row block.
template <typename V, typename X, typename A, int TILE, int STAGES, class Epi>
__device__ __forceinline__ void spmv_tile(const CsrView<V>& M, int s, const X* __restrict__ x,
                                          SpmvSmem<V, A, TILE, STAGES>& sm, Epi& epi) {
    const int t = threadIdx.x;
    const int lane = t & 31, warp = t >> 5;
    SpmvStage<V, TILE>& st = sm.st[s];
    const int32_t r0 = sm.meta[s][0], r1 = sm.meta[s][1];
    const int32_t z0 = sm.meta[s][2], z1 = sm.meta[s][3];
    const int nr = r1 - r0;
    const int32_t a0 = z0 & ~7;
    const int32_t roff = r0 - (r0 & ~3);  // row r0's slot in the staged row_ptr
    const int cnt = z1 - a0;
    A* prod = prod_slots<V, A, TILE>(st);

    // products: every gather of this thread is issued before any is used
    // (one L2 round trip per block)
    constexpr int kPer = (TILE + 16 + kThreads - 1) / kThreads;
    {
        const int e0 = (z0 - a0) + t;
        int c[kPer];
        A v[kPer];
#pragma unroll
        for (int q = 0; q < kPer; ++q) {
            const int e = e0 + q * kThreads;
            c[q] = e < cnt ? st.col[e] : -1;
            v[q] = e < cnt ? widen<V, A>(st.val[e]) : A(0);
        }
        A xv[kPer];
#pragma unroll
        for (int q = 0; q < kPer; ++q) xv[q] = c[q] >= 0 ? static_cast<A>(__ldg(x + c[q])) : A(0);
#pragma unroll
        for (int q = 0; q < kPer; ++q) {
            const int e = e0 + q * kThreads;
            if (e < cnt) prod[e] = mul_rn(v[q], xv[q]);
        }
    }
    __syncthreads();

    // thread-per-row reduction; flag the long rows
    bool is_long = false;
    if (t < nr) {
        const int32_t s0 = st.rp[roff + t] - a0, s1 = st.rp[roff + t + 1] - a0;
        if (s1 - s0 <= M.short_max) {
            // serial CSR-order sum; loads batched four at a time
            A acc = A(0);
            int32_t j = s0;
            for (; j + 4 <= s1; j += 4) {
                const A p0 = prod[j], p1 = prod[j + 1], p2 = prod[j + 2], p3 = prod[j + 3];
                acc = add_rn(add_rn(add_rn(add_rn(acc, p0), p1), p2), p3);
            }
            for (; j < s1; ++j) acc = add_rn(acc, prod[j]);
            epi(r0 + t, acc);
        } else {
            is_long = true;
        }
    }
    // Returns with the stage free when no row needs a warp (the common case
    // for stencils: one barrier).
    if (!__syncthreads_or(is_long)) return;

    // deterministic list of long rows in row order (ballot + warp prefix)
    const unsigned m = __ballot_sync(0xffffffffu, is_long);
    if (lane == 0) sm.warp_cnt[warp] = __popc(m);
    __syncthreads();
    int base = 0, nl = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
        const int cw = sm.warp_cnt[w];
        if (w < warp) base += cw;
        nl += cw;
    }
    if (is_long) sm.long_rows[base + __popc(m & ((1u << lane) - 1u))] = t;
    __syncthreads();

    // warp-per-row reduction of the long rows
    for (int q = warp; q < nl; q += kWarps) {
        const int tt = sm.long_rows[q];
        const int32_t s0 = st.rp[roff + tt] - a0, s1 = st.rp[roff + tt + 1] - a0;
        A acc = A(0);
        for (int32_t j = s0 + lane; j < s1; j += 32) acc += prod[j];
        acc = warp_sum(acc);
        if (lane == 0) epi(r0 + tt, acc);
    }
    __syncthreads();
}

// The persistent pipelined loop over this CTA's row blocks.  Returns false if
// a bounded wait gave up (the error word is set; the caller must not use its
// partial results).  Call from all threads.
template <typename V, typename X, typename A, int TILE, int STAGES, class Epi>
__device__ __forceinline__ bool spmv_pipeline(const CsrView<V>& M, const X* __restrict__ x,
                                              SpmvSmem<V, A, TILE, STAGES>& sm, Epi& epi,
                                              unsigned int* err) {
    const int t = threadIdx.x;
    if (t == 0) {
#pragma unroll
        for (int s = 0; s < STAGES; ++s) mbar_init(&sm.bar[s], 1);
        fence_mbar_init();
    }
    __syncthreads();
    // Thread 0 issues; it holds the descriptor of the next block to issue in
    // registers, loaded one block ahead so its latency is off the critical path.
    int4 next_desc = make_int4(0, 0, 0, 0);
    if (t == 0) {
#pragma unroll
        for (int s = 0; s < STAGES; ++s) {
            const int64_t b = int64_t(blockIdx.x) + int64_t(s) * gridDim.x;
            if (b < M.nblk) spmv_issue<V, A, TILE, STAGES>(M, __ldg(M.desc + b), sm, s);
        }
        const int64_t nb = int64_t(blockIdx.x) + int64_t(STAGES) * gridDim.x;
        if (nb < M.nblk) next_desc = __ldg(M.desc + nb);
    }
    uint32_t parity = 0;  // bit s: phase parity to wait for on stage s
    int s = 0;
    for (int64_t b = blockIdx.x; b < M.nblk; b += gridDim.x) {
        const bool ok = mbar_wait_bounded(&sm.bar[s], (parity >> s) & 1u);
        if (__syncthreads_or(!ok)) {
            // Give up: report, then wait (bounded) for this CTA's copies still
            // in flight so none lands in shared memory after exit.
            if (t == 0) atomicOr(err, kErrWaitTimeout);
            for (int q = 0; q < STAGES; ++q) {
                const int sq = (s + q) % STAGES;
                if (b + int64_t(q) * gridDim.x < M.nblk)
                    mbar_wait_bounded(&sm.bar[sq], (parity >> sq) & 1u);
            }
            return false;
        }
        parity ^= 1u << s;
        const int32_t z0 = sm.meta[s][2], z1 = sm.meta[s][3];
        if (z1 - z0 > TILE) {
            spmv_long_row<V, X, A, TILE, STAGES>(M, sm.meta[s][0], z0, z1, x, sm, epi);
            __syncthreads();
        } else {
            spmv_tile<V, X, A, TILE, STAGES>(M, s, x, sm, epi);  // ends with a barrier
        }
        // stage s and meta[s] are free again
        if (t == 0) {
            const int64_t nb = b + int64_t(STAGES) * gridDim.x;
            if (nb < M.nblk) {
                fence_proxy_async_smem();  // products were written over stage s
                spmv_issue<V, A, TILE, STAGES>(M, next_desc, sm, s);
                const int64_t nn = nb + gridDim.x;
                if (nn < M.nblk) next_desc = __ldg(M.desc + nn);
            }
        }
        s = (s + 1 == STAGES) ? 0 : s + 1;
    }
    return true;
}

// Epilogue: y[row] = value.
template <typename X, typename A>
struct StoreEpi {
    X* __restrict__ y;
    __device__ __forceinline__ void operator()(int32_t row, A v) { y[row] = static_cast<X>(v); }
};

// Dynamic shared memory of the pipelined kernels.
template <typename V, typename A, int TILE, int STAGES>
constexpr size_t spmv_smem_bytes() {
    return sizeof(SpmvSmem<V, A, TILE, STAGES>);
}

}  // namespace nm
