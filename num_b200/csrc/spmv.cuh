// spmv.cuh -- device body of the row-block CSR SpMV, shared by the plain SpMV
// kernel and the fused CG kernel.
//
// Persistent, warp-specialised CTAs of 288 threads walk the row blocks
// b = blockIdx.x + k*gridDim.x:
//
//  * one producer warp (warp 8, one lane) brings each block's col_idx,
//    values, row_ptr slice and x windows into a ring of STAGES shared-memory
//    stages with TMA bulk copies (cp.async.bulk); a `full` mbarrier per stage
//    counts the transaction bytes, an `empty` mbarrier per stage counts the
//    consumer warps that have released it, so the producer runs up to STAGES
//    blocks ahead of the consumers;
//  * eight consumer warps (256 threads, named barrier 1) compute the block
//    from the staged operands and the staged x window entries (x[col] from
//    global memory when the block has no windows): rows with <= short_max
//    nonzeros are summed by one thread each, serially in CSR order
//    (bit-identical to the reference's serial row loop,
//    src/spmv_kernel.hpp:90-97); longer rows by one warp each.  A block that
//    is one row with more than TILE nonzeros is read straight from global
//    memory by all consumers and reduced with a deterministic sum.
//
// A block without warp rows costs the consumers no barrier at all: each warp
// releases the stage on its own.
//
// The epilogue functor receives (row, value) exactly once per row, on one
// consumer thread; CG uses it to store Ap and to accumulate p.Ap on the fly.
// An epilogue with kBlockSums also gets one sum per row block: each consumer
// warp reduces its threads' take() values and parks the warp's sum in the
// stage's slot before releasing the stage; the producer, once the stage is
// released, adds the eight warp sums in warp order and hands the block sum to
// finish_block(b, d, sum) -- no barrier or atomic on the consumers' path.
//
// Alignment (TMA bulk copies need 16-byte aligned addresses and sizes): the
// staged nonzero range is [z0 & ~7, (z1 + 7) & ~7), the row_ptr range
// [r0 & ~3, (r1 + 4) & ~3), x windows start and end on multiples of 4 elements
// inside [0, ncols & ~3); the device arrays are padded so these never leave
// the allocation (see upload in csr.cu), and windows are used only when x is
// 16-byte aligned.
//
// Every mbarrier wait is bounded (mbar_wait_bounded).  When one gives up the
// kernel sets the device error word; that consumer stops waiting and stops
// touching staged data (but keeps the CTA's barrier schedule), and the
// producer waits (bounded again) for its copies still in flight before the
// CTA exits.
#pragma once

#include <type_traits>

#include "csr.cuh"

namespace nm {

constexpr int kConsumers = kThreads;        // 8 consumer warps
constexpr int kCtaThreads = kThreads + 32;  // + 1 producer warp
constexpr int kProducerWarp = kWarps;

// Barrier among the 256 consumer threads only (id 1; id 0 is __syncthreads).
__device__ __forceinline__ void consumer_sync() {
    asm volatile("bar.sync 1, %0;" ::"n"(kConsumers) : "memory");
}

__device__ __forceinline__ bool consumer_sync_or(bool pred) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred q, o;\n\t"
        "setp.ne.u32 q, %1, 0;\n\t"
        "bar.red.or.pred o, 1, %2, q;\n\t"
        "selp.u32 %0, 1, 0, o;\n\t}"
        : "=r"(r)
        : "r"(static_cast<uint32_t>(pred)), "n"(kConsumers)
        : "memory");
    return r != 0;
}

// Deterministic sum over the consumer threads; valid in consumer thread 0.
template <typename T>
__device__ __forceinline__ T consumer_sum(T v, T* scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_sum(v);
    if (lane == 0) scratch[warp] = v;
    consumer_sync();
    T s = T(0);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int w = 0; w < kWarps; ++w) s += scratch[w];
    }
    consumer_sync();
    return s;
}

template <typename V, typename X, int TILE>
struct alignas(16) SpmvStage {
    int32_t col[TILE + 16];
    V val[TILE + 16];
    int32_t rp[kThreads + 8];
    X xw[xwin_capacity(TILE)];  // the block's x windows, back to back
};

// With XR the stage also holds the same windows of a second vector xr: the
// pipeline then multiplies by x' = fma(beta, x, xr), formed as it is read.
template <typename V, typename X, int TILE>
struct alignas(16) SpmvStageXR : SpmvStage<V, X, TILE> {
    X xrw[xwin_capacity(TILE)];
};

template <typename V, typename X, typename A, int TILE, int STAGES, bool XR = false>
struct SpmvSmem {
    std::conditional_t<XR, SpmvStageXR<V, X, TILE>, SpmvStage<V, X, TILE>> st[STAGES];
    uint64_t full[STAGES];
    uint64_t empty[STAGES];
    BlockDesc meta[STAGES];  // descriptor of the block in each stage
    int32_t long_rows[kThreads];
    int32_t warp_cnt[kWarps];
    A red[kWarps + 1];
    double blk_red[STAGES][kWarps];  // per-warp epilogue sums of the block in each stage
    int64_t bid[STAGES];             // index of the block in each stage
};

__device__ __forceinline__ BlockDesc load_desc(const BlockDesc* p) {
    const int4* q = reinterpret_cast<const int4*>(p);
    BlockDesc d;
    d.rz = __ldg(q);
    d.xs = __ldg(q + 1);
    d.xl = __ldg(q + 2);
    d.aux = __ldg(q + 3);
    return d;
}

// Every block is computed.
struct AllBlocks {
    __device__ __forceinline__ bool operator()(const BlockDesc&) const { return true; }
};

// Producer: stage the block described by d into stage s (its nonzeros,
// row_ptr slice and, when M.stage_x, its x windows).  A block the gate
// rejected (d.aux.z = 1, decided when the descriptor was loaded) is not
// staged; it reaches the consumers marked skipped.
template <typename V, typename X, typename A, int TILE, int STAGES, bool XR = false>
__device__ __forceinline__ void spmv_issue(const CsrView<V>& M, const X* __restrict__ x,
                                           BlockDesc d, SpmvSmem<V, X, A, TILE, STAGES, XR>& sm,
                                           int s, const X* __restrict__ xr = nullptr) {
    const int32_t r0 = d.rz.x, r1 = d.rz.y, z0 = d.rz.z, z1 = d.rz.w;
    const bool skip = d.aux.z != 0;
    const bool long_row = z1 - z0 > TILE;
    const bool stage_x = !skip && !long_row && M.stage_x && d.xs.x >= 0;
    d.aux.w = stage_x ? 1 : 0;  // x windows staged (xs / xl keep the descriptor's values)
    sm.meta[s] = d;
    if (skip || long_row) {  // nothing staged (long rows are read from global)
        mbar_arrive_expect_tx(&sm.full[s], 0u);
        return;
    }
    const int32_t a0 = z0 & ~7, a1 = (z1 + 7) & ~7;
    const int32_t ra0 = r0 & ~3, ra1 = (r1 + 4) & ~3;
    const uint32_t ncol = static_cast<uint32_t>(a1 - a0);
    const uint32_t nrp = static_cast<uint32_t>(ra1 - ra0);
    const uint32_t nxw = stage_x ? static_cast<uint32_t>(d.xl.x + d.xl.y + d.xl.z + d.xl.w) : 0u;
    const uint32_t bytes = ncol * uint32_t(sizeof(int32_t) + sizeof(V)) + nrp * 4u +
                           nxw * uint32_t(sizeof(X)) * (XR ? 2u : 1u);
    auto& st = sm.st[s];
    mbar_arrive_expect_tx(&sm.full[s], bytes);
    if (ncol) {
        bulk_g2s(st.col, M.col_idx + a0, ncol * 4u, &sm.full[s]);
        bulk_g2s(st.val, M.values + a0, ncol * uint32_t(sizeof(V)), &sm.full[s]);
    }
    bulk_g2s(st.rp, M.row_ptr + ra0, nrp * 4u, &sm.full[s]);
    if (stage_x) {
        const int32_t ws[kXSeg] = {d.xs.x, d.xs.y, d.xs.z, d.xs.w};
        const int32_t wl[kXSeg] = {d.xl.x, d.xl.y, d.xl.z, d.xl.w};
        int32_t off = 0;
#pragma unroll
        for (int k = 0; k < kXSeg; ++k) {
            if (wl[k] > 0) {
                bulk_g2s(st.xw + off, x + ws[k], uint32_t(wl[k]) * uint32_t(sizeof(X)),
                         &sm.full[s]);
                if constexpr (XR)
                    bulk_g2s(st.xrw + off, xr + ws[k], uint32_t(wl[k]) * uint32_t(sizeof(X)),
                             &sm.full[s]);
            }
            off += wl[k];
        }
    }
}

// x entries that TMA did not stage: the read-only path, or L2 when x changes
// within the kernel (M.coherent_x).
template <typename V, typename X>
__device__ __forceinline__ X load_x(const CsrView<V>& M, const X* p) {
    return M.coherent_x ? __ldcg(p) : __ldg(p);
}

// Entry c of the multiplied vector: x[c], or with XR fma(beta, x[c], xr[c]).
template <bool XR, typename V, typename X>
__device__ __forceinline__ X load_xop(const CsrView<V>& M, const X* x, const X* xr, X beta,
                                      int32_t c) {
    if constexpr (XR) {
        static_assert(std::is_same_v<X, double>, "a formed x' is FP64 only");
        return fma(beta, load_x(M, x + c), load_x(M, xr + c));
    } else {
        return load_x(M, x + c);
    }
}

// One long row (nnz > TILE) straight from global memory, all consumers.
template <typename V, typename X, typename A, int TILE, int STAGES, bool XR, class Epi>
__device__ __forceinline__ void spmv_long_row(const CsrView<V>& M, bool ok, int32_t r0,
                                              int32_t z0, int32_t z1, const X* __restrict__ x,
                                              SpmvSmem<V, X, A, TILE, STAGES, XR>& sm, Epi& epi,
                                              const X* __restrict__ xr, X beta) {
    const int t = threadIdx.x;
    A s = A(0);
    for (int32_t j = (z0 & ~3) + 4 * t; ok && j < z1; j += 4 * kConsumers) {
        const int4 c = ld_stream(reinterpret_cast<const int4*>(M.col_idx + j));
        A v[4];
        Load4<V, A>::run(M.values, j, v);
        const int32_t cc[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int32_t jj = j + q;
            if (jj >= z0 && jj < z1)
                s += v[q] * static_cast<A>(load_xop<XR>(M, x, xr, beta, cc[q]));
        }
    }
    s = consumer_sum(s, sm.red);
    if (t == 0 && ok) epi(r0, s);
}

// Consumers: one staged multi-row block, straight from the staged operands.
// A row with <= short_max nonzeros is summed by one thread serially in CSR
// order; longer rows by a warp.  `ok` = this thread saw the stage complete;
// a thread that did not touches no staged data but takes the same barriers
// (the control flow depends only on the descriptor d).
// Where a gathered block keeps its products: in place of the values when they
// have the accumulator's width, else (BF16 values, FP32 accumulation) in place
// of the column indices.
template <typename V, typename X, typename A, int TILE>
__device__ __forceinline__ A* prod_slots(SpmvStage<V, X, TILE>& st) {
    if constexpr (sizeof(V) == sizeof(A)) {
        return reinterpret_cast<A*>(st.val);
    } else {
        static_assert(sizeof(A) == sizeof(int32_t), "products need a 4-byte slot");
        return reinterpret_cast<A*>(st.col);
    }
}

template <typename V, typename X, typename A, int TILE, int STAGES, bool XR, class Epi>
__device__ __forceinline__ void spmv_rows(const CsrView<V>& M, int s, bool ok, const BlockDesc& d,
                                          const X* __restrict__ x,
                                          SpmvSmem<V, X, A, TILE, STAGES, XR>& sm, Epi& epi,
                                          const X* __restrict__ xr, X beta) {
    const int t = threadIdx.x;
    const int lane = t & 31, warp = t >> 5;
    auto& st = sm.st[s];
    const int32_t r0 = d.rz.x, z0 = d.rz.z;
    const int nr = d.rz.y - r0;
    const int32_t a0 = z0 & ~7;
    const int32_t roff = r0 - (r0 & ~3);  // row r0's slot in the staged row_ptr
    // column -> staged x slot: window k holds columns [xs_k, xs_k + xl_k)
    const int32_t dl0 = -d.xs.x, dl1 = d.xl.x - d.xs.y, dl2 = d.xl.x + d.xl.y - d.xs.z,
                  dl3 = d.xl.x + d.xl.y + d.xl.z - d.xs.w;
    auto xval = [&](int32_t c) -> A {
        const int32_t dl = c >= d.xs.w ? dl3 : (c >= d.xs.z ? dl2 : (c >= d.xs.y ? dl1 : dl0));
        if constexpr (XR)
            return static_cast<A>(fma(beta, st.xw[c + dl], st.xrw[c + dl]));
        else
            return static_cast<A>(st.xw[c + dl]);
    };

    // A block without staged x windows (scattered columns) gathers first:
    // each consumer reads its share of the block's columns and values into
    // registers, issues all of its x loads at once, and parks the products
    // v_j * x[col_j] in the stage; after a consumer barrier the rows add the
    // products in CSR order (the same operations, in the same order, as
    // multiplying in the row loop).  Whether a block gathers is decided from
    // fields the producer leaves unchanged (the descriptor's windows and
    // M.stage_x), so consumers that gave up on the stage take the same
    // barrier.
    const bool gather = !(M.stage_x && d.xs.x >= 0);
    A* prod = prod_slots<V, X, A, TILE>(st);
    if (gather) {
        if (ok) {
            constexpr int G = (TILE + kConsumers - 1) / kConsumers;
            const int32_t j0 = z0 - a0 + t, j1 = d.rz.w - a0;
            int32_t c[G];
            A v[G], xv[G];
#pragma unroll
            for (int g = 0; g < G; ++g) {
                const int32_t j = j0 + g * kConsumers;
                c[g] = j < j1 ? st.col[j] : 0;
                v[g] = j < j1 ? widen<V, A>(st.val[j]) : A(0);
            }
#pragma unroll
            for (int g = 0; g < G; ++g)
                // through L2 (ld.global.cg): scattered columns rarely hit L1,
                // and skipping it raises the gather rate (power-law rows:
                // 299 -> 248 us per SpMV)
                if (j0 + g * kConsumers < j1) {
                    if constexpr (XR)
                        xv[g] = static_cast<A>(fma(beta, __ldcg(x + c[g]), __ldcg(xr + c[g])));
                    else
                        xv[g] = static_cast<A>(__ldcg(x + c[g]));
                }
#pragma unroll
            for (int g = 0; g < G; ++g) {
                const int32_t j = j0 + g * kConsumers;
                if (j < j1) prod[j] = mul_rn(v[g], xv[g]);
            }
        }
        consumer_sync();
    }

    bool is_long = false;
    if (ok && t < nr) {
        const int32_t s0 = st.rp[roff + t] - a0, s1 = st.rp[roff + t + 1] - a0;
        if (s1 - s0 <= M.short_max) {
            A acc = A(0);
            if (gather) {
                for (int32_t j = s0; j < s1; ++j) acc = add_rn(acc, prod[j]);
            } else {
                // serial CSR-order sum, operands fetched four at a time
                int32_t j = s0;
                for (; j + 4 <= s1; j += 4) {
                    int32_t c[4];
                    A v[4], xv[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        c[q] = st.col[j + q];
                        v[q] = widen<V, A>(st.val[j + q]);
                    }
#pragma unroll
                    for (int q = 0; q < 4; ++q) xv[q] = xval(c[q]);
#pragma unroll
                    for (int q = 0; q < 4; ++q) acc = add_rn(acc, mul_rn(v[q], xv[q]));
                }
                for (; j < s1; ++j)
                    acc = add_rn(acc, mul_rn(widen<V, A>(st.val[j]), xval(st.col[j])));
            }
            epi(r0 + t, acc);
        } else {
            is_long = true;
        }
    }
    if (d.aux.x == 0) return;  // no warp rows in this block

    // deterministic list of long rows in row order (ballot + warp prefix)
    const unsigned m = __ballot_sync(0xffffffffu, is_long);
    if (lane == 0) sm.warp_cnt[warp] = __popc(m);
    consumer_sync();
    int base = 0, nl = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
        const int cw = sm.warp_cnt[w];
        if (w < warp) base += cw;
        nl += cw;
    }
    if (is_long) sm.long_rows[base + __popc(m & ((1u << lane) - 1u))] = t;
    consumer_sync();

    // warp-per-row reduction of the long rows
    for (int q = warp; q < nl; q += kWarps) {
        const int tt = sm.long_rows[q];
        A acc = A(0);
        if (ok) {
            const int32_t s0 = st.rp[roff + tt] - a0, s1 = st.rp[roff + tt + 1] - a0;
            if (gather) {
                for (int32_t j = s0 + lane; j < s1; j += 32) acc += prod[j];
            } else {
                for (int32_t j = s0 + lane; j < s1; j += 32)
                    acc += mul_rn(widen<V, A>(st.val[j]), xval(st.col[j]));
            }
        }
        acc = warp_sum(acc);
        if (lane == 0 && ok) epi(r0 + tt, acc);
    }
    // long_rows / warp_cnt are next written after a consumer barrier of a later
    // block, which every warp reaches only after leaving this loop.
}

// The persistent pipelined loop over this CTA's row blocks, for all 288
// threads.  Returns false on the threads of a CTA where a bounded wait gave
// up (the error word is set; partial results must not be used).  On return
// no TMA copy into this CTA's shared memory is pending.
// With XR the vector multiplied is x' = fma(beta, x, xr), formed from staged
// windows of both (or gathered pairs) as it is read.
template <typename V, typename X, typename A, int TILE, int STAGES, bool XR = false, class Epi,
          class Gate = AllBlocks>
__device__ __forceinline__ bool spmv_pipeline(CsrView<V> M, const X* __restrict__ x,
                                              SpmvSmem<V, X, A, TILE, STAGES, XR>& sm, Epi& epi,
                                              unsigned int* err, const Gate& gate = Gate(),
                                              const X* __restrict__ xr = nullptr,
                                              X beta = X(0)) {
    const int t = threadIdx.x;
    const int warp = t >> 5, lane = t & 31;
    if (M.nblk_dev) M.nblk = __ldg(M.nblk_dev);
    if (t == 0) {
#pragma unroll
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&sm.full[s], 1);
            mbar_init(&sm.empty[s], kWarps);
        }
        fence_mbar_init();
    }
    __syncthreads();

    if (warp == kProducerWarp) {
        if (lane != 0) return true;
        // ---- producer ----
        uint32_t full_par = 0, empty_par = 0;  // bit s: parity of the next phase
        uint32_t used = 0;                     // bit s: stage s has been issued into
        bool ok = true;
        int s = 0;
        int64_t k = 0;
        // descriptors (with the gate's verdict in aux.z) are loaded one block ahead
        auto fetch = [&](int64_t bb) {
            BlockDesc dd = load_desc(M.desc + bb);
            dd.aux.z = gate(dd) ? 0 : 1;
            return dd;
        };
        // the block sum of the (released) block in stage q, to the epilogue
        auto finish = [&](int q) {
            if constexpr (Epi::kBlockSums) {
                double sum = 0.0;
#pragma unroll
                for (int w = 0; w < kWarps; ++w) sum += sm.blk_red[q][w];
                epi.finish_block(sm.bid[q], sm.meta[q], sum);
            }
        };
        BlockDesc next{};
        if (int64_t(blockIdx.x) < M.nblk) next = fetch(blockIdx.x);
        for (int64_t b = blockIdx.x; b < M.nblk; b += gridDim.x, ++k) {
            const BlockDesc d = next;
            if (b + gridDim.x < M.nblk) next = fetch(b + gridDim.x);
            if (k >= STAGES) {
                if (!mbar_wait_bounded(&sm.empty[s], (empty_par >> s) & 1u)) {
                    atomicOr(err, kErrWaitTimeout);
                    ok = false;
                    break;
                }
                empty_par ^= 1u << s;
                finish(s);
            }
            sm.bid[s] = b;
            spmv_issue<V, X, A, TILE, STAGES, XR>(M, x, d, sm, s, xr);
            full_par ^= 1u << s;
            used |= 1u << s;
            s = (s + 1 == STAGES) ? 0 : s + 1;
        }
        if constexpr (Epi::kBlockSums) {
            // the blocks still in the ring: wait for their release, finish them
            for (int q = 0; ok && q < STAGES; ++q) {
                if (!(used & (1u << q))) continue;
                if (!mbar_wait_bounded(&sm.empty[q], (empty_par >> q) & 1u)) {
                    atomicOr(err, kErrWaitTimeout);
                    ok = false;
                    break;
                }
                finish(q);
            }
        }
        // Drain: every stage's last copy has landed before the CTA may exit.
        for (int q = 0; q < STAGES; ++q)
            if (used & (1u << q)) mbar_wait_bounded(&sm.full[q], ((full_par >> q) & 1u) ^ 1u);
        return ok;
    }

    // ---- consumers ----
    // A consumer whose bounded wait gave up stops touching staged data and
    // waiting, but keeps taking the same barriers until the loop ends.
    uint32_t full_par = 0;
    bool failed = false;
    int s = 0;
    for (int64_t b = blockIdx.x; b < M.nblk; b += gridDim.x) {
        bool ok = false;
        if (!failed) {
            ok = mbar_wait_bounded(&sm.full[s], (full_par >> s) & 1u);
            if (!ok) {
                failed = true;
                atomicOr(err, kErrWaitTimeout);
            }
        }
        full_par ^= 1u << s;
        const BlockDesc d = ok ? sm.meta[s] : load_desc(M.desc + b);
        // A block the producer skipped (nothing staged) runs the same barrier
        // schedule as any other -- it depends only on d.rz and d.aux.x, equal in
        // the staged and the global descriptor -- with data access off, so
        // consumers that saw the stage and consumers that gave up stay in step.
        const bool active = ok && d.aux.z == 0;
        if (d.rz.w - d.rz.z > TILE)
            spmv_long_row<V, X, A, TILE, STAGES, XR>(M, active, d.rz.x, d.rz.z, d.rz.w, x, sm,
                                                     epi, xr, beta);
        else
            spmv_rows<V, X, A, TILE, STAGES, XR>(M, s, active, d, x, sm, epi, xr, beta);
        if constexpr (Epi::kBlockSums) {
            const double v = warp_sum(epi.take());
            if (lane == 0) sm.blk_red[s][warp] = v;  // published by the arrival below
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&sm.empty[s]);  // this warp is done with stage s
        s = (s + 1 == STAGES) ? 0 : s + 1;
    }
    return !failed;
}

// Epilogue: y[row] = value.
template <typename X, typename A>
struct StoreEpi {
    static constexpr bool kBlockSums = false;
    X* __restrict__ y;
    __device__ __forceinline__ void operator()(int32_t row, A v) { y[row] = static_cast<X>(v); }
    __device__ __forceinline__ double take() { return 0.0; }
    __device__ __forceinline__ void finish_block(int64_t, const BlockDesc&, double) {}
};

// Dynamic shared memory of the pipelined kernels.
template <typename V, typename X, typename A, int TILE, int STAGES, bool XR = false>
constexpr size_t spmv_smem_bytes() {
    return sizeof(SpmvSmem<V, X, A, TILE, STAGES, XR>);
}

}  // namespace nm
