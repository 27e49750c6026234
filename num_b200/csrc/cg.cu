// cg.cu -- conjugate gradient with device-resident scalars.
//
// Same algorithm, stopping rule and iteration count as cg_solve_local
// (src/cg_solver.hpp:133-196) and, with the breakdown guard, as
// cg_solve_distributed at one rank (src/cg_solver.hpp:38-125).  The reference
// runs 5 launches, 5 fences and 2 device->host scalar copies per iteration;
// here one iteration is three kernels that never return to the host:
//
//   K1 spmv_pap : Ap = A p fused with p.Ap (row epilogue); last CTA: alpha
//   K2 update_xr: x += alpha p, r -= alpha Ap, r.r; last CTA: stopping test,
//                 beta, iteration count
//   K3 update_p : p = r + beta p
//
// Each kernel returns at once when the solve is done, so the host enqueues
// iterations in CUDA-graph chunks and polls the done flag between chunks.
// HBM per iteration: 12 nnz + 4(n+1) (matrix) + 8n (p gather, L2-resident
// in steady state) + 8n (Ap write) in K1; 4 reads + 2 writes of n doubles in
// K2; 2 reads + 1 write in K3 -- 12 nnz + 4(n+1) + 88 n bytes.
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "cg.cuh"
#include "spmv.cuh"

namespace nm {

__global__ void __launch_bounds__(kThreads)
    cg_init_kernel(int64_t n, CgState* st, const double* __restrict__ Ap, double* __restrict__ r,
                   double* __restrict__ p, double* partials) {
    __shared__ double red[kWarps];
    const double* __restrict__ b = st->b;
    double srr = 0.0, sbb = 0.0;
    for (int64_t i = int64_t(blockIdx.x) * kThreads + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * kThreads) {
        const double bi = b[i];
        const double ri = fma(-1.0, Ap[i], bi);  // r = -1*Ap + b
        r[i] = ri;
        p[i] = ri;
        srr = fma(ri, ri, srr);
        sbb = fma(bi, bi, sbb);
    }
    double part[2];
    part[0] = block_sum(srr, red);
    part[1] = block_sum(sbb, red);
    double tot[2];
    if (grid_reduce_last<2>(part, partials, &st->counter, tot, red)) {
        const double rr = tot[0];
        double bnorm = sqrt(tot[1]);
        if (bnorm == 0.0) bnorm = 1.0;
        st->bnorm = bnorm;
        st->rr = rr;
        st->iter = 0;
        st->status = kCgOk;
        const double rel = sqrt(rr) / bnorm;
        if (rel < st->tol) {
            st->done = 1; st->converged = 1; st->iters = 0; st->final_res = rel;
        } else if (st->max_iter <= 0) {
            st->done = 1; st->converged = 0; st->iters = st->max_iter; st->final_res = rel;
        } else {
            st->done = 0; st->converged = 0;
        }
    }
}

// Row epilogue of K1: store Ap and accumulate p.Ap; the producer hands one
// sum per row block to partials[block].
struct PApEpi {
    static constexpr bool kBlockSums = true;
    double* __restrict__ Ap;
    const double* __restrict__ p;
    double* __restrict__ part;
    double dot;
    __device__ __forceinline__ void operator()(int32_t row, double v) {
        Ap[row] = v;
        dot = fma(__ldg(p + row), v, dot);
    }
    __device__ __forceinline__ double take() {
        const double d = dot;
        dot = 0.0;
        return d;
    }
    __device__ __forceinline__ void finish_block(int64_t b, const BlockDesc&, double sum) {
        part[b] = sum;
    }
};

template <int TILE, int STAGES>
__global__ void __launch_bounds__(kCtaThreads)
    cg_spmv_pap_kernel(const CsrView<double> M, CgState* st, const double* __restrict__ p,
                       double* __restrict__ Ap, double* partials, unsigned int* err) {
    if (__ldcg(&st->done)) return;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    auto& sm = *reinterpret_cast<SpmvSmem<double, double, double, TILE, STAGES>*>(smem_raw);
    __shared__ bool am_last;
    PApEpi epi{Ap, p, partials, 0.0};
    const bool ok = spmv_pipeline<double, double, double, TILE, STAGES>(M, p, sm, epi, err);
    if (!ok && threadIdx.x == 0) {
        // A bounded wait gave up: end the solve; every CTA still arrives below
        // so the arrival counter stays consistent.
        atomicExch(&st->status, kCgDeviceError);
        atomicExch(&st->done, 1);
    }
    // the last CTA to arrive adds the per-block sums in the fixed order
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        am_last = atomicAdd(&st->counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!am_last) return;
    __threadfence();
    const double pAp_t = reduce256(partials, M.nblk, sm.red);
    if (threadIdx.x == 0) {
        st->counter = 0u;
        const double pAp = pAp_t;
        st->pAp = pAp;
        if (st->guard && fabs(pAp) < 1e-300) {
            st->status = kCgBreakdown;
            st->done = 1;
            st->converged = 0;
            st->iters = st->iter;
            st->final_res = sqrt(st->rr) / st->bnorm;
        } else {
            st->alpha = st->rr / pAp;
        }
    }
}

__global__ void __launch_bounds__(kThreads, 8)
    cg_update_xr_kernel(int64_t n, CgState* st, const double* __restrict__ p,
                        const double* __restrict__ Ap, double* __restrict__ r, double* partials) {
    if (__ldcg(&st->done)) return;
    __shared__ double red[kWarps];
    const double alpha = __ldcg(&st->alpha);
    double* __restrict__ x = st->x;
    double s = 0.0;
    const int64_t S = int64_t(gridDim.x) * kThreads;
    if (n <= S) {  // one element per thread: the order the persistent solves share
        const int64_t i = int64_t(blockIdx.x) * kThreads + threadIdx.x;
        if (i < n) {
            const double pi = p[i];
            x[i] = fma(alpha, pi, x[i]);            // x = alpha*p + x
            const double ri = fma(-alpha, Ap[i], r[i]);  // r = -alpha*Ap + r
            r[i] = ri;
            s = fma(ri, ri, s);
        }
    } else {
        // Larger systems (the CUDA-graph path alone): four consecutive
        // elements per thread and step, p, Ap, r read 16 bytes at a time (the
        // workspace vectors are 256-byte aligned), x element by element (the
        // caller's vector may be 8-byte aligned only); r.r in element order.
        for (int64_t q = int64_t(blockIdx.x) * kThreads + threadIdx.x; 4 * q < n; q += S) {
            const int64_t i0 = 4 * q;
            if (i0 + 4 <= n) {
                const double2 p01 = *reinterpret_cast<const double2*>(p + i0);
                const double2 p23 = *reinterpret_cast<const double2*>(p + i0 + 2);
                const double2 a01 = *reinterpret_cast<const double2*>(Ap + i0);
                const double2 a23 = *reinterpret_cast<const double2*>(Ap + i0 + 2);
                const double2 r01 = *reinterpret_cast<const double2*>(r + i0);
                const double2 r23 = *reinterpret_cast<const double2*>(r + i0 + 2);
                const double pv[4] = {p01.x, p01.y, p23.x, p23.y};
                const double av[4] = {a01.x, a01.y, a23.x, a23.y};
                const double rv0[4] = {r01.x, r01.y, r23.x, r23.y};
                double xv[4], rv[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) xv[e] = x[i0 + e];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    x[i0 + e] = fma(alpha, pv[e], xv[e]);     // x = alpha*p + x
                    rv[e] = fma(-alpha, av[e], rv0[e]);      // r = -alpha*Ap + r
                    s = fma(rv[e], rv[e], s);
                }
                *reinterpret_cast<double2*>(r + i0) = make_double2(rv[0], rv[1]);
                *reinterpret_cast<double2*>(r + i0 + 2) = make_double2(rv[2], rv[3]);
            } else {
                for (int64_t i = i0; i < n; ++i) {
                    const double pi = p[i];
                    x[i] = fma(alpha, pi, x[i]);
                    const double ri = fma(-alpha, Ap[i], r[i]);
                    r[i] = ri;
                    s = fma(ri, ri, s);
                }
            }
        }
    }
    double part[1] = {block_sum(s, red)};
    double tot[1];
    if (grid_reduce_last<1>(part, partials, &st->counter, tot, red)) {
        const double rr_new = tot[0];
        const int32_t it = st->iter + 1;
        st->iter = it;
        const double rel = sqrt(rr_new) / st->bnorm;
        if (rel < st->tol) {
            st->done = 1; st->converged = 1; st->iters = it; st->final_res = rel;
        } else {
            if (it >= st->max_iter) {
                st->done = 1; st->converged = 0; st->iters = st->max_iter; st->final_res = rel;
            }
            st->beta = rr_new / st->rr;
            st->rr = rr_new;
        }
    }
}

__global__ void __launch_bounds__(kThreads)
    cg_update_p_kernel(int64_t n, const CgState* st, double* __restrict__ p,
                       const double* __restrict__ r) {
    if (__ldcg(&st->done)) return;
    const double beta = __ldcg(&st->beta);
    for (int64_t i = int64_t(blockIdx.x) * kThreads + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * kThreads)
        p[i] = fma(beta, p[i], r[i]);  // p = 1*r + beta*p
}

// ---------------------------------------------------------------------------
// Persistent CG: the whole iteration loop in one cooperative launch.
//
// The grid is the SpMV grid of the three-kernel path (every CTA resident, so a
// grid-wide barrier can be met), and each phase reproduces that path exactly:
//   A  the same SpMV pipeline with the same p.Ap epilogue and CTA sum; every
//      CTA then reduces the CTA sums in the order the three-kernel path's
//      last CTA uses (stride blockDim over gridDim);
//   B  x, r update and r.r over "virtual CTAs" v = blockIdx.x, + gridDim.x,
//      ... < grid_vec of 256 threads, with cg_update_xr_kernel's element
//      mapping and CTA sum, and the same final reduction;
//   C  p = r + beta p (elementwise) -- or, in the two-barrier form, folded
//      into the next iteration's phase A (see CoopFormPApEpi).
// So the iterates are bit-identical to nm_cg_local's graph path.  Every CTA
// computes the scalars itself (identically); CTA 0 publishes the final state.
// Data written inside the kernel is read with ld.global.cg (L2), never through
// the non-coherent read-only path.  Three (two) grid barriers per iteration
// replace the kernel boundaries; each wait is bounded (kWaitLimitNs): a CTA that gives
// up sets the error word and the state to kCgDeviceError and leaves, and the
// others give up at their next barrier.
// ---------------------------------------------------------------------------

struct CoopPApEpi {
    static constexpr bool kBlockSums = true;
    double* __restrict__ Ap;
    const double* __restrict__ p;
    double* __restrict__ part;  // p.Ap per row block
    double dot;
    __device__ __forceinline__ void operator()(int32_t row, double v) {
        Ap[row] = v;
        dot = fma(__ldcg(p + row), v, dot);
    }
    __device__ __forceinline__ double take() {
        const double d = dot;
        dot = 0.0;
        return d;
    }
    __device__ __forceinline__ void finish_block(int64_t b, const BlockDesc&, double sum) {
        part[b] = sum;
    }
};

// Row epilogue of the two-barrier form: the row's new direction
// p'[row] = fma(beta, p[row], r[row]) (what the three-kernel path's p update
// computes) goes to the other p buffer, then Ap and p'.Ap as in CoopPApEpi.
struct CoopFormPApEpi {
    static constexpr bool kBlockSums = true;
    double* __restrict__ Ap;
    const double* __restrict__ p;
    const double* __restrict__ r;
    double* __restrict__ pn;
    double* __restrict__ part;
    double beta;
    double dot;
    __device__ __forceinline__ void operator()(int32_t row, double v) {
        Ap[row] = v;
        const double pr = fma(beta, __ldcg(p + row), __ldcg(r + row));
        pn[row] = pr;
        dot = fma(pr, v, dot);
    }
    __device__ __forceinline__ double take() {
        const double d = dot;
        dot = 0.0;
        return d;
    }
    __device__ __forceinline__ void finish_block(int64_t b, const BlockDesc&, double sum) {
        part[b] = sum;
    }
};

// Step 1 of the CUDA-graph path in its formed version (where the two sets of
// staged windows fit the SM): the SpMV multiplies by p' = fma(beta, p_in, r)
// formed from staged windows of both -- the operation the p update kernel
// performs, on the same operands, in every CTA that reads a column -- each
// row's owner writes p'[row] to p_out, and step 2 updates x with p_out; the
// p update kernel goes.  The buffers alternate by iteration; the first
// iteration of a solve forms fma(0, p0, r0) = r0 = p0 (beta is 0 in the
// initial state), so the iterates are those of the three-kernel form.
template <int TILE, int STAGES>
__global__ void __launch_bounds__(kCtaThreads)
    cg_spmv_pap_formed_kernel(const CsrView<double> M, CgState* st,
                              const double* __restrict__ p_in, double* __restrict__ p_out,
                              const double* __restrict__ r, double* __restrict__ Ap,
                              double* partials, unsigned int* err) {
    if (__ldcg(&st->done)) return;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    auto& sm = *reinterpret_cast<SpmvSmem<double, double, double, TILE, STAGES, true>*>(smem_raw);
    __shared__ bool am_last;
    const double beta = __ldcg(&st->beta);
    CoopFormPApEpi epi{Ap, p_in, r, p_out, partials, beta, 0.0};
    const bool ok = spmv_pipeline<double, double, double, TILE, STAGES, true>(
        M, p_in, sm, epi, err, AllBlocks(), r, beta);
    if (!ok && threadIdx.x == 0) {
        // A bounded wait gave up: end the solve; every CTA still arrives below
        // so the arrival counter stays consistent.
        atomicExch(&st->status, kCgDeviceError);
        atomicExch(&st->done, 1);
    }
    // the last CTA to arrive adds the per-block sums in the fixed order
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        am_last = atomicAdd(&st->counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!am_last) return;
    __threadfence();
    const double pAp = reduce256(partials, M.nblk, sm.red);
    if (threadIdx.x == 0) {
        st->counter = 0u;
        st->pAp = pAp;
        if (st->guard && fabs(pAp) < 1e-300) {
            st->status = kCgBreakdown;
            st->done = 1;
            st->converged = 0;
            st->iters = st->iter;
            st->final_res = sqrt(st->rr) / st->bnorm;
        } else {
            st->alpha = st->rr / pAp;
        }
    }
}

// FORMED: the two-barrier form.  Phase C disappears: the next iteration's
// SpMV multiplies by p' = fma(beta, p, r) formed from staged windows of p and
// r (the same operation on the same operands in every CTA that reads a
// column), and each row's owner writes p'[row] to the other p buffer for
// phase B; the buffers alternate.  The first iteration forms p' = fma(0, p0,
// r0) = r0 = p0.  Same iterates as the three-barrier form, one grid barrier
// fewer per iteration, at the cost of a second set of staged windows.
template <int TILE, int STAGES, bool FORMED>
__global__ void __launch_bounds__(kCtaThreads, 2)
    cg_coop_kernel(CsrView<double> M, CgState* st, double* p, double* p2, double* Ap, double* r,
                   double* part_a, double* part_b, int grid_vec, int64_t n, unsigned int* err) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    auto& sm = *reinterpret_cast<SpmvSmem<double, double, double, TILE, STAGES, FORMED>*>(smem_raw);
    __shared__ double bcast[2];
    __shared__ bool flag;
    const int t = threadIdx.x;
    // the state after cg_init_kernel
    if (__ldcg(&st->done)) return;
    double* __restrict__ x = st->x;
    const double bnorm = __ldcg(&st->bnorm), tol = __ldcg(&st->tol);
    const int32_t max_iter = __ldcg(&st->max_iter), guard = __ldcg(&st->guard);
    double rr = __ldcg(&st->rr);
    int32_t iter = __ldcg(&st->iter);
    M.coherent_x = 1;
    bool failed = false;
    double beta_prev = 0.0;  // FORMED: beta of the previous iteration
    for (;;) {
        // ---- A: Ap = A p, p.Ap (FORMED: p' = fma(beta_prev, p, r) formed on the fly) ----
        double* pa_vec = p;  // the direction of this iteration
        bool ok;
        if constexpr (FORMED) {
            pa_vec = p2;
            CoopFormPApEpi epi{Ap, p, r, p2, part_a, beta_prev, 0.0};
            ok = spmv_pipeline<double, double, double, TILE, STAGES, true>(M, p, sm, epi, err,
                                                                          AllBlocks(), r,
                                                                          beta_prev);
        } else {
            CoopPApEpi epi{Ap, p, part_a, 0.0};
            ok = spmv_pipeline<double, double, double, TILE, STAGES>(M, p, sm, epi, err);
        }
        __syncthreads();
        if (t == 0) {  // the ring's barriers are initialised again by the next SpMV
#pragma unroll
            for (int q = 0; q < STAGES; ++q) {
                asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(&sm.full[q]))
                             : "memory");
                asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(&sm.empty[q]))
                             : "memory");
            }
        }
        if (!ok) atomicExch(&st->status, kCgDeviceError);
        // the producer left one p.Ap sum per row block in part_a
        if (!grid_barrier(&st->bar_count, &st->bar_gen, err, &st->status, &flag)) { failed = true; break; }
        const double pAp = reduce256(part_a, M.nblk, sm.red);
        if (t == 0) bcast[0] = pAp;
        __syncthreads();
        const double pAp_all = bcast[0];
        if (guard && fabs(pAp_all) < 1e-300) {
            if (blockIdx.x == 0 && t == 0) {
                st->pAp = pAp_all;
                st->status = kCgBreakdown;
                st->converged = 0;
                st->iters = iter;
                st->final_res = sqrt(rr) / bnorm;
                st->done = 1;
            }
            return;
        }
        const double alpha = rr / pAp_all;
        // ---- B: x += alpha p, r -= alpha Ap, r.r (virtual CTAs of 256 threads) ----
        for (int v = blockIdx.x; v < grid_vec; v += gridDim.x) {
            double sv = 0.0;
            if (t < kThreads) {
                for (int64_t i = int64_t(v) * kThreads + t; i < n; i += int64_t(grid_vec) * kThreads) {
                    const double pi = __ldcg(pa_vec + i);
                    x[i] = fma(alpha, pi, __ldcg(x + i));
                    const double ri = fma(-alpha, __ldcg(Ap + i), __ldcg(r + i));
                    r[i] = ri;
                    sv = fma(ri, ri, sv);
                }
            }
            const double pv = block_sum8(sv, sm.red);
            if (t == 0) part_b[v] = pv;
        }
        if (!grid_barrier(&st->bar_count, &st->bar_gen, err, &st->status, &flag)) { failed = true; break; }
        const double rr_new0 = reduce256(part_b, grid_vec, sm.red);
        if (t == 0) bcast[1] = rr_new0;
        __syncthreads();
        const double rr_new = bcast[1];
        ++iter;
        const double rel = sqrt(rr_new) / bnorm;
        if (rel < tol) {
            if (blockIdx.x == 0 && t == 0) {
                st->iter = iter; st->converged = 1; st->iters = iter; st->final_res = rel;
                st->rr = rr_new; st->done = 1;
            }
            return;
        }
        const double beta = rr_new / rr;
        rr = rr_new;
        if (iter >= max_iter) {
            if (blockIdx.x == 0 && t == 0) {
                st->iter = iter; st->converged = 0; st->iters = max_iter; st->final_res = rel;
                st->beta = beta; st->rr = rr; st->done = 1;
            }
            return;
        }
        if constexpr (FORMED) {
            // the next SpMV forms p from this iteration's direction and r
            double* const q = p;
            p = p2;
            p2 = q;
            beta_prev = beta;
        } else {
            // ---- C: p = r + beta p ----
            for (int64_t i = int64_t(blockIdx.x) * blockDim.x + t; i < n;
                 i += int64_t(gridDim.x) * blockDim.x)
                p[i] = fma(beta, __ldcg(p + i), __ldcg(r + i));
            if (!grid_barrier(&st->bar_count, &st->bar_gen, err, &st->status, &flag)) { failed = true; break; }
        }
    }
    if (failed && t == 0) {
        atomicExch(&st->status, kCgDeviceError);
        atomicExch(&st->done, 1);
    }
}

namespace {
std::atomic<int> g_cg_persistent{1};  // nm_cg_set_persistent
// Largest system solved by the persistent launch; larger ones keep the graph
// path (their vector phases need more CTAs than the SpMV grid has).
constexpr int64_t kCoopMaxRows = 262144;
}  // namespace

namespace {

// Pinned host slots for the CG state copies: slabs allocated once
// (portable pinned memory, kept until exit) and handed out per workspace, so
// a solve on a new matrix pays no page-locking and its teardown no pinned free.
class PinnedSlots {
  public:
    CgState* get() {
        std::lock_guard<std::mutex> g(mu_);
        if (free_.empty()) {
            constexpr int kSlab = 256;
            void* slab = nullptr;
            if (cudaHostAlloc(&slab, sizeof(CgState) * kSlab, cudaHostAllocPortable) != cudaSuccess)
                return nullptr;
            auto* c = static_cast<CgState*>(slab);
            for (int i = kSlab - 1; i >= 0; --i) free_.push_back(c + i);
        }
        CgState* out = free_.back();
        free_.pop_back();
        return out;
    }
    void put(CgState* c) {
        if (!c) return;
        std::lock_guard<std::mutex> g(mu_);
        free_.push_back(c);
    }

  private:
    std::mutex mu_;
    std::vector<CgState*> free_;
};

PinnedSlots& pinned_slots() {
    static PinnedSlots* s = new PinnedSlots();  // never destroyed: slots outlive statics
    return *s;
}

}  // namespace

CgWorkspace::~CgWorkspace() {
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
    if (cap_stream) cudaStreamDestroy(cap_stream);
    cudaFree(dmem);
    if (res_mem) cudaFree(res_mem);
    if (cl_mem) cudaFree(cl_mem);
    pinned_slots().put(h_in);
    pinned_slots().put(h_out);
}

namespace {

template <int TILE, int STAGES>
int prepare_cg_spmv(int* occ) {
    return prepare_kernel(reinterpret_cast<const void*>(cg_spmv_pap_kernel<TILE, STAGES>),
                          kCtaThreads, spmv_smem_bytes<double, double, double, TILE, STAGES>(),
                          occ);
}

template <int TILE, int STAGES>
int prepare_cg_spmv_formed(int* occ) {
    return prepare_kernel(
        reinterpret_cast<const void*>(cg_spmv_pap_formed_kernel<TILE, STAGES>), kCtaThreads,
        spmv_smem_bytes<double, double, double, TILE, STAGES, true>(), occ);
}

template <int TILE>
int prepare_cg_spmv_formed_s(int stages, int* occ) {
    if (stages == 4) return prepare_cg_spmv_formed<TILE, 4>(occ);
    return stages == 3 ? prepare_cg_spmv_formed<TILE, 3>(occ) : prepare_cg_spmv_formed<TILE, 2>(occ);
}

template <int TILE, int STAGES, bool FORMED>
int prepare_coop(int* occ) {
    return prepare_kernel(reinterpret_cast<const void*>(cg_coop_kernel<TILE, STAGES, FORMED>),
                          kCtaThreads,
                          spmv_smem_bytes<double, double, double, TILE, STAGES, FORMED>(), occ);
}

template <int TILE, bool FORMED>
int prepare_coop_s(int stages, int* occ) {
    if (stages == 4) return prepare_coop<TILE, 4, FORMED>(occ);
    return stages == 3 ? prepare_coop<TILE, 3, FORMED>(occ) : prepare_coop<TILE, 2, FORMED>(occ);
}

template <bool FORMED>
int prepare_coop_t(int tile, int stages, int* occ) {
    switch (tile) {
        case 1024: return prepare_coop_s<1024, FORMED>(stages, occ);
        case 4096: return prepare_coop_s<4096, FORMED>(stages, occ);
        default: return prepare_coop_s<2048, FORMED>(stages, occ);
    }
}

template <int TILE>
int prepare_cg_spmv_s(int stages, int* occ) {
    if (stages == 4) return prepare_cg_spmv<TILE, 4>(occ);
    return stages == 3 ? prepare_cg_spmv<TILE, 3>(occ) : prepare_cg_spmv<TILE, 2>(occ);
}

int ensure_workspace(nm_csr* A, CgWorkspace** out) {
    if (A->cg) {
        *out = A->cg.get();
        return NM_OK;
    }
    auto ws = std::make_unique<CgWorkspace>();
    const int64_t n = A->nrows;
    ws->n = n;
    // Above the persistent solves' limit only the CUDA-graph path runs: its
    // vector kernels take two CTAs per SM (fewer CTA sums for each last-CTA
    // reduction; 1 M rows: 37.8 us per iteration against 44.9 us with eight);
    // below it, one element per thread, the order every path shares.
    ws->grid_vec = n > kCoopMaxRows ? sm_count() * 2 : vec_grid(n);
    ws->h_in = pinned_slots().get();
    ws->h_out = pinned_slots().get();
    if (!ws->h_in || !ws->h_out) return fail(NM_ERR_NOMEM, "cg: no pinned host memory");
    // Load the iteration kernels and set their shared-memory attributes now
    // (lazy module loading), not during graph capture.
    cudaFuncAttributes fa;
    NM_CUDA_TRY(cudaFuncGetAttributes(&fa, cg_update_xr_kernel));
    NM_CUDA_TRY(cudaFuncGetAttributes(&fa, cg_update_p_kernel));
    int occ = 0, st = NM_OK;
    switch (A->tune.tile) {
        case 1024: st = prepare_cg_spmv_s<1024>(A->tune.stages, &occ); break;
        case 4096: st = prepare_cg_spmv_s<4096>(A->tune.stages, &occ); break;
        default: st = prepare_cg_spmv_s<2048>(A->tune.stages, &occ); break;
    }
    if (st != NM_OK) return st;
    ws->grid_spmv = spmv_grid(A, occ);
    {
        int occ_g = 0;
        switch (A->tune.tile) {
            case 1024: st = prepare_cg_spmv_formed_s<1024>(A->tune.stages, &occ_g); break;
            case 4096: st = prepare_cg_spmv_formed_s<4096>(A->tune.stages, &occ_g); break;
            default: st = prepare_cg_spmv_formed_s<2048>(A->tune.stages, &occ_g); break;
        }
        if (st != NM_OK) return st;
        ws->graph_formed = occ_g > 0;
        if (ws->graph_formed) ws->grid_spmv_f = spmv_grid(A, occ_g);
    }
    // K1 leaves one sum per row block, K2 one per vector CTA, the initial
    // kernel two per vector CTA; the persistent solve keeps the block sums and
    // the vector sums side by side
    ws->partials_cap = static_cast<int>(A->nblk) + 2 * ws->grid_vec;
    {
        // r, p, Ap, p2, the CTA partial sums and the state in one allocation
        // (each part 256-byte aligned)
        auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
        const size_t vb = up(sizeof(double) * size_t(n));
        const size_t pb = up(sizeof(double) * size_t(ws->partials_cap));
        NM_CUDA_TRY(cudaMalloc(&ws->dmem, 4 * vb + pb + up(sizeof(CgState))));
        auto* base = static_cast<unsigned char*>(ws->dmem);
        ws->r = reinterpret_cast<double*>(base);
        ws->p = reinterpret_cast<double*>(base + vb);
        ws->Ap = reinterpret_cast<double*>(base + 2 * vb);
        ws->p2 = reinterpret_cast<double*>(base + 3 * vb);
        ws->partials = reinterpret_cast<double*>(base + 4 * vb);
        ws->st = reinterpret_cast<CgState*>(base + 4 * vb + pb);  // written by every solve
    }
    {
        // The persistent solve runs on the same grid, every CTA resident.
        int dev = 0, coop_ok = 0, occ_c = 0, occ_f = 0;
        NM_CUDA_TRY(cudaGetDevice(&dev));
        NM_CUDA_TRY(cudaDeviceGetAttribute(&coop_ok, cudaDevAttrCooperativeLaunch, dev));
        st = prepare_coop_t<false>(A->tune.tile, A->tune.stages, &occ_c);
        if (st != NM_OK) return st;
        st = prepare_coop_t<true>(A->tune.tile, A->tune.stages, &occ_f);
        if (st != NM_OK) return st;
        // Large systems keep the graph path: their update phases need more CTAs
        // than the SpMV grid has.  The two-barrier form stages twice the
        // windows, so fewer of its CTAs fit an SM; where the grid does not fit
        // it, the three-barrier form runs.
        const bool fits = coop_ok && n <= kCoopMaxRows;
        ws->coop_formed = fits && int64_t(occ_f) * sm_count() >= ws->grid_spmv;
        ws->coop = ws->coop_formed || (fits && int64_t(occ_c) * sm_count() >= ws->grid_spmv);
        if (coop_ok) {
            st = plan_resident(A, ws.get());
            if (st != NM_OK) return st;
        }
        st = plan_cluster(A, ws.get());
        if (st != NM_OK) return st;
    }
    ws->err = device_error_word();
    if (!ws->err) return fail(NM_ERR_CUDA, "cg: cannot map the device error word");
    A->cg = std::move(ws);
    *out = A->cg.get();
    return NM_OK;
}

// One iteration of the CUDA-graph path: three kernels, or (graph_formed) two,
// the direction read from p (parity 0) or p2 (parity 1) and formed into the
// other buffer.
template <int TILE, int STAGES>
void launch_iteration_t(const nm_csr* A, CgWorkspace* ws, cudaStream_t s, int parity) {
    CsrView<double> M = A->view<double>();
    M.stage_x = 1;  // p, p2 and r are workspace vectors (256-byte aligned)
    if (ws->graph_formed) {
        double* p_in = parity ? ws->p2 : ws->p;
        double* p_out = parity ? ws->p : ws->p2;
        cg_spmv_pap_formed_kernel<TILE, STAGES>
            <<<ws->grid_spmv_f, kCtaThreads,
               spmv_smem_bytes<double, double, double, TILE, STAGES, true>(), s>>>(
                M, ws->st, p_in, p_out, ws->r, ws->Ap, ws->partials, ws->err);
        cg_update_xr_kernel<<<ws->grid_vec, kThreads, 0, s>>>(ws->n, ws->st, p_out, ws->Ap,
                                                              ws->r, ws->partials);
        return;
    }
    cg_spmv_pap_kernel<TILE, STAGES>
        <<<ws->grid_spmv, kCtaThreads, spmv_smem_bytes<double, double, double, TILE, STAGES>(), s>>>(
            M, ws->st, ws->p, ws->Ap, ws->partials, ws->err);
    cg_update_xr_kernel<<<ws->grid_vec, kThreads, 0, s>>>(ws->n, ws->st, ws->p, ws->Ap, ws->r,
                                                          ws->partials);
    cg_update_p_kernel<<<ws->grid_vec, kThreads, 0, s>>>(ws->n, ws->st, ws->p, ws->r);
}

template <int TILE>
void launch_iteration_s(const nm_csr* A, CgWorkspace* ws, cudaStream_t s, int parity) {
    if (A->tune.stages == 4) launch_iteration_t<TILE, 4>(A, ws, s, parity);
    else if (A->tune.stages == 3) launch_iteration_t<TILE, 3>(A, ws, s, parity);
    else launch_iteration_t<TILE, 2>(A, ws, s, parity);
}

void launch_iteration(const nm_csr* A, CgWorkspace* ws, cudaStream_t s, int parity) {
    switch (A->tune.tile) {
        case 1024: launch_iteration_s<1024>(A, ws, s, parity); break;
        case 4096: launch_iteration_s<4096>(A, ws, s, parity); break;
        default: launch_iteration_s<2048>(A, ws, s, parity); break;
    }
}

// A CUDA graph of `iters` CG iterations (2 or 3 kernels each), captured once
// per workspace and chunk length, replayed on the caller's stream.
int chunk_graph(const nm_csr* A, CgWorkspace* ws, int iters, cudaGraphExec_t* out) {
    auto it = ws->graphs.find(iters);
    if (it != ws->graphs.end()) {
        *out = it->second;
        return NM_OK;
    }
    cudaGraph_t g = nullptr;
    if (!ws->cap_stream)
        NM_CUDA_TRY(cudaStreamCreateWithFlags(&ws->cap_stream, cudaStreamNonBlocking));
    NM_CUDA_TRY(cudaStreamBeginCapture(ws->cap_stream, cudaStreamCaptureModeThreadLocal));
    // chunks are of even length, so every chunk starts with the direction in p
    for (int i = 0; i < iters; ++i) launch_iteration(A, ws, ws->cap_stream, i & 1);
    cudaError_t e = cudaStreamEndCapture(ws->cap_stream, &g);
    if (e != cudaSuccess) return fail(NM_ERR_CUDA, "CG graph capture failed: %s", cudaGetErrorString(e));
    cudaGraphExec_t ex = nullptr;
    e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess)
        return fail(NM_ERR_CUDA, "CG graph instantiate failed: %s", cudaGetErrorString(e));
    ws->graphs[iters] = ex;
    *out = ex;
    return NM_OK;
}

template <int TILE, int STAGES, bool FORMED>
int launch_coop_t(const nm_csr* A, CgWorkspace* ws, cudaStream_t s) {
    CsrView<double> M = A->view<double>();
    M.stage_x = 1;  // p, p2 and r are workspace vectors (256-byte aligned)
    double* part_a = ws->partials;
    double* part_b = ws->partials + A->nblk;
    int grid_vec = ws->grid_vec;
    int64_t n = ws->n;
    void* args[] = {&M,     &ws->st, &ws->p,    &ws->p2, &ws->Ap, &ws->r,
                    &part_a, &part_b, &grid_vec, &n,      &ws->err};
    NM_CUDA_TRY(cudaLaunchCooperativeKernel(
        reinterpret_cast<const void*>(cg_coop_kernel<TILE, STAGES, FORMED>),
        dim3(ws->grid_spmv), dim3(kCtaThreads), args,
        spmv_smem_bytes<double, double, double, TILE, STAGES, FORMED>(), s));
    return NM_OK;
}

template <int TILE, bool FORMED>
int launch_coop_s(const nm_csr* A, CgWorkspace* ws, cudaStream_t s) {
    if (A->tune.stages == 4) return launch_coop_t<TILE, 4, FORMED>(A, ws, s);
    if (A->tune.stages == 3) return launch_coop_t<TILE, 3, FORMED>(A, ws, s);
    return launch_coop_t<TILE, 2, FORMED>(A, ws, s);
}

template <bool FORMED>
int launch_coop_f(const nm_csr* A, CgWorkspace* ws, cudaStream_t s) {
    switch (A->tune.tile) {
        case 1024: return launch_coop_s<1024, FORMED>(A, ws, s);
        case 4096: return launch_coop_s<4096, FORMED>(A, ws, s);
        default: return launch_coop_s<2048, FORMED>(A, ws, s);
    }
}

int launch_coop(const nm_csr* A, CgWorkspace* ws, cudaStream_t s) {
    return ws->coop_formed ? launch_coop_f<true>(A, ws, s) : launch_coop_f<false>(A, ws, s);
}

}  // namespace

// Runs one CG solve on `s`; synchronises `s` before returning.
int cg_run(nm_csr* A, const double* b, double* x, double tol, int32_t max_iter, int guard,
           nm_cg_result* res, cudaStream_t s) {
    if (A->dtype != NM_F64) return fail(NM_ERR_TYPE, "cg: float64 matrices only");
    if (A->nrows != A->ncols) return fail(NM_ERR_INVALID, "cg: matrix must be square");
    if (!b || !x || !res) return fail(NM_ERR_INVALID, "cg: NULL argument");
    std::lock_guard<std::mutex> lock(A->cg_mutex);
    CgWorkspace* ws = nullptr;
    int st = ensure_workspace(A, &ws);
    if (st != NM_OK) return st;

    CgState* h = ws->h_in;
    std::memset(h, 0, sizeof(CgState));
    h->b = b;
    h->x = x;
    h->tol = tol;
    h->max_iter = max_iter;
    h->guard = guard;
    NM_CUDA_TRY(cudaMemcpyAsync(ws->st, h, sizeof(CgState), cudaMemcpyHostToDevice, s));
    // r = b - A x0, p = r, ||b||, r.r, early exit.
    st = launch_spmv(A, x, ws->Ap, s);
    if (st != NM_OK) return st;
    cg_init_kernel<<<ws->grid_vec, kThreads, 0, s>>>(ws->n, ws->st, ws->Ap, ws->r, ws->p,
                                                     ws->partials);
    NM_CHECK_LAUNCH();

    const int mode = g_cg_persistent.load();
    // mode 1: the cluster solve where it applies (6.0 us per iteration on the
    // 256^2 Laplacian), else the TMA-pipelined persistent solve where it fits
    // (9.8 us there), else the resident one (10.8 us); 2, 3, 4: the second,
    // the third, the first only; 0: graph chunks
    const bool cluster = ws->cluster && (mode == 4 || mode == 1);
    const bool resident = !cluster && ws->resident && (mode == 3 || (mode == 1 && !ws->coop));
    const bool coop = cluster || resident || (ws->coop && (mode == 1 || mode == 2));
    if (coop) {
        // the whole iteration loop in one persistent launch
        st = cluster ? launch_cluster(A, ws, s)
                     : (resident ? launch_resident(A, ws, s) : launch_coop(A, ws, s));
        if (st != NM_OK) return st;
        ws->last_path = cluster ? 4 : (resident ? 3 : (ws->coop_formed ? 2 : 1));
        NM_CUDA_TRY(cudaMemcpyAsync(ws->h_out, ws->st, sizeof(CgState), cudaMemcpyDeviceToHost, s));
        NM_CUDA_TRY(cudaStreamSynchronize(s));
    }
    // Otherwise iterate in graph chunks of growing length; poll `done` in between.
    int chunk = 8;
    if (!coop) ws->last_path = 0;
    for (; !coop;) {
        NM_CUDA_TRY(cudaMemcpyAsync(ws->h_out, ws->st, sizeof(CgState), cudaMemcpyDeviceToHost, s));
        NM_CUDA_TRY(cudaStreamSynchronize(s));
        if (ws->h_out->done) break;
        cudaGraphExec_t ex = nullptr;
        st = chunk_graph(A, ws, chunk, &ex);
        if (st != NM_OK) return st;
        NM_CUDA_TRY(cudaGraphLaunch(ex, s));
        if (chunk < 64) chunk *= 2;
    }
    const CgState& o = *ws->h_out;
    st = nm_check_device_errors();
    if (st != NM_OK) return st;
    if (o.status == kCgDeviceError)
        return fail(NM_ERR_RUNTIME, "cg: a device wait gave up; the solve was abandoned");
    if (o.status == kCgBreakdown)
        return fail(NM_ERR_RUNTIME, "CG: p'Ap is near zero - A may not be SPD");
    res->iters = o.iters;
    res->final_res = o.final_res;
    res->converged = o.converged;
    return NM_OK;
}

}  // namespace nm

extern "C" int nm_cg_last_path(const nm_csr* A, int32_t* path) {
    nm::clear_error();
    if (!A || !path) return nm::fail(NM_ERR_INVALID, "nm_cg_last_path: NULL argument");
    *path = A->cg ? A->cg->last_path : -1;
    return NM_OK;
}

extern "C" int nm_cg_set_persistent(int32_t enable) {
    nm::clear_error();
    if (enable < 0 || enable > 4)
        return nm::fail(NM_ERR_INVALID, "nm_cg_set_persistent: 0 to 4");
    nm::g_cg_persistent.store(enable);
    return NM_OK;
}

extern "C" int nm_cg_local(nm_csr* A, const double* b, double* x, double tol, int32_t max_iter,
                           nm_cg_result* result, void* stream) {
    nm::clear_error();
    if (!A) return nm::fail(NM_ERR_INVALID, "nm_cg_local: NULL matrix");
    return nm::cg_run(A, b, x, tol, max_iter, 0, result, static_cast<cudaStream_t>(stream));
}

// ---------------------------------------------------------------------------
// CG that allocates nothing: nm_cg_local_static.
//
// Who needs it: callers that cannot call cudaMalloc when they solve -- a
// process whose device memory is already claimed by another allocator (a
// framework's caching pool or a serving engine that reserves nearly all of
// HBM at start-up, where a new cudaMalloc fails or fragments the pool), and
// latency-critical loops, where cudaMalloc / cudaFree synchronise the whole
// device and stall every other stream.  nm_cg_local caches a workspace per
// matrix, allocated on first use; this variant instead takes r, p, Ap, the
// CTA partial sums, the device-resident CG state and the error word from one
// file-scope device array that is part of the loaded library (about 8.4 MB,
// held until the process exits by every GPU on which this file's module has
// been loaded).  Under CUDA's default lazy module loading the driver loads the
// module, and so reserves the array, on the first use of this file's kernels
// or symbols on a device -- normally the first call of this entry point or of
// nm_cg_local there; with CUDA_MODULE_LOADING=EAGER it happens when the
// library is loaded.  A caller whose own pool will claim nearly all of HBM
// makes one call (a solve of any small matrix) on each device before that
// pool takes its memory.
//
// It runs the same kernels in the same order with the same grids as
// nm_cg_local (launched directly instead of through cached CUDA graphs, and
// polling the state through plain copies instead of pinned buffers), so the
// two give the same iterates.  Limits: n <= kStaticCgMaxRows rows (larger
// matrices are rejected with NM_ERR_INVALID); every call reuses the one
// array, so it keeps the previous call's contents (the state, the arrival
// counter and the error word are reset at the start of each call) and calls
// that overlap on the GPU would race -- this entry point serialises its host
// callers and synchronises `stream` before returning.
// ---------------------------------------------------------------------------
namespace nm {
namespace {

constexpr int64_t kStaticCgMaxRows = 262144;
// one p.Ap sum per row block (at most one block per row) or two sums per
// vector CTA, whichever is more
constexpr int kStaticCgMaxPartials = static_cast<int>(kStaticCgMaxRows) + 4096;
constexpr size_t kStaticErrOff = 512;      // error word, after the CgState
constexpr size_t kStaticPartOff = 1024;    // CTA partial sums
constexpr size_t kStaticVecOff = kStaticPartOff + sizeof(double) * kStaticCgMaxPartials;
constexpr size_t kStaticVecBytes = sizeof(double) * size_t(kStaticCgMaxRows);
constexpr size_t kStaticBytes = kStaticVecOff + 3 * kStaticVecBytes;
static_assert(sizeof(CgState) <= kStaticErrOff, "CgState must fit its slot");
static_assert(kStaticVecOff % 256 == 0 && kStaticVecBytes % 256 == 0, "vector alignment");

// The scratch itself.  In host code this name is only a stand-in for the
// symbol: its device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_cg_static_scratch[kStaticBytes];

constexpr int kStaticMaxDevices = 64;
struct StaticCgDevice {
    bool ready;
    unsigned char* base;  // device address of g_cg_static_scratch on this device
    int sms;
    int occ[3][3];        // CTAs per SM of cg_spmv_pap_kernel<tile, stages>; 0 = not set up
};
std::mutex g_static_mu;
StaticCgDevice g_static_dev[kStaticMaxDevices];

template <int TILE, int STAGES>
int static_attr(int* occ) {
    const void* fn = reinterpret_cast<const void*>(cg_spmv_pap_kernel<TILE, STAGES>);
    const size_t smem = spmv_smem_bytes<double, double, double, TILE, STAGES>();
    if (smem > 48 * 1024)
        NM_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem)));
    NM_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     cudaSharedmemCarveoutMaxShared));
    NM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, fn, kCtaThreads, smem));
    if (*occ < 1) return fail(NM_ERR_CUDA, "nm_cg_local_static: kernel does not fit on an SM");
    return NM_OK;
}

// Once per device, with that device current: the scratch array's device
// address and the kernel attributes.  Caller holds g_static_mu.
int static_setup(int dev, StaticCgDevice** out) {
    if (dev < 0 || dev >= kStaticMaxDevices)
        return fail(NM_ERR_INVALID, "nm_cg_local_static: device %d not supported", dev);
    StaticCgDevice& d = g_static_dev[dev];
    if (!d.ready) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_cg_static_scratch);
        if (e != cudaSuccess || !p)
            return fail(NM_ERR_CUDA, "nm_cg_local_static: cudaGetSymbolAddress failed: %s",
                        cudaGetErrorString(e));
        NM_CUDA_TRY(cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev));
        d.base = static_cast<unsigned char*>(p);
        d.ready = true;
    }
    *out = &d;
    return NM_OK;
}

struct StaticCgLaunch {
    CsrView<double> M;
    CgState* st;
    double *r, *p, *Ap, *partials;
    unsigned int* err;
    int64_t n;
    int grid_spmv, grid_vec;
};

template <int TILE, int STAGES>
int static_spmv_pap(const StaticCgLaunch& L, const double* v, cudaStream_t s) {
    CsrView<double> M = L.M;
    M.stage_x = (reinterpret_cast<uintptr_t>(v) % 16) == 0;
    cg_spmv_pap_kernel<TILE, STAGES>
        <<<L.grid_spmv, kCtaThreads, spmv_smem_bytes<double, double, double, TILE, STAGES>(), s>>>(
            M, L.st, v, L.Ap, L.partials, L.err);
    NM_CHECK_LAUNCH();
    return NM_OK;
}

template <int TILE>
int static_spmv_stages(int stages, const StaticCgLaunch& L, const double* v, cudaStream_t s) {
    if (stages == 4) return static_spmv_pap<TILE, 4>(L, v, s);
    return stages == 3 ? static_spmv_pap<TILE, 3>(L, v, s) : static_spmv_pap<TILE, 2>(L, v, s);
}

int static_spmv_dispatch(int tile, int stages, const StaticCgLaunch& L, const double* v,
                         cudaStream_t s) {
    switch (tile) {
        case 1024: return static_spmv_stages<1024>(stages, L, v, s);
        case 4096: return static_spmv_stages<4096>(stages, L, v, s);
        default: return static_spmv_stages<2048>(stages, L, v, s);
    }
}

template <int TILE>
int static_attr_stages(int stages, int* occ) {
    if (stages == 4) return static_attr<TILE, 4>(occ);
    return stages == 3 ? static_attr<TILE, 3>(occ) : static_attr<TILE, 2>(occ);
}

// Waits for `s` when it goes out of scope, whatever the return path, once
// armed.  Declared after the lock, so it runs before the lock is released: a
// call that fails after enqueueing work leaves nothing on the GPU that could
// overlap the next call's use of the shared array.  The wait's own status is
// ignored (the call already reports the first error).
struct StaticStreamDrain {
    cudaStream_t s;
    bool armed = false;
    ~StaticStreamDrain() {
        if (armed) (void)cudaStreamSynchronize(s);
    }
};

}  // namespace
}  // namespace nm

extern "C" int nm_cg_local_static(const nm_csr* A, const double* b, double* x, double tol,
                                  int32_t max_iter, nm_cg_result* result, void* stream) {
    using namespace nm;
    clear_error();
    if (!A || !b || !x || !result) return fail(NM_ERR_INVALID, "nm_cg_local_static: NULL argument");
    if (A->dtype != NM_F64) return fail(NM_ERR_TYPE, "nm_cg_local_static: float64 matrices only");
    if (A->nrows != A->ncols) return fail(NM_ERR_INVALID, "nm_cg_local_static: matrix must be square");
    if (int64_t(A->nrows) > kStaticCgMaxRows)
        return fail(NM_ERR_INVALID,
                    "nm_cg_local_static: %d rows exceed the fixed scratch of %lld rows; use "
                    "nm_cg_local",
                    A->nrows, static_cast<long long>(kStaticCgMaxRows));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    std::lock_guard<std::mutex> lock(g_static_mu);
    int dev = 0;
    NM_CUDA_TRY(cudaGetDevice(&dev));
    StaticCgDevice* d = nullptr;
    int st = static_setup(dev, &d);
    if (st != NM_OK) return st;

    const int ti = A->tune.tile == 1024 ? 0 : (A->tune.tile == 4096 ? 2 : 1);
    const int si = A->tune.stages - 2;
    if (d->occ[ti][si] == 0) {  // kernel attributes of this variant, once per device
        switch (ti) {
            case 0: st = static_attr_stages<1024>(A->tune.stages, &d->occ[ti][si]); break;
            case 2: st = static_attr_stages<4096>(A->tune.stages, &d->occ[ti][si]); break;
            default: st = static_attr_stages<2048>(A->tune.stages, &d->occ[ti][si]); break;
        }
        if (st != NM_OK) {
            d->occ[ti][si] = 0;
            return st;
        }
    }
    const int mult = A->tune.grid_mult > 0 ? A->tune.grid_mult : d->occ[ti][si];
    StaticCgLaunch L;
    L.M = A->view<double>();
    L.n = A->nrows;
    L.grid_spmv = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(int64_t(d->sms) * mult, A->nblk)));
    L.grid_vec = static_cast<int>(std::max<int64_t>(
        1, std::min<int64_t>((L.n + kThreads - 1) / kThreads, int64_t(d->sms) * 8)));
    if (std::max<int64_t>(A->nblk, 2 * int64_t(L.grid_vec)) > kStaticCgMaxPartials)
        return fail(NM_ERR_INVALID, "nm_cg_local_static: %d row blocks exceed the scratch",
                    A->nblk);
    L.st = reinterpret_cast<CgState*>(d->base);
    L.err = reinterpret_cast<unsigned int*>(d->base + kStaticErrOff);
    L.partials = reinterpret_cast<double*>(d->base + kStaticPartOff);
    L.r = reinterpret_cast<double*>(d->base + kStaticVecOff);
    L.p = reinterpret_cast<double*>(d->base + kStaticVecOff + kStaticVecBytes);
    L.Ap = reinterpret_cast<double*>(d->base + kStaticVecOff + 2 * kStaticVecBytes);

    // Reset the header (state, arrival counter, error word) left by the last call.
    unsigned char hdr[kStaticPartOff];
    std::memset(hdr, 0, sizeof hdr);
    CgState h;
    std::memset(&h, 0, sizeof h);
    h.b = b;
    h.x = x;
    h.tol = tol;
    h.max_iter = max_iter;
    h.guard = 0;
    std::memcpy(hdr, &h, sizeof h);
    StaticStreamDrain drain{s};
    drain.armed = true;  // from here on every return waits for `s` first
    NM_CUDA_TRY(cudaMemcpyAsync(d->base, hdr, sizeof hdr, cudaMemcpyHostToDevice, s));

    // Ap = A x0 through the fused kernel (its x0.Ax0 by-product is unused;
    // the state's alpha it leaves is overwritten before any use), then
    // r = b - Ap, p = r, ||b||, r.r and the early exit.
    st = static_spmv_dispatch(A->tune.tile, A->tune.stages, L, x, s);
    if (st != NM_OK) return st;
    cg_init_kernel<<<L.grid_vec, kThreads, 0, s>>>(L.n, L.st, L.Ap, L.r, L.p, L.partials);
    NM_CHECK_LAUNCH();

    int chunk = 8;
    CgState o;
    unsigned int errw = 0;
    for (;;) {
        NM_CUDA_TRY(cudaMemcpyAsync(hdr, d->base, sizeof hdr, cudaMemcpyDeviceToHost, s));
        NM_CUDA_TRY(cudaStreamSynchronize(s));
        std::memcpy(&o, hdr, sizeof o);
        std::memcpy(&errw, hdr + kStaticErrOff, sizeof errw);
        if (o.done || errw) break;
        for (int i = 0; i < chunk; ++i) {
            st = static_spmv_dispatch(A->tune.tile, A->tune.stages, L, L.p, s);
            if (st != NM_OK) return st;
            cg_update_xr_kernel<<<L.grid_vec, kThreads, 0, s>>>(L.n, L.st, L.p, L.Ap, L.r,
                                                               L.partials);
            cg_update_p_kernel<<<L.grid_vec, kThreads, 0, s>>>(L.n, L.st, L.p, L.r);
        }
        NM_CHECK_LAUNCH();
        if (chunk < 64) chunk *= 2;
    }
    if (errw || o.status == kCgDeviceError)
        return fail(NM_ERR_RUNTIME,
                    "nm_cg_local_static: a device wait gave up; the solve was abandoned");
    result->iters = o.iters;
    result->final_res = o.final_res;
    result->converged = o.converged;
    return NM_OK;
}
