// cg_resident.cu -- plain CG with the matrix resident on chip for small systems.
//
// Same algorithm, stopping rule and iterates as cg_solve_local
// (src/cg_solver.hpp:133-196) and as this library's other CG paths, bit for
// bit.  For systems of up to 262,144 rows whose row-block partition is whole
// 256-row tiles (every row at most 8 nonzeros, e.g. the 2-D / 3-D stencil
// Laplacians) one cooperative launch runs the whole solve:
//
//  * CTA c owns B consecutive tiles; thread t of the CTA owns row t of each.
//    The CTA's rows of A are read once per solve into shared memory (an ELL
//    layout: entry e of row t at [e][t]), and x, r, p, Ap of its rows live in
//    registers for the whole solve.
//  * Per iteration the CTA forms the window of this iteration's direction it
//    multiplies by -- every column its rows touch -- as p_k = fma(beta, p_{k-1},
//    r_k) from the global copies of p_{k-1} and r_k (the operation the p update
//    of the other paths performs, so every CTA forms the same bits), multiplies
//    from shared memory (thread rows, serial CSR-order sums), and publishes the
//    rows' new p (one of two alternating buffers) and, in the second half, r.
//  * The two dot products per iteration are the grid's only synchronisation:
//    each CTA publishes one sum per tile into a slot array with a release
//    store, and every CTA waits for all slots (one warp polls them with relaxed
//    loads, then an acquire fence) and adds them in
//    the fixed order of reduce256.  A slot holds a signalling NaN until its sum
//    arrives -- no arithmetic result has those bits -- so the data carries the
//    barrier: no arrival counter and no second round trip.  Three slot buffers
//    rotate; a CTA clears its own slot of the buffer after next when it
//    publishes, which is safe because every CTA has read that buffer before
//    it published into the one in between.
//
// The per-tile sums and their order are those of the other paths (p.Ap per
// row block with the SpMV pipeline's warp-sum order, r.r per 256-row tile), so
// nm_cg_local gives the same iterates whichever path runs.  Every wait is
// bounded (kWaitLimitNs); a CTA that gives up sets the error word and the
// state to kCgDeviceError and leaves, and the others give up in turn.
#include <algorithm>
#include <vector>

#include "cg.cuh"

namespace nm {
namespace {

// A slot that holds no sum yet: a signalling NaN (quiet bit clear).  Every
// published sum is the result of a floating-point addition, which never
// returns a signalling NaN.
constexpr uint64_t kSlotEmpty = 0x7FF0DEADBEEF0001ull;
constexpr int kResMaxWidth = 8;  // nonzeros of the longest row
constexpr int kResMaxSlots = 1024;  // row blocks: 32 per polling lane

struct ResArgs {
    const int32_t* row_ptr;
    const int32_t* col_idx;
    const double* values;
    const int4* cta;  // per CTA: first row, end row, window start, window end
    CgState* st;
    double* P0;  // p_0 (from the initial kernel), then p_2, p_4, ...
    double* P1;  // p_1, p_3, ...
    double* R;   // r_k
    double* slots;  // 3 buffers of nblk sums
    unsigned int* err;
    int32_t nblk;
    int32_t width;  // ELL width: nonzeros of the longest row
};

__device__ __forceinline__ void st_release(double* p, double v) {
    asm volatile("st.release.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(__double_as_longlong(v))
                 : "memory");
}
__device__ __forceinline__ void st_relaxed_bits(double* p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__global__ void fill_slots_kernel(double* slots, int64_t count) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count;
         i += int64_t(gridDim.x) * blockDim.x)
        reinterpret_cast<unsigned long long*>(slots)[i] = kSlotEmpty;
}

// One sum per owned tile (per thread: d[q] for tile q): a shuffle tree per
// warp, the eight warp sums in warp order, published into slot blk0 + q of
// `cur` with a release store after the CTA's writes; the thread also clears
// its slot of `nxt`.
template <int B>
__device__ __forceinline__ void publish(const double (&d)[B], double (*scr)[kWarps], int nown,
                                        int blk0, double* cur, double* nxt) {
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
#pragma unroll
    for (int q = 0; q < B; ++q) {
        const double v = warp_sum(d[q]);
        if (lane == 0) scr[q][warp] = v;
    }
    __syncthreads();  // also orders every thread's global writes before the release
    if (t < nown) {
        double sum = 0.0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) sum += scr[t][w];
        st_relaxed_bits(nxt + blk0 + t, kSlotEmpty);
        st_release(cur + blk0 + t, sum);
    }
}

__device__ __forceinline__ uint64_t ld_relaxed_bits(const double* p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Waits for every slot of `cur` and returns their total in reduce256's order
// (every thread gets it).  One warp polls -- lane l the slots l, l + 32, ...,
// with relaxed loads, the outstanding ones re-read together, each sum parked
// in shared memory as it arrives -- and, once all have, a fence gives it
// acquire order; the CTA then adds the parked sums in the fixed order.
// Returns false in every thread when the
// wait gave up.
__device__ __forceinline__ bool gather_total(const double* cur, int nblk, double* red,
                                             double* bc, unsigned int* err, double* out,
                                             bool* okf, double* sv) {
    const int t = threadIdx.x;
    if (t < 32) {
        bool ok = true;
        uint32_t pending = 0;
        for (int j = 0; j < 32; ++j)
            if (t + 32 * j < nblk) pending |= 1u << j;
        const uint64_t t0 = global_timer_ns();
        for (uint32_t it = 0; pending; ++it) {
            uint64_t v[32];
#pragma unroll
            for (int j = 0; j < 32; ++j)
                if (pending & (1u << j)) v[j] = ld_relaxed_bits(cur + t + 32 * j);
#pragma unroll
            for (int j = 0; j < 32; ++j)
                if ((pending & (1u << j)) && v[j] != kSlotEmpty) {
                    pending &= ~(1u << j);
                    sv[t + 32 * j] = __longlong_as_double(static_cast<long long>(v[j]));
                }
            if (pending && (it & 63u) == 63u &&
                (global_timer_ns() - t0 > kWaitLimitNs || it > (1u << 28))) {
                atomicOr(err, kErrWaitTimeout);
                ok = false;
                break;
            }
        }
        __threadfence();  // acquire: the publishers' writes before their release stores
        const bool all = __all_sync(0xffffffffu, ok);
        if (t == 0) *okf = all;
    }
    __syncthreads();
    const bool all_ok = *okf;
    double s = 0.0;
    if (all_ok && t < kThreads)
        for (int i = t; i < nblk; i += kThreads) s += sv[i];
    const double tot = block_sum8(s, red);
    if (t == 0) *bc = tot;
    __syncthreads();
    *out = *bc;
    return all_ok;
}

template <int B>
__global__ void __launch_bounds__(kThreads) cg_resident_kernel(ResArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int W = a.width;
    double* ellv = reinterpret_cast<double*>(smem_raw);                      // [B*W][256]
    int32_t* ellc = reinterpret_cast<int32_t*>(ellv + B * W * kThreads);     // [B*W][256]
    double* win = reinterpret_cast<double*>(ellc + B * W * kThreads);        // [window]
    __shared__ double scr[B][kWarps];
    __shared__ double red[kWarps + 1];
    __shared__ double bc;
    __shared__ bool okf;
    __shared__ double sv[kResMaxSlots];  // the sums of the phase, as the polling warp saw them
    const int t = threadIdx.x;
    CgState* st = a.st;
    if (__ldcg(&st->done)) return;  // the initial kernel decided already
    const int4 cta = a.cta[blockIdx.x];
    const int32_t row0 = cta.x, row1 = cta.y, lo = cta.z, wlen = cta.w - cta.z;
    const int blk0 = row0 / kThreads;
    const int nown = (row1 - row0 + kThreads - 1) / kThreads;
    double* __restrict__ xg = st->x;
    const double bnorm = __ldcg(&st->bnorm), tol = __ldcg(&st->tol);
    const int32_t max_iter = __ldcg(&st->max_iter), guard = __ldcg(&st->guard);
    double rr = __ldcg(&st->rr);
    int32_t iter = __ldcg(&st->iter);

    double x[B], r[B], p[B], ap[B];
    int len[B];
#pragma unroll
    for (int q = 0; q < B; ++q) {
        const int32_t row = row0 + q * kThreads + t;
        len[q] = 0;
        x[q] = r[q] = p[q] = ap[q] = 0.0;
        if (row < row1) {
            const int32_t z0 = __ldg(a.row_ptr + row);
            len[q] = __ldg(a.row_ptr + row + 1) - z0;
            for (int e = 0; e < len[q]; ++e) {
                ellv[(q * W + e) * kThreads + t] = __ldg(a.values + z0 + e);
                ellc[(q * W + e) * kThreads + t] = __ldg(a.col_idx + z0 + e) - lo;
            }
            x[q] = __ldcg(xg + row);
            r[q] = __ldcg(a.R + row);
            p[q] = __ldcg(a.P0 + row);
        }
    }

    double beta = 0.0;
    int phase = 0;  // reduction phases so far (two per iteration)
    bool failed = false, write_x = true;
    int status = kCgOk;
    for (int k = 0;; ++k) {
        // ---- A: window of p_k, Ap = A p_k, p_k . Ap ----
        const double* Pold = (k & 1) ? a.P0 : a.P1;  // p_{k-1}
        double* Pnew = (k & 1) ? a.P1 : a.P0;        // p_k (p_0 is in P0 already)
        for (int w = t; w < wlen; w += kThreads) {
            const int32_t j = lo + w;
            win[w] = k == 0 ? __ldcg(a.P0 + j) : fma(beta, __ldcg(Pold + j), __ldcg(a.R + j));
        }
        if (k > 0) {
#pragma unroll
            for (int q = 0; q < B; ++q) {
                const int32_t row = row0 + q * kThreads + t;
                if (row < row1) {
                    p[q] = fma(beta, p[q], r[q]);  // p = 1*r + beta*p
                    Pnew[row] = p[q];
                }
            }
        }
        __syncthreads();
        double d[B];
#pragma unroll
        for (int q = 0; q < B; ++q) {
            double acc = 0.0;
            const double* vq = ellv + q * W * kThreads + t;
            const int32_t* cq = ellc + q * W * kThreads + t;
            for (int e = 0; e < len[q]; ++e)
                acc = add_rn(acc, mul_rn(vq[e * kThreads], win[cq[e * kThreads]]));
            ap[q] = acc;
            d[q] = fma(p[q], acc, 0.0);
        }
        double* cur = a.slots + (phase % 3) * a.nblk;
        double* nxt = a.slots + ((phase + 1) % 3) * a.nblk;
        publish<B>(d, scr, nown, blk0, cur, nxt);
        double pAp;
        if (!gather_total(cur, a.nblk, red, &bc, a.err, &pAp, &okf, sv)) {
            failed = true;
            break;
        }
        ++phase;
        if (guard && fabs(pAp) < 1e-300) {
            status = kCgBreakdown;
            if (blockIdx.x == 0 && t == 0) {
                st->pAp = pAp;
                st->converged = 0;
                st->iters = iter;
                st->final_res = sqrt(rr) / bnorm;
            }
            break;
        }
        const double alpha = rr / pAp;

        // ---- B: x += alpha p, r -= alpha Ap, r . r ----
        double s[B];
#pragma unroll
        for (int q = 0; q < B; ++q) {
            const int32_t row = row0 + q * kThreads + t;
            s[q] = 0.0;
            if (row < row1) {
                x[q] = fma(alpha, p[q], x[q]);       // x = alpha*p + x
                r[q] = fma(-alpha, ap[q], r[q]);     // r = -alpha*Ap + r
                a.R[row] = r[q];
                s[q] = fma(r[q], r[q], 0.0);
            }
        }
        cur = a.slots + (phase % 3) * a.nblk;
        nxt = a.slots + ((phase + 1) % 3) * a.nblk;
        publish<B>(s, scr, nown, blk0, cur, nxt);
        double rr_new;
        if (!gather_total(cur, a.nblk, red, &bc, a.err, &rr_new, &okf, sv)) {
            failed = true;
            break;
        }
        ++phase;
        ++iter;
        const double rel = sqrt(rr_new) / bnorm;
        if (rel < tol) {
            if (blockIdx.x == 0 && t == 0) {
                st->iter = iter; st->converged = 1; st->iters = iter; st->final_res = rel;
                st->rr = rr_new;
            }
            break;
        }
        beta = rr_new / rr;
        rr = rr_new;
        if (iter >= max_iter) {
            if (blockIdx.x == 0 && t == 0) {
                st->iter = iter; st->converged = 0; st->iters = max_iter; st->final_res = rel;
                st->beta = beta; st->rr = rr;
            }
            break;
        }
    }
    if (failed) {
        write_x = false;
        if (t == 0) {
            atomicExch(&st->status, kCgDeviceError);
            atomicExch(&st->done, 1);
        }
        return;
    }
    if (write_x) {
#pragma unroll
        for (int q = 0; q < B; ++q) {
            const int32_t row = row0 + q * kThreads + t;
            if (row < row1) xg[row] = x[q];
        }
    }
    if (blockIdx.x == 0 && t == 0) {
        if (status != kCgOk) st->status = status;
        st->done = 1;
    }
}

template <int B>
const void* resident_fn() {
    return reinterpret_cast<const void*>(cg_resident_kernel<B>);
}

const void* resident_kernel_for(int B) {
    switch (B) {
        case 1: return resident_fn<1>();
        case 2: return resident_fn<2>();
        case 3: return resident_fn<3>();
        case 4: return resident_fn<4>();
        case 5: return resident_fn<5>();
        case 6: return resident_fn<6>();
        case 7: return resident_fn<7>();
        default: return resident_fn<8>();
    }
}

}  // namespace

int plan_resident(const nm_csr* A, CgWorkspace* ws) {
    ws->resident = false;
    const int64_t n = A->nrows;
    if (n > kResidentMaxRows || A->tune.max_rows != kThreads) return NM_OK;
    if (int64_t(A->h_row_ptr.size()) != n + 1 || A->h_col_idx.size() < size_t(A->nnz)) return NM_OK;
    // every row short enough that each row block is one whole 256-row tile
    const int wcap = std::min({A->tune.short_max, A->tune.tile / kThreads, kResMaxWidth});
    const int32_t* rp = A->h_row_ptr.data();
    const int32_t* ci = A->h_col_idx.data();
    int W = 1;
    for (int64_t i = 0; i < n; ++i) {
        const int len = rp[i + 1] - rp[i];
        if (len > wcap) return NM_OK;
        W = std::max(W, len);
    }
    const int64_t nblk = (n + kThreads - 1) / kThreads;
    if (A->nblk != nblk || nblk > kResMaxSlots) return NM_OK;
    const int sms = sm_count();
    const int B = static_cast<int>((nblk + sms - 1) / sms);
    if (B < 1 || B > kResidentMaxTiles) return NM_OK;
    const int G = static_cast<int>((nblk + B - 1) / B);
    std::vector<int4> cta(G);
    int64_t win_max = 0;
    for (int c = 0; c < G; ++c) {
        const int32_t r0 = c * B * kThreads;
        const int32_t r1 = static_cast<int32_t>(std::min<int64_t>(n, int64_t(c + 1) * B * kThreads));
        int32_t lo = r0, hi = r1;
        for (int32_t i = r0; i < r1; ++i)
            for (int32_t z = rp[i]; z < rp[i + 1]; ++z) {
                lo = std::min(lo, ci[z]);
                hi = std::max(hi, ci[z] + 1);
            }
        cta[c] = make_int4(r0, r1, lo, hi);
        win_max = std::max<int64_t>(win_max, hi - lo);
    }
    const size_t smem = size_t(B) * W * kThreads * (sizeof(double) + sizeof(int32_t)) +
                        size_t(win_max) * sizeof(double);
    if (smem > kResidentMaxSmem) return NM_OK;
    const void* fn = resident_kernel_for(B);
    NM_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(smem)));
    int occ = 0;
    NM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, kThreads, smem));
    if (int64_t(occ) * sms < G) return NM_OK;
    const size_t cta_bytes = (size_t(G) * sizeof(int4) + 255) & ~size_t(255);
    NM_CUDA_TRY(cudaMalloc(&ws->res_mem, cta_bytes + 3 * size_t(nblk) * sizeof(double)));
    ws->res_cta = static_cast<int4*>(ws->res_mem);
    ws->res_slots = reinterpret_cast<double*>(static_cast<unsigned char*>(ws->res_mem) + cta_bytes);
    NM_CUDA_TRY(cudaMemcpy(ws->res_cta, cta.data(), G * sizeof(int4), cudaMemcpyHostToDevice));
    ws->res_tiles = B;
    ws->res_grid = G;
    ws->res_width = W;
    ws->res_smem = smem;
    ws->resident = true;
    return NM_OK;
}

int launch_resident(const nm_csr* A, CgWorkspace* ws, cudaStream_t s) {
    const int64_t nslots = 3 * int64_t(A->nblk);
    fill_slots_kernel<<<static_cast<int>(std::min<int64_t>((nslots + 255) / 256, 64)), 256, 0, s>>>(
        ws->res_slots, nslots);
    NM_CHECK_LAUNCH();
    ResArgs a;
    a.row_ptr = A->d_row_ptr;
    a.col_idx = A->d_col_idx;
    a.values = static_cast<const double*>(A->d_values);
    a.cta = ws->res_cta;
    a.st = ws->st;
    a.P0 = ws->p;
    a.P1 = ws->p2;
    a.R = ws->r;
    a.slots = ws->res_slots;
    a.err = ws->err;
    a.nblk = A->nblk;
    a.width = ws->res_width;
    void* args[] = {&a};
    NM_CUDA_TRY(cudaLaunchCooperativeKernel(resident_kernel_for(ws->res_tiles), dim3(ws->res_grid),
                                            dim3(kThreads), args, ws->res_smem, s));
    return NM_OK;
}

}  // namespace nm
