// cg_cluster.cu -- plain CG of a small system in one thread-block cluster.
//
// Same algorithm, stopping rule and iterates as cg_solve_local
// (src/cg_solver.hpp:133-196) and as this library's other CG paths, bit for
// bit.  A system of up to 65,536 rows of at most kClusterMaxWidth nonzeros
// each, whose row-block partition is whole 256-row tiles, is solved by one
// cluster of kClusterCtas CTAs on as many SMs, in one launch:
//
//  * CTA c of the cluster owns rows [c * RC, (c + 1) * RC), RC = 256 R; its
//    thread t owns rows t, t + 256, ..., so each 256-row tile is the CTA's 8
//    warps, one row per lane -- the tile and warp structure of the other
//    paths' sums.
//    The CTA's matrix values sit in shared memory for the whole solve, its
//    column indices and its rows of r in registers, its rows of p and Ap in
//    shared memory, x in global memory.
//  * The direction p_k of the CTA's rows is kept in its shared memory; an
//    SpMV reads a column's p_k from the owning CTA's shared memory over the
//    cluster's distributed shared memory, so no vector goes through L2.
//  * Each of the two dot products is summed per 256-row tile in the CTA and
//    published in the CTA's shared memory; after a cluster barrier every CTA
//    reads all tile sums (one per thread, from the owning CTAs) and adds them
//    in reduce256's order.  Three hardware cluster barriers per iteration
//    (after the new direction, after each set of tile sums) replace the
//    global-memory synchronisation of the grid-wide paths.
#include <cooperative_groups.h>

#include <algorithm>
#include <vector>

#include "cg.cuh"

namespace cg = cooperative_groups;

namespace nm {
namespace {

constexpr int kClusterCtas = 16;
constexpr int kClusterThreads = 256;
constexpr int kClusterMaxR = 16;       // rows per thread
constexpr int kClusterMaxWidth = 8;    // nonzeros of the longest row

// A double from CTA `rank` of the cluster at its shared-memory address `sa`
// (the same offset this CTA uses: every CTA lays out its memory alike).
__device__ __forceinline__ double ld_cluster_f64(uint32_t sa, uint32_t rank) {
    uint32_t ra;
    double v;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(ra) : "r"(sa), "r"(rank));
    asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(ra) : "memory");
    return v;
}

__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\t"
                 "barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

struct ClusterArgs {
    const int32_t* row_ptr;
    const int32_t* col_idx;
    const double* values;
    CgState* st;
    const double* P0;  // p_0 = r_0 (the initial kernel)
    const double* R0;  // r_0
    int32_t n;
    int32_t width;
    int32_t nblk;      // 256-row tiles
};

// Tile sums of one value per owned row: row t + 256 q is lane t % 32 of warp
// t / 32 of the CTA's tile q.  tile_part parks the warp's shuffle-tree sum of
// tile q; tile_finish adds each tile's 8 warp sums in warp order into ts[q].
__device__ __forceinline__ void tile_part(int q, double d, double (*scr)[kWarps]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const double v = warp_sum(d);
    if (lane == 0) scr[q][warp] = v;
}

template <int R>
__device__ __forceinline__ void tile_finish(double (*scr)[kWarps], double* ts) {
    const int t = threadIdx.x;
    __syncthreads();
    if (t < R) {
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) s += scr[t][w];
        ts[t] = s;
    }
}

// After a cluster barrier: the total of every CTA's tile sums, reduce256's
// order (thread t takes tile t; the 256 values by block_sum8).
template <int R>
__device__ __forceinline__ double cluster_total(double* ts, int nblk, double* red, double* bc) {
    const int t = threadIdx.x;
    double s = 0.0;
    if (t < nblk) {
        const uint32_t owner = uint32_t(t) / R;
        s = ld_cluster_f64(smem_u32(ts) + (uint32_t(t) - owner * R) * 8u, owner);
    }
    const double tot = block_sum8(s, red);
    if (t == 0) *bc = tot;
    __syncthreads();
    const double out = *bc;
    return out;
}

template <int R>
__global__ void __launch_bounds__(kClusterThreads, 1) cg_cluster_kernel(ClusterArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int RC = kClusterThreads * R;        // rows per CTA
    const int W = a.width;
    double* vals = reinterpret_cast<double*>(smem_raw);  // [R][W][256]
    double* ps = vals + R * W * kClusterThreads;          // [RC] this CTA's p_k
    double* aps = ps + RC;                                // [RC] its (A p_k), owner-private
    const uint32_t ps_sa = smem_u32(ps);
    __shared__ double scr[R][kWarps];
    __shared__ double ts_a[R], ts_b[R];  // tile sums of p.Ap and r.r
    __shared__ double red[kWarps + 1];
    __shared__ double bc;
    const int t = threadIdx.x;
    const int rank = static_cast<int>(cg::this_cluster().block_rank());
    CgState* st = a.st;
    if (__ldcg(&st->done)) return;  // the same in every CTA: no barrier is skipped unevenly
    const int32_t row0 = rank * RC;
    double* __restrict__ xg = st->x;
    const double bnorm = __ldcg(&st->bnorm), tol = __ldcg(&st->tol);
    const int32_t max_iter = __ldcg(&st->max_iter), guard = __ldcg(&st->guard);
    double rr = __ldcg(&st->rr);
    int32_t iter = __ldcg(&st->iter);

    // column indices (< 65,536) two to a register, row lengths 4 bits each
    uint32_t colp[R][kClusterMaxWidth / 2];
    uint32_t lens = 0u;
    double r[R];
#pragma unroll
    for (int q = 0; q < R; ++q) {
        const int32_t row = row0 + t + kClusterThreads * q;
        double p0 = 0.0;
        r[q] = 0.0;
#pragma unroll
        for (int e = 0; e < kClusterMaxWidth / 2; ++e) colp[q][e] = 0u;
        if (row < a.n) {
            const int32_t z0 = __ldg(a.row_ptr + row);
            const int len = __ldg(a.row_ptr + row + 1) - z0;
            lens |= uint32_t(len) << (4 * q);
#pragma unroll
            for (int e = 0; e < kClusterMaxWidth; ++e)
                if (e < len) {
                    const uint32_t c = static_cast<uint32_t>(__ldg(a.col_idx + z0 + e));
                    colp[q][e >> 1] |= (e & 1) ? (c << 16) : c;
                    vals[(q * W + e) * kClusterThreads + t] = __ldg(a.values + z0 + e);
                }
            r[q] = __ldcg(a.R0 + row);
            p0 = __ldcg(a.P0 + row);
        }
        ps[t + kClusterThreads * q] = p0;
    }

    double beta = 0.0;
    int status = kCgOk;
    for (int k = 0;; ++k) {
        // ---- the new direction, in this CTA's shared memory ----
#pragma unroll
        for (int q = 0; q < R; ++q)
            if (k > 0) {
                double& pq = ps[t + kClusterThreads * q];
                pq = fma(beta, pq, r[q]);  // p = 1*r + beta*p
            }
        cluster_sync_all();
        // ---- Ap = A p (thread rows, serial CSR-order sums), p.Ap per tile ----
#pragma unroll
        for (int q = 0; q < R; ++q) {
            double acc = 0.0;
            const int len = int((lens >> (4 * q)) & 15u);
#pragma unroll
            for (int e = 0; e < kClusterMaxWidth; ++e)
                if (e < len) {
                    const uint32_t c = (colp[q][e >> 1] >> ((e & 1) * 16)) & 0xffffu;
                    const uint32_t owner = c / RC;
                    acc = add_rn(acc, mul_rn(vals[(q * W + e) * kClusterThreads + t],
                                             ld_cluster_f64(ps_sa + (c - owner * RC) * 8u,
                                                            owner)));
                }
            aps[t + kClusterThreads * q] = acc;
            tile_part(q, fma(ps[t + kClusterThreads * q], acc, 0.0), scr);
        }
        tile_finish<R>(scr, ts_a);
        cluster_sync_all();
        const double pAp = cluster_total<R>(ts_a, a.nblk, red, &bc);
        if (guard && fabs(pAp) < 1e-300) {
            status = kCgBreakdown;
            if (rank == 0 && t == 0) {
                st->pAp = pAp;
                st->converged = 0;
                st->iters = iter;
                st->final_res = sqrt(rr) / bnorm;
            }
            break;
        }
        const double alpha = rr / pAp;
        // ---- x += alpha p, r -= alpha Ap, r.r per tile ----
#pragma unroll
        for (int q = 0; q < R; ++q) {
            const int32_t row = row0 + t + kClusterThreads * q;
            double sq = 0.0;
            if (row < a.n) {
                r[q] = fma(-alpha, aps[t + kClusterThreads * q], r[q]);  // r = -alpha*Ap + r
                sq = fma(r[q], r[q], 0.0);
            }
            tile_part(q, sq, scr);
        }
        tile_finish<R>(scr, ts_b);
#pragma unroll
        for (int q = 0; q < R; ++q) {  // off the critical path: before the barrier wait
            const int32_t row = row0 + t + kClusterThreads * q;
            if (row < a.n) xg[row] = fma(alpha, ps[t + kClusterThreads * q], xg[row]);  // x = alpha*p + x
        }
        cluster_sync_all();
        const double rr_new = cluster_total<R>(ts_b, a.nblk, red, &bc);
        ++iter;
        const double rel = sqrt(rr_new) / bnorm;
        if (rel < tol) {
            if (rank == 0 && t == 0) {
                st->iter = iter; st->converged = 1; st->iters = iter; st->final_res = rel;
                st->rr = rr_new;
            }
            break;
        }
        beta = rr_new / rr;
        rr = rr_new;
        if (iter >= max_iter) {
            if (rank == 0 && t == 0) {
                st->iter = iter; st->converged = 0; st->iters = max_iter; st->final_res = rel;
                st->beta = beta; st->rr = rr;
            }
            break;
        }
    }
    // No CTA may leave while another can still read its shared memory.
    cluster_sync_all();
    if (rank == 0 && t == 0) {
        if (status != kCgOk) st->status = status;
        st->done = 1;
    }
}

template <int R>
const void* cluster_fn() {
    return reinterpret_cast<const void*>(cg_cluster_kernel<R>);
}

const void* cluster_kernel_for(int R) {
    switch (R) {
        case 1: return cluster_fn<1>();
        case 2: return cluster_fn<2>();
        case 3: return cluster_fn<3>();
        case 4: return cluster_fn<4>();
        case 5: return cluster_fn<5>();
        case 6: return cluster_fn<6>();
        case 7: return cluster_fn<7>();
        case 8: return cluster_fn<8>();
        case 9: return cluster_fn<9>();
        case 10: return cluster_fn<10>();
        case 11: return cluster_fn<11>();
        case 12: return cluster_fn<12>();
        case 13: return cluster_fn<13>();
        case 14: return cluster_fn<14>();
        case 15: return cluster_fn<15>();
        default: return cluster_fn<16>();
    }
}

size_t cluster_smem(int R, int W) {
    return size_t(R) * W * kClusterThreads * sizeof(double) +
           2 * size_t(R) * kClusterThreads * sizeof(double);
}

}  // namespace

int plan_cluster(const nm_csr* A, CgWorkspace* ws) {
    ws->cluster = false;
    const int64_t n = A->nrows;
    if (n > int64_t(kClusterCtas) * kClusterThreads * kClusterMaxR) return NM_OK;
    if (A->tune.max_rows != kThreads) return NM_OK;
    if (int64_t(A->h_row_ptr.size()) != n + 1) return NM_OK;
    const int wcap = std::min({A->tune.short_max, A->tune.tile / kThreads, kClusterMaxWidth});
    const int32_t* rp = A->h_row_ptr.data();
    int W = 1;
    for (int64_t i = 0; i < n; ++i) {
        const int len = rp[i + 1] - rp[i];
        if (len > wcap) return NM_OK;
        W = std::max(W, len);
    }
    if (A->nblk != (n + kThreads - 1) / kThreads) return NM_OK;  // whole 256-row tiles
    const int R = static_cast<int>(
        (n + int64_t(kClusterCtas) * kClusterThreads - 1) / (int64_t(kClusterCtas) * kClusterThreads));
    const size_t smem = cluster_smem(R, W);
    int dev = 0, cl = 0, smem_max = 0;
    NM_CUDA_TRY(cudaGetDevice(&dev));
    NM_CUDA_TRY(cudaDeviceGetAttribute(&cl, cudaDevAttrClusterLaunch, dev));
    NM_CUDA_TRY(cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const void* fn = cluster_kernel_for(R);
    cudaFuncAttributes fa;
    NM_CUDA_TRY(cudaFuncGetAttributes(&fa, fn));
    if (!cl || smem + fa.sharedSizeBytes > size_t(smem_max)) return NM_OK;
    NM_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    NM_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(smem)));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kClusterCtas);
    cfg.blockDim = dim3(kClusterThreads);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = kClusterCtas;
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, fn, &cfg) != cudaSuccess || clusters < 1) {
        cudaGetLastError();  // not schedulable here: the other paths run
        return NM_OK;
    }
    ws->cluster = true;
    ws->cl_rows_per_thread = R;
    ws->cl_width = W;
    ws->cl_smem = smem;
    return NM_OK;
}

int launch_cluster(const nm_csr* A, CgWorkspace* ws, cudaStream_t s) {
    ClusterArgs a;
    a.row_ptr = A->d_row_ptr;
    a.col_idx = A->d_col_idx;
    a.values = static_cast<const double*>(A->d_values);
    a.st = ws->st;
    a.P0 = ws->p;
    a.R0 = ws->r;
    a.n = A->nrows;
    a.width = ws->cl_width;
    a.nblk = A->nblk;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kClusterCtas);
    cfg.blockDim = dim3(kClusterThreads);
    cfg.dynamicSmemBytes = ws->cl_smem;
    cfg.stream = s;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = kClusterCtas;
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    void* args[] = {&a};
    NM_CUDA_TRY(cudaLaunchKernelExC(&cfg, cluster_kernel_for(ws->cl_rows_per_thread), args));
    return NM_OK;
}

}  // namespace nm
