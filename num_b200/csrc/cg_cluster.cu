// cg_cluster.cu -- plain CG of a small system in one thread-block cluster.
//
// Same algorithm, stopping rule and iterates as cg_solve_local
// (src/cg_solver.hpp:133-196) and as this library's other CG paths, bit for
// bit.  A system of up to 65,536 rows of at most kClusterMaxWidth nonzeros
// each, whose row-block partition is whole 256-row tiles, is solved by one
// cluster of kClusterCtas CTAs on as many SMs, in one launch:
//
//  * CTA c of the cluster owns rows [c * RC, (c + 1) * RC), RC = NT R for NT
//    threads; thread t owns rows t, t + NT, ..., so each 256-row tile is 8
//    warps of the CTA, one row per lane -- the tile and warp structure of the
//    other paths' sums.
//  * The CTA's rows of A sit in shared memory for the whole solve, their
//    column indices renumbered into the CTA's extended direction: its own
//    rows of p, then a halo of the entries of p its rows read from other
//    CTAs.  After updating its rows of r each CTA stores every entry of r
//    another CTA's halo holds straight into that CTA's shared memory over
//    distributed shared memory (lists built once on the host), and each CTA
//    forms the new direction for its own rows and its halo alike -- the
//    same fma on the same doubles as the owner -- so the SpMV reads only its
//    own shared memory and no vector goes through L2.
//  * When every value of A is a float exactly (a stencil's integer
//    coefficients, say) the values are held as floats -- each converts back
//    to the same double -- with 16-bit column numbers beside them, x and r
//    stay in registers, and 1024 threads run per CTA.  Otherwise the values
//    are doubles, the column numbers sit in registers, x is updated in global
//    memory, and 512 threads run per CTA.
//  * Each of the two dot products is summed per 256-row tile in the CTA and
//    the tile sums are stored into every CTA of the cluster; after the
//    cluster barrier warp 0 of each CTA adds all of them in reduce256's order
//    from its own shared memory and derives the scalars for the CTA.  Two
//    hardware cluster barriers per iteration (after each set of tile sums)
//    replace the global-memory synchronisation of the grid-wide paths.
#include <cooperative_groups.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include <utility>
#include <vector>

#include "cg.cuh"

namespace cg = cooperative_groups;

namespace nm {
namespace {

constexpr int kClusterCtas = 16;
constexpr int kClusterMaxWidth = 8;  // nonzeros of the longest row
constexpr int kMaxPushes = 8192;     // halo stores a CTA makes per iteration
// The kernel is compiled for width classes of 3, 5, 7 and 8 nonzeros per row;
// the largest rows per thread of each class keeps the CTA's rows of A, p, Ap
// and the halo within an SM's shared memory and (with doubles) the column
// numbers within the registers a thread of a 512-thread CTA has.
constexpr int kWidthClasses[4] = {3, 5, 7, 8};
constexpr int kClassMaxR32[4] = {4, 4, 3, 3};  // float values, 1024 threads
constexpr int kClassMaxR64[4] = {8, 8, 5, 5};  // double values, 512 threads

template <bool F32V>
constexpr int cluster_threads() {
    return F32V ? 1024 : 512;
}

__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\t"
                 "barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// Stores v at shared-memory address `sa` (this CTA's offset; every CTA lays
// out its memory alike) of CTA `rank` of the cluster.
__device__ __forceinline__ void st_cluster_f64(uint32_t sa, uint32_t rank, double v) {
    uint32_t ra;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(ra) : "r"(sa), "r"(rank));
    asm volatile("st.shared::cluster.f64 [%0], %1;" ::"r"(ra), "d"(v) : "memory");
}

struct ClusterArgs {
    const int32_t* row_ptr;
    const uint16_t* lcol;      // column numbers in the owning CTA's extended direction
    const double* values;
    const int32_t* push_off;   // [kClusterCtas][NT + 1]: a thread's range of push_ent
    const uint32_t* push_ent;  // q | dest << 3 | halo slot << 7
    CgState* st;
    const double* P0;  // p_0 = r_0 (the initial kernel)
    const double* R0;  // r_0
    int32_t n;
    int32_t width;
    int32_t nblk;   // 256-row tiles
    int32_t halo;   // halo slots of every CTA (the most any CTA needs)
    int32_t pmax;   // push entries of the CTA with the most
};

// The warp sums of P values per lane at once (P a power of two <= 8): the
// same pairing as warp_sum's shuffle tree, value by value -- stage o adds the
// partials of lanes l and l ^ o -- but at each of the first log2(P) stages a
// lane keeps half of its values and hands the partner the other half, so the
// P trees take P - 1 + 5 - log2(P) shuffles instead of 5 P.  Afterwards v[0]
// of lane l holds the sum of value (l >> (5 - log2 P)) & (P - 1).
template <int P>
__device__ __forceinline__ void multi_warp_sum(double (&v)[P]) {
    const int lane = threadIdx.x & 31;
    int o = 16;
#pragma unroll
    for (int cnt = P; cnt > 1; cnt >>= 1, o >>= 1) {
        const bool hi = (lane & o) != 0;
        const int half = cnt >> 1;
#pragma unroll
        for (int j = 0; j < half; ++j) {
            const double send = hi ? v[j] : v[j + half];
            const double keep = hi ? v[j + half] : v[j];
            v[j] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
    }
#pragma unroll
    for (; o > 0; o >>= 1) v[0] += __shfl_xor_sync(0xffffffffu, v[0], o);
}

constexpr int pow2_at_least(int r) { return r <= 1 ? 1 : (r <= 2 ? 2 : (r <= 4 ? 4 : 8)); }
constexpr int log2_of(int p) { return p <= 1 ? 0 : 1 + log2_of(p / 2); }

// Tile sums of one value per owned row (row t + NT q is lane t % 32 of warp
// (t / 32) % 8 of the CTA's tile (NT / 256) q + t / 256): every warp's R
// shuffle trees at once, parked in scr[tile][warp in tile].
template <int R, int NT>
__device__ __forceinline__ void tile_parts(const double (&d)[R], double (*scr)[kWarps]) {
    constexpr int P = pow2_at_least(R);
    constexpr int SH = 5 - log2_of(P);
    double v[P];
#pragma unroll
    for (int q = 0; q < P; ++q) v[q] = q < R ? d[q] : 0.0;
    multi_warp_sum<P>(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int q = (lane >> SH) & (P - 1);
    if ((lane & ((1 << SH) - 1)) == 0 && q < R)
        scr[q * (NT / kThreads) + warp / kWarps][warp % kWarps] = v[0];
}

// After a CTA barrier on scr: each tile's 8 warp sums added in warp order
// from 0.0, and the tile sum stored at entry tile0 + tile of `ts_sa` in every
// CTA of the cluster -- one (tile, destination) pair per thread.
template <int KT>
__device__ __forceinline__ void push_tiles(double (*scr)[kWarps], uint32_t ts_sa, int tile0) {
    const int t = threadIdx.x;
    if (t < KT * kClusterCtas) {
        const int tile = t % KT, dest = t / KT;
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) s += scr[tile][w];
        st_cluster_f64(ts_sa + uint32_t(tile0 + tile) * 8u, uint32_t(dest), s);
    }
}

// After the cluster barrier: the total of the cluster's tile sums (this
// CTA's copy `ts`, nblk <= 256 of them) in reduce256's order, by one warp --
// lane l takes tiles l + 32 w as virtual warp w's lane, the
// eight virtual warps' trees run at once and their sums are added in order
// from 0.0, block_sum8's order.
__device__ __forceinline__ double cluster_total(const double* ts, int nblk) {
    const int lane = threadIdx.x & 31;
    double v[8];
#pragma unroll
    for (int w = 0; w < 8; ++w) v[w] = lane + 32 * w < nblk ? ts[lane + 32 * w] : 0.0;
    multi_warp_sum<8>(v);  // lane 4 w holds virtual warp w's sum
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < 8; ++w) s += __shfl_sync(0xffffffffu, v[0], 4 * w);
    return s;
}

template <int R, int WM, bool F32V>
__global__ void __launch_bounds__(cluster_threads<F32V>(), 1) cg_cluster_kernel(ClusterArgs a) {
    constexpr int NT = cluster_threads<F32V>();
    constexpr int RC = NT * R;                // rows per CTA
    constexpr int KT = R * (NT / kThreads);   // 256-row tiles per CTA
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int W = a.width;  // <= WM: the stride of A in shared memory
    double* pe = reinterpret_cast<double*>(smem_raw);  // [RC + halo]: own rows of p_k, the halo
    double* hr = pe + RC + a.halo;                     // [halo] the halo's entries of r_k
    double* aps = hr + a.halo;                         // [RC] own rows of A p_k
    // [R][W][NT] values (doubles, or floats followed by 16-bit column numbers)
    double* vald = aps + RC;
    float* valf = reinterpret_cast<float*>(aps + RC);
    uint32_t* pent = F32V ? reinterpret_cast<uint32_t*>(valf + R * W * NT)
                          : reinterpret_cast<uint32_t*>(vald + R * W * NT);  // [pmax]
    uint16_t* colh = reinterpret_cast<uint16_t*>(pent + a.pmax);
    const uint32_t pe_sa = smem_u32(pe), hr_sa = smem_u32(hr);
    __shared__ double scr[KT][kWarps];
    __shared__ double sc[4];  // the scalars warp 0 derives from a total
    __shared__ double ts_a[kClusterCtas * KT], ts_b[kClusterCtas * KT];  // every CTA's tiles
    const int t = threadIdx.x;
    const uint32_t rank = cg::this_cluster().block_rank();
    CgState* st = a.st;
    if (__ldcg(&st->done)) return;  // the same in every CTA: no barrier is skipped unevenly
    const int32_t row0 = int32_t(rank) * RC;
    const int tile0 = int(rank) * KT;
    double* __restrict__ xg = st->x;
    const double bnorm = __ldcg(&st->bnorm), tol = __ldcg(&st->tol);
    const int32_t max_iter = __ldcg(&st->max_iter), guard = __ldcg(&st->guard);
    double rr = __ldcg(&st->rr);
    int32_t iter = __ldcg(&st->iter);

    // this CTA's halo stores: its entries in shared memory, a thread's range
    const int32_t* po = a.push_off + rank * (NT + 1);
    const int32_t pbase = __ldg(po);
    const int32_t ptotal = __ldg(po + NT) - pbase;
    for (int j = t; j < ptotal; j += NT) pent[j] = __ldg(a.push_ent + pbase + j);
    const int32_t pj0 = __ldg(po + t) - pbase, pj1 = __ldg(po + t + 1) - pbase;

    constexpr int kColWords = F32V ? 1 : (WM + 1) / 2;
    uint32_t colp[R][kColWords];  // doubles: column numbers two to a word
    uint32_t lens = 0u;           // R <= 8 rows of 4 bits
    double r[R], x[R];
#pragma unroll
    for (int q = 0; q < R; ++q) {
        const int32_t row = row0 + t + NT * q;
        double p0 = 0.0;
        r[q] = 0.0;
        x[q] = 0.0;
#pragma unroll
        for (int e = 0; e < kColWords; ++e) colp[q][e] = 0u;
        if (row < a.n) {
            const int32_t z0 = __ldg(a.row_ptr + row);
            const int len = __ldg(a.row_ptr + row + 1) - z0;
            lens |= uint32_t(len) << (4 * q);
#pragma unroll
            for (int e = 0; e < WM; ++e)
                if (e < len) {
                    const uint32_t c = __ldg(a.lcol + z0 + e);
                    const int at = (q * W + e) * NT + t;
                    if constexpr (F32V) {
                        valf[at] = static_cast<float>(__ldg(a.values + z0 + e));
                        colh[at] = static_cast<uint16_t>(c);
                    } else {
                        colp[q][e >> 1] |= (e & 1) ? (c << 16) : c;
                        vald[at] = __ldg(a.values + z0 + e);
                    }
                }
            r[q] = __ldcg(a.R0 + row);
            p0 = __ldcg(a.P0 + row);
            if constexpr (F32V) x[q] = xg[row];
        }
        pe[t + NT * q] = p0;
    }
    for (int j = t; j < 2 * a.halo; j += NT) pe[RC + j] = 0.0;  // the halo's p and r
    // Every CTA of the cluster running, its push entries in place, before the
    // first store into another CTA's shared memory; then p_0's halo.
    cluster_sync_all();
    for (int j = pj0; j < pj1; ++j) {
        const uint32_t e = pent[j];
        st_cluster_f64(pe_sa + (RC + (e >> 7)) * 8u, (e >> 3) & 15u, pe[t + NT * (e & 7u)]);
    }
    cluster_sync_all();

    // Per iteration two cluster barriers: after the p.Ap tile sums, and after
    // the r.r tile sums together with the r entries of every halo.  Each CTA
    // forms p_{k+1} = r + beta p_k for its own rows and for its halo alike
    // (the same fma on the same doubles as the owner), so the direction needs
    // no barrier of its own.
    double beta = 0.0;
    int status = kCgOk;
    for (int k = 0;; ++k) {
        // ---- the new direction, own rows and halo, in this CTA's shared memory ----
        if (k > 0) {
            double pv[R];
#pragma unroll
            for (int q = 0; q < R; ++q) pv[q] = pe[t + NT * q];
#pragma unroll
            for (int q = 0; q < R; ++q) pv[q] = fma(beta, pv[q], r[q]);  // p = 1*r + beta*p
#pragma unroll
            for (int q = 0; q < R; ++q) pe[t + NT * q] = pv[q];
            for (int j = t; j < a.halo; j += NT) pe[RC + j] = fma(beta, pe[RC + j], hr[j]);
            __syncthreads();
        }
        // ---- Ap = A p (thread rows, serial CSR-order sums), p.Ap per tile ----
        double d[R];
#pragma unroll
        for (int q = 0; q < R; ++q) {
            double acc = 0.0;
            const int len = int((lens >> (4 * q)) & 15u);
#pragma unroll
            for (int e = 0; e < WM; ++e)
                if (e < len) {
                    const int at = (q * W + e) * NT + t;
                    uint32_t c;
                    double v;
                    if constexpr (F32V) {
                        c = colh[at];
                        v = static_cast<double>(valf[at]);
                    } else {
                        c = (colp[q][e >> 1] >> ((e & 1) * 16)) & 0xffffu;
                        v = vald[at];
                    }
                    acc = add_rn(acc, mul_rn(v, pe[c]));
                }
            aps[t + NT * q] = acc;
            d[q] = fma(pe[t + NT * q], acc, 0.0);
        }
        tile_parts<R, NT>(d, scr);
        __syncthreads();
        push_tiles<KT>(scr, smem_u32(ts_a), tile0);
        cluster_sync_all();
        if (t < 32) {  // warp 0: p.Ap, alpha, the breakdown test
            const double pAp = cluster_total(ts_a, a.nblk);
            if (t == 0) {
                sc[0] = pAp;
                sc[1] = rr / pAp;
                sc[2] = (guard && fabs(pAp) < 1e-300) ? 1.0 : 0.0;
            }
        }
        __syncthreads();
        if (sc[2] != 0.0) {
            status = kCgBreakdown;
            if (rank == 0 && t == 0) {
                st->pAp = sc[0];
                st->converged = 0;
                st->iters = iter;
                st->final_res = sqrt(rr) / bnorm;
            }
            break;
        }
        const double alpha = sc[1];
        // ---- x += alpha p, r -= alpha Ap, r.r per tile, r's halo entries ----
#pragma unroll
        for (int q = 0; q < R; ++q) {
            const int32_t row = row0 + t + NT * q;
            d[q] = 0.0;
            if (row < a.n) {
                r[q] = fma(-alpha, aps[t + NT * q], r[q]);  // r = -alpha*Ap + r
                d[q] = fma(r[q], r[q], 0.0);
                if constexpr (F32V) x[q] = fma(alpha, pe[t + NT * q], x[q]);  // x = alpha*p + x
            }
        }
        for (int j = pj0; j < pj1; ++j) {
            const uint32_t e = pent[j], eq = e & 7u;
            double v = r[0];
#pragma unroll
            for (int q = 1; q < R; ++q) v = eq == uint32_t(q) ? r[q] : v;
            st_cluster_f64(hr_sa + (e >> 7) * 8u, (e >> 3) & 15u, v);
        }
        tile_parts<R, NT>(d, scr);
        if constexpr (!F32V) {
#pragma unroll
            for (int q = 0; q < R; ++q) {
                const int32_t row = row0 + t + NT * q;
                if (row < a.n) xg[row] = fma(alpha, pe[t + NT * q], xg[row]);  // x = alpha*p + x
            }
        }
        __syncthreads();
        push_tiles<KT>(scr, smem_u32(ts_b), tile0);
        cluster_sync_all();
        if (t < 32) {  // warp 0: r.r, the stopping test, beta
            const double rr_new = cluster_total(ts_b, a.nblk);
            if (t == 0) {
                sc[0] = rr_new;
                sc[1] = sqrt(rr_new) / bnorm;
                sc[2] = rr_new / rr;
            }
        }
        __syncthreads();
        const double rr_new = sc[0], rel = sc[1];
        ++iter;
        if (rel < tol) {
            if (rank == 0 && t == 0) {
                st->iter = iter; st->converged = 1; st->iters = iter; st->final_res = rel;
                st->rr = rr_new;
            }
            break;
        }
        beta = sc[2];
        rr = rr_new;
        if (iter >= max_iter) {
            if (rank == 0 && t == 0) {
                st->iter = iter; st->converged = 0; st->iters = max_iter; st->final_res = rel;
                st->beta = beta; st->rr = rr;
            }
            break;
        }
    }
    if constexpr (F32V) {
#pragma unroll
        for (int q = 0; q < R; ++q) {
            const int32_t row = row0 + t + NT * q;
            if (row < a.n) xg[row] = x[q];
        }
    }
    // No CTA may leave while another can still read or write its shared memory.
    cluster_sync_all();
    if (rank == 0 && t == 0) {
        if (status != kCgOk) st->status = status;
        st->done = 1;
    }
}

template <int WM, bool F32V, int... Rs>
const void* cluster_fn(int R, std::integer_sequence<int, Rs...>) {
    const void* fns[] = {reinterpret_cast<const void*>(cg_cluster_kernel<Rs + 1, WM, F32V>)...};
    return fns[R - 1];
}

// The instance for R rows per thread of width class `cls`.
template <bool F32V>
const void* cluster_kernel_for(int cls, int R) {
    constexpr const int* mr = F32V ? kClassMaxR32 : kClassMaxR64;
    switch (cls) {
        case 0: return cluster_fn<3, F32V>(R, std::make_integer_sequence<int, mr[0]>{});
        case 1: return cluster_fn<5, F32V>(R, std::make_integer_sequence<int, mr[1]>{});
        case 2: return cluster_fn<7, F32V>(R, std::make_integer_sequence<int, mr[2]>{});
        default: return cluster_fn<8, F32V>(R, std::make_integer_sequence<int, mr[3]>{});
    }
}

const void* cluster_kernel_for(bool f32v, int cls, int R) {
    return f32v ? cluster_kernel_for<true>(cls, R) : cluster_kernel_for<false>(cls, R);
}

}  // namespace

int plan_cluster(const nm_csr* A, CgWorkspace* ws) {
    ws->cluster = false;
    const int64_t n = A->nrows;
    if (n > int64_t(kClusterCtas) * 1024 * 4) return NM_OK;
    if (A->tune.max_rows != kThreads) return NM_OK;
    if (int64_t(A->h_row_ptr.size()) != n + 1) return NM_OK;
    if (A->nblk != (n + kThreads - 1) / kThreads) return NM_OK;  // whole 256-row tiles
    const int wcap = std::min({A->tune.short_max, A->tune.tile / kThreads, kClusterMaxWidth});
    const int32_t* rp = A->h_row_ptr.data();
    const int32_t* ci = A->h_col_idx.data();
    int W = 1;
    for (int64_t i = 0; i < n; ++i) {
        const int len = rp[i + 1] - rp[i];
        if (len > wcap) return NM_OK;
        W = std::max(W, len);
    }
    int cls = 0;
    while (kWidthClasses[cls] < W) ++cls;  // W <= kClusterMaxWidth, the last class
    // Values that are floats exactly (a stencil's integers, say) are held as
    // floats: less shared memory, the same doubles on the way back.
    const int64_t nnz = rp[n];
    std::vector<double> hv(static_cast<size_t>(nnz));
    NM_CUDA_TRY(cudaMemcpy(hv.data(), A->d_values, sizeof(double) * size_t(nnz),
                           cudaMemcpyDeviceToHost));
    bool f32v = true;
    for (const double v : hv)
        if (static_cast<double>(static_cast<float>(v)) != v) {
            f32v = false;
            break;
        }
    const int NT = f32v ? cluster_threads<true>() : cluster_threads<false>();
    const int64_t per_r = int64_t(kClusterCtas) * NT;
    const int R = static_cast<int>((n + per_r - 1) / per_r);
    if (R > (f32v ? kClassMaxR32 : kClassMaxR64)[cls]) return NM_OK;
    const int32_t RC = NT * R;

    // Each CTA's columns in its extended direction: its own rows, then one
    // halo slot per other column it reads; and for every such slot a store
    // by the thread that owns the column's row.
    std::vector<uint16_t> lcol(static_cast<size_t>(nnz));
    std::vector<int32_t> slot_of(static_cast<size_t>(n), -1);  // a CTA's halo slot of a column
    std::vector<int32_t> touched;
    std::vector<std::pair<int32_t, uint32_t>> pushes;  // (owner CTA * NT + thread, entry)
    int32_t halo = 0;
    for (int c = 0; c < kClusterCtas; ++c) {
        const int64_t r0 = int64_t(c) * RC, r1 = std::min<int64_t>(r0 + RC, n);
        for (int64_t i = r0; i < r1; ++i)
            for (int32_t z = rp[i]; z < rp[i + 1]; ++z) {
                const int32_t col = ci[z];
                if (col >= r0 && col < r0 + RC) {
                    lcol[size_t(z)] = static_cast<uint16_t>(col - r0);
                    continue;
                }
                int32_t slot = slot_of[size_t(col)];
                if (slot < 0) {
                    slot = int32_t(touched.size());
                    if (RC + slot > 0xffff) return NM_OK;  // beyond 16-bit column numbers
                    slot_of[size_t(col)] = slot;
                    touched.push_back(col);
                    const int32_t o = col / RC, lr = col - o * RC;
                    pushes.emplace_back(o * NT + lr % NT,
                                        uint32_t(lr / NT) | uint32_t(c) << 3 | uint32_t(slot) << 7);
                }
                lcol[size_t(z)] = static_cast<uint16_t>(RC + slot);
            }
        halo = std::max(halo, int32_t(touched.size()));
        for (const int32_t col : touched) slot_of[size_t(col)] = -1;
        touched.clear();
    }
    // the stores grouped by owning thread (counting sort; each thread's in
    // the order found)
    std::vector<int32_t> push_off(size_t(kClusterCtas) * (NT + 1), 0);
    std::vector<int32_t> per_thread(size_t(kClusterCtas) * NT + 1, 0);
    for (const auto& pr : pushes) ++per_thread[size_t(pr.first) + 1];
    for (size_t k = 1; k < per_thread.size(); ++k) per_thread[k] += per_thread[k - 1];
    std::vector<uint32_t> push_ent(pushes.size());
    {
        std::vector<int32_t> fill(per_thread.begin(), per_thread.end() - 1);
        for (const auto& pr : pushes) push_ent[size_t(fill[size_t(pr.first)]++)] = pr.second;
    }
    int32_t pmax = 0;
    for (int o = 0; o < kClusterCtas; ++o) {
        for (int t = 0; t <= NT; ++t)
            push_off[size_t(o) * (NT + 1) + t] = per_thread[size_t(o) * NT + t];
        pmax = std::max(pmax, per_thread[size_t(o + 1) * NT] - per_thread[size_t(o) * NT]);
    }
    if (pmax > kMaxPushes) return NM_OK;

    const size_t held = size_t(R) * W * NT;  // entries of A a CTA holds
    const size_t smem = sizeof(double) * (2 * size_t(RC) + 2 * size_t(halo)) +
                        (f32v ? held * sizeof(float) : held * sizeof(double)) +
                        sizeof(uint32_t) * size_t(pmax) +
                        (f32v ? held * sizeof(uint16_t) : 0);
    int dev = 0, cl = 0, smem_max = 0;
    NM_CUDA_TRY(cudaGetDevice(&dev));
    NM_CUDA_TRY(cudaDeviceGetAttribute(&cl, cudaDevAttrClusterLaunch, dev));
    NM_CUDA_TRY(cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const void* fn = cluster_kernel_for(f32v, cls, R);
    if (!cl) return NM_OK;
    // Per device and kernel instance, once: its static shared memory, the
    // cluster-size and shared-memory attributes (set to the device's
    // maximum), and per dynamic size whether a cluster can be scheduled.
    static std::mutex cache_mu;
    static std::map<std::pair<int, const void*>, size_t> static_smem;
    static std::map<std::tuple<int, const void*, size_t>, bool> schedulable;
    std::lock_guard<std::mutex> lock(cache_mu);
    auto si = static_smem.find({dev, fn});
    if (si == static_smem.end()) {
        cudaFuncAttributes fa;
        NM_CUDA_TRY(cudaFuncGetAttributes(&fa, fn));
        NM_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        NM_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         smem_max - static_cast<int>(fa.sharedSizeBytes)));
        si = static_smem.emplace(std::make_pair(dev, fn), fa.sharedSizeBytes).first;
    }
    if (smem + si->second > size_t(smem_max)) return NM_OK;
    const auto key = std::make_tuple(dev, fn, smem);
    auto sc = schedulable.find(key);
    if (sc != schedulable.end()) {
        if (!sc->second) return NM_OK;
    } else {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(kClusterCtas);
        cfg.blockDim = dim3(NT);
        cfg.dynamicSmemBytes = smem;
        cudaLaunchAttribute attr;
        attr.id = cudaLaunchAttributeClusterDimension;
        attr.val.clusterDim.x = kClusterCtas;
        attr.val.clusterDim.y = 1;
        attr.val.clusterDim.z = 1;
        cfg.attrs = &attr;
        cfg.numAttrs = 1;
        int clusters = 0;
        const bool ok = cudaOccupancyMaxActiveClusters(&clusters, fn, &cfg) == cudaSuccess &&
                        clusters >= 1;
        if (!ok) cudaGetLastError();  // not schedulable here: the other paths run
        schedulable.emplace(key, ok);
        if (!ok) return NM_OK;
    }

    // column numbers, push offsets and entries in one device allocation
    const size_t b_lcol = (sizeof(uint16_t) * size_t(nnz) + 255) & ~size_t(255);
    const size_t b_off = (sizeof(int32_t) * push_off.size() + 255) & ~size_t(255);
    const size_t b_ent = sizeof(uint32_t) * std::max<size_t>(push_ent.size(), 1);
    void* mem = nullptr;
    NM_CUDA_TRY(cudaMalloc(&mem, b_lcol + b_off + b_ent));
    char* base = static_cast<char*>(mem);
    cudaError_t e = cudaMemcpy(base, lcol.data(), sizeof(uint16_t) * size_t(nnz),
                               cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(base + b_lcol, push_off.data(), sizeof(int32_t) * push_off.size(),
                       cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !push_ent.empty())
        e = cudaMemcpy(base + b_lcol + b_off, push_ent.data(), sizeof(uint32_t) * push_ent.size(),
                       cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(mem);
        NM_CUDA_TRY(e);
    }
    if (ws->cl_mem) cudaFree(ws->cl_mem);
    ws->cl_mem = mem;
    ws->cl_lcol = reinterpret_cast<uint16_t*>(base);
    ws->cl_push_off = reinterpret_cast<int32_t*>(base + b_lcol);
    ws->cl_push_ent = reinterpret_cast<uint32_t*>(base + b_lcol + b_off);
    ws->cluster = true;
    ws->cl_rows_per_thread = R;
    ws->cl_class = cls;
    ws->cl_f32v = f32v;
    ws->cl_width = W;
    ws->cl_halo = halo;
    ws->cl_pmax = pmax;
    ws->cl_smem = smem;
    return NM_OK;
}

int launch_cluster(const nm_csr* A, CgWorkspace* ws, cudaStream_t s) {
    ClusterArgs a;
    a.row_ptr = A->d_row_ptr;
    a.lcol = ws->cl_lcol;
    a.values = static_cast<const double*>(A->d_values);
    a.push_off = ws->cl_push_off;
    a.push_ent = ws->cl_push_ent;
    a.st = ws->st;
    a.P0 = ws->p;
    a.R0 = ws->r;
    a.n = static_cast<int32_t>(A->nrows);
    a.width = ws->cl_width;
    a.nblk = static_cast<int32_t>(A->nblk);
    a.halo = ws->cl_halo;
    a.pmax = ws->cl_pmax;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kClusterCtas);
    cfg.blockDim = dim3(ws->cl_f32v ? cluster_threads<true>() : cluster_threads<false>());
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
    NM_CUDA_TRY(cudaLaunchKernelExC(
        &cfg, cluster_kernel_for(ws->cl_f32v, ws->cl_class, ws->cl_rows_per_thread), args));
    return NM_OK;
}

}  // namespace nm
