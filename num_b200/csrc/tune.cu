// tune.cu -- the SpMV autotuner: times candidate row-block partitions and
// launch shapes of one matrix on the device and keeps the fastest.
//
// Search space (every candidate is a valid nm_tuning):
//   tile      1024, 2048, 4096   nonzeros per multi-row block (smem stage size)
//   short_max 32, 64             rows up to this length are thread-per-row
//   stages    2, 3, 4            TMA ring depth (skipped when it does not fit)
//   grid_mult 0 (all resident CTAs), 1, 2 CTAs per SM
//   and, once each, the warp-gather and sliced gather kernels (which ignore
//   the four above)
// max_rows stays at its default (one consumer thread per row of a block).
// tile and short_max change the descriptors (a host rebuild per pair);
// stages and grid_mult only change the launch.  short_max never goes below
// 32, so every row of <= 32 nonzeros keeps the serial CSR summation order.
#include <algorithm>
#include <mutex>
#include <vector>

#include "csr.cuh"

namespace nm {
namespace {

// Average time of `reps` launches after `warm` untimed ones, in microseconds.
int time_spmv(const nm_csr* A, const void* x, void* y, cudaStream_t s, int warm, int reps,
              cudaEvent_t e0, cudaEvent_t e1, float* us) {
    for (int i = 0; i < warm; ++i) {
        const int st = launch_spmv(A, x, y, s);
        if (st != NM_OK) return st;
    }
    NM_CUDA_TRY(cudaEventRecord(e0, s));
    for (int i = 0; i < reps; ++i) {
        const int st = launch_spmv(A, x, y, s);
        if (st != NM_OK) return st;
    }
    NM_CUDA_TRY(cudaEventRecord(e1, s));
    NM_CUDA_TRY(cudaEventSynchronize(e1));
    float ms = 0.f;
    NM_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
    *us = ms * 1000.f / float(reps);
    return NM_OK;
}

struct EventPair {
    cudaEvent_t a = nullptr, b = nullptr;
    ~EventPair() {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
};

}  // namespace
}  // namespace nm

extern "C" int nm_csr_autotune(nm_csr* A, const void* x, void* y, void* stream,
                               double budget_ms, nm_tuning* best, nm_tune_trial* trials,
                               int32_t cap, int32_t* ntrials) {
    using namespace nm;
    clear_error();
    if (!A || !x || !y || !best) return fail(NM_ERR_INVALID, "nm_csr_autotune: NULL argument");
    if (cap > 0 && !trials) return fail(NM_ERR_INVALID, "nm_csr_autotune: NULL trials");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const nm_tuning start = A->tune;
    int dev = 0, smem_max = 0;
    NM_CUDA_TRY(cudaGetDevice(&dev));
    NM_CUDA_TRY(cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    reset_cg(A);  // its graphs hold the descriptors rebuilt below
    EventPair ev;
    NM_CUDA_TRY(cudaEventCreate(&ev.a));
    NM_CUDA_TRY(cudaEventCreate(&ev.b));
    // Launches per candidate: about budget_ms / (candidates x SpMV time).
    float t0 = 0.f;
    int st = time_spmv(A, x, y, s, 2, 3, ev.a, ev.b, &t0);
    if (st != NM_OK) return st;
    constexpr int kCandidates = 3 * 2 * 3 * 3 + 1;
    const double budget_us = (budget_ms > 0 ? budget_ms : 200.0) * 1000.0;
    const int reps = int(std::max(3.0, std::min(200.0, budget_us / kCandidates / std::max(1.f, t0))));
    const int32_t tiles[] = {1024, 2048, 4096};
    const int32_t shorts[] = {32, 64};
    const int32_t stages[] = {2, 3, 4};
    const int32_t grids[] = {0, 1, 2};
    nm_tuning win = start;
    float win_us = 0.f;
    bool have = false;
    int32_t n = 0;
    for (int32_t tile : tiles)
        for (int32_t sm : shorts) {
            nm_tuning t = start;
            t.tile = tile;
            t.short_max = sm;
            t.max_rows = kDefaultMaxRows;
            t.stages = 2;
            t.grid_mult = 0;
            t.kernel = NM_KERNEL_BLOCKS;
            A->tune = t;
            st = rebuild_blocks(A);
            if (st != NM_OK) break;
            for (int32_t stg : stages)
                for (int32_t g : grids) {
                    if (st != NM_OK) break;
                    const size_t need = spmv_smem_for(A->dtype, tile, stg);
                    if (need == 0 || need > size_t(smem_max)) continue;  // does not fit an SM
                    A->tune.stages = stg;
                    A->tune.grid_mult = g;
                    float us = 0.f;
                    st = time_spmv(A, x, y, s, 1, reps, ev.a, ev.b, &us);
                    if (st != NM_OK) continue;  // ends both loops
                    if (n < cap) trials[n] = nm_tune_trial{A->tune, us};
                    ++n;
                    if (!have || us < win_us) {
                        win = A->tune;
                        win_us = us;
                        have = true;
                    }
                }
            if (st != NM_OK) break;
        }
    for (const int kern : {int(NM_KERNEL_GATHER), int(NM_KERNEL_SLICED)}) {
        if (st != NM_OK) break;
        nm_tuning t = start;
        t.kernel = kern;
        A->tune = t;
        st = rebuild_blocks(A);
        // a matrix whose sliced copy would pad too much runs the gather kernel
        // under NM_KERNEL_SLICED: nothing new to time
        if (st == NM_OK && kern == NM_KERNEL_SLICED && !A->sell_ready) break;
        float us = 0.f;
        if (st == NM_OK) st = time_spmv(A, x, y, s, 1, reps, ev.a, ev.b, &us);
        if (st == NM_OK) {
            if (n < cap) trials[n] = nm_tune_trial{A->tune, us};
            ++n;
            if (!have || us < win_us) {
                win = A->tune;
                win_us = us;
                have = true;
            }
        }
    }
    if (ntrials) *ntrials = n;
    // Install the winner (or put the starting tuning back on failure).
    const nm_tuning fin = (st == NM_OK && have) ? win : start;
    const int err = st;
    A->tune = fin;
    st = rebuild_blocks(A);
    if (err != NM_OK) return err;
    if (st != NM_OK) return st;
    *best = fin;
    return NM_OK;
}
