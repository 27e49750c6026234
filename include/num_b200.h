/*
 * num_b200.h -- C ABI of the num_b200 sparse library (CSR SpMV, multi-RHS and
 * many-matrix SpMV, CG and its vector ops, halo pack/unpack), built for
 * NVIDIA B200 (sm_100a).
 *
 * This is the drop-in boundary for the `kokkos_spmv` Python module of
 * w-jiwonchoi/num (src/bindings.cpp).  Every entry point takes plain pointers
 * and sizes; device buffers are raw CUDA device pointers and `stream` is a
 * cudaStream_t (NULL = the legacy default stream).  Entry points that only
 * enqueue work return as soon as it is enqueued; the ones that return a host
 * scalar (nm_dot, nm_norm2, nm_cg_*) synchronise `stream` first.
 *
 * Every function returns an nm_status; on failure nm_last_error() returns a
 * message for the calling thread.  The Python binding maps NM_ERR_INVALID to
 * ValueError, NM_ERR_TYPE to TypeError and the rest to RuntimeError, which are
 * the exception types of the reference binding.
 */
#ifndef NUM_B200_H
#define NUM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status, dtypes, result records ------------------------------------ */

enum nm_status {
    NM_OK = 0,
    NM_ERR_INVALID = 1,   /* bad size / shape / index: std::invalid_argument   */
    NM_ERR_TYPE = 2,      /* unsupported dtype                                  */
    NM_ERR_RUNTIME = 3,   /* algorithmic failure (e.g. CG breakdown guard)      */
    NM_ERR_CUDA = 4,      /* CUDA runtime error                                 */
    NM_ERR_NOMEM = 5      /* device allocation failed                           */
};

enum nm_dtype { NM_F64 = 0, NM_F32 = 1, NM_BF16 = 2 };

/* CGResult (src/cg_solver.hpp:22-26). */
typedef struct {
    int32_t iters;
    double final_res;
    int32_t converged;
} nm_cg_result;

/* Row-block partition parameters of the SpMV kernels (see nm_csr_set_tuning). */
typedef struct {
    int32_t tile;       /* max nonzeros of a multi-row block; longer rows get a CTA */
    int32_t max_rows;   /* max rows of a block (<= 256)                             */
    int32_t short_max;  /* rows with <= short_max nonzeros: one thread; else a warp */
    int32_t grid_mult;  /* CTAs launched per SM by the persistent SpMV grid (0: auto) */
    int32_t stages;     /* TMA pipeline depth of the SpMV kernels: 2, 3 or 4          */
    int32_t kernel;     /* plain SpMV kernel: NM_KERNEL_AUTO / _BLOCKS / _GATHER      */
} nm_tuning;

/* nm_tuning.kernel.  BLOCKS: the row-block TMA pipeline.  GATHER: one warp per
 * 32 rows streaming the nonzeros and gathering x through L2, every row summed
 * serially in CSR order (for scattered columns).  SLICED: the same serial row
 * sums from a copy of the matrix sorted by row length and stored as
 * column-major 32-row slices, lane per row (built when first selected; a
 * matrix it would pad to more than twice its nonzeros runs GATHER instead).
 * AUTO: GATHER when at least 3/4 of the nonzeros lie in row blocks without x
 * windows and no row has more than 4096 nonzeros, else BLOCKS.  The
 * autotuner times all three.  CG and the batched engine always use the
 * row-block pipeline. */
enum nm_kernel { NM_KERNEL_AUTO = 1, NM_KERNEL_BLOCKS = 2, NM_KERNEL_GATHER = 3,
                 NM_KERNEL_SLICED = 4 };

typedef struct nm_csr nm_csr;    /* device CSR matrix (CrsMatrixHandle)   */
typedef struct nm_dist nm_dist;  /* one rank's slice (DistCrsHandle)      */

/* ---- errors / context ----------------------------------------------------- */

/* Message of the last failing call on this thread ("" if none). */
const char* nm_last_error(void);

/* Library version string. */
const char* nm_version(void);

/* init(device_id) (src/bindings.cpp:53-66): selects the device and creates
 * its context.  This library is one process per GPU; rank/size are 0/1 here
 * (the Python layer reports torch.distributed's values when it is set up). */
int nm_init(int device_id, int32_t* rank, int32_t* size);

/* finalize() (src/bindings.cpp:68-70): releases cached workspaces. */
int nm_finalize(void);

/* Reads and clears the current device's error word.  Kernels that stage data
 * with TMA wait on mbarriers with a time limit (~2 s); one that gives up sets
 * the word and exits instead of hanging.  Call after synchronising the stream;
 * returns NM_ERR_RUNTIME if any kernel gave up since the last call. */
int nm_check_device_errors(void);

/* Failure-detection hook for tests (no counterpart in the reference, whose
 * kernels have no bounded waits).  Runs the library's own bounded wait
 * routine in a kernel where the wait cannot complete -- kind 0: an mbarrier
 * that expects one arrival more than it gets (one CTA); kind 1: a grid
 * barrier of `ctas` (1..64) co-resident CTAs that expects one CTA more --
 * with the wait limited to limit_ms (0 < limit_ms <= 2000) instead of the
 * library's ~2 s.  Nothing else is pending, so the kernel returns on its own
 * once the wait gives up.  Synchronises `stream`; *waited_ms (may be NULL)
 * receives the longest wait.  Returns NM_ERR_RUNTIME when the wait gave up,
 * as set up, leaving the device error word set for nm_check_device_errors;
 * NM_OK would mean the wait completed. */
int nm_test_wait_timeout(int32_t kind, int32_t ctas, double limit_ms, double* waited_ms,
                         void* stream);

/* ---- CSR matrix ------------------------------------------------------------ */

/* CrsMatrixHandle ctor (src/crs_matrix.hpp:45-72) / upload_csr
 * (src/bindings.cpp:97-108).  Copies host CSR arrays (int32 row_ptr[n+1],
 * int32 col_idx[nnz], values[nnz] of `dtype`) to the device and builds the
 * row-block partition.  nnz = row_ptr[nrows].  Non-positive dims, a row_ptr
 * that does not start at 0 or decreases, and column indices outside
 * [0, ncols) return NM_ERR_INVALID. */
int nm_csr_create(const int32_t* row_ptr, const int32_t* col_idx, const void* values,
                  int dtype, int32_t nrows, int32_t ncols, nm_csr** out);

/* Many independent CSR matrices (no counterpart in the reference): matrix m
 * has dims (nrows[m], ncols[m]) and its own CSR arrays, concatenated in
 * matrix order: row_ptr holds count segments of nrows[m]+1 entries (each
 * starting at 0), col_idx/values hold the nonzeros with LOCAL column indices.
 * The result is one block-diagonal device matrix; x and y of nm_spmv are the
 * per-matrix vectors concatenated in matrix order, so one launch multiplies
 * every matrix. */
int nm_csr_create_batched(int32_t count, const int32_t* nrows, const int32_t* ncols,
                          const int32_t* row_ptr, const int32_t* col_idx,
                          const void* values, int dtype, nm_csr** out);

/* The 5-point 2-D (dim 2; values 4 / -1) or 7-point 3-D (dim 3; 6 / -1)
 * Dirichlet Laplacian on an L^dim grid, x fastest, assembled on the device:
 * the same arrays as python/matrix_generators.py make_laplacian_2d (:16-37)
 * and make_laplacian_3d_fast (:68-80) followed by upload_csr
 * (src/bindings.cpp:97-123), without building them on the host or copying
 * them over PCIe (row_ptr and col_idx are read back once for the row-block
 * partition).  Values are stored as `dtype`.  dim other than 2 / 3, L <= 0,
 * or L^dim rows / nonzeros beyond the int32 offsets return NM_ERR_INVALID. */
int nm_csr_laplacian(int32_t dim, int32_t L, int dtype, nm_csr** out);

/* Copies the device arrays back to host buffers: row_ptr[nrows+1],
 * col_idx[nnz], values[nnz] in the stored dtype (many-matrix handles: the
 * block-diagonal matrix with global column indices).  Addition: the
 * reference's CrsMatrix has no read-back. */
int nm_csr_export(const nm_csr* A, int32_t* row_ptr, int32_t* col_idx, void* values);

/* Frees the device copy (handle destructor). */
int nm_csr_destroy(nm_csr* A);

/* Read-only properties nrows/ncols/nnz (src/bindings.cpp:79-88), the value
 * dtype, and the number of row blocks. */
int nm_csr_info(const nm_csr* A, int32_t* nrows, int32_t* ncols, int32_t* nnz,
                int32_t* dtype, int32_t* nblocks);

/* Replaces pick_rows_per_team (src/spmv_kernel.hpp:102-109): sets the
 * row-block partition parameters and rebuilds the partition.  tile,
 * max_rows, short_max, stages and kernel <= 0 (grid_mult < 0) keep their
 * current values; grid_mult 0 selects the automatic grid.  Defaults: 2048,
 * 256, 32, 0, 2, NM_KERNEL_AUTO. */
int nm_csr_set_tuning(nm_csr* A, const nm_tuning* t);
int nm_csr_get_tuning(const nm_csr* A, nm_tuning* t);

/* The plain-SpMV kernel nm_spmv runs on A under its tuning (AUTO resolved):
 * NM_KERNEL_BLOCKS, NM_KERNEL_GATHER or NM_KERNEL_SLICED. */
int nm_csr_spmv_kernel(const nm_csr* A, int32_t* kernel);

/* One timed candidate of nm_csr_autotune. */
typedef struct {
    nm_tuning tuning;
    float us;  /* average device time of one SpMV under `tuning` */
} nm_tune_trial;

/* SpMV autotuner (no reference counterpart; the reference's partition is
 * fixed).  Times y = A*x on `stream` under every candidate tile (1024, 2048,
 * 4096), short_max (32, 64), stages (2, 3, 4; those whose shared memory fits)
 * and grid_mult (0, 1, 2) of the row-block kernel, and the warp-gather
 * kernel, spending about budget_ms of device time (<= 0:
 * 200 ms), installs the fastest on A and returns it in *best.  x is read; y
 * is overwritten.  trials[0..min(cap, *ntrials)) receive every timing (trials
 * may be NULL when cap is 0).  Synchronises `stream`. */
int nm_csr_autotune(nm_csr* A, const void* x, void* y, void* stream, double budget_ms,
                    nm_tuning* best, nm_tune_trial* trials, int32_t cap, int32_t* ntrials);

/* Copies the row-block boundaries (nblocks+1 entries) and, if bins != NULL,
 * the per-row reduction bin (0 thread, 1 warp, 2 CTA) to host memory. */
int nm_csr_row_blocks(const nm_csr* A, int32_t* blk, int32_t cap, int8_t* bins);

/* Host only (needs no GPU): the row-block partition nm_csr_create builds for
 * row_ptr under tuning t (NULL = defaults); *nblk receives the block count,
 * blk its nblk+1 boundaries, bins (optional) the per-row reduction bin. */
int nm_row_blocks_host(const int32_t* row_ptr, int32_t nrows, const nm_tuning* t,
                       int32_t* blk, int32_t cap, int8_t* bins, int32_t* nblk);

/* ---- SpMV ------------------------------------------------------------------ */

/* spmv(A, x, y) (src/bindings.cpp:152-170; launch_spmv_custom and
 * launch_spmv_kokkoskernels, src/spmv_kernel.hpp:118-180): y = A*x.
 * F64 matrices take double x/y; F32 and BF16 matrices take float x/y and
 * accumulate in FP32. */
int nm_spmv(const nm_csr* A, const void* x, void* y, void* stream);

/* y = A*x for x[ncols] and y[nrows] in HOST memory (element types as for
 * nm_spmv): copies x in, multiplies, copies y out and returns when y is
 * written -- the work is ordered after what is already queued on `stream`,
 * and `stream` is synchronised before the call returns, also after an error.
 * The row blocks run in chunks, each as soon as the part of x its nonzeros
 * read has arrived, and each chunk's rows of y are copied out while later
 * chunks compute, so for banded matrices the two transfers overlap
 * (page-locked x and y let the copies run at the full link rate).  The handle
 * keeps device copies of x and y (allocated on the first call, freed with the
 * handle); calls on one handle run one after the other.  Not callable on a
 * stream that is being captured (it synchronises the stream).  Addition: the
 * reference's spmv takes device arrays only (src/bindings.cpp:152-183); this
 * is the call for a host-side caller, who would otherwise copy x in and y out
 * around nm_spmv. */
int nm_spmv_host(const nm_csr* A, const void* x, void* y, void* stream);

/* batch_spmv(A, X, Y) (src/bindings.cpp:186-200; launch_batch_spmv,
 * src/batch_spmv_kernel.hpp:120-174): Y(nrows,k) = A * X(ncols,k), both
 * row-major.  F64 matrices only (as in the reference). */
int nm_batch_spmv(const nm_csr* A, const double* X, double* Y, int32_t k, void* stream);

/* ---- vector ops (src/vec_ops.hpp) ------------------------------------------- */

/* vec_axpy (src/vec_ops.hpp:16-26): z = alpha*x + y, one FMA. */
int nm_axpy(int64_t n, double alpha, const double* x, const double* y, double* z,
            void* stream);
/* vec_axpy2 (src/vec_ops.hpp:31-42): z = alpha*x + beta*y = fma(beta, y, alpha*x). */
int nm_axpy2(int64_t n, double alpha, const double* x, double beta, const double* y,
             double* z, void* stream);
/* vec_local_dot (src/vec_ops.hpp:47-59): deterministic sum of x[i]*y[i]. */
int nm_dot(int64_t n, const double* x, const double* y, double* result, void* stream);
/* vec_local_norm2 (src/vec_ops.hpp:64-69). */
int nm_norm2(int64_t n, const double* x, double* result, void* stream);
/* vec_copy / vec_fill / vec_scale (src/vec_ops.hpp:74-100). */
int nm_copy(int64_t n, const double* src, double* dst, void* stream);
int nm_fill(int64_t n, double value, double* x, void* stream);
int nm_scale(int64_t n, double alpha, double* x, void* stream);

/* ---- CG -------------------------------------------------------------------- */

/* Process-wide choice of how nm_cg_local / nm_dist_cg_single iterate:
 * 1 (default) one persistent launch per solve for systems of at most 262,144
 * rows -- the cluster solve where it applies (systems of at most 65,536 rows
 * of at most 8 nonzeros on one 16-CTA thread-block cluster: the rows of A in
 * shared memory, each CTA's halo of the direction kept current over
 * distributed shared memory, two hardware cluster barriers per iteration),
 * else the TMA-pipelined persistent solve where its SpMV grid is
 * co-resident, else the resident solve (matrix rows and vectors kept on
 * chip, two grid-wide sums per iteration; rows of at most 8 nonzeros);
 * 2 the TMA-pipelined persistent solve only; 3 the resident solve only;
 * 4 the cluster solve only; 0 CUDA-graph chunks of two kernels per
 * iteration, the SpMV forming p = r + beta p as it reads it (also what 2 to 4
 * run where their path does not apply).  All
 * give the same iterates, bit for bit (every dot product is summed in one
 * fixed order: per row block or 256-row tile, then over the blocks).  Other
 * values: NM_ERR_INVALID.  No reference counterpart (an implementation
 * switch). */
int nm_cg_set_persistent(int32_t enable);

/* How the last nm_cg_local / nm_dist_cg_single solve on A iterated: 0 the
 * CUDA-graph chunks, 1 the TMA-pipelined persistent solve (three grid
 * barriers per iteration), 2 the same in its two-barrier form, 3 the resident
 * solve, 4 the cluster solve; -1 before A's first solve.  No reference
 * counterpart. */
int nm_cg_last_path(const nm_csr* A, int32_t* path);

/* cg_solve_local (src/cg_solver.hpp:133-196; src/bindings.cpp:273-290):
 * unpreconditioned CG, x in/out, same stopping rule and iteration count.
 * The iteration runs on the device with device-resident scalars; the
 * workspace is cached on the matrix.  F64 matrices. */
int nm_cg_local(nm_csr* A, const double* b, double* x, double tol, int32_t max_iter,
                nm_cg_result* result, void* stream);

/* CG that allocates nothing.  No counterpart in the reference.  For callers
 * that cannot call cudaMalloc when they solve: processes whose device memory
 * is already claimed by another allocator (a framework's caching pool, a
 * serving engine that reserves nearly all of HBM), and latency-critical loops
 * where cudaMalloc / cudaFree would synchronise the device.  Same algorithm,
 * kernels and result as nm_cg_local, but every scratch vector comes from one
 * fixed device array that is part of the library (about 8.4 MB, held until
 * exit) instead of a per-matrix workspace.  The driver reserves that array
 * on a device when it loads the CG code there: under CUDA's default lazy
 * module loading that is the first call of nm_cg_local_static or nm_cg_local
 * on the device (with CUDA_MODULE_LOADING=EAGER, when the library loads), so
 * a caller whose pool will claim nearly all of HBM makes one call (a solve
 * of any small matrix) on each device before that pool takes its memory.
 * A is a handle made earlier with nm_csr_create; b, x as in nm_cg_local.
 * Limit: A->nrows <= 262,144 (larger matrices: NM_ERR_INVALID).  The first
 * call on a device looks up the array's device address, and the first call
 * with each tile / stage setting sets that kernel's attributes; those first
 * calls must not overlap a global-mode stream capture on any thread.  The
 * entry point waits on `stream` for the solve's progress, so it cannot be
 * called on a stream that is being captured.  All calls
 * share the one array (the state is reset at the start of each call); calls
 * that overlap on the GPU would race, so this entry point serialises its host
 * callers and synchronises `stream` before returning, on error returns too. */
int nm_cg_local_static(const nm_csr* A, const double* b, double* x, double tol,
                       int32_t max_iter, nm_cg_result* result, void* stream);

/* ---- batched / mixed-precision / served solver (no counterpart in the reference) */

typedef struct nm_solver nm_solver;

/* Solver options.  inner: value precision of the inner iterations -- NM_F64
 * (plain FP64 Jacobi-PCG, no refinement), NM_F32 or NM_BF16 (FP32 vectors and
 * accumulation, FP64 iterative refinement).  precond: 1 Jacobi, 0 none.
 * inner_rtol: relative reduction of one inner solve (default 1e-3; ignored
 * for NM_F64).  max_outer: refinement steps before giving up (default 30). */
typedef struct {
    int32_t inner;
    int32_t precond;
    double inner_rtol;
    int32_t max_outer;
    double cont_window; /* a refinement step keeps the Krylov direction while the
                           true residual is within this factor of the inner
                           solve's estimate (default 2; <= 0 keeps the default) */
} nm_solver_opts;

/* Process-wide choice of how a step's inner iterations run: 0 (default) a
 * CUDA graph whose loop body launches the SpMV, update and p update of every
 * live system as kernels; 1 one persistent cooperative launch per step (the
 * same phases separated by grid barriers, ending as soon as no system
 * iterates), when the device supports it.  Both give the same bits.  Other
 * values: NM_ERR_INVALID. */
int nm_solver_set_persistent(int32_t enable);

/* A solver with a device arena for up to max_rows rows and max_nnz nonzeros
 * in total over max_systems concurrently resident systems. */
int nm_solver_create(int64_t max_rows, int64_t max_nnz, int32_t max_systems,
                     const nm_solver_opts* opts, nm_solver** out);
int nm_solver_destroy(nm_solver* S);

/* Admit one SPD system A x = b (host CSR, FP64; x0 may be NULL for zero) with
 * its own tolerance |b - A x| / |b| < tol and iteration cap.  Returns
 * NM_ERR_NOMEM when its rows or nonzeros do not fit the free arena or no
 * slot is free (admission by free device memory); *slot identifies it. */
int nm_solver_admit(nm_solver* S, const int32_t* row_ptr, const int32_t* col_idx,
                    const double* values, int32_t n, const double* b, const double* x0,
                    double tol, int32_t max_iter, int32_t* slot);

/* Admit systems in order, preparing them in parallel on the host, until one
 * does not fit (FIFO): *admitted = how many were admitted, slots[0..admitted)
 * their slots.  Returns NM_OK when the rest merely did not fit. */
int nm_solver_admit_batch(nm_solver* S, int32_t count, const int32_t* const* row_ptr,
                          const int32_t* const* col_idx, const double* const* values,
                          const int32_t* n, const double* const* b, double tol, int32_t max_iter,
                          int32_t* slots, int32_t* admitted);

/* One step of the batch: the pending refinement steps, then up to `iters`
 * inner iterations of every active system (rounded up to a multiple of 8; in
 * groups of 8, the device ends the step early once no system is iterating --
 * every live one has converged or awaits its refinement step), then the
 * systems' states are read back; *n_done = systems that finished in this
 * step.  Synchronous. */
int nm_solver_step(nm_solver* S, int32_t iters, int32_t* n_done);

/* nm_solver_step in two halves, so that host work overlaps the device:
 * _begin enqueues the step and returns; nm_solver_admit / _admit_batch may run
 * meanwhile (their host preparation overlaps the iterations, their uploads go
 * on a separate stream; the systems join at the next step); _end waits and
 * reads the states back.  nm_solver_take is refused between the two. */
int nm_solver_step_begin(nm_solver* S, int32_t iters);
int nm_solver_step_end(nm_solver* S, int32_t* n_done);

/* Engine counters since creation: steps run, list rebuilds, chunk graph
 * captures and full instantiations, outer (refinement) launches, inner
 * iterations run; host seconds spent per part of a step (list upload,
 * outer launch, capture, waiting in nm_solver_step_end, state scan) and of
 * admission (parallel preparation, upload enqueue); device seconds of all
 * steps and milliseconds of the last one. */
typedef struct {
    int64_t steps, list_uploads, graph_captures, graph_instantiations, outer_launches,
        inner_iterations;
    double s_lists, s_outer, s_capture, s_run, s_scan;
    double s_admit_prep, s_admit_commit, s_device, last_step_ms;
    int64_t last_step_iters;  /* inner iterations the last step ran */
} nm_solver_counters;
int nm_solver_counters_get(const nm_solver* S, nm_solver_counters* out);

/* State of a slot: phase (1 refining, 2 iterating, 3 done), result (iters =
 * inner iterations, final_res = |b - A x| / |b| of the last refinement
 * step), refinement steps taken. */
int nm_solver_status(const nm_solver* S, int32_t slot, int32_t* phase, nm_cg_result* result,
                     int32_t* outer);

/* Copy the solution to host memory (x_host may be NULL) and free the slot. */
int nm_solver_take(nm_solver* S, int32_t slot, double* x_host);

/* nm_solver_take for `count` distinct slots at once: x_host[k] (NULL, or
 * x_host itself NULL: discard) receives the solution of slots[k]; one stream
 * synchronisation for all.  Not between step_begin and step_end. */
int nm_solver_take_batch(nm_solver* S, int32_t count, const int32_t* slots,
                         double* const* x_host);

/* Solve an admitted system again (same matrix): b_host (NULL: keep b) and
 * x0_host (NULL: zero) are copied in, the iteration state is reset, and the
 * system rejoins at the next step.  Not between step_begin and step_end. */
int nm_solver_resolve(nm_solver* S, int32_t slot, const double* b_host, const double* x0_host);

/* Copy of a system's current x (the system stays admitted).  Synchronous. */
int nm_solver_solution(nm_solver* S, int32_t slot, double* x_host);

/* The cudaStream_t the solver's steps run on (for timing with events). */
int nm_solver_stream(const nm_solver* S, void** stream);

/* Largest free row and nonzero ranges, active systems, free slots. */
int nm_solver_info(const nm_solver* S, int64_t* free_rows, int64_t* free_nnz, int32_t* active,
                   int32_t* free_slots);

/* ---- distributed slice, halo pack / unpack -------------------------------- */

/* distribute_csr (src/dist_spmv.hpp:27-100; build_ghost_map
 * src/halo_exchange.hpp:38-130; build_send_indices :154-191) for rank `rank`
 * of `size`: even block-row split, local CSR with columns remapped to
 * [0, local_n + n_ghost), ghost lists per owner rank (ascending ids, offsets
 * in owner-rank order) and send index lists.  Host work plus one upload. */
int nm_dist_create(const int32_t* row_ptr, const int32_t* col_idx, const double* values,
                   int32_t global_nrows, int32_t global_ncols, int32_t rank, int32_t size,
                   nm_dist** out);
int nm_dist_destroy(nm_dist* D);

/* Host only (needs no GPU): the same partition and halo plan as
 * nm_dist_create without any device upload.  Such a handle answers the
 * info / plan / local_host queries; compute entry points reject it. */
int nm_dist_plan(const int32_t* row_ptr, const int32_t* col_idx, const double* values,
                 int32_t global_nrows, int32_t global_ncols, int32_t rank, int32_t size,
                 nm_dist** out);

/* Host copy of the remapped local CSR (row_ptr local_n+1, col_idx/values
 * local_nnz); pass NULL arrays to query *local_nnz first. */
int nm_dist_local_host(const nm_dist* D, int32_t* local_nnz, int32_t* row_ptr,
                       int32_t* col_idx, double* values);

/* DistCrsMatrix properties (src/bindings.cpp:90-94) plus the halo sizes. */
int nm_dist_info(const nm_dist* D, int32_t* global_nrows, int32_t* row_start,
                 int32_t* row_end, int32_t* n_ghost, int32_t* total_send,
                 int32_t* n_send_nbrs, int32_t* n_recv_nbrs);

/* Host copies of the exchange plan: per neighbour its rank, count and offset
 * (send: offset into the packed send buffer; recv: offset of its ghosts in
 * x_ghost), and the flat lists (send: LOCAL indices packed in neighbour
 * order; recv: GLOBAL ghost ids in ghost order).  Arrays sized from
 * nm_dist_info. */
int nm_dist_send_plan(const nm_dist* D, int32_t* nbr_rank, int32_t* count, int32_t* offset,
                      int32_t* send_idx);
int nm_dist_recv_plan(const nm_dist* D, int32_t* nbr_rank, int32_t* count, int32_t* offset,
                      int32_t* ghost_ids);

/* The local matrix (columns in [0, local_n + n_ghost)); owned by D. */
int nm_dist_local(const nm_dist* D, const nm_csr** local);

/* halo_pack (src/halo_exchange.hpp:228-233): send_buf[i] = x_local[send_idx[i]]. */
int nm_halo_pack(const nm_dist* D, const double* x_local, double* send_buf, void* stream);

/* halo_scatter (src/halo_exchange.hpp:289-298) for all neighbours at once:
 * x_ext[local_n + off_r + i] = recv_buf[off_r + i], with recv_buf holding the
 * neighbours' values back to back in ghost order. */
int nm_halo_unpack(const nm_dist* D, const double* recv_buf, double* x_ext, void* stream);

/* distributed_spmv local part (src/dist_spmv.hpp:118-163): y_local = A_local *
 * x_ext, x_ext = [x_local | x_ghost].  With no ghosts x_ext may be x_local. */
int nm_dist_spmv_local(const nm_dist* D, const double* x_ext, double* y_local, void* stream);

/* The same product in two parts, so that the halo exchange can overlap the
 * first (addition: the reference describes this overlap as future work,
 * src/halo_exchange.hpp:28-33).  nm_dist_spmv_interior writes the rows whose
 * columns are all owned, reading x_local only (no ghost needed, so it may run
 * while the halo is in flight); nm_dist_spmv_boundary writes the other rows,
 * reading x_ext = [x_local | x_ghost] after the unpack.  Together they write
 * every row of y_local once, each row by the row-block kernel (rows of <= 32
 * nonzeros summed serially in CSR order).  nm_dist_row_split reports the
 * two row counts (also for host-only plans). */
int nm_dist_spmv_interior(const nm_dist* D, const double* x_local, double* y_local,
                          void* stream);
int nm_dist_spmv_boundary(const nm_dist* D, const double* x_ext, double* y_local, void* stream);
int nm_dist_row_split(const nm_dist* D, int32_t* n_interior, int32_t* n_boundary);

/* cg_solve_distributed (src/cg_solver.hpp:38-125) at one rank (no ghosts):
 * CG of nm_cg_local plus the reference's breakdown guard |p.Ap| < 1e-300,
 * reported as NM_ERR_RUNTIME "CG: p'Ap is near zero - A may not be SPD". */
int nm_dist_cg_single(nm_dist* D, const double* b, double* x, double tol, int32_t max_iter,
                      nm_cg_result* result, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* NUM_B200_H */
