/*
 * oracle.c -- CPU restatement of the reference sparse hot path (w-jiwonchoi/num,
 * module `kokkos_spmv`).  TEST INFRASTRUCTURE ONLY: the parity tests, the smoke
 * check and the bench's CPU-baseline / reference arm use it as the checker or as
 * the timed CPU stand-in for the reference's Kokkos-OpenMP build (which cannot be
 * built here: Kokkos, KokkosKernels, MPI and nanobind are absent).  The product
 * (num_b200) never links, loads or calls this file.
 *
 * Parity pins: see tests/test_oracle_golden.py -- every known answer held by the
 * reference's own tests (tests/test_spmv_kernel.cpp, tests/test_cg.cpp) and
 * SciPy fixtures made from the reference's python/matrix_generators.py.
 *
 * Build: oracle/Makefile  (gcc -O3 -fopenmp -ffp-contract=off -shared).
 * -ffp-contract=off keeps `acc += v * x` as a rounded product followed by a
 * rounded sum, which is the serial order of the reference's flat functor.
 * Where the reference's CUDA build would contract an expression into an FMA
 * (vec_ops.hpp axpy / axpy2 under nvcc's default -fmad=true) the oracle calls
 * fma() explicitly, with the operand placement written at each site, so the
 * device kernels can be compared bit for bit on those ops.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* CSR SpMV, serial row order.                                               */
/* Follows SpMVFunctorFlat::operator() (src/spmv_kernel.hpp:90-97) and the   */
/* host dense_spmv helper (tests/test_spmv_kernel.cpp:44-56):                */
/*   acc = 0; for j in [rowptr[i], rowptr[i+1]): acc += values[j]*x[colind[j]] */
/* ------------------------------------------------------------------------ */
void or_spmv_f64(int nrows, const int32_t *rowptr, const int32_t *colind,
                 const double *vals, const double *x, double *y)
{
    for (int i = 0; i < nrows; ++i) {
        double acc = 0.0;
        for (int32_t j = rowptr[i]; j < rowptr[i + 1]; ++j)
            acc += vals[j] * x[colind[j]];
        y[i] = acc;
    }
}

/* Same loop, rows split statically over OpenMP threads (the Kokkos OpenMP
 * RangePolicy mapping); each row keeps the serial order, so the result is
 * bit-identical to or_spmv_f64.  Used as the timed CPU baseline. */
void or_spmv_f64_omp(int nrows, const int32_t *rowptr, const int32_t *colind,
                     const double *vals, const double *x, double *y)
{
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nrows; ++i) {
        double acc = 0.0;
        for (int32_t j = rowptr[i]; j < rowptr[i + 1]; ++j)
            acc += vals[j] * x[colind[j]];
        y[i] = acc;
    }
}

/* FP32 values, FP32 x/y, FP32 accumulation (the precision the FP32 device
 * kernel computes in).  Serial order. */
void or_spmv_f32(int nrows, const int32_t *rowptr, const int32_t *colind,
                 const float *vals, const float *x, float *y)
{
    for (int i = 0; i < nrows; ++i) {
        float acc = 0.0f;
        for (int32_t j = rowptr[i]; j < rowptr[i + 1]; ++j)
            acc += vals[j] * x[colind[j]];
        y[i] = acc;
    }
}

void or_spmv_f32_omp(int nrows, const int32_t *rowptr, const int32_t *colind,
                     const float *vals, const float *x, float *y)
{
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nrows; ++i) {
        float acc = 0.0f;
        for (int32_t j = rowptr[i]; j < rowptr[i + 1]; ++j)
            acc += vals[j] * x[colind[j]];
        y[i] = acc;
    }
}

int or_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void or_set_num_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ------------------------------------------------------------------------ */
/* Multi-RHS SpMV  Y(N,k) = A * X(ncols,k), both row-major (LayoutRight).     */
/* Follows BatchSpMVFunctorMDRange::operator() (src/batch_spmv_kernel.hpp:    */
/* 95-102): one serial accumulation per (row i, column b).                   */
/* ------------------------------------------------------------------------ */
void or_batch_spmv_f64(int nrows, int k, const int32_t *rowptr,
                       const int32_t *colind, const double *vals,
                       const double *X, double *Y)
{
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nrows; ++i) {
        for (int b = 0; b < k; ++b) {
            double acc = 0.0;
            for (int32_t j = rowptr[i]; j < rowptr[i + 1]; ++j)
                acc += vals[j] * X[(int64_t)colind[j] * k + b];
            Y[(int64_t)i * k + b] = acc;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Vector ops (src/vec_ops.hpp).                                             */
/* ------------------------------------------------------------------------ */

/* vec_axpy (src/vec_ops.hpp:16-26): z = alpha*x + y, as fma(alpha, x, y). */
void or_axpy(int n, double alpha, const double *x, const double *y, double *z)
{
    for (int i = 0; i < n; ++i) z[i] = fma(alpha, x[i], y[i]);
}

/* vec_axpy2 (src/vec_ops.hpp:31-42): z = alpha*x + beta*y, evaluated as
 * fma(beta, y, alpha*x).  CG calls it as (1, r, beta, p, p), which makes it
 * the single-rounding p = fma(beta, p, r). */
void or_axpy2(int n, double alpha, const double *x, double beta,
              const double *y, double *z)
{
    for (int i = 0; i < n; ++i) z[i] = fma(beta, y[i], alpha * x[i]);
}

/* vec_local_dot (src/vec_ops.hpp:47-59), serial order. */
double or_dot(int n, const double *x, const double *y)
{
    double acc = 0.0;
    for (int i = 0; i < n; ++i) acc += x[i] * y[i];
    return acc;
}

/* vec_local_norm2 (src/vec_ops.hpp:64-69). */
double or_norm2(int n, const double *x) { return sqrt(or_dot(n, x, x)); }

/* vec_scale (src/vec_ops.hpp:94-100). */
void or_scale(int n, double alpha, double *x)
{
    for (int i = 0; i < n; ++i) x[i] *= alpha;
}

/* ------------------------------------------------------------------------ */
/* cg_solve_local (src/cg_solver.hpp:133-196), unpreconditioned CG with the  */
/* recursive residual, strict `<` stopping test on sqrt(r.r)/||b||,          */
/* ||b|| == 0 -> 1, and iters = iter + 1 on convergence.                     */
/* ------------------------------------------------------------------------ */
typedef struct {
    int    iters;
    double final_res;
    int    converged;
} or_cg_result;

void or_cg_local(int n, const int32_t *rowptr, const int32_t *colind,
                 const double *vals, const double *b, double *x, double tol,
                 int max_iter, or_cg_result *res)
{
    double *r  = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    double *p  = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    double *Ap = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));

    or_spmv_f64(n, rowptr, colind, vals, x, Ap);      /* Ap = A*x0      :144-146 */
    or_axpy(n, -1.0, Ap, b, r);                       /* r = -Ap + b    :147-148 */
    memcpy(p, r, sizeof(double) * (size_t)n);         /* p = r          :150     */

    double b_norm2 = or_norm2(n, b);                  /* :152-153 */
    if (b_norm2 == 0.0) b_norm2 = 1.0;
    double r_dot = or_dot(n, r, r);                   /* :155-156 */

    if (sqrt(r_dot) / b_norm2 < tol) {                /* :158-159 */
        res->iters = 0;
        res->final_res = sqrt(r_dot) / b_norm2;
        res->converged = 1;
        goto done;
    }

    for (int iter = 0; iter < max_iter; ++iter) {     /* :161-192 */
        or_spmv_f64(n, rowptr, colind, vals, p, Ap);
        double pAp = or_dot(n, p, Ap);
        double alpha = r_dot / pAp;
        or_axpy(n, alpha, p, x, x);                   /* x = alpha*p + x   */
        or_axpy(n, -alpha, Ap, r, r);                 /* r = -alpha*Ap + r */
        double r_dot_new = or_dot(n, r, r);
        double rel_res = sqrt(r_dot_new) / b_norm2;
        if (rel_res < tol) {
            res->iters = iter + 1;
            res->final_res = rel_res;
            res->converged = 1;
            goto done;
        }
        double beta = r_dot_new / r_dot;
        r_dot = r_dot_new;
        or_axpy2(n, 1.0, r, beta, p, p);              /* p = r + beta*p    */
    }
    /* :194-195 */
    res->iters = max_iter;
    res->final_res = sqrt(or_dot(n, r, r)) / b_norm2;
    res->converged = 0;
done:
    free(r);
    free(p);
    free(Ap);
}

/* ------------------------------------------------------------------------ */
/* Jacobi-preconditioned CG in FP64.  No counterpart in the reference (it    */
/* has no preconditioner); restated from the textbook PCG recurrence        */
/* (Saad, Iterative Methods for Sparse Linear Systems, 2nd ed., Alg. 9.1)    */
/* with the reference's stopping rule: strict `<` on sqrt(r.r)/||b||.        */
/*   z = D^-1 r, rz = r.z, p = z;                                            */
/*   alpha = rz / p.Ap; x += alpha p; r -= alpha Ap; test; z = D^-1 r;       */
/*   rz' = r.z; beta = rz'/rz; p = z + beta p.                               */
/* The diagonal inverse is applied as a product with dinv[i] = 1/a_ii.       */
/* ------------------------------------------------------------------------ */
void or_jacobi_dinv(int n, const int32_t *rowptr, const int32_t *colind,
                    const double *vals, double *dinv)
{
    for (int i = 0; i < n; ++i) {
        double d = 0.0;
        for (int32_t j = rowptr[i]; j < rowptr[i + 1]; ++j)
            if (colind[j] == i) d += vals[j];
        dinv[i] = (d != 0.0) ? 1.0 / d : 1.0;
    }
}

void or_pcg_jacobi(int n, const int32_t *rowptr, const int32_t *colind,
                   const double *vals, const double *b, double *x, double tol,
                   int max_iter, or_cg_result *res)
{
    size_t sz = sizeof(double) * (size_t)(n > 0 ? n : 1);
    double *r = (double *)malloc(sz), *p = (double *)malloc(sz);
    double *Ap = (double *)malloc(sz), *z = (double *)malloc(sz);
    double *dinv = (double *)malloc(sz);
    or_jacobi_dinv(n, rowptr, colind, vals, dinv);

    or_spmv_f64(n, rowptr, colind, vals, x, Ap);
    or_axpy(n, -1.0, Ap, b, r);
    for (int i = 0; i < n; ++i) z[i] = dinv[i] * r[i];
    memcpy(p, z, sz);
    double b_norm2 = or_norm2(n, b);
    if (b_norm2 == 0.0) b_norm2 = 1.0;
    double rr = or_dot(n, r, r);
    double rz = or_dot(n, r, z);
    if (sqrt(rr) / b_norm2 < tol) {
        res->iters = 0; res->final_res = sqrt(rr) / b_norm2; res->converged = 1;
        goto done;
    }
    for (int iter = 0; iter < max_iter; ++iter) {
        or_spmv_f64(n, rowptr, colind, vals, p, Ap);
        double pAp = or_dot(n, p, Ap);
        double alpha = rz / pAp;
        or_axpy(n, alpha, p, x, x);
        or_axpy(n, -alpha, Ap, r, r);
        rr = or_dot(n, r, r);
        double rel = sqrt(rr) / b_norm2;
        if (rel < tol) {
            res->iters = iter + 1; res->final_res = rel; res->converged = 1;
            goto done;
        }
        for (int i = 0; i < n; ++i) z[i] = dinv[i] * r[i];
        double rz_new = or_dot(n, r, z);
        double beta = rz_new / rz;
        rz = rz_new;
        or_axpy2(n, 1.0, z, beta, p, p);
    }
    res->iters = max_iter;
    res->final_res = sqrt(or_dot(n, r, r)) / b_norm2;
    res->converged = 0;
done:
    free(r); free(p); free(Ap); free(z); free(dinv);
}

/* ------------------------------------------------------------------------ */
/* Threaded CG for the timed CPU baseline only (never a parity reference):   */
/* the same recurrences as or_cg_local (precond = 0) and or_pcg_jacobi       */
/* (precond = 1), with every SpMV and vector loop an OpenMP static parallel  */
/* for, as the reference's Kokkos-OpenMP RangePolicy kernels run on the      */
/* host (src/spmv_kernel.hpp:170-180, src/vec_ops.hpp:16-69); the dot        */
/* products reduce in OpenMP's order.                                        */
/* ------------------------------------------------------------------------ */
static double omp_dot(int n, const double *x, const double *y)
{
    double acc = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : acc)
    for (int i = 0; i < n; ++i) acc += x[i] * y[i];
    return acc;
}

void or_cg_omp(int n, const int32_t *rowptr, const int32_t *colind, const double *vals,
               const double *b, double *x, double tol, int max_iter, int precond,
               or_cg_result *res)
{
    size_t sz = sizeof(double) * (size_t)(n > 0 ? n : 1);
    double *r = (double *)malloc(sz), *p = (double *)malloc(sz);
    double *Ap = (double *)malloc(sz), *z = (double *)malloc(sz);
    double *dinv = (double *)malloc(sz);
    if (precond) or_jacobi_dinv(n, rowptr, colind, vals, dinv);
    or_spmv_f64_omp(n, rowptr, colind, vals, x, Ap);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        r[i] = b[i] - Ap[i];
        z[i] = precond ? dinv[i] * r[i] : r[i];
        p[i] = z[i];
    }
    double b_norm2 = sqrt(omp_dot(n, b, b));
    if (b_norm2 == 0.0) b_norm2 = 1.0;
    double rr = omp_dot(n, r, r);
    double rz = precond ? omp_dot(n, r, z) : rr;
    if (sqrt(rr) / b_norm2 < tol) {
        res->iters = 0; res->final_res = sqrt(rr) / b_norm2; res->converged = 1;
        goto done;
    }
    for (int iter = 0; iter < max_iter; ++iter) {
        or_spmv_f64_omp(n, rowptr, colind, vals, p, Ap);
        double alpha = rz / omp_dot(n, p, Ap);
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) {
            x[i] = fma(alpha, p[i], x[i]);
            r[i] = fma(-alpha, Ap[i], r[i]);
        }
        rr = omp_dot(n, r, r);
        double rel = sqrt(rr) / b_norm2;
        if (rel < tol) {
            res->iters = iter + 1; res->final_res = rel; res->converged = 1;
            goto done;
        }
        double rz_new = rr;
        if (precond) {
#pragma omp parallel for schedule(static)
            for (int i = 0; i < n; ++i) z[i] = dinv[i] * r[i];
            rz_new = omp_dot(n, r, z);
        }
        double beta = rz_new / rz;
        rz = rz_new;
        const double *zz = precond ? z : r;
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) p[i] = fma(beta, p[i], zz[i]);
    }
    res->iters = max_iter;
    res->final_res = sqrt(omp_dot(n, r, r)) / b_norm2;
    res->converged = 0;
done:
    free(r); free(p); free(Ap); free(z); free(dinv);
}

/* ------------------------------------------------------------------------ */
/* Row-block partition ("binning") of the device SpMV.  No counterpart in    */
/* the reference (its only dispatch input is the global average, see         */
/* pick_rows_per_team, src/spmv_kernel.hpp:102-109).  This is the CPU        */
/* restatement of the device library's rule, checked bit-exact against it:   */
/*   - a row with more than `tile` nonzeros is a block of its own            */
/*     (block-per-row);                                                      */
/*   - otherwise consecutive rows are packed greedily into a block while the */
/*     block holds at most `max_rows` rows and at most `tile` nonzeros;      */
/*     inside such a block a row with <= short_max nonzeros is reduced by    */
/*     one thread, a longer one by one warp.                                 */
/* blk receives nblk+1 row boundaries (blk[0] = 0, blk[nblk] = nrows).       */
/* bins (optional, length nrows) receives 0 thread / 1 warp / 2 block.       */
/* Returns nblk, or -1 if cap is too small.                                  */
/* ------------------------------------------------------------------------ */
int or_row_blocks(int nrows, const int32_t *rowptr, int tile, int max_rows,
                  int short_max, int32_t *blk, int cap, int8_t *bins)
{
    int nb = 0;
    if (cap < 1) return -1;
    blk[0] = 0;
    int r = 0;
    while (r < nrows) {
        int len = rowptr[r + 1] - rowptr[r];
        if (len > tile) {
            if (bins) bins[r] = 2;
            ++r;
        } else {
            int start = r;
            int nz = 0;
            while (r < nrows && r - start < max_rows) {
                int l = rowptr[r + 1] - rowptr[r];
                if (nz + l > tile) break;
                if (bins) bins[r] = (int8_t)(l <= short_max ? 0 : 1);
                nz += l;
                ++r;
            }
        }
        if (nb + 1 >= cap) return -1;
        blk[++nb] = r;
    }
    return nb;
}

/* ------------------------------------------------------------------------ */
/* Halo pack / scatter kernels (src/halo_exchange.hpp:228-233, :289-298).    */
/* ------------------------------------------------------------------------ */
void or_halo_pack(int total_send, const int32_t *send_idx, const double *x_local,
                  double *send_buf)
{
    for (int i = 0; i < total_send; ++i) send_buf[i] = x_local[send_idx[i]];
}

void or_halo_scatter(int count, int offset, const double *rbuf, double *x_ghost)
{
    for (int i = 0; i < count; ++i) x_ghost[offset + i] = rbuf[i];
}
