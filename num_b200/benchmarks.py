"""SpMV and CG benchmark harness with the interface of the reference's
python/benchmark_spmv.py and python/benchmark_cg.py, run on this library's
drop-in module with torch CUDA tensors where those scripts use cupy.

    python -m num_b200.benchmarks spmv --N 1000000 --batch 128
    python -m num_b200.benchmarks cg --matrix laplacian_3d --N 1000000
    torchrun --nproc-per-node 4 -m num_b200.benchmarks spmv --backend kokkos_dist

Same flags, printed table and CSV columns as the reference scripts:
  spmv  backend, N, nnz, elapsed_us, bw_GB_s, gflops (+ k for batch rows),
        bytes = 12 nnz + 8 k N + 8 N (benchmark_spmv.py:108-114), the median of
        --repeat timed calls after a warm-up (:90-102), timed with CUDA events;
  cg    N, nnz, backend, elapsed_s, iters, residual, converged, b = ones, one
        timed solve after a warm-up solve (benchmark_cg.py:152-184).
Backends: scipy (scipy_cpu / scipy_cg), kokkos (kokkos_kk_1gpu), kokkos_custom
(kokkos_custom_1gpu; the same B200 kernels), kokkos_dist (ranks of a
torch.distributed job), batch (kokkos_batch_k<k>).  jax, petsc and the
mpi4py launch are not installed here; their rows are reported as skipped.
Matrices: the reference registry's five (matrix_generators.py:234-260):
laplacian_2d, laplacian_3d, lattice_gauge, random_sparse and power_law, sized
from --N as it does (L = int(N**0.5) for the 2-D grids, round(N**(1/3)) for
the 3-D one, N rows for the others), with the same arrays
(num_b200.generators).
CSV files go to --out (default ./benchmark_results), named spmv_<time>.csv /
cg_<time>.csv like the reference's.
"""
from __future__ import annotations

import argparse
import csv
import sys
import time
from datetime import datetime
from pathlib import Path

import numpy as np

from .generators import MATRICES

SKIPPED_BACKENDS = {"jax": "jax is not installed", "petsc": "petsc4py is not installed"}


def get_matrix(name: str, N: int):
    """The reference registry's matrices and sizing (a host CSR)."""
    from . import generators as gen
    return gen.get_matrix(name, N)


def spmv_metrics(elapsed_s: float, N: int, nnz: int, k: int = 1) -> dict:
    """benchmark_spmv.py:108-114: bytes 12 nnz + 8 k N + 8 N, flops 2 nnz k."""
    mem_bytes = nnz * 12 + k * N * 8 + N * 8
    return {"elapsed_us": elapsed_s * 1e6, "bw_GB_s": mem_bytes / elapsed_s / 1e9,
            "gflops": 2 * nnz * k / elapsed_s / 1e9}


def measure_gpu(fn, warmup: int = 20, repeat: int = 100) -> float:
    """Median seconds of `repeat` calls of fn, each timed with CUDA events on
    the current stream after `warmup` untimed calls."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    times = []
    for _ in range(repeat):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        e1.synchronize()
        times.append(e0.elapsed_time(e1) * 1e-3)
    return float(np.median(times))


def measure_cpu(fn, warmup: int = 5, repeat: int = 100) -> float:
    for _ in range(warmup):
        fn()
    times = []
    for _ in range(repeat):
        t0 = time.perf_counter()
        fn()
        times.append(time.perf_counter() - t0)
    return float(np.median(times))


def _upload(kspmv, A):
    return kspmv.upload_csr(A.row_ptr, A.col_idx, A.values, A.nrows, A.ncols)


def _write_csv(out: Path, stem: str, rows: list[dict]) -> Path:
    out.mkdir(parents=True, exist_ok=True)
    path = out / f"{stem}_{datetime.now().strftime('%Y%m%d_%H%M%S')}.csv"
    keys, seen = [], set()
    for row in rows:
        for k in row:
            if k not in seen:
                keys.append(k)
                seen.add(k)
    with open(path, "w", newline="") as f:
        w = csv.DictWriter(f, fieldnames=keys, extrasaction="ignore")
        w.writeheader()
        w.writerows(rows)
    return path


def _gpu_ready():
    try:
        import torch
        return torch.cuda.is_available()
    except ImportError:  # pragma: no cover
        return False


_OWN_GROUP = []  # the process group this module created (destroyed by main)


def _init_ranks():
    """(rank, size, kspmv or None): the drop-in module on this rank's GPU
    (rank % GPUs, as the reference scripts assign devices)."""
    import os
    from datetime import timedelta
    rank, size = 0, 1
    if not _gpu_ready():
        return rank, size, None
    import torch
    if int(os.environ.get("WORLD_SIZE", "1")) > 1 and not torch.distributed.is_initialized():
        # a short timeout: a rank that stops answering ends the others' next
        # collective with an error instead of a long hang
        torch.distributed.init_process_group("nccl", timeout=timedelta(seconds=120))
        _OWN_GROUP.append(True)
    from . import kokkos_spmv as kspmv
    if torch.distributed.is_initialized():
        rank, size = torch.distributed.get_rank(), torch.distributed.get_world_size()
    kspmv.init(rank % torch.cuda.device_count())
    return rank, size, kspmv


# ---- SpMV --------------------------------------------------------------------------------

def run_spmv(argv=None) -> list[dict]:
    p = argparse.ArgumentParser(description="SpMV benchmark (reference interface)")
    p.add_argument("--N", type=int, default=100_000)
    p.add_argument("--matrix", default="laplacian_3d", choices=list(MATRICES))
    p.add_argument("--batch", type=int, default=0,
                   help="If > 0, also run batch SpMV with this many RHS vectors")
    p.add_argument("--repeat", type=int, default=100)
    p.add_argument("--backend", nargs="+",
                   default=["scipy", "jax", "kokkos", "kokkos_custom", "kokkos_dist"])
    p.add_argument("--no-csv", action="store_true")
    p.add_argument("--out", default="benchmark_results")
    args = p.parse_args(argv)

    rank, size, kspmv = _init_ranks()
    A = get_matrix(args.matrix, args.N)
    N, nnz = A.nrows, A.nnz
    x = np.random.default_rng(42).standard_normal(A.ncols)
    rows: list[dict] = []
    if rank == 0:
        print(f"\nSpMV Benchmark — {args.matrix}  N={N:,}  nnz={nnz:,}  nnz/row={nnz / N:.1f}")
        print("-" * 78)
        print(f"{'Backend':<32} {'Time(μs)':>10} {'BW(GB/s)':>10} {'GFLOPS':>8}")
        print("-" * 78)

    def report(tag, m):
        if not m or rank != 0:
            return
        print(f"  {tag:<30} {m['elapsed_us']:>10.1f} {m['bw_GB_s']:>10.2f} {m['gflops']:>8.2f}")
        rows.append({"backend": tag, "N": N, "nnz": nnz, **m})

    def skip(tag, why):
        if rank == 0:
            print(f"  [SKIP] {tag}: {why}", file=sys.stderr)

    if "scipy" in args.backend and rank == 0:
        S = A.to_scipy()
        report("scipy_cpu", spmv_metrics(measure_cpu(lambda: S @ x, 5, args.repeat), N, nnz))
    for b, why in SKIPPED_BACKENDS.items():
        if b in args.backend:
            skip(f"{b}_1gpu", why)
    gpu_wanted = {"kokkos", "kokkos_custom", "kokkos_dist"} & set(args.backend) or args.batch > 0
    if gpu_wanted and kspmv is None:
        skip("kokkos_*", "no CUDA device")
    if kspmv is not None and rank == 0:
        import torch
        dev = torch.device("cuda", torch.cuda.current_device())
        for b, tag, kk in (("kokkos", "kokkos_kk_1gpu", True),
                           ("kokkos_custom", "kokkos_custom_1gpu", False)):
            if b in args.backend:
                M = _upload(kspmv, A)
                xt = torch.tensor(x, device=dev)
                yt = torch.zeros(N, dtype=torch.float64, device=dev)
                t = measure_gpu(lambda: kspmv.spmv(M, xt, yt, kokkoskernels=kk), 20, args.repeat)
                report(tag, spmv_metrics(t, N, nnz))
    if "kokkos_dist" in args.backend and size > 1 and kspmv is not None:
        import torch
        Ad = kspmv.distribute_csr(A.row_ptr, A.col_idx, A.values, A.nrows, A.ncols)
        n_loc = Ad.local_row_end - Ad.local_row_start
        xl = torch.ones(n_loc, dtype=torch.float64, device="cuda")
        yl = torch.zeros(n_loc, dtype=torch.float64, device="cuda")
        for _ in range(5):
            kspmv.dist_spmv(Ad, xl, yl)
        torch.cuda.synchronize()
        torch.distributed.barrier()
        reps = min(args.repeat, 50)
        t0 = time.perf_counter()
        for _ in range(reps):
            kspmv.dist_spmv(Ad, xl, yl)
        torch.cuda.synchronize()
        torch.distributed.barrier()
        m = spmv_metrics((time.perf_counter() - t0) / reps, N, nnz)
        report(f"kokkos_dist_{size}gpu", {**m, "n_ranks": size})
    if args.batch > 0 and rank == 0:
        k = args.batch
        print(f"\n  --- Batch SpMV (k={k}) ---")
        if "jax" in args.backend:
            skip(f"jax_vmap_k{k}", SKIPPED_BACKENDS["jax"])
        if kspmv is not None:
            import torch
            M = _upload(kspmv, A)
            g = torch.Generator(device="cuda").manual_seed(0)
            X = torch.randn(A.ncols, k, dtype=torch.float64, device="cuda", generator=g)
            Y = torch.zeros(N, k, dtype=torch.float64, device="cuda")
            t = measure_gpu(lambda: kspmv.batch_spmv(M, X, Y), 20, args.repeat)
            report(f"kokkos_batch_k{k}", {**spmv_metrics(t, N, nnz, k=k), "k": k})
    if not args.no_csv and rank == 0 and rows:
        print(f"\n  Results saved to {_write_csv(Path(args.out), 'spmv', rows)}")
    return rows


# ---- CG ----------------------------------------------------------------------------------

def run_cg(argv=None) -> list[dict]:
    p = argparse.ArgumentParser(description="CG benchmark (reference interface)")
    p.add_argument("--N", type=int, default=100_000)
    p.add_argument("--matrix", default="laplacian_3d", choices=list(MATRICES))
    p.add_argument("--tol", type=float, default=1e-8)
    p.add_argument("--maxiter", type=int, default=2000)
    p.add_argument("--no-csv", action="store_true")
    p.add_argument("--no-petsc", action="store_true")
    p.add_argument("--backend", nargs="+", default=["scipy", "kokkos", "kokkos_dist"])
    p.add_argument("--out", default="benchmark_results")
    args = p.parse_args(argv)

    rank, size, kspmv = _init_ranks()
    A = get_matrix(args.matrix, args.N)
    N, nnz = A.nrows, A.nnz
    b = np.ones(N, dtype=np.float64)
    rows: list[dict] = []
    if rank == 0:
        print(f"\nCG Benchmark — {args.matrix}  N={N:,}  nnz={nnz:,}  tol={args.tol:.0e}  np={size}")
        if not args.no_petsc:
            print("  (petsc_cg skipped — petsc4py not installed)")
        print("-" * 78)
        print(f"  {'Backend':<30} {'Time(s)':>9} {'Iters':>7} {'Residual':>12} Converged")
        print("-" * 78)

    def report(m):
        if not m or rank != 0:
            return
        conv = "YES" if m.get("converged") else "NO "
        print(f"  {m['backend']:<30} {m['elapsed_s']:>9.3f} {m.get('iters', '-'):>7} "
              f"{m.get('residual', float('nan')):>12.3e} {conv}")
        rows.append({"N": N, "nnz": nnz, **m})

    if "scipy" in args.backend and rank == 0:
        import scipy.sparse.linalg as spla
        S = A.to_scipy()
        its = [0]

        def cb(_):
            its[0] += 1
        t0 = time.perf_counter()
        xs, info = spla.cg(S, b, rtol=args.tol, maxiter=args.maxiter, callback=cb)
        el = time.perf_counter() - t0
        report({"backend": "scipy_cg", "elapsed_s": el, "iters": its[0],
                "residual": float(np.linalg.norm(b - S @ xs) / np.linalg.norm(b)),
                "converged": info == 0})
    if kspmv is not None and "kokkos" in args.backend and rank == 0:
        import torch
        M = _upload(kspmv, A)
        bt = torch.tensor(b, device="cuda")

        def solve():
            xt = torch.zeros(N, dtype=torch.float64, device="cuda")
            return kspmv.cg_solve_local(M, bt, xt, tol=args.tol, max_iter=args.maxiter)
        solve()  # warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = solve()
        torch.cuda.synchronize()
        report({"backend": "kspmv_cg_1gpu", "elapsed_s": time.perf_counter() - t0,
                "iters": res["iters"], "residual": res["residual"],
                "converged": res["converged"]})
    if kspmv is not None and "kokkos_dist" in args.backend and size > 1:
        import torch
        Ad = kspmv.distribute_csr(A.row_ptr, A.col_idx, A.values, A.nrows, A.ncols)
        lo, hi = Ad.local_row_start, Ad.local_row_end
        bl = torch.tensor(b[lo:hi], device="cuda")

        def dsolve():
            xl = torch.zeros(hi - lo, dtype=torch.float64, device="cuda")
            return kspmv.cg_solve(Ad, bl, xl, tol=args.tol, max_iter=args.maxiter)
        dsolve()
        torch.cuda.synchronize()
        torch.distributed.barrier()
        t0 = time.perf_counter()
        res = dsolve()
        torch.cuda.synchronize()
        torch.distributed.barrier()
        report({"backend": f"kspmv_cg_{size}gpu", "elapsed_s": time.perf_counter() - t0,
                "iters": res["iters"], "residual": res["residual"],
                "converged": res["converged"]})
    if not args.no_csv and rank == 0 and rows:
        print(f"\n  Results saved to {_write_csv(Path(args.out), 'cg', rows)}")
    return rows


def main(argv=None) -> int:
    argv = list(sys.argv[1:] if argv is None else argv)
    if not argv or argv[0] not in ("spmv", "cg"):
        print("usage: python -m num_b200.benchmarks {spmv,cg} [options]", file=sys.stderr)
        return 2
    try:
        (run_spmv if argv[0] == "spmv" else run_cg)(argv[1:])
    finally:
        if _OWN_GROUP:
            import torch
            torch.distributed.destroy_process_group()
            _OWN_GROUP.clear()
    return 0


if __name__ == "__main__":
    sys.exit(main())
