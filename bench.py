#!/usr/bin/env python
"""Benchmark of the sparse hot path on B200.

Default workload (one step = one FP64 CSR SpMV, y = A x):
  3-D 7-point Laplacian on a 160^3 grid: n = 4,096,000, nnz = 28,518,400,
  int32 indices, FP64 values, x ~ U[-1, 1] (default_rng(1)).
  Algorithmic bytes per SpMV = 12 nnz + 4 (n + 1) + 8 n (x) + 8 n (y)
  = 424.14 MB, larger than the 126 MB L2, so no flush is needed between steps.
  The default line also carries a `secondary` object: plain FP64 CG solves/s
  on the 256^2 Laplacian, the 160^3 matrix setup time (host build + upload
  against on-device assembly) and a served-CG sample (see serve_c5).

Other workloads (--workload):
  spmv_c2a_fp32, spmv_c2b[_fp32], spmv_c1     one SpMV per step
  spmv_c3[_fp32]    4,096 banded SPD matrices (n log-uniform in [32, 4096],
                    seed 2) multiplied in one launch per step
  batch_c2_k128     one multi-RHS SpMV Y = A X per step (100^3 Laplacian,
                    128 right-hand sides), the drop-in batch_spmv
  cg_c1             one plain FP64 CG solve per step (256^2 Laplacian,
                    b = A 1, x0 = 0, tol 1e-8), the drop-in cg_solve_local
  cg_c4_fp64 / cg_c4_fp32 / cg_c4_bf16
                    one Jacobi-PCG solve per step of the 128^3 variable-
                    coefficient Poisson system (seed 3) to 1e-10 through the
                    batched engine: FP64, or FP32 / BF16 values with FP64
                    iterative refinement
  serve_c5          one pass of a served request stream per step (Poisson
                    arrivals, seed 4; Laplacians and banded SPD systems),
                    FP32 inner + FP64 refinement, tol 1e-8, continuous
                    batching; compared with the plain FP64 drop-in run one
                    request at a time

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME]
    python bench.py --impl reference ...   # the reference's CPU path (oracle port)

Multi-GPU (torchrun, one rank per GPU): every rank runs the same workload on
its own GPU (independent replicas, weak scaling, no data-path collective);
value = total work of all ranks / max-over-ranks time.
Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "CG solves/s + p99 latency at rel-res 1e-8 vs plain FP64 CG; SpMV HBM GB/s"

# name -> (description, kind, precision)
WORKLOADS = {
    "spmv_c2a": ("3-D 7-point Laplacian 160^3, FP64 CSR SpMV", "spmv", "fp64"),
    "spmv_c2a_fp32": ("3-D 7-point Laplacian 160^3, FP32 CSR SpMV", "spmv", "fp32"),
    "spmv_c2b": ("power-law rows n=2,000,000 mean 16 sigma 1.2, FP64 CSR SpMV", "spmv", "fp64"),
    "spmv_c2b_fp32": ("power-law rows n=2,000,000 mean 16 sigma 1.2, FP32 CSR SpMV", "spmv",
                      "fp32"),
    "spmv_c1": ("2-D 5-point Laplacian 256^2, FP64 CSR SpMV", "spmv", "fp64"),
    "spmv_c3": ("4,096 banded SPD matrices n log-U[32,4096] (seed 2), FP64 SpMV of all in one "
                "launch", "spmv", "fp64"),
    "spmv_c3_fp32": ("4,096 banded SPD matrices n log-U[32,4096] (seed 2), FP32 SpMV of all in "
                     "one launch", "spmv", "fp32"),
    "batch_c2_k128": ("3-D 7-point Laplacian 100^3, multi-RHS SpMV Y = A X with 128 columns, "
                      "FP64", "batch", "fp64"),
    "cg_c1": ("2-D 5-point Laplacian 256^2, plain FP64 CG, b = A*1, x0 = 0, tol 1e-8", "cg",
              "fp64"),
    "cg_1m": ("2-D 5-point Laplacian 1024^2 (1,048,576 rows: the CUDA-graph path), plain FP64 "
              "CG, b = A*1, x0 = 0, tol 1e-8", "cg", "fp64"),
    "vec_c2a": ("CG vector ops at 4,096,000 elements: axpy, axpy2 and dot per step", "vec",
                "fp64"),
    "halo_c2a": ("halo pack + unpack of the 160^3 Laplacian split into 8 row slabs (8 virtual "
                 "ranks on one GPU)", "halo", "fp64"),
    "cg_c4_fp64": ("3-D variable-coefficient Poisson 128^3 (seed 3), Jacobi PCG FP64 to 1e-10",
                   "engine", "fp64"),
    "cg_c4_fp32": ("3-D variable-coefficient Poisson 128^3 (seed 3), Jacobi PCG FP32 + FP64 "
                   "iterative refinement to 1e-10", "engine", "fp32"),
    "cg_c4_bf16": ("3-D variable-coefficient Poisson 128^3 (seed 3), Jacobi PCG BF16 values + "
                   "FP64 iterative refinement to 1e-10", "engine", "bf16"),
    "serve_c5": ("served CG stream (seed 4): 50/50 2-D Laplacian side log-U[32,1024] or banded "
                 "SPD n log-U[256,65536], b ~ N(0,1), Jacobi PCG to 1e-8, FP32 inner + FP64 "
                 "refinement, continuous batching", "serve", "fp32"),
}


def spmv_stream_ms(kspmv, M, xh, xd0, yd0, dt, stream, steps, dev):
    """Device ms per step of a stream of SpMVs through the public API, each
    step copying its x in from pinned host memory and its y out: copy-in,
    SpMV and copy-out on separate streams with two device and host buffers,
    ordered by events."""
    import torch
    xd = [xd0, torch.empty_like(xd0)]
    yd = [yd0, torch.empty_like(yd0)]
    yh = [torch.empty(yd0.shape[0], dtype=dt).pin_memory() for _ in range(2)]
    s_in, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    ev = lambda: torch.cuda.Event()  # noqa: E731
    x_ready, y_ready, y_out = [ev(), ev()], [ev(), ev()], [ev(), ev()]

    def run(n):
        for i in range(n):
            b = i & 1
            with torch.cuda.stream(s_in):
                s_in.wait_event(y_ready[b])  # the SpMV that read xd[b] is done
                xd[b].copy_(xh, non_blocking=True)
                x_ready[b].record(s_in)
            stream.wait_event(x_ready[b])
            stream.wait_event(y_out[b])      # yd[b] of step i-2 is on the host
            with torch.cuda.stream(stream):
                kspmv.spmv(M, xd[b], yd[b], async_=True)
            y_ready[b].record(stream)
            with torch.cuda.stream(s_out):
                s_out.wait_event(y_ready[b])
                yh[b].copy_(yd[b], non_blocking=True)
                y_out[b].record(s_out)

    run(4)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s_in.wait_event(e0)
    s_out.wait_event(e0)
    run(steps)
    s_out.wait_event(y_ready[(steps - 1) & 1])
    e1.record(s_out)
    torch.cuda.synchronize(dev)
    return e0.elapsed_time(e1) / steps


def make_workload(name):
    from num_b200 import generators as gen
    if name.startswith("spmv_c2a"):
        A = gen.laplacian_3d(160)
        seed = 1
    elif name.startswith("spmv_c2b"):
        A = gen.power_law(2_000_000, seed=1001)
        seed = 1
    elif name in ("spmv_c1", "cg_c1"):
        A = gen.laplacian_2d(256)
        seed = 0
    elif name == "cg_1m":
        A = gen.laplacian_2d(1024)
        seed = 0
    elif name.startswith("spmv_c3"):
        mats, xs = gen.banded_batch(4096, seed=2)
        return mats, np.concatenate(xs)
    else:
        raise SystemExit(f"unknown workload {name}")
    x = np.random.default_rng(seed).uniform(-1.0, 1.0, A.ncols)
    return A, x


def block_diagonal(mats):
    """One host CSR holding the matrices on the diagonal (for byte counts and
    the CPU legs)."""
    from num_b200.generators import Csr
    rps, cis, vals = [np.zeros(1, np.int64)], [], []
    r = z = 0
    for A in mats:
        rps.append(A.row_ptr[1:].astype(np.int64) + z)
        cis.append(A.col_idx.astype(np.int64) + r)
        vals.append(A.values)
        r += A.nrows
        z += A.nnz
    return Csr(np.concatenate(rps).astype(np.int32), np.concatenate(cis).astype(np.int32),
               np.concatenate(vals), r, r)


def spmv_bytes(A, precision):
    from num_b200.generators import spmv_bytes as sb
    vb = {"fp64": 8, "fp32": 4, "bf16": 2}[precision]
    xb = 8 if precision == "fp64" else 4
    return sb(A.nnz, A.nrows, A.ncols, vb, xb)


def cg_iter_bytes(nnz, n, vb, tb):
    """Algorithmic bytes of one CG iteration as the library runs it (three
    kernels): SpMV with p.Ap (values + int32 columns + row_ptr, the gathered
    p once, Ap written), the x/r update with r.r (x, p, r, Ap read; x, r
    written) and the p update (r, p read; p written) -- 11 vector passes of
    tb bytes.  With a Jacobi preconditioner (the engine) the update also reads
    the inverse diagonal and the correction d and writes z: 13 passes."""
    return (vb + 4) * nnz + 4 * (n + 1) + 11 * tb * n


def engine_iter_bytes(nnz, n, vb, tb):
    """One inner iteration of the batched engine: SpMV with p.Ap (values +
    columns + row_ptr, p gathered once, Ap written); update (p, Ap, r, d,
    D^-1 read; d, r, z written); p update (z, p read; p written)."""
    return (vb + 4) * nnz + 4 * (n + 1) + 13 * tb * n


def engine_outer_bytes(nnz, n, tb):
    """One refinement step: x += s d (d, x read, x written: 16 + tb), the FP64
    residual SpMV (values, columns, row_ptr; x gathered, b read, r64 written:
    24), the inner start (r64, D^-1 read; r, z, d written: 8 + 4 tb) and
    p = z + g p (z, p read, p written: 3 tb)."""
    return 12 * nnz + 4 * (n + 1) + (48 + 8 * tb) * n


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs, burst copy)"
    return 6650.0, "fallback 6.65 TB/s"


def traffic_for(workload):
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        d = json.loads(p.read_text())
        v = d.get(workload)
        if isinstance(v, dict):
            return v.get("bytes_per_launch")
        return v
    return None


# ---- clocks during the timed region -------------------------------------------------

class ClockSampler:
    """Samples SM clock and clock-event reasons with NVML every ~10 ms."""

    REASONS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap",
               0x8: "hw_slowdown", 0x10: "sync_boost", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown",
               0x100: "display_clock_setting"}

    def __init__(self, device_index):
        self.samples = []
        self.max_mhz = None
        self._stop = threading.Event()
        self._h = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            h = None
            try:
                import torch
                pr = torch.cuda.get_device_properties(device_index)
                bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
                h = pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())
            except Exception:
                h = pynvml.nvmlDeviceGetHandleByIndex(0)
            self._h = h
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self._h = None

    def _run(self):
        nv = self.nv
        while not self._stop.is_set():
            try:
                mhz = nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM)
                try:
                    rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                except AttributeError:
                    rs = nv.nvmlDeviceGetCurrentClocksThrottleReasons(self._h)
                util = nv.nvmlDeviceGetUtilizationRates(self._h).gpu
                self.samples.append((mhz, rs, util))
            except Exception:
                pass
            time.sleep(0.01)

    def __enter__(self):
        if self._h is not None:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        if self._h is not None:
            self._stop.set()
            self._t.join()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": [], "samples": 0}
        mhz = [s[0] for s in self.samples]
        bits = 0
        for s in self.samples:
            bits |= int(s[1])
        reasons = [n for b, n in self.REASONS.items() if bits & b and n != "gpu_idle"]
        return {"sm_mhz": statistics.median(mhz), "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(self.samples)}


def dtype_name(precision):
    return {"fp64": "f64", "fp32": "f32", "bf16": "bf16/f32"}[precision]


def max_over_ranks(values, world, dev):
    if world == 1:
        return [float(v) for v in values]
    import torch
    import torch.distributed as dist
    t = torch.tensor(values, dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def base_line(args, world, value, unit, ms_per_step, precision, config, higher=True):
    return {
        "metric": METRIC, "value": value, "unit": unit, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_per_step, 6), "higher_is_better": higher,
        "scaling": "weak", "vs_baseline": None, "dtype": dtype_name(precision),
        "data": "synthetic", "config": config,
    }


# ---- our arm: SpMV ---------------------------------------------------------------------

def spmv_config(desc, name, A, precision):
    """The SpMV workload's config keys, the same in both arms."""
    return {"workload": desc, "name": name, "nrows": A.nrows, "nnz": A.nnz,
            "index": "int32", "values": precision, "bytes_per_step": spmv_bytes(A, precision),
            "bytes_formula": "(value bytes + 4)*nnz + 4*(n+1) + x bytes*ncols + y bytes*nrows"}


def sustained(step, stream, dev, min_ms=400.0):
    """Back-to-back steps for at least min_ms of device time, timed as one
    event pair: keeps the GPU under load long enough for the clock sampler to
    take ~20+ samples around the timed region, and reports the sustained rate
    beside the per-step events."""
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(10):
        step()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    est = max(e0.elapsed_time(e1) / 10, 1e-3)
    n = int(min(200000, max(10, min_ms / est)))
    e0.record(stream)
    for _ in range(n):
        step()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    return n, e0.elapsed_time(e1)


def run_spmv(args, rank, world, local_rank):
    import torch

    from num_b200 import _lib
    from num_b200 import kokkos_spmv as kspmv

    dev = torch.device("cuda", local_rank)
    desc, _, precision = WORKLOADS[args.workload]
    A, x = make_workload(args.workload)
    if isinstance(A, list):  # many matrices, one launch
        mats = A
        M = kspmv.upload_csr_batched([m.astuple() for m in mats], precision=precision)
        A = block_diagonal(mats)
        batch = {"matrices": len(mats), "api": "upload_csr_batched"}
    else:
        M = kspmv.upload_csr(A.row_ptr, A.col_idx, A.values, A.nrows, A.ncols,
                             precision=precision)
        batch = None
    if args.tile or args.short_max or args.stages or args.grid_mult >= 0:
        tuned = kspmv.tune(M, tile=args.tile, short_max=args.short_max, stages=args.stages,
                           grid_mult=args.grid_mult)
        tuned["chosen_by"] = "command line"
    else:
        # the project's autotuner picks the partition and launch shape
        at = kspmv.autotune(M, budget_ms=200, cache=False)
        tuned = {k: at[k] for k in ("tile", "max_rows", "short_max", "grid_mult", "stages",
                                    "kernel")}
        tuned["chosen_by"] = f"autotune ({len(at['trials'])} candidates timed)"
        best = {}
        for tr in at["trials"]:
            best[tr["kernel"]] = min(best.get(tr["kernel"], float("inf")), tr["us"])
        tuned["best_us_by_kernel"] = best
    dt = torch.float64 if precision == "fp64" else torch.float32
    xd = torch.tensor(x, dtype=dt, device=dev)
    yd = torch.empty(A.nrows, dtype=dt, device=dev)
    lib = _lib.load()
    stream = torch.cuda.current_stream(dev)
    s = stream.cuda_stream
    nbytes = spmv_bytes(A, precision)

    def step():
        st = lib.nm_spmv(M._h, xd.data_ptr(), yd.data_ptr(), s)
        if st:
            _lib.check(st, "nm_spmv")

    # Operands smaller than L2: flush it between steps (a 256 MB write, outside
    # the per-step events) and time the steps alone.
    flush = torch.empty(64 << 20, dtype=torch.float32, device=dev) if nbytes < 126e6 else None
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    barrier(world)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        sus_n, sus_ms = sustained(step, stream, dev)
        torch.cuda.synchronize(dev)
        t0.record(stream)
        for k in range(args.steps):
            if flush is not None:
                flush.zero_()
            ev[k][0].record(stream)
            step()
            ev[k][1].record(stream)
        t1.record(stream)
        torch.cuda.synchronize(dev)
    barrier(world)
    total_ms = t0.elapsed_time(t1)
    kern_ms = [a.elapsed_time(b) for a, b in ev]
    if flush is not None:
        total_ms = sum(kern_ms)
    kern_avg_ms = sum(kern_ms) / len(kern_ms)
    total_ms, kern_avg_ms = max_over_ranks([total_ms, kern_avg_ms], world, dev)
    ms_per_step = total_ms / args.steps

    # e2e through the public API with host buffers: spmv_host (C ABI
    # nm_spmv_host) copies pinned x in, multiplies and copies y out, the row
    # blocks in chunks so that the copy-out runs beside the copy-in; and, for
    # comparison, the same copies made by the caller around the device-buffer
    # spmv, one after the other.
    e2e_steps = max(3, min(args.steps, 50))
    xh = torch.tensor(x, dtype=dt).pin_memory()
    yh = torch.empty(A.nrows, dtype=dt).pin_memory()

    def timed_e2e(one):
        for _ in range(2):
            one()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(e2e_steps):
            one()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return max_over_ranks([e0.elapsed_time(e1) / e2e_steps], world, dev)[0]

    def around_spmv():
        xd.copy_(xh, non_blocking=True)
        kspmv.spmv(M, xd, yd)
        yh.copy_(yd, non_blocking=True)
        stream.synchronize()

    sep_ms = timed_e2e(around_spmv)
    y_dev = yh.clone()
    yh.fill_(float("nan"))
    e2e_ms = timed_e2e(lambda: kspmv.spmv_host(M, xh, yh))
    if not torch.equal(yh, y_dev):
        raise RuntimeError("spmv_host result differs from the device-buffer spmv")
    pipe_ms = max_over_ranks([spmv_stream_ms(kspmv, M, xh, xd, yd, dt, stream, e2e_steps, dev)],
                             world, dev)[0]

    if rank != 0:
        return None
    peak, peak_src = measured_peak()
    achieved = nbytes / (kern_avg_ms * 1e-3) / 1e9
    config = spmv_config(desc, args.workload, A, precision)
    config.update({
        "l2": ("inputs larger than L2 (no flush): %.1f MB per step > 126 MB" % (nbytes / 1e6)
               if flush is None else "inputs smaller than L2 (%.1f MB): L2 flushed (256 MB "
               "write) between steps, steps timed alone" % (nbytes / 1e6)),
        "parallelism": f"replicas x{world}", "tuning": tuned,
    })
    if batch:
        config["batch"] = batch
    line = base_line(args, world, round(world * nbytes / (ms_per_step * 1e-3) / 1e9, 2), "GB/s",
                     ms_per_step, precision, config)
    line.update({
        "roofline": {
            "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_source": peak_src,
            "frac_of_8TBs_spec": round(achieved / 8000.0, 4),
            "traffic": traffic_for(args.workload),
            "kernel": ("nm::spmv_gather_kernel (warp per 32 rows, x gathered through L2)"
                       if kspmv.spmv_kernel(M) == "gather"
                       else "nm::spmv_kernel (row-block CSR SpMV)"),
            "kernel_avg_us": round(kern_avg_ms * 1e3, 3),
        },
        "e2e": {
            "value": round(nbytes / (e2e_ms * 1e-3) / 1e9, 2), "unit": "GB/s",
            "h2d_bytes_per_step": int(xh.numel() * xh.element_size()),
            "d2h_bytes_per_step": int(yh.numel() * yh.element_size()),
            "ms_per_step": round(e2e_ms, 4), "steps": e2e_steps,
            "api": "num_b200.kokkos_spmv.spmv_host (C ABI nm_spmv_host) on pinned host x/y",
            "mode": "synchronous per call, like the reference's spmv (fence before return); "
                    "x in as pieces, row blocks in chunks, each chunk's y out while later "
                    "chunks compute; y checked equal to the device-buffer spmv's",
        },
        "e2e_copies_around_spmv": {
            "value": round(nbytes / (sep_ms * 1e-3) / 1e9, 2), "unit": "GB/s",
            "ms_per_step": round(sep_ms, 4), "steps": e2e_steps,
            "api": "pinned x copied in, kokkos_spmv.spmv (C ABI nm_spmv), y copied out, "
                   "one after the other",
        },
        "e2e_pipelined": {
            "value": round(nbytes / (pipe_ms * 1e-3) / 1e9, 2), "unit": "GB/s",
            "ms_per_step": round(pipe_ms, 4), "steps": e2e_steps,
            "mode": "a stream of SpMVs: every step still copies its x in and its y out "
                    "(same bytes); copy-in, SpMV and copy-out on three CUDA streams with "
                    "double buffers, so one step's copy-out overlaps the next one's copy-in",
            "api": "kokkos_spmv.spmv(..., async_=True)",
        },
        "gpu_launches": args.steps,
        "clocks": clk.summary(),
        "sustained": {"steps": sus_n, "ms": round(sus_ms, 3),
                      "value": round(world * nbytes * sus_n / (sus_ms * 1e-3) / 1e9, 2),
                      "unit": "GB/s",
                      "note": "back-to-back steps (no L2 flush) right before the timed region, "
                              "inside the clock sampler's window"},
        "reference_metric_gbs": round(
            (12 * A.nnz + 16 * A.nrows) / (kern_avg_ms * 1e-3) / 1e9, 1)
        if precision == "fp64" else None,
    })
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_spmv(A, x, precision, budget_s=args.cpu_seconds)
    if world == 1 and args.workload == "spmv_c2a" and not args.no_secondary:
        line["secondary"] = secondary(local_rank)
    return line


# ---- our arm: multi-RHS SpMV (the drop-in batch_spmv) -----------------------------------

def batch_bytes(A, k):
    """12 nnz + 4 (n+1) for the matrix, X read once (k doubles per column
    index), Y written once (k doubles per row)."""
    return 12 * A.nnz + 4 * (A.nrows + 1) + 8 * k * (A.ncols + A.nrows)


def run_batch(args, rank, world, local_rank):
    import torch

    from num_b200 import _lib
    from num_b200 import generators as gen
    from num_b200 import kokkos_spmv as kspmv
    dev = torch.device("cuda", local_rank)
    desc, _, precision = WORKLOADS[args.workload]
    k = 128
    A = gen.laplacian_3d(100)
    M = kspmv.upload_csr(A.row_ptr, A.col_idx, A.values, A.nrows, A.ncols)
    g = torch.Generator(device=dev).manual_seed(1)
    X = torch.rand((A.ncols, k), dtype=torch.float64, device=dev, generator=g) * 2 - 1
    Y = torch.empty((A.nrows, k), dtype=torch.float64, device=dev)
    lib = _lib.load()
    stream = torch.cuda.current_stream(dev)
    s = stream.cuda_stream
    nbytes = batch_bytes(A, k)

    def step():
        st = lib.nm_batch_spmv(M._h, X.data_ptr(), Y.data_ptr(), k, s)
        if st:
            _lib.check(st, "nm_batch_spmv")

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    barrier(world)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        sus_n, sus_ms = sustained(step, stream, dev)
        t0.record(stream)
        for i in range(args.steps):
            ev[i][0].record(stream)
            step()
            ev[i][1].record(stream)
        t1.record(stream)
        torch.cuda.synchronize(dev)
    barrier(world)
    total_ms = t0.elapsed_time(t1)
    kern_avg_ms = sum(a.elapsed_time(b) for a, b in ev) / args.steps
    total_ms, kern_avg_ms = max_over_ranks([total_ms, kern_avg_ms], world, dev)
    ms_per_step = total_ms / args.steps
    # e2e: pinned X in, Y out, through kokkos_spmv.batch_spmv
    Xh = X.cpu().pin_memory()
    Yh = torch.empty_like(Y, device="cpu").pin_memory()
    e_steps = 5
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e_steps):
        X.copy_(Xh, non_blocking=True)
        kspmv.batch_spmv(M, X, Y)
        Yh.copy_(Y, non_blocking=True)
        stream.synchronize()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    e_ms = max_over_ranks([e0.elapsed_time(e1) / e_steps], world, dev)[0]
    lib_ref = cusparse_spmm_reference(A, X, dev, stream)
    if rank != 0:
        return None
    peak, peak_src = measured_peak()
    achieved = nbytes / (kern_avg_ms * 1e-3) / 1e9
    if "us" in lib_ref:
        lib_ref["gbs"] = round(nbytes / (lib_ref["us"] * 1e-6) / 1e9, 1)
        lib_ref["library_us_over_ours"] = round(lib_ref["us"] / (kern_avg_ms * 1e3), 3)
    config = {"workload": desc, "name": args.workload, "nrows": A.nrows, "nnz": A.nnz, "k": k,
              "bytes_per_step": nbytes,
              "bytes_formula": "12*nnz + 4*(n+1) + 8*k*(ncols + nrows)",
              "l2": "inputs larger than L2 (%.0f MB per step)" % (nbytes / 1e6),
              "parallelism": f"replicas x{world}",
              "api": "kokkos_spmv.batch_spmv (C ABI nm_batch_spmv), X and Y row-major"}
    line = base_line(args, world, round(world * nbytes / (ms_per_step * 1e-3) / 1e9, 2),
                     "GB/s", ms_per_step, precision, config)
    line.update({
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                     "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_source": peak_src,
                     "traffic": None, "kernel": "nm::batch_spmv_kernel",
                     "kernel_avg_us": round(kern_avg_ms * 1e3, 3),
                     "reference_formula_gbs": round(
                         (12 * A.nnz + 8 * k * A.nrows + 8 * A.nrows) / (kern_avg_ms * 1e-3) / 1e9, 1)},
        "e2e": {"value": round(nbytes / (e_ms * 1e-3) / 1e9, 2), "unit": "GB/s",
                "h2d_bytes_per_step": int(Xh.numel() * 8), "d2h_bytes_per_step": int(Yh.numel() * 8),
                "ms_per_step": round(e_ms, 3),
                "api": "kokkos_spmv.batch_spmv with pinned X / Y copies"},
        "gpu_launches": args.steps,
        "clocks": clk.summary(),
        "sustained": {"steps": sus_n, "ms": round(sus_ms, 3),
                      "value": round(world * nbytes * sus_n / (sus_ms * 1e-3) / 1e9, 2),
                      "unit": "GB/s",
                      "note": "back-to-back steps right before the timed region, inside the "
                              "clock sampler's window"},
        "library_reference": lib_ref,
    })
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_batch(A, k, budget_s=args.cpu_seconds)
    return line


def cusparse_spmm_reference(A, X, dev, stream, steps=20):
    """The library the reference's batch_spmv calls for k >= 32 (cuSPARSE
    SpMM through KokkosKernels, src/batch_spmv_kernel.hpp:157-170), timed on
    the same matrix and X: torch's CSR @ dense product, which runs cuSPARSE
    SpMM.  Reported beside our kernel; not used on our path."""
    import torch
    try:
        S = torch.sparse_csr_tensor(torch.tensor(A.row_ptr.astype(np.int64), device=dev),
                                    torch.tensor(A.col_idx.astype(np.int64), device=dev),
                                    torch.tensor(A.values, device=dev),
                                    size=(A.nrows, A.ncols))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            for _ in range(3):
                Y = S @ X
            e0.record(stream)
            for _ in range(steps):
                Y = S @ X
            e1.record(stream)
        torch.cuda.synchronize(dev)
        return {"us": round(e0.elapsed_time(e1) * 1e3 / steps, 2),
                "what": "cuSPARSE SpMM via torch.sparse_csr_tensor @ dense (the library "
                        "KokkosKernels calls for k >= 32), same matrix and X",
                "output_contiguous": bool(Y.is_contiguous())}
    except Exception as e:  # the comparison is optional
        return {"unavailable": f"{type(e).__name__}: {e}"}


def cpu_baseline_batch(A, k, budget_s=10.0):
    from oracle import oracle
    L = oracle.lib()
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    X = np.random.default_rng(1).uniform(-1, 1, (A.ncols, k))
    Y = np.empty((A.nrows, k))
    rp, ci, v = (np.ascontiguousarray(a) for a in (A.row_ptr, A.col_idx, A.values))
    run = lambda: L.or_batch_spmv_f64(A.nrows, k, rp.ctypes.data, ci.ctypes.data,
                                      v.ctypes.data, X.ctypes.data, Y.ctypes.data)
    run()
    times = []
    t_end = time.perf_counter() + budget_s
    while time.perf_counter() < t_end and len(times) < 100:
        t = time.perf_counter()
        run()
        times.append(time.perf_counter() - t)
    med = statistics.median(times)
    return {"value": round(batch_bytes(A, k) / med / 1e9, 3), "unit": "GB/s", "cores": threads,
            "kind": "port",
            "sample": f"full product, {len(times)} runs, median {med * 1e3:.1f} ms; "
                      "oracle/oracle.c or_batch_spmv_f64 (OpenMP rows, serial per (row, column))"}


# ---- our arm: plain CG (the drop-in cg_solve_local) ------------------------------------

def cg_c1_measure(dev, steps, warmup, with_clock=True, local_rank=0, name="cg_c1"):
    """Device-timed plain FP64 CG solves (b = A 1 resident, x zeroed on the
    device each step) and the same through the public API with host copies."""
    import torch

    from num_b200 import kokkos_spmv as kspmv
    A, _ = make_workload(name)
    M = kspmv.upload_csr(A.row_ptr, A.col_idx, A.values, A.nrows, A.ncols)
    bh = A.to_scipy() @ np.ones(A.ncols)
    b = torch.tensor(bh, device=dev)
    x = torch.zeros(A.nrows, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    for _ in range(warmup):
        x.zero_()
        info = kspmv.cg_solve_local(M, b, x, tol=1e-8, max_iter=5000)
    torch.cuda.synchronize(dev)
    # the operands (11.5 MB) fit L2: flush it before every solve (outside the
    # per-solve events)
    flush = torch.empty(64 << 20, dtype=torch.float32, device=dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    iters = 0
    clk = ClockSampler(local_rank) if with_clock else None
    if clk:
        clk.__enter__()
        # back-to-back solves for ~0.4 s before the timed ones: the sampler
        # sees the GPU under this load for 20+ samples
        t_end = time.perf_counter() + 0.4
        while time.perf_counter() < t_end:
            x.zero_()
            kspmv.cg_solve_local(M, b, x, tol=1e-8, max_iter=5000)
    for k in range(steps):
        x.zero_()
        flush.zero_()
        ev[k][0].record(stream)
        info = kspmv.cg_solve_local(M, b, x, tol=1e-8, max_iter=5000)
        ev[k][1].record(stream)
        iters += info["iters"]
    torch.cuda.synchronize(dev)
    if clk:
        clk.__exit__()
    ms = sum(a.elapsed_time(c) for a, c in ev)
    xs = x.cpu().numpy()
    err = float(np.abs(xs - 1.0).max())
    # e2e: pinned b in, x out, every solve
    bp = torch.tensor(bh).pin_memory()
    xp = torch.empty(A.nrows, dtype=torch.float64).pin_memory()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_steps = max(3, min(steps, 20))
    e0.record(stream)
    for _ in range(e_steps):
        b.copy_(bp, non_blocking=True)
        x.zero_()
        kspmv.cg_solve_local(M, b, x, tol=1e-8, max_iter=5000)
        xp.copy_(x, non_blocking=True)
        stream.synchronize()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    e_ms = e0.elapsed_time(e1) / e_steps
    from num_b200 import _lib
    path = C.c_int32(-1)
    _lib.load().nm_cg_last_path(M._h, C.byref(path))
    return {"A": A, "ms": ms, "iters": iters, "info": info, "max_err_vs_ones": err,
            "e2e_ms": e_ms, "h2d": bp.numel() * 8, "d2h": xp.numel() * 8,
            "clocks": clk.summary() if clk else None, "path": CG_PATHS.get(path.value),
            "path_id": path.value}


CG_PATHS = {0: "CUDA-graph chunks of 2 kernels per iteration (the p update formed in the "
               "SpMV)",
            1: "persistent TMA-pipelined solve, 3 grid barriers per iteration",
            2: "persistent TMA-pipelined solve, 2 grid barriers per iteration",
            3: "resident solve (matrix rows and vectors on chip, 2 grid-wide sums per "
               "iteration)",
            4: "cluster solve (one 16-CTA thread-block cluster: the rows of A in shared "
               "memory, each CTA's halo of the direction kept current over distributed "
               "shared memory, 2 hardware cluster barriers per iteration)"}


def run_cg(args, rank, world, local_rank):
    import torch
    dev = torch.device("cuda", local_rank)
    desc, _, precision = WORKLOADS[args.workload]
    barrier(world)
    r = cg_c1_measure(dev, args.steps, args.warmup, local_rank=local_rank, name=args.workload)
    barrier(world)
    ms, e2e_ms = max_over_ranks([r["ms"], r["e2e_ms"]], world, dev)
    if rank != 0:
        return None
    A = r["A"]
    it_per_solve = r["iters"] / args.steps
    per_it = cg_iter_bytes(A.nnz, A.nrows, 8, 8)
    peak, peak_src = measured_peak()
    achieved = per_it * r["iters"] / (r["ms"] * 1e-3) / 1e9
    ms_per = ms / args.steps
    config = {"workload": desc, "name": args.workload, "nrows": A.nrows, "nnz": A.nnz,
              "tol": 1e-8, "iters_per_solve": it_per_solve,
              "final_residual": r["info"]["residual"], "max_abs_err_vs_ones": r["max_err_vs_ones"],
              "l2": "operands fit L2 (%.1f MB): L2 flushed before every solve, solves timed "
                    "alone; within a solve the iterations run from L2" % (per_it / 1e6),
              "parallelism": f"replicas x{world}",
              "api": "kokkos_spmv.cg_solve_local (C ABI nm_cg_local)",
              "path": r["path"], "cg_mode": args.cg_mode}
    line = base_line(args, world, round(world * 1e3 / ms_per, 3), "solves/s", ms_per, precision,
                     config)
    line.update({
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_source": peak_src,
                     "traffic": None, "kernel": "whole CG iteration (SpMV+p.Ap, x/r update, "
                     "p update)", "bytes_per_iteration": per_it,
                     "us_per_iteration": round(r["ms"] * 1e3 / r["iters"], 3)},
        "e2e": {"value": round(1e3 / e2e_ms, 3), "unit": "solves/s",
                "h2d_bytes_per_step": r["h2d"], "d2h_bytes_per_step": r["d2h"],
                "ms_per_step": round(e2e_ms, 4),
                "api": "kokkos_spmv.cg_solve_local with pinned b copied in and x copied out"},
        # per solve: A x0, the initial kernel, then one persistent launch, or
        # two kernels per iteration on the CUDA-graph path
        "gpu_launches": int(3 * args.steps if r["path_id"] in (1, 2, 3, 4)
                            else r["iters"] * 2 + 2 * args.steps),
        "clocks": r["clocks"],
    })
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_cg(A, A.to_scipy() @ np.ones(A.ncols), 1e-8,
                                               budget_s=args.cpu_seconds, precond=False)
    return line


# ---- our arm: the batched engine on one large system (C4) --------------------------------

def run_engine(args, rank, world, local_rank):
    import torch

    from num_b200 import generators as gen
    from num_b200.solver import BatchSolver
    dev = torch.device("cuda", local_rank)
    desc, _, precision = WORKLOADS[args.workload]
    A, b = gen.varcoef_poisson_3d(128, seed=3)
    S = BatchSolver(A.nrows + 4096, A.nnz + 4096, 4, precision=precision)
    slot = S.admit(A, b, tol=1e-10, max_iter=20000)
    ext = torch.cuda.ExternalStream(S.stream(), device=dev)
    chunk = 64

    def solve_once():
        S.resolve(slot)
        while slot in S.active:
            S.step(chunk)

    while slot in S.active:  # the first solve (admission was outside)
        S.step(chunk)
    for _ in range(max(0, args.warmup - 1)):
        solve_once()
    torch.cuda.synchronize(dev)
    barrier(world)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        # back-to-back solves for ~0.4 s before the timed ones: the sampler
        # sees the GPU under this load for 20+ samples
        t_end = time.perf_counter() + 0.4
        while time.perf_counter() < t_end:
            solve_once()
        torch.cuda.synchronize(dev)
        c0 = S.counters()
        t0.record(ext)
        for _ in range(args.steps):
            solve_once()
        t1.record(ext)
        torch.cuda.synchronize(dev)
    c1 = S.counters()
    ms = t0.elapsed_time(t1)
    st = S.status(slot)
    x, _ = S.take(slot)
    true_res = float(np.linalg.norm(b - A.to_scipy() @ x) / np.linalg.norm(b))
    # e2e: the whole public-API solve per step (admission from host arrays,
    # steps, x copied back, slot freed)
    e_steps = max(1, min(args.steps, 3))
    e0 = time.perf_counter()
    for _ in range(e_steps):
        (xe, ie), = S.solve([(A, b)], tol=1e-10, max_iter=20000, chunk=chunk)
    e_ms = (time.perf_counter() - e0) * 1e3 / e_steps
    err_fp64 = None
    if precision != "fp64":
        # untimed: the same system by the FP64 engine, the reference solution
        # the mixed-precision result is compared with
        R = BatchSolver(A.nrows + 4096, A.nnz + 4096, 4, precision="fp64")
        (x64, _), = R.solve([(A, b)], tol=1e-10, max_iter=20000, chunk=chunk)
        err_fp64 = float(np.linalg.norm(x - x64) / np.linalg.norm(x64))
        del R
    barrier(world)
    ms, e_ms = max_over_ranks([ms, e_ms], world, dev)
    if rank != 0:
        return None
    vb = {"fp64": 8, "fp32": 4, "bf16": 2}[precision]
    tb = 8 if precision == "fp64" else 4
    its = (c1["inner_iterations"] - c0["inner_iterations"]) / args.steps  # enqueued
    outer = st["outer"]
    per_solve = st["iters"] * engine_iter_bytes(A.nnz, A.nrows, vb, tb) + \
        outer * engine_outer_bytes(A.nnz, A.nrows, tb)
    peak, peak_src = measured_peak()
    dev_s = (c1["s_device"] - c0["s_device"]) / args.steps
    ms_per = ms / args.steps
    achieved = per_solve / dev_s / 1e9 if dev_s > 0 else None
    config = {"workload": desc, "name": args.workload, "nrows": A.nrows, "nnz": A.nnz,
              "tol": 1e-10, "inner_iterations": st["iters"], "outer_steps": outer,
              "iterations_enqueued_per_solve": its, "residual": st["residual"],
              "true_residual_fp64": true_res, "converged": st["converged"],
              "rel_error_vs_fp64_solution": err_fp64,
              "chunk": chunk, "engine_mode": args.engine_mode,
              "parallelism": f"replicas x{world}",
              "api": "num_b200.solver.BatchSolver (C ABI nm_solver_*): admit once, "
                     "nm_solver_resolve + steps per solve",
              "l2": "inputs larger than L2 (%.0f MB of matrix values + indices)" %
                    ((vb + 4) * A.nnz / 1e6)}
    line = base_line(args, world, round(world * 1e3 / ms_per, 4), "solves/s", ms_per, precision,
                     config)
    line.update({
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1) if achieved else None,
                     "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4) if achieved else None,
                     "peak_source": peak_src, "traffic": None,
                     "kernel": "whole engine iteration (SpMV+p.Ap, update, p update) + "
                               "refinement steps, device time of the steps",
                     "bytes_per_solve": per_solve},
        "e2e": {"value": round(1e3 / e_ms, 4), "unit": "solves/s",
                "h2d_bytes_per_step": int(A.nnz * (12 + vb) + A.nrows * 16),
                "d2h_bytes_per_step": int(A.nrows * 8), "ms_per_step": round(e_ms, 3),
                "api": "BatchSolver.solve: admission from host arrays, steps, take"},
        # per inner iteration of the one large system: SpMV, alpha, update, p
        # update; one control kernel per 8-iteration body; the refinement steps
        "gpu_launches": int((c1["inner_iterations"] - c0["inner_iterations"]) * 4 +
                            (c1["inner_iterations"] - c0["inner_iterations"]) // 8 +
                            (c1["outer_launches"] - c0["outer_launches"]) * 6),
        "clocks": clk.summary(),
    })
    if world == 1 and not args.no_cpu_baseline:
        # the CPU solves in FP64: scale to the FP64 Jacobi-PCG iteration count
        # of this system (692, equal to the FP64 engine's)
        got = {}
        line["cpu_baseline"] = cpu_baseline_cg(A, b, 1e-10, budget_s=args.cpu_seconds,
                                               precond=True, full_iters=692, out=got)
        # the engine's solution against the oracle's FP64 Jacobi-PCG one (an
        # untimed full solve when the timing above scaled a partial one)
        xo = got.get("x")
        if xo is None:
            from oracle import oracle
            _, xo = oracle.cg_omp(A.row_ptr, A.col_idx, A.values, b, tol=1e-10, max_iter=20000,
                                  precond=True)
        line["config"]["rel_error_vs_oracle_solution"] = float(
            np.linalg.norm(x - xo) / np.linalg.norm(xo))
    return line


# ---- our arm: served request stream (C5) -----------------------------------------------

def served_bytes(requests, rec, precision):
    """Algorithmic bytes of the engine iterations a served pass ran: per
    request its inner iterations times engine_iter_bytes and its refinement
    steps times engine_outer_bytes."""
    vb = {"fp64": 8, "fp32": 4, "bf16": 2}[precision]
    tb = 8 if precision == "fp64" else 4
    tot = 0
    for (_, A, _, _), r in zip(requests, rec):
        tot += r["iters"] * engine_iter_bytes(A.nnz, A.nrows, vb, tb)
        tot += r.get("outer", 0) * engine_outer_bytes(A.nnz, A.nrows, tb)
    return tot


def serve_measure(dev, requests, runs, warmup, arena_bytes, with_plain=True, local_rank=0,
                  precision="fp32", precond="jacobi", check_limit=None, plain_passes=2):
    """Served runs of the stream on one solver, and the plain drop-in.

    Streams longer than check_limit requests (None: no limit) check the true
    FP64 residual, and compare with the plain drop-in's solution, on their
    first check_limit requests only, and warm up on those too (all arriving
    at once) instead of on whole passes."""
    import torch

    from num_b200 import serve
    from num_b200.solver import BatchSolver, arena_for
    rows, nnz = arena_for(arena_bytes, nnz_per_row=5.0, precision=precision)
    S = BatchSolver(rows, nnz, 1024, precision=precision, precond=precond)
    ext = torch.cuda.ExternalStream(S.stream(), device=dev)
    head = requests if check_limit is None or len(requests) <= check_limit else \
        [(0.0, A, b, k) for (_, A, b, k) in requests[:check_limit]]
    errs = []
    sols = {}

    def check_fn(i, x, info):
        _, A, b, _ = head[i]
        errs.append(float(np.linalg.norm(b - A.to_scipy() @ x) / np.linalg.norm(b)))
        sols[i] = np.array(x, copy=True)

    # untimed: one pass that checks every result's true FP64 residual, and the
    # warm-up passes
    serve.serve(head, S, tol=1e-8, chunk=16, check=check_fn)
    for _ in range(max(0, warmup - 1)):
        serve.serve(head, S, tol=1e-8, chunk=16)
    stats, recs = [], []
    c0 = S.counters()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clk = ClockSampler(local_rank)
    with clk:
        t0.record(ext)
        for k in range(runs):
            st, rec = serve.serve(requests, S, tol=1e-8, chunk=16)
            stats.append(st)
            recs.append(rec)
        t1.record(ext)
        torch.cuda.synchronize(dev)
    c1 = S.counters()
    alg = sum(served_bytes(requests, rec, precision) for rec in recs)
    out = {"ms": t0.elapsed_time(t1), "stats": stats, "ctr0": c0, "ctr1": c1,
           "algorithmic_bytes": alg, "max_true_residual": max(errs) if errs else None,
           "checked": len(head), "clocks": clk.summary()}
    del S
    if with_plain:
        # the plain drop-in's pass time varies with host work (uploads, frees):
        # compare against the better of the passes
        runs_p = [serve.serve_plain(requests, tol=1e-8)[0] for _ in range(plain_passes)]
        pst = max(runs_p, key=lambda r: r["solves_per_s"])
        pst["passes_solves_per_s"] = [round(r["solves_per_s"], 3) for r in runs_p]
        out["plain"] = pst
        # untimed: the served results of the checked requests against the
        # plain FP64 drop-in's solutions of the same requests
        rel = []

        def cmp_fn(i, x, info):
            if i in sols:
                rel.append(float(np.linalg.norm(sols[i] - x) / max(np.linalg.norm(x), 1e-300)))
        serve.serve_plain(head, tol=1e-8, check=cmp_fn)
        out["max_rel_error_vs_fp64"] = max(rel) if rel else None
    return out


def run_serve(args, rank, world, local_rank):
    import torch

    from num_b200 import serve
    dev = torch.device("cuda", local_rank)
    desc, _, _ = WORKLOADS[args.workload]
    precision = args.serve_precision
    requests = serve.make_requests(args.requests, rate=args.rate, seed=4, pool=args.pool)
    big = len(requests) > 1000
    barrier(world)
    r = serve_measure(dev, requests, args.steps, args.warmup, args.arena_gb * 1e9,
                      local_rank=local_rank, precision=precision, precond=args.serve_precond,
                      check_limit=300 if big else None, plain_passes=1 if big else 2,
                      with_plain=not args.no_plain)
    barrier(world)
    ms = max_over_ranks([r["ms"]], world, dev)[0]
    if rank != 0:
        return None
    n = len(requests)
    ms_per = ms / args.steps
    solves_s = n / (ms_per * 1e-3)
    c0, c1 = r["ctr0"], r["ctr1"]
    p50 = statistics.median(s["p50_ms"] for s in r["stats"])
    p99 = statistics.median(s["p99_ms"] for s in r["stats"])
    tot_rows = sum(q[1].nrows for q in requests)
    tot_nnz = sum(q[1].nnz for q in requests)
    inner = {"fp32": "fp32 values + vectors, FP64 refinement",
             "bf16": "bf16 values, fp32 vectors, FP64 refinement",
             "fp64": "fp64 values + vectors, no refinement"}[precision]
    config = {"workload": desc, "name": args.workload, "requests": n,
              "arrival_rate_per_s": args.rate if args.rate > 0 else "all at t=0 (saturated)",
              "distinct_systems": min(n, args.pool) if args.pool else n,
              "rows_total": tot_rows, "nnz_total": tot_nnz, "tol": 1e-8,
              "arena_gb_cap": args.arena_gb, "inner": inner,
              "preconditioner": args.serve_precond,
              "max_true_residual_fp64": r["max_true_residual"],
              "checked_requests": r["checked"],
              "max_rel_error_vs_fp64_dropin": r.get("max_rel_error_vs_fp64"),
              "parallelism": f"replicas x{world}",
              "api": "num_b200.serve.serve over BatchSolver (nm_solver_* C ABI)"}
    if big:
        config["note"] = ("requests i >= pool reuse system i mod pool (an i.i.d. sample of "
                          "the distribution); every request has its own Poisson arrival; "
                          "residual / error checks and warm-up on the first 300 requests")
    line = base_line(args, world, round(world * solves_s, 3), "solves/s", ms_per, precision,
                     config)
    peak, peak_src = measured_peak()
    dev_s = (c1["s_device"] - c0["s_device"]) / args.steps
    achieved = r["algorithmic_bytes"] / args.steps / dev_s / 1e9 if dev_s > 0 else None
    line.update({
        "latency_ms": {"p50": round(p50, 3), "p99": round(p99, 3)},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1) if achieved else None,
                     "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4) if achieved else None,
                     "peak_source": peak_src, "traffic": None,
                     "kernel": "served engine steps: summed algorithmic bytes of every "
                               "request's inner iterations and refinement steps over the "
                               "steps' device time",
                     "device_busy_s_per_pass": round(dev_s, 4),
                     "device_busy_frac": round(dev_s / (ms_per * 1e-3), 4)},
        "e2e": {"value": round(world * solves_s, 3), "unit": "solves/s",
                "h2d_bytes_per_step": int(tot_nnz * 16 + tot_rows * 12),
                "d2h_bytes_per_step": int(tot_rows * 8),
                "note": "the served loop is end to end by construction: every request's "
                        "matrix and b come from host memory and x goes back"},
        # at least SpMV, update, p update per inner iteration (alpha too while
        # a large system is live), one control kernel per 8-iteration body,
        # the refinement steps
        "gpu_launches": int((c1["inner_iterations"] - c0["inner_iterations"]) * 3 +
                            (c1["inner_iterations"] - c0["inner_iterations"]) // 8 +
                            (c1["outer_launches"] - c0["outer_launches"]) * 6),
        "clocks": r["clocks"],
    })
    if "plain" in r:
        plain = r["plain"]
        line["plain_fp64_drop_in"] = {
            "solves_per_s": round(plain["solves_per_s"], 3), "p50_ms": round(plain["p50_ms"], 3),
            "p99_ms": round(plain["p99_ms"], 3), "passes": plain["passes_solves_per_s"],
            "note": "the better of the passes",
            "api": "kokkos_spmv.upload_csr + cg_solve_local, one request at a time in "
                   "arrival order"}
        line["ratio_vs_plain"] = round(solves_s / plain["solves_per_s"], 3)
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_serve(requests, budget_s=args.cpu_seconds)
    return line


def setup_c2a_measure(dev):
    """Setup of the 160^3 Laplacian handle, wall clock, the better of two runs:
    host generator + upload_csr (host arrays, validation, host-to-device copy,
    partition) against kokkos_spmv.laplacian (assembly on the device, row_ptr
    and columns read back for the partition)."""
    import torch

    from num_b200 import generators as gen
    from num_b200 import kokkos_spmv as k
    gen_s, up_s, dev_s = [], [], []
    for _ in range(2):
        t0 = time.perf_counter()
        A = gen.laplacian_3d(160)
        t1 = time.perf_counter()
        M = k.upload_csr(*A.astuple())
        torch.cuda.synchronize(dev)
        t2 = time.perf_counter()
        gen_s.append(t1 - t0)
        up_s.append(t2 - t1)
        del M, A
        t0 = time.perf_counter()
        M = k.laplacian(3, 160)
        torch.cuda.synchronize(dev)
        dev_s.append(time.perf_counter() - t0)
        del M
    host = min(g + u for g, u in zip(gen_s, up_s))
    return {"host_generate_s": round(min(gen_s), 4), "host_upload_s": round(min(up_s), 4),
            "device_laplacian_s": round(min(dev_s), 4), "speedup": round(host / min(dev_s), 2),
            "api": "generators.laplacian_3d + kokkos_spmv.upload_csr vs kokkos_spmv.laplacian"}


def secondary(local_rank):
    """Short CG and serving numbers for the default line."""
    import torch

    from num_b200 import serve
    dev = torch.device("cuda", local_rank)
    out = {}
    r = cg_c1_measure(dev, 20, 3, with_clock=False)
    out["cg_c1_plain_fp64"] = {"solves_per_s": round(20e3 / r["ms"], 2),
                               "us_per_iteration": round(r["ms"] * 1e3 / r["iters"], 3),
                               "iters": r["info"]["iters"], "residual": r["info"]["residual"],
                               "e2e_solves_per_s": round(1e3 / r["e2e_ms"], 2)}
    out["setup_c2a"] = setup_c2a_measure(dev)
    requests = serve.make_requests(200, rate=0.0, seed=4)
    # two timed passes on each side, the better one of each (host wall clock
    # of the pass, as serve / serve_plain report it)
    s = serve_measure(dev, requests, 2, 2, 64e9)
    st = max(s["stats"], key=lambda r: r["solves_per_s"])
    out["serve_c5_sample"] = {
        "requests": 200, "arrivals": "all at t=0 (saturated)",
        "served_fp32_ir_solves_per_s": round(st["solves_per_s"], 2),
        "served_passes": [round(r["solves_per_s"], 3) for r in s["stats"]],
        "p50_ms": round(st["p50_ms"], 2), "p99_ms": round(st["p99_ms"], 2),
        "plain_fp64_solves_per_s": round(s["plain"]["solves_per_s"], 2),
        "plain_passes": s["plain"]["passes_solves_per_s"],
        "plain_p50_ms": round(s["plain"]["p50_ms"], 2),
        "plain_p99_ms": round(s["plain"]["p99_ms"], 2),
        "ratio_vs_plain": round(st["solves_per_s"] / s["plain"]["solves_per_s"], 3),
        "comparison": "the better of two passes on each side",
        "max_true_residual_fp64": s["max_true_residual"],
        "max_rel_error_vs_fp64_dropin": s.get("max_rel_error_vs_fp64")}
    return out


# ---- CPU legs (oracle port of the reference's CPU path) --------------------------------------

def cpu_spmv_setup(A, x, precision):
    from oracle import oracle
    L = oracle.lib()
    rp = np.ascontiguousarray(A.row_ptr)
    ci = np.ascontiguousarray(A.col_idx)
    if precision == "fp64":
        v = np.ascontiguousarray(A.values)
        xx = np.ascontiguousarray(x, np.float64)
        y = np.empty(A.nrows)
        fn, es = L.or_spmv_f64_omp, 8
    else:
        v = np.ascontiguousarray(A.values, np.float32)
        xx = np.ascontiguousarray(x, np.float32)
        y = np.empty(A.nrows, np.float32)
        fn, es = L.or_spmv_f32_omp, 4
    keep = (rp, ci, v, xx, y)

    def run(r0, r1):
        fn(r1 - r0, rp.ctypes.data + 4 * r0, ci.ctypes.data, v.ctypes.data, xx.ctypes.data,
           y.ctypes.data + es * r0)
    return run, keep, oracle


def slice_bytes(A, r0, r1, precision):
    vb = 8 if precision == "fp64" else 4
    nz = int(A.row_ptr[r1] - A.row_ptr[r0])
    return (vb + 4) * nz + 4 * (r1 - r0 + 1) + vb * (r1 - r0) * 2


def cpu_baseline_spmv(A, x, precision, budget_s=10.0):
    run, keep, oracle = cpu_spmv_setup(A, x, precision)
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    run(0, A.nrows)
    times = []
    t_end = time.perf_counter() + budget_s
    while time.perf_counter() < t_end and len(times) < 1000:
        t = time.perf_counter()
        run(0, A.nrows)
        times.append(time.perf_counter() - t)
    med = statistics.median(times)
    nbytes = spmv_bytes(A, precision)
    return {"value": round(nbytes / med / 1e9, 3), "unit": "GB/s", "cores": threads,
            "kind": "port",
            "sample": f"full matrix, {len(times)} SpMVs in ~{budget_s:.0f} s, median "
                      f"{med * 1e3:.2f} ms; oracle/oracle.c or_spmv_*_omp (OpenMP static rows)"}


def cpu_baseline_cg(A, b, tol, budget_s=10.0, precond=False, full_iters=None, out=None):
    """Threaded CPU CG (oracle/oracle.c or_cg_omp).  When one solve would take
    longer than the budget, a capped number of iterations is timed and the
    solve time scaled to the full iteration count.  out (a dict): receives
    the last full solve's x under "x" when full solves were timed."""
    from oracle import oracle
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    t = time.perf_counter()
    info, _ = oracle.cg_omp(A.row_ptr, A.col_idx, A.values, b, tol=tol, max_iter=20,
                            precond=precond)
    t20 = (time.perf_counter() - t) / max(1, info["iters"])
    est_iters = full_iters or 1000
    if t20 * est_iters < budget_s / 3:
        times, iters = [], None
        t_end = time.perf_counter() + budget_s
        while time.perf_counter() < t_end and len(times) < 200:
            t = time.perf_counter()
            info, xo = oracle.cg_omp(A.row_ptr, A.col_idx, A.values, b, tol=tol,
                                     max_iter=20000, precond=precond)
            times.append(time.perf_counter() - t)
            iters = info["iters"]
            if out is not None:
                out["x"] = xo
        med = statistics.median(times)
        sample = (f"{len(times)} full solves ({iters} iterations each) in ~{budget_s:.0f} s, "
                  f"median {med * 1e3:.2f} ms")
    else:
        cap = max(5, int(budget_s / 2 / max(t20, 1e-9)))
        t = time.perf_counter()
        info, _ = oracle.cg_omp(A.row_ptr, A.col_idx, A.values, b, tol=1e-300, max_iter=cap,
                                precond=precond)
        per_it = (time.perf_counter() - t) / cap
        med = per_it * est_iters
        sample = (f"{cap} iterations timed ({per_it * 1e3:.2f} ms each), scaled to the "
                  f"{est_iters} iterations of the full solve")
    kind = "Jacobi PCG" if precond else "CG"
    return {"value": round(1.0 / med, 4), "unit": "solves/s", "cores": threads, "kind": "port",
            "sample": f"{sample}; oracle/oracle.c or_cg_omp ({kind}, OpenMP loops)"}


def cpu_baseline_serve(requests, budget_s=10.0):
    """Threaded CPU Jacobi-PCG of the requests one at a time, in arrival order,
    for about budget_s seconds."""
    from oracle import oracle
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    order = sorted(range(len(requests)), key=lambda i: requests[i][0])
    done, t0 = 0, time.perf_counter()
    for i in order:
        _, A, b, _ = requests[i]
        oracle.cg_omp(A.row_ptr, A.col_idx, A.values, b, tol=1e-8, max_iter=100000, precond=True)
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    return {"value": round(done / el, 3), "unit": "solves/s", "cores": threads, "kind": "port",
            "sample": f"the first {done} of {len(requests)} requests in arrival order, solved "
                      f"one at a time in {el:.1f} s (oracle/oracle.c or_cg_omp, Jacobi PCG)"}


# ---- the reference arm ---------------------------------------------------------------------

def run_reference(args, rank, world):
    if rank != 0:
        return None
    desc, kind, precision = WORKLOADS[args.workload]
    threads = os.cpu_count() or 1
    note = "the reference's Kokkos-OpenMP build is not buildable here; oracle/oracle.c port"
    if kind == "spmv":
        A, x = make_workload(args.workload)
        if isinstance(A, list):
            A = block_diagonal(A)
        run, keep, oracle = cpu_spmv_setup(A, x, precision)
        oracle.set_threads(threads)
        t = time.perf_counter()
        run(0, A.nrows)
        full = time.perf_counter() - t
        per_step = 60.0 / max(1, args.steps + args.warmup)
        rows = int(max(1024, min(A.nrows, A.nrows * per_step / max(full, 1e-9))))
        pos = 0

        def step():
            nonlocal pos
            r0 = pos
            r1 = min(A.nrows, r0 + rows)
            run(r0, r1)
            pos = 0 if r1 >= A.nrows else r1
            return slice_bytes(A, r0, r1, precision)

        for _ in range(args.warmup):
            step()
        tot_b = 0
        t0 = time.perf_counter()
        for _ in range(args.steps):
            tot_b += step()
        el = time.perf_counter() - t0
        val, unit = tot_b / el / 1e9, "GB/s"
        sample = (f"row slices of {rows} of {A.nrows} rows per step ({rows / A.nrows:.1%} of one "
                  f"SpMV), or_spmv_*_omp on {threads} threads ({note})")
        cfg = spmv_config(desc, args.workload, A, precision)
        ms_step = el / args.steps * 1e3
    elif kind == "batch":
        from num_b200 import generators as gen
        A = gen.laplacian_3d(100)
        cb = cpu_baseline_batch(A, 128, budget_s=min(60.0, 2.0 * (args.steps + args.warmup)))
        val, unit, sample = cb["value"], "GB/s", cb["sample"] + f" ({note})"
        cfg = {"workload": desc, "name": args.workload, "nrows": A.nrows, "nnz": A.nnz, "k": 128,
               "bytes_per_step": batch_bytes(A, 128),
               "bytes_formula": "12*nnz + 4*(n+1) + 8*k*(ncols + nrows)"}
        ms_step = batch_bytes(A, 128) / (val * 1e9) * 1e3
    elif kind in ("cg", "engine"):
        from num_b200 import generators as gen
        if kind == "cg":
            A, _ = make_workload(args.workload)
            b, tol, pre, iters = A.to_scipy() @ np.ones(A.ncols), 1e-8, False, None
        else:
            A, b = gen.varcoef_poisson_3d(128, seed=3)
            tol, pre, iters = 1e-10, True, 692
        per_step_budget = 60.0 / max(1, args.steps + args.warmup)
        cb = cpu_baseline_cg(A, b, tol, budget_s=per_step_budget * args.steps, precond=pre,
                             full_iters=iters)
        val, unit, sample = cb["value"], "solves/s", cb["sample"] + f" ({note})"
        cfg = {"workload": desc, "name": args.workload, "nrows": A.nrows, "nnz": A.nnz,
               "tol": tol}
        ms_step = 1e3 / val
    elif kind == "vec":
        from oracle import oracle
        n = VEC_N
        rng = np.random.default_rng(5)
        x, y = rng.random(n), rng.random(n)
        t0 = time.perf_counter()
        reps = 0
        while time.perf_counter() - t0 < min(30.0, 1.0 * (args.steps + args.warmup)):
            z = oracle.axpy(0.5, x, y)
            w = oracle.axpy2(0.25, x, -0.5, z)
            oracle.dot(x, w)
            reps += 1
        el = (time.perf_counter() - t0) / reps
        val, unit = vec_bytes(n) / el / 1e9, "GB/s"
        sample = (f"{reps} steps of axpy + axpy2 + dot on {n} doubles, oracle/oracle.c "
                  f"(serial loops) ({note})")
        cfg = {"workload": desc, "name": args.workload, "n": n, "bytes_per_step": vec_bytes(n)}
        ms_step = el * 1e3
    elif kind == "halo":
        from oracle import oracle
        A, parts = halo_workload()
        x = np.random.default_rng(6).uniform(-1, 1, A.ncols)
        t0 = time.perf_counter()
        reps = 0
        while time.perf_counter() - t0 < min(30.0, 1.0 * (args.steps + args.warmup)):
            for p in parts:
                buf = oracle.halo_pack(p["send_idx"], x[p["row_start"]:p["row_end"]])
                ext = np.empty(p["local_n"] + p["n_ghost"])
                ext[p["local_n"]:] = x[p["ghost_ids"]]  # unpack of the received ghosts
                del buf, ext
            reps += 1
        el = (time.perf_counter() - t0) / reps
        nbytes = sum(halo_bytes(p["total_send"], p["n_ghost"]) for p in parts)
        val, unit = nbytes / el / 1e9, "GB/s"
        sample = f"{reps} steps over {len(parts)} slabs, oracle.halo_pack + numpy scatter ({note})"
        cfg = {"workload": desc, "name": args.workload, "ranks": len(parts),
               "bytes_per_step": nbytes}
        ms_step = el * 1e3
    else:  # serve
        from num_b200 import serve
        requests = serve.make_requests(args.requests, rate=args.rate, seed=4, pool=args.pool)
        cb = cpu_baseline_serve(requests, budget_s=60.0)
        val, unit, sample = cb["value"], "solves/s", cb["sample"] + f" ({note})"
        cfg = {"workload": desc, "name": args.workload, "requests": len(requests)}
        ms_step = 1e3 / val
    cfg["parallelism"] = "cpu"
    return {
        "metric": METRIC, "value": round(val, 4), "unit": unit, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": dtype_name(precision if kind == "spmv" else "fp64"), "data": "synthetic",
        "config": cfg, "impl": "reference",
        "cpu_baseline": {"value": round(val, 4), "unit": unit, "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": round(val, 4), "unit": unit, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


# ---- CG vector ops and halo pack / unpack (their own kernels, measured alone) ----------

VEC_N = 4_096_000  # the 160^3 system's length


def vec_bytes(n):
    """axpy (x, y read, z written) + axpy2 (same) + dot (x, y read)."""
    return 24 * n + 24 * n + 16 * n


def halo_bytes(total_send, n_ghost):
    """pack: index, gathered x entry, buffer entry per sent value; unpack:
    buffer entry read, ghost slot written."""
    return total_send * (4 + 8 + 8) + n_ghost * 16


def halo_workload(P=8):
    """The 160^3 Laplacian's halo plan for P row slabs (the library's host-only
    planner, nm_dist_plan): per rank its row range, send index list (local)
    and ghost ids."""
    from num_b200 import _lib
    from num_b200 import generators as gen
    lib = _lib.load()
    A = gen.laplacian_3d(160)
    rp, ci, v = (np.ascontiguousarray(a) for a in (A.row_ptr, A.col_idx, A.values))
    parts = []
    for r in range(P):
        h = C.c_void_p()
        _lib.check(lib.nm_dist_plan(rp.ctypes.data, ci.ctypes.data, v.ctypes.data, A.nrows,
                                    A.ncols, r, P, C.byref(h)), "nm_dist_plan")
        info = [C.c_int32() for _ in range(7)]
        _lib.check(lib.nm_dist_info(h, *[C.byref(i) for i in info]), "nm_dist_info")
        gn, rs, re, ng, ts, nsn, nrn = (i.value for i in info)
        send_idx = np.empty(max(ts, 1), np.int32)
        ghost_ids = np.empty(max(ng, 1), np.int32)
        a1, a2, a3 = (np.empty(max(nsn, 1), np.int32) for _ in range(3))
        _lib.check(lib.nm_dist_send_plan(h, a1.ctypes.data, a2.ctypes.data, a3.ctypes.data,
                                         send_idx.ctypes.data), "send plan")
        b1, b2, b3 = (np.empty(max(nrn, 1), np.int32) for _ in range(3))
        _lib.check(lib.nm_dist_recv_plan(h, b1.ctypes.data, b2.ctypes.data, b3.ctypes.data,
                                         ghost_ids.ctypes.data), "recv plan")
        lib.nm_dist_destroy(h)
        parts.append({"row_start": rs, "row_end": re, "local_n": re - rs, "n_ghost": ng,
                      "total_send": ts, "send_idx": send_idx[:ts], "ghost_ids": ghost_ids[:ng]})
    return A, parts


def time_ops(ops, stream, steps, warmup):
    """Each op of `ops` (name -> callable enqueueing one kernel) timed with
    its own CUDA events over `steps` rounds after `warmup` rounds; returns
    (ms of the whole timed region, {name: average ms})."""
    import torch
    for _ in range(warmup):
        for f in ops.values():
            f()
    torch.cuda.synchronize()
    ev = {k: [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(steps)] for k in ops}
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for i in range(steps):
        for k, f in ops.items():
            ev[k][i][0].record(stream)
            f()
            ev[k][i][1].record(stream)
    t1.record(stream)
    torch.cuda.synchronize()
    avg = {k: sum(a.elapsed_time(b) for a, b in v) / steps for k, v in ev.items()}
    return t0.elapsed_time(t1), avg


def run_vec(args, rank, world, local_rank):
    import torch

    from num_b200 import _lib
    dev = torch.device("cuda", local_rank)
    desc, _, precision = WORKLOADS[args.workload]
    n = VEC_N
    g = torch.Generator(device=dev).manual_seed(5)
    x = torch.rand(n, dtype=torch.float64, device=dev, generator=g)
    y = torch.rand(n, dtype=torch.float64, device=dev, generator=g)
    z, w = torch.empty_like(x), torch.empty_like(x)
    lib = _lib.load()
    stream = torch.cuda.current_stream(dev)
    s = stream.cuda_stream
    res = C.c_double()
    ops = {
        "axpy": lambda: lib.nm_axpy(n, 0.5, x.data_ptr(), y.data_ptr(), z.data_ptr(), s),
        "axpy2": lambda: lib.nm_axpy2(n, 0.25, x.data_ptr(), -0.5, z.data_ptr(), w.data_ptr(),
                                      s),
        "dot": lambda: lib.nm_dot(n, x.data_ptr(), w.data_ptr(), C.byref(res), s),
    }
    # inputs (3 x 33 MB) are smaller than L2: a 256 MB write before each round
    flush = torch.empty(64 << 20, dtype=torch.float32, device=dev)
    ops = {"flush": flush.zero_, **ops}
    with ClockSampler(local_rank) as clk:
        # ~0.5 s of back-to-back rounds (the dot synchronises each one) so the
        # sampler sees the GPU under this load for 20+ samples
        t_end = time.perf_counter() + 0.5
        while time.perf_counter() < t_end:
            for f in ops.values():
                f()
        total_ms, avg = time_ops(ops, stream, args.steps, args.warmup)
    step_ms = avg["axpy"] + avg["axpy2"] + avg["dot"]
    step_ms = max_over_ranks([step_ms], world, dev)[0]
    if rank != 0:
        return None
    nbytes = vec_bytes(n)
    peak, peak_src = measured_peak()
    config = {"workload": desc, "name": args.workload, "n": n, "bytes_per_step": nbytes,
              "bytes_formula": "axpy 24n + axpy2 24n + dot 16n",
              "l2": "operands (3 x 33 MB) smaller than L2: L2 flushed (256 MB write) before "
                    "each round, ops timed alone",
              "parallelism": f"replicas x{world}",
              "api": "C ABI nm_axpy / nm_axpy2 / nm_dot (the dot returns its value to the "
                     "host, as vec_local_dot does)"}
    line = base_line(args, world, round(world * nbytes / (step_ms * 1e-3) / 1e9, 2), "GB/s",
                     step_ms, precision, config)
    per = {k: {"us": round(avg[k] * 1e3, 2),
               "gbs": round((24 if k != "dot" else 16) * n / (avg[k] * 1e-3) / 1e9, 1)}
           for k in ("axpy", "axpy2", "dot")}
    line.update({
        "roofline": {"bound": "hbm", "achieved": per["axpy2"]["gbs"], "peak": peak,
                     "unit": "GB/s", "frac": round(per["axpy2"]["gbs"] / peak, 4),
                     "peak_source": peak_src, "traffic": None,
                     "kernel": "nm::axpy2_kernel (24 B per element)", "per_op": per},
        "e2e": {"value": line["value"], "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 8,
                "note": "the dot's value comes back to the host every step; the vectors are "
                        "device operands of the CG, never host data"},
        "gpu_launches": 3 * args.steps,
        "clocks": clk.summary(),
    })
    return line


def run_halo(args, rank, world, local_rank):
    import torch

    from num_b200 import _lib
    dev = torch.device("cuda", local_rank)
    desc, _, precision = WORKLOADS[args.workload]
    A, parts = halo_workload()
    lib = _lib.load()
    stream = torch.cuda.current_stream(dev)
    s = stream.cuda_stream
    rp, ci, v = (np.ascontiguousarray(a) for a in (A.row_ptr, A.col_idx, A.values))
    x = torch.tensor(np.random.default_rng(6).uniform(-1, 1, A.ncols), device=dev)
    handles, bufs = [], []
    for r, p in enumerate(parts):
        h = C.c_void_p()
        _lib.check(lib.nm_dist_create(rp.ctypes.data, ci.ctypes.data, v.ctypes.data, A.nrows,
                                      A.ncols, r, len(parts), C.byref(h)), "nm_dist_create")
        handles.append(h)
        send = torch.empty(max(p["total_send"], 1), dtype=torch.float64, device=dev)
        recv = torch.rand(max(p["n_ghost"], 1), dtype=torch.float64, device=dev)
        ext = torch.empty(p["local_n"] + p["n_ghost"], dtype=torch.float64, device=dev)
        bufs.append((x[p["row_start"]:p["row_end"]], send, recv, ext))
    def enqueue(kind, st):
        for h, (xl, send, recv, ext) in zip(handles, bufs):
            if kind == "pack":
                _lib.check(lib.nm_halo_pack(h, xl.data_ptr(), send.data_ptr(), st),
                           "nm_halo_pack")
            else:
                _lib.check(lib.nm_halo_unpack(h, recv.data_ptr(), ext.data_ptr(), st),
                           "nm_halo_unpack")

    # The 8 packs and the 8 unpacks each captured as one CUDA graph and
    # replayed: per-launch host overhead (~5 us through ctypes) would otherwise
    # sit between the events of kernels that run for ~2-5 us.
    graphs = {}
    side = torch.cuda.Stream(dev)
    for kind in ("pack", "unpack"):
        enqueue(kind, s)  # first launches outside capture (lazy module loading)
        torch.cuda.synchronize(dev)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=side):
            enqueue(kind, side.cuda_stream)
        graphs[kind] = g
    # inputs (13 MB per step) fit L2: a 256 MB write before each round
    flush = torch.empty(64 << 20, dtype=torch.float32, device=dev)
    ops = {"flush": flush.zero_, "pack": graphs["pack"].replay,
           "unpack": graphs["unpack"].replay}
    with ClockSampler(local_rank) as clk:
        sustained(lambda: (graphs["pack"].replay(), graphs["unpack"].replay()), stream, dev)
        total_ms, avg = time_ops(ops, stream, args.steps, args.warmup)
    step_ms = avg["pack"] + avg["unpack"]
    step_ms = max_over_ranks([step_ms], world, dev)[0]
    del graphs
    for h in handles:
        lib.nm_dist_destroy(h)
    if rank != 0:
        return None
    nbytes = sum(halo_bytes(p["total_send"], p["n_ghost"]) for p in parts)
    pack_us = avg["pack"] * 1e3
    unpack_us = avg["unpack"] * 1e3
    pack_b = sum(p["total_send"] * 20 for p in parts)
    peak, peak_src = measured_peak()
    pack_gbs = pack_b / (pack_us * 1e-6) / 1e9
    config = {"workload": desc, "name": args.workload, "ranks": len(parts),
              "send_total": sum(p["total_send"] for p in parts),
              "ghost_total": sum(p["n_ghost"] for p in parts), "bytes_per_step": nbytes,
              "bytes_formula": "pack 20 B per sent value + unpack 16 B per ghost",
              "l2": "operands (13 MB per step) smaller than L2: L2 flushed (256 MB write) "
                    "before each round",
              "timing": "the 8 packs, then the 8 unpacks, each one CUDA-graph replay "
                        "timed with CUDA events",
              "parallelism": f"replicas x{world}",
              "api": "C ABI nm_halo_pack / nm_halo_unpack on nm_dist_create slabs"}
    line = base_line(args, world, round(world * nbytes / (step_ms * 1e-3) / 1e9, 2), "GB/s",
                     step_ms, precision, config)
    line.update({
        "roofline": {"bound": "hbm", "achieved": round(pack_gbs, 1), "peak": peak,
                     "unit": "GB/s", "frac": round(pack_gbs / peak, 4), "peak_source": peak_src,
                     "traffic": None, "kernel": "nm::halo_pack_kernel",
                     "pack_us_per_step": round(pack_us, 2),
                     "unpack_us_per_step": round(unpack_us, 2),
                     "note": "each launch moves ~0.5-1 MB: launch and DRAM latency, not "
                             "bandwidth, bound it"},
        "e2e": {"value": line["value"], "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0,
                "note": "halo buffers are device operands of the distributed SpMV"},
        "gpu_launches": 2 * len(parts) * args.steps,
        "clocks": clk.summary(),
    })
    return line


DEFAULT_STEPS = {"spmv": 2000, "batch": 100, "cg": 50, "engine": 5, "serve": 3, "vec": 200,
                 "halo": 200}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=0, help="0: the workload's default")
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="spmv_c2a", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the CG / serving summary of the default line")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--tile", type=int, default=0, help="row-block tile (0: library default)")
    ap.add_argument("--stages", type=int, default=0, help="TMA pipeline depth (0: default)")
    ap.add_argument("--short-max", type=int, default=0)
    ap.add_argument("--grid-mult", type=int, default=-1)
    ap.add_argument("--requests", type=int, default=200, help="serve_c5: requests per pass")
    ap.add_argument("--rate", type=float, default=0.0,
                    help="serve_c5: Poisson arrival rate (req/s); 0 = all at t=0")
    ap.add_argument("--arena-gb", type=float, default=64.0, help="serve_c5: arena cap")
    ap.add_argument("--pool", type=int, default=1000,
                    help="serve_c5: distinct systems; longer streams reuse them")
    ap.add_argument("--serve-precision", default="fp32", choices=["fp32", "bf16", "fp64"],
                    help="serve_c5: the engine's inner precision")
    ap.add_argument("--serve-precond", default="jacobi", choices=["jacobi", "none"],
                    help="serve_c5: the engine's preconditioner")
    ap.add_argument("--no-plain", action="store_true",
                    help="serve_c5: skip the plain FP64 drop-in comparison")
    ap.add_argument("--cg-mode", type=int, default=1, choices=[0, 1, 2, 3, 4],
                    help="nm_cg_set_persistent: 1 persistent (default), 2 the TMA-pipelined "
                         "persistent solve only, 3 the resident solve only, 0 CUDA-graph "
                         "chunks")
    ap.add_argument("--engine-mode", default="graph", choices=["persistent", "graph"],
                    help="nm_solver_set_persistent: one cooperative launch per engine step, or "
                         "a CUDA graph of kernels")
    args = ap.parse_args()
    kind = WORKLOADS[args.workload][1]
    if args.steps <= 0:
        args.steps = DEFAULT_STEPS[kind]
    if args.warmup < 3:
        args.warmup = 3
    if kind in ("engine", "serve") and args.warmup > 3:
        args.warmup = 3  # whole solves / passes: three are plenty

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        line = run_reference(args, rank, world)
        if line:
            print(json.dumps(line), flush=True)
        return
    import torch
    torch.cuda.set_device(local_rank)
    from num_b200 import _lib
    from num_b200 import kokkos_spmv as kspmv
    kspmv.init(local_rank)
    _lib.check(_lib.load().nm_cg_set_persistent(args.cg_mode), "nm_cg_set_persistent")
    _lib.check(_lib.load().nm_solver_set_persistent(1 if args.engine_mode == "persistent" else 0),
               "nm_solver_set_persistent")
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    try:
        run = {"spmv": run_spmv, "batch": run_batch, "cg": run_cg, "engine": run_engine,
               "serve": run_serve, "vec": run_vec, "halo": run_halo}[kind]
        line = run(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    if line:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
