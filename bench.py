#!/usr/bin/env python
"""Benchmark of the sparse hot path on B200.

Default workload (one step = one FP64 CSR SpMV, y = A x):
  3-D 7-point Laplacian on a 160^3 grid: n = 4,096,000, nnz = 28,518,400,
  int32 indices, FP64 values, x ~ U[-1, 1] (default_rng(1)).
  Algorithmic bytes per SpMV = 12 nnz + 4 (n + 1) + 8 n (x) + 8 n (y)
  = 424.14 MB, larger than the 126 MB L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME]
    python bench.py --impl reference ...   # the reference's CPU path (oracle port)

Multi-GPU (torchrun, one rank per GPU): every rank runs the same workload on
its own GPU (independent replicas, weak scaling, no data-path collective);
value = total bytes of all ranks / max-over-ranks time.
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

WORKLOADS = {
    "spmv_c2a": ("3-D 7-point Laplacian 160^3, FP64 CSR SpMV", "fp64"),
    "spmv_c2a_fp32": ("3-D 7-point Laplacian 160^3, FP32 CSR SpMV", "fp32"),
    "spmv_c2b": ("power-law rows n=2,000,000 mean 16 sigma 1.2, FP64 CSR SpMV", "fp64"),
    "spmv_c2b_fp32": ("power-law rows n=2,000,000 mean 16 sigma 1.2, FP32 CSR SpMV", "fp32"),
    "spmv_c1": ("2-D 5-point Laplacian 256^2, FP64 CSR SpMV", "fp64"),
}


def make_workload(name):
    from num_b200 import generators as gen
    if name.startswith("spmv_c2a"):
        A = gen.laplacian_3d(160)
        seed = 1
    elif name.startswith("spmv_c2b"):
        A = gen.power_law(2_000_000, seed=1001)
        seed = 1
    elif name == "spmv_c1":
        A = gen.laplacian_2d(256)
        seed = 0
    else:
        raise SystemExit(f"unknown workload {name}")
    x = np.random.default_rng(seed).uniform(-1.0, 1.0, A.ncols)
    return A, x


def spmv_bytes(A, precision):
    from num_b200.generators import spmv_bytes as sb
    vb = {"fp64": 8, "fp32": 4, "bf16": 2}[precision]
    xb = 8 if precision == "fp64" else 4
    return sb(A.nnz, A.nrows, A.ncols, vb, xb)


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


# ---- our arm ---------------------------------------------------------------------------

def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist

    from num_b200 import _lib
    from num_b200 import kokkos_spmv as kspmv

    kspmv.init(local_rank)
    dev = torch.device("cuda", local_rank)
    desc, precision = WORKLOADS[args.workload]
    A, x = make_workload(args.workload)
    M = kspmv.upload_csr(A.row_ptr, A.col_idx, A.values, A.nrows, A.ncols, precision=precision)
    tuned = kspmv.tune(M, tile=args.tile, short_max=args.short_max, stages=args.stages,
                       grid_mult=args.grid_mult)
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

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        torch.cuda.synchronize(dev)
        t0.record(stream)
        for k in range(args.steps):
            ev[k][0].record(stream)
            step()
            ev[k][1].record(stream)
        t1.record(stream)
        torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    total_ms = t0.elapsed_time(t1)
    kern_ms = [a.elapsed_time(b) for a, b in ev]
    kern_avg_ms = sum(kern_ms) / len(kern_ms)
    t = torch.tensor([total_ms, kern_avg_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms, kern_avg_ms = float(t[0]), float(t[1])
    ms_per_step = total_ms / args.steps

    # correctness spot check (outside the timed region)
    if rank == 0 and args.workload == "spmv_c1":
        pass

    # e2e through the public drop-in API: pinned host x -> device, spmv, y -> pinned host
    e2e_steps = max(3, min(args.steps, 50))
    xh = torch.tensor(x, dtype=dt).pin_memory()
    yh = torch.empty(A.nrows, dtype=dt).pin_memory()
    for _ in range(2):
        xd.copy_(xh, non_blocking=True)
        kspmv.spmv(M, xd, yd)
        yh.copy_(yd, non_blocking=True)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        xd.copy_(xh, non_blocking=True)
        kspmv.spmv(M, xd, yd)
        yh.copy_(yd, non_blocking=True)
        stream.synchronize()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    e2e_ms = e0.elapsed_time(e1) / e2e_steps
    te = torch.tensor([e2e_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_ms = float(te[0])

    if rank != 0:
        return None
    peak, peak_src = measured_peak()
    achieved = nbytes / (kern_avg_ms * 1e-3) / 1e9
    line = {
        "metric": METRIC,
        "value": round(world * nbytes / (ms_per_step * 1e-3) / 1e9, 2),
        "unit": "GB/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_per_step, 6),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if precision == "fp64" else ("f32" if precision == "fp32" else "bf16/f32"),
        "data": "synthetic",
        "config": {
            "workload": desc, "name": args.workload, "nrows": A.nrows, "nnz": A.nnz,
            "index": "int32", "values": precision,
            "bytes_per_step": nbytes,
            "bytes_formula": "12*nnz + 4*(n+1) + 8*ncols + 8*nrows (fp64)",
            "l2": "inputs larger than L2 (no flush): %.1f MB per step > 126 MB" % (nbytes / 1e6),
            "parallelism": f"replicas x{world}",
            "tuning": tuned,
        },
        "roofline": {
            "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_source": peak_src,
            "frac_of_8TBs_spec": round(achieved / 8000.0, 4),
            "traffic": traffic_for(args.workload),
            "kernel": "nm::spmv_kernel (row-block CSR SpMV)",
            "kernel_avg_us": round(kern_avg_ms * 1e3, 3),
        },
        "e2e": {
            "value": round(nbytes / (e2e_ms * 1e-3) / 1e9, 2), "unit": "GB/s",
            "h2d_bytes_per_step": int(xh.numel() * xh.element_size()),
            "d2h_bytes_per_step": int(yh.numel() * yh.element_size()),
            "ms_per_step": round(e2e_ms, 4), "steps": e2e_steps,
            "api": "num_b200.kokkos_spmv.spmv (C ABI nm_spmv) with pinned host x/y copies",
        },
        "gpu_launches": args.steps,
        "clocks": clk.summary(),
        "reference_metric_gbs": round(
            (12 * A.nnz + 16 * A.nrows) / (kern_avg_ms * 1e-3) / 1e9, 1) if precision == "fp64" else None,
    }
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(A, x, precision, budget_s=args.cpu_seconds)
    return line


# ---- CPU leg (oracle port of the reference's CPU path) --------------------------------------

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


def cpu_baseline(A, x, precision, budget_s=10.0):
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


def run_reference(args, rank, world):
    if rank != 0:
        return None
    desc, precision = WORKLOADS[args.workload]
    A, x = make_workload(args.workload)
    run, keep, oracle = cpu_spmv_setup(A, x, precision)
    threads = os.cpu_count() or 1
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
    val = tot_b / el / 1e9
    sample = (f"row slices of {rows} of {A.nrows} rows per step ({rows / A.nrows:.1%} of one SpMV), "
              f"oracle/oracle.c or_spmv_*_omp on {threads} threads (the reference's Kokkos-OpenMP "
              f"build is not buildable here)")
    return {
        "metric": METRIC, "value": round(val, 3), "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(el / args.steps * 1e3, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if precision == "fp64" else "f32", "data": "synthetic",
        "config": {"workload": desc, "name": args.workload, "nrows": A.nrows, "nnz": A.nnz,
                   "parallelism": "cpu"},
        "impl": "reference",
        "cpu_baseline": {"value": round(val, 3), "unit": "GB/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": round(val, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="spmv_c2a", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--tile", type=int, default=0, help="row-block tile (0: library default)")
    ap.add_argument("--stages", type=int, default=0, help="TMA pipeline depth (0: default)")
    ap.add_argument("--short-max", type=int, default=0)
    ap.add_argument("--grid-mult", type=int, default=-1)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        line = run_reference(args, rank, world)
        if line:
            print(json.dumps(line), flush=True)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    try:
        line = run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    if line:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
