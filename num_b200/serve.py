"""Serving CG solve requests: continuous batching on the solver engine, and the
plain FP64 CG drop-in run one request at a time for comparison.

A request is (arrival time in seconds, A, b).  `serve` runs a real-time loop:
every loop iteration starts one engine step (pending refinement steps + `chunk`
lockstep iterations of all live solves) and, while the device runs it, admits
the requests that have arrived, in arrival order, while the arena has room for
them (admission by free device memory; they join at the next step); then it
waits for the step, retires finished solves and records their latency (finish
- arrival).  `serve_plain` solves the same requests one at a time, in arrival
order, with the drop-in FP64 CG (`kokkos_spmv.cg_solve_local` semantics: upload,
solve, copy back).
"""
from __future__ import annotations

import math
import time

import numpy as np

from . import generators as gen


def make_requests(count: int, rate: float, seed: int = 4, side_range=(32, 1024),
                  banded_range=(256, 65536), pool: int | None = None):
    """The served workload: Poisson arrivals at `rate` req/s (rate <= 0: all at
    t = 0); each request with equal probability a 2-D 5-point Laplacian with
    side log-uniform in side_range, or a banded SPD matrix (half-bandwidth
    uniform in 1..8, 2 mirrored off-band entries per row, diagonal 1.05 x the
    off-diagonal row sum) with n log-uniform in banded_range; b ~ N(0, 1).

    pool: when count exceeds it, only the first `pool` requests draw their own
    system (A, b) -- an i.i.d. sample of the distribution -- and request i
    reuses system i mod pool, while every request still draws its own arrival
    time.  A 20,000-request stream would otherwise hold ~100 GB of host CSR
    arrays.  The first `pool` requests are those of the unpooled stream."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(count):
        if rate > 0:
            t += rng.exponential(1.0 / rate)
        if pool is not None and i >= pool:
            _, A, b, kind = out[i % pool]
            out.append((t, A, b, kind))
            continue
        if rng.random() < 0.5:
            side = int(round(math.exp(rng.uniform(math.log(side_range[0]),
                                                  math.log(side_range[1])))))
            A = gen.laplacian_2d(side)
            kind = f"laplace2d:{side}"
        else:
            n = int(round(math.exp(rng.uniform(math.log(banded_range[0]),
                                               math.log(banded_range[1])))))
            A = gen.banded_spd(n, int(rng.integers(1, 9)), rng)
            kind = f"banded:{n}"
        b = rng.standard_normal(A.nrows)
        out.append((t, A, b, kind))
    return out


def _stats(lat, t0, t_end, n_done):
    lat = np.asarray(lat)
    return {"completed": int(n_done), "seconds": t_end - t0,
            "solves_per_s": n_done / max(t_end - t0, 1e-12),
            "p50_ms": float(np.percentile(lat, 50) * 1e3) if lat.size else None,
            "p99_ms": float(np.percentile(lat, 99) * 1e3) if lat.size else None,
            "mean_ms": float(lat.mean() * 1e3) if lat.size else None}


def serve(requests, solver, tol: float = 1e-8, max_iter: int = 100000, chunk: int = 8,
          check=None, batch: int = 16):
    """Continuous batching.  Returns (stats, per-request records).  `batch`:
    requests prepared per admission call (in parallel on the host)."""
    order = sorted(range(len(requests)), key=lambda i: requests[i][0])
    queue = []  # arrived, not yet admitted (FIFO)
    nxt = 0
    live = {}   # slot -> request index
    rec = [None] * len(requests)
    t0 = time.perf_counter()
    def arrivals():
        nonlocal nxt
        now = time.perf_counter() - t0
        while nxt < len(order) and requests[order[nxt]][0] <= now:
            queue.append(order[nxt])
            nxt += 1

    def admit(count):
        got = solver.admit_many([requests[i][1:3] for i in queue[:count]], tol=tol,
                                max_iter=max_iter)
        for slot, i in zip(got, queue):
            live[slot] = i
        del queue[: len(got)]
        return len(got) == min(count, len(queue) + len(got))  # False: no room

    def admit_budgeted(budget):
        # admit in small batches while the device is still busy with the step
        t_start = time.perf_counter()
        while queue and time.perf_counter() - t_start < budget:
            if not admit(batch):
                break
            arrivals()

    def step_iters():
        # While requests wait, size the step so that its device time covers
        # the host time of admitting the next batch, with 1.5x headroom (both
        # estimated: device ms per iteration of the last step, host seconds
        # spent in admission calls per admitted row so far).
        if not queue:
            return chunk, 0.0
        c = solver.counters()
        rows_done = max(1, solver.rows_admitted)
        spent = solver.seconds["admit"]
        per_row = spent / rows_done if spent > 0 else 1e-7
        nxt_rows = sum(requests[i][1].nrows for i in queue[:batch])
        need = 1.5 * per_row * nxt_rows
        last = c["last_step_ms"] * 1e-3
        per_it = last / max(1, c["last_step_iters"]) if last > 0 else 0.0
        if per_it <= 0:
            return chunk * 4, need
        it = int(min(64 * chunk, max(chunk, need / per_it)))
        return it, need

    while nxt < len(order) or queue or live:
        arrivals()
        if not live:
            if queue:
                admit(batch)  # a first batch to start the device
            if not live:
                if nxt < len(order):  # idle until the next arrival
                    time.sleep(max(0.0, requests[order[nxt]][0] - (time.perf_counter() - t0)))
                continue
        iters, budget = step_iters()
        solver.step_begin(iters)
        arrivals()
        admit_budgeted(max(budget, 1e-3))  # host preparation overlaps the step on the device
        done = solver.step_end()
        for slot, (x, info) in zip(done, solver.take_many(done)):
            i = live.pop(slot)
            t_fin = time.perf_counter() - t0
            rec[i] = {"latency": t_fin - requests[i][0], "finish": t_fin, **info}
            if check is not None:
                check(i, x, info)
    lat = [r["latency"] for r in rec]
    t_first = min(r[0] for r in requests)
    t_end = max(r["finish"] for r in rec)
    return _stats(lat, t_first, t_end, len(rec)), rec


def serve_plain(requests, tol: float = 1e-8, max_iter: int = 100000, check=None,
                device: int = 0):
    """The plain FP64 CG drop-in, one request at a time in arrival order."""
    import torch

    from . import kokkos_spmv as kspmv
    kspmv.init(device)
    dev = torch.device("cuda", device)
    order = sorted(range(len(requests)), key=lambda i: requests[i][0])
    rec = [None] * len(requests)
    t0 = time.perf_counter()
    for i in order:
        t_arr, A, b, _ = requests[i]
        wait = t_arr - (time.perf_counter() - t0)
        if wait > 0:
            time.sleep(wait)
        M = kspmv.upload_csr(A.row_ptr, A.col_idx, A.values, A.nrows, A.ncols)
        bt = torch.from_numpy(np.ascontiguousarray(b)).to(dev, non_blocking=False)
        xt = torch.zeros(A.nrows, dtype=torch.float64, device=dev)
        info = kspmv.cg_solve_local(M, bt, xt, tol=tol, max_iter=max_iter)
        x = xt.cpu().numpy()
        t_fin = time.perf_counter() - t0
        rec[i] = {"latency": t_fin - t_arr, "finish": t_fin, **info}
        if check is not None:
            check(i, x, info)
        del M
    lat = [r["latency"] for r in rec]
    t_first = min(r[0] for r in requests)
    t_end = max(r["finish"] for r in rec)
    return _stats(lat, t_first, t_end, len(rec)), rec
