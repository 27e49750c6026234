"""Distributed SpMV and CG: halo exchange plan and per-iteration orchestration.

Restates the reference's distributed path (src/dist_spmv.hpp:118-163,
src/halo_exchange.hpp:209-303, src/cg_solver.hpp:38-125) for one process per
GPU over torch.distributed:

  * the plan (who sends which entries to whom) comes from the library's
    distribute_csr restatement (nm_dist_create / nm_dist_plan);
  * pack  : the library kernel gathers x_local[send_idx] into a send buffer;
  * exchange: one batched isend/irecv per neighbour (NCCL on GPUs, gloo on
    CPU), at most one message per ordered pair of ranks per exchange, so
    messages match by (peer, order) as the reference's tag-42 Isend/Irecv do;
  * unpack: the library kernel writes the received values behind the owned
    entries of x_ext = [x_local | x_ghost];
  * SpMV on x_ext with the remapped local matrix -- on GPUs in two parts:
    the rows whose columns are all owned are multiplied from x_local while
    the exchange is in flight, the rows with ghost columns after the unpack
    (the overlap the reference describes as future work,
    src/halo_exchange.hpp:28-33).

With one rank there are no ghosts: dist_spmv is the local SpMV on x_local
directly (the reference still allocates and fills x_ext per call, which is
skipped), and cg_solve is the library's device-resident CG with the
reference's breakdown guard.

The CG recurrence below (`cg_distributed`) is written against a small `ops`
interface so that the identical control flow runs on GPUs (DeviceOps: library
kernels + torch.distributed all_reduce) and, in the CPU test suite, with CPU
stand-ins over gloo.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _lib

try:
    import torch
    import torch.distributed as dist
except ImportError:  # pragma: no cover
    torch = None
    dist = None


@dataclass
class HaloPlan:
    rank: int
    size: int
    row_start: int
    row_end: int
    n_ghost: int
    total_send: int
    send_rank: np.ndarray   # neighbour ranks we send to (ascending)
    send_count: np.ndarray
    send_off: np.ndarray    # offsets into the packed send buffer
    send_idx: np.ndarray    # LOCAL indices packed, neighbour order
    recv_rank: np.ndarray   # owner ranks we receive from (ascending)
    recv_count: np.ndarray
    recv_off: np.ndarray    # offsets of their ghosts in x_ghost
    ghost_ids: np.ndarray   # GLOBAL ids of the ghosts, ghost order

    @property
    def local_n(self) -> int:
        return self.row_end - self.row_start

    @classmethod
    def from_handle(cls, h, info=None, rank: int | None = None, size: int | None = None):
        lib = _lib.load()
        vals = [C.c_int32() for _ in range(7)]
        _lib.check(lib.nm_dist_info(h, *map(C.byref, vals)))
        _, rs, re, ng, ts, nsn, nrn = (v.value for v in vals)
        s_rank, s_cnt, s_off = (np.empty(nsn, np.int32) for _ in range(3))
        s_idx = np.empty(ts, np.int32)
        r_rank, r_cnt, r_off = (np.empty(nrn, np.int32) for _ in range(3))
        g_ids = np.empty(ng, np.int32)
        _lib.check(lib.nm_dist_send_plan(h, s_rank.ctypes.data, s_cnt.ctypes.data,
                                         s_off.ctypes.data, s_idx.ctypes.data))
        _lib.check(lib.nm_dist_recv_plan(h, r_rank.ctypes.data, r_cnt.ctypes.data,
                                         r_off.ctypes.data, g_ids.ctypes.data))
        if rank is None:
            from . import kokkos_spmv
            rank, size = kokkos_spmv.rank(), kokkos_spmv.size()
        return cls(rank, size, rs, re, ng, ts, s_rank, s_cnt, s_off, s_idx, r_rank, r_cnt, r_off,
                   g_ids)


def plan_host(rowptr, colind, values, n: int, ncols: int, rank: int, size: int):
    """Host-only plan of rank `rank` of `size` (no GPU needed): (HaloPlan,
    local CSR (rowptr, colind, values) with remapped columns)."""
    lib = _lib.load()
    rowptr = np.ascontiguousarray(rowptr, np.int32)
    colind = np.ascontiguousarray(colind, np.int32)
    values = np.ascontiguousarray(values, np.float64)
    h = C.c_void_p()
    _lib.check(lib.nm_dist_plan(rowptr.ctypes.data, colind.ctypes.data, values.ctypes.data, int(n),
                                int(ncols), int(rank), int(size), C.byref(h)), "nm_dist_plan")
    try:
        plan = HaloPlan.from_handle(h, rank=rank, size=size)
        lnnz = C.c_int32()
        _lib.check(lib.nm_dist_local_host(h, C.byref(lnnz), None, None, None))
        lrp = np.empty(plan.local_n + 1, np.int32)
        lci = np.empty(lnnz.value, np.int32)
        lv = np.empty(lnnz.value, np.float64)
        _lib.check(lib.nm_dist_local_host(h, None, lrp.ctypes.data, lci.ctypes.data,
                                          lv.ctypes.data))
    finally:
        lib.nm_dist_destroy(h)
    return plan, (lrp, lci, lv)


def exchange_start(plan: HaloPlan, send_buf, recv_buf, group=None) -> list:
    """Post the exchange (src/halo_exchange.hpp:237-285): each neighbour's
    packed segment sent, each owner's ghost segment received, as one batch of
    P2P ops.  Returns the requests for exchange_wait."""
    ops = []
    for r, c, o in zip(plan.recv_rank, plan.recv_count, plan.recv_off):
        ops.append(dist.P2POp(dist.irecv, recv_buf[int(o):int(o) + int(c)], int(r), group))
    for r, c, o in zip(plan.send_rank, plan.send_count, plan.send_off):
        ops.append(dist.P2POp(dist.isend, send_buf[int(o):int(o) + int(c)], int(r), group))
    return dist.batch_isend_irecv(ops) if ops else []


def exchange_wait(reqs) -> None:
    """Complete the exchange (with NCCL: the current stream waits for it)."""
    for req in reqs:
        req.wait()


def exchange(plan: HaloPlan, send_buf, recv_buf, group=None) -> None:
    """The whole halo exchange: exchange_start then exchange_wait."""
    exchange_wait(exchange_start(plan, send_buf, recv_buf, group))


class DeviceOps:
    """Library kernels on one GPU + torch.distributed for the reductions and
    the halo.  Buffers are torch CUDA float64 tensors."""

    def __init__(self, A_dist, group=None):
        self.A = A_dist
        self.plan = A_dist.plan()
        self.group = group
        self.lib = _lib.load()
        n = self.plan.local_n
        dev = torch.device("cuda", torch.cuda.current_device())
        self.x_ext = torch.zeros(n + self.plan.n_ghost, dtype=torch.float64, device=dev)
        self.send_buf = torch.empty(max(self.plan.total_send, 1), dtype=torch.float64, device=dev)
        self.recv_buf = torch.empty(max(self.plan.n_ghost, 1), dtype=torch.float64, device=dev)

    def _s(self):
        return torch.cuda.current_stream().cuda_stream

    def spmv(self, x, y):
        p = self.plan
        if p.n_ghost == 0 and p.total_send == 0:
            _lib.check(self.lib.nm_dist_spmv_local(self.A._h, x.data_ptr(), y.data_ptr(),
                                                   self._s()), "dist_spmv")
            return
        _lib.check(self.lib.nm_halo_pack(self.A._h, x.data_ptr(), self.send_buf.data_ptr(),
                                         self._s()), "halo_pack")
        reqs = exchange_start(p, self.send_buf, self.recv_buf, self.group)
        # while the halo is in flight: the rows without ghost columns, and the
        # owned part of x_ext (x_ext_fill_local, src/dist_spmv.hpp:139-142)
        _lib.check(self.lib.nm_dist_spmv_interior(self.A._h, x.data_ptr(), y.data_ptr(),
                                                  self._s()), "dist_spmv")
        self.x_ext[: p.local_n].copy_(x)
        exchange_wait(reqs)
        _lib.check(self.lib.nm_halo_unpack(self.A._h, self.recv_buf.data_ptr(),
                                           self.x_ext.data_ptr(), self._s()), "halo_unpack")
        _lib.check(self.lib.nm_dist_spmv_boundary(self.A._h, self.x_ext.data_ptr(), y.data_ptr(),
                                                  self._s()), "dist_spmv")

    def dot(self, x, y) -> float:
        out = C.c_double()
        _lib.check(self.lib.nm_dot(x.shape[0], x.data_ptr(), y.data_ptr(), C.byref(out),
                                   self._s()), "dot")
        return out.value

    def allreduce_sum(self, v: float) -> float:
        t = torch.tensor([v], dtype=torch.float64, device=self.x_ext.device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
        return float(t.item())

    def axpy(self, a, x, y, z):
        _lib.check(self.lib.nm_axpy(x.shape[0], a, x.data_ptr(), y.data_ptr(), z.data_ptr(),
                                    self._s()), "axpy")

    def axpy2(self, a, x, b, y, z):
        _lib.check(self.lib.nm_axpy2(x.shape[0], a, x.data_ptr(), b, y.data_ptr(), z.data_ptr(),
                                     self._s()), "axpy2")

    def copy(self, src, dst):
        dst.copy_(src)

    def empty_like(self, v):
        return torch.empty_like(v)


def cg_distributed(ops, b, x, tol: float = 1e-10, max_iter: int = 1000) -> dict:
    """cg_solve_distributed (src/cg_solver.hpp:38-125), step for step:
    r = b - A x0; p = r; ||b|| (0 -> 1); early exit; per iteration one halo
    SpMV, p.Ap with the |p.Ap| < 1e-300 guard, x/r updates, r.r, the strict
    `<` test returning iter+1, beta, p = r + beta p."""
    r = ops.empty_like(b)
    p = ops.empty_like(b)
    Ap = ops.empty_like(b)
    ops.spmv(x, Ap)
    ops.axpy(-1.0, Ap, b, r)
    ops.copy(r, p)
    b_norm2 = math.sqrt(ops.allreduce_sum(ops.dot(b, b)))
    if b_norm2 == 0.0:
        b_norm2 = 1.0
    r_dot = ops.allreduce_sum(ops.dot(r, r))
    if math.sqrt(r_dot) / b_norm2 < tol:
        return {"iters": 0, "residual": math.sqrt(r_dot) / b_norm2, "converged": True}
    for it in range(max_iter):
        ops.spmv(p, Ap)
        pAp = ops.allreduce_sum(ops.dot(p, Ap))
        if abs(pAp) < 1e-300:
            raise RuntimeError("CG: p'Ap is near zero — A may not be SPD")
        alpha = r_dot / pAp
        ops.axpy(alpha, p, x, x)
        ops.axpy(-alpha, Ap, r, r)
        r_dot_new = ops.allreduce_sum(ops.dot(r, r))
        rel_res = math.sqrt(r_dot_new) / b_norm2
        if rel_res < tol:
            return {"iters": it + 1, "residual": rel_res, "converged": True}
        beta = r_dot_new / r_dot
        r_dot = r_dot_new
        ops.axpy2(1.0, r, beta, p, p)
    final = ops.allreduce_sum(ops.dot(r, r))
    return {"iters": max_iter, "residual": math.sqrt(final) / b_norm2, "converged": False}


def dist_spmv(A_dist, x_local, y_local) -> None:
    from ._arrays import device_array
    xt = device_array(x_local, "float64", "x_local")
    yt = device_array(y_local, "float64", "y_local")
    n = A_dist.local_row_end - A_dist.local_row_start
    if xt.shape[0] != n or yt.shape[0] != n:
        raise ValueError("dist_spmv: x_local / y_local length != local rows")
    ops = _ops_for(A_dist)
    ops.spmv(xt, yt)
    torch.cuda.current_stream(yt.device).synchronize()
    _lib.check(_lib.load().nm_check_device_errors(), "dist_spmv")


def _ops_for(A_dist):
    ops = getattr(A_dist, "_ops", None)
    if ops is None:
        ops = DeviceOps(A_dist)
        A_dist._ops = ops
    return ops


def cg_solve(A_dist, b, x, tol: float, max_iter: int) -> dict:
    from ._arrays import device_array, stream_of
    bt = device_array(b, "float64", "b")
    xt = device_array(x, "float64", "x")
    n = A_dist.local_row_end - A_dist.local_row_start
    if bt.shape[0] != n or xt.shape[0] != n:
        raise ValueError("cg_solve: b / x length != local rows")
    if A_dist.n_ghost == 0 and A_dist.total_send == 0 and _world() == 1:
        res = _lib.CgResult()
        _lib.check(_lib.load().nm_dist_cg_single(A_dist._h, bt.data_ptr(), xt.data_ptr(),
                                                 float(tol), int(max_iter), C.byref(res),
                                                 stream_of(xt)), "cg_solve")
        return {"iters": int(res.iters), "residual": float(res.final_res),
                "converged": bool(res.converged)}
    out = cg_distributed(_ops_for(A_dist), bt, xt, float(tol), int(max_iter))
    torch.cuda.current_stream(xt.device).synchronize()
    return out


def _world() -> int:
    if dist is not None and dist.is_available() and dist.is_initialized():
        return dist.get_world_size()
    return 1
