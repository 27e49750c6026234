"""The multi-rank path at world size 2 (and 3) on CPU with gloo.

Each process builds its rank's plan with the library's host-only
distribute_csr restatement (nm_dist_plan), exchanges halos with the product's
`halo.exchange` (batched isend/irecv) and runs the product's distributed CG
recurrence (`halo.cg_distributed`).  The kernels are replaced by CPU stand-ins
from the oracle (this machine has no GPU); the host logic under test is the
plan, the exchange schedule and the CG control flow with its all-reduces.
Results must equal the oracle's single-process restatement with P virtual
ranks: the halos bit for bit; the CG iteration counts exactly, and at two
ranks the iterates bit for bit (a 2-rank all-reduce sums in the oracle's rank
order; with more ranks the order is the collective's, as with MPI_Allreduce).
"""
import datetime
import os
import socket
import traceback

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _row_subset(rp, ci, v, rows):
    """CSR of the given rows of (rp, ci, v), rows in the given order."""
    lens = (rp[rows + 1] - rp[rows]).astype(np.int64)
    srp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    take = np.concatenate([np.arange(rp[r], rp[r + 1]) for r in rows]) if len(rows) else \
        np.empty(0, np.int64)
    return srp, ci[take].astype(np.int32), v[take]


class CpuOps:
    """Oracle-backed stand-ins for DeviceOps (same interface and the same
    overlapped order: the exchange is posted, the rows without ghost columns
    are multiplied from x_local, then the exchange completes and the rows with
    ghost columns are multiplied from x_ext)."""

    def __init__(self, plan, local_csr, oracle, halo):
        self.plan, self.csr, self.o, self.halo = plan, local_csr, oracle, halo
        self.send = torch.zeros(max(plan.total_send, 1), dtype=torch.float64)
        self.recv = torch.zeros(max(plan.n_ghost, 1), dtype=torch.float64)
        rp, ci, v = local_csr
        n = plan.local_n
        ghost = np.array([bool((ci[rp[i]:rp[i + 1]] >= n).any()) for i in range(n)], bool)
        self.irows, self.brows = np.flatnonzero(~ghost), np.flatnonzero(ghost)
        self.icsr = _row_subset(rp, ci, v, self.irows)
        self.bcsr = _row_subset(rp, ci, v, self.brows)

    def spmv(self, x, y):
        p = self.plan
        self.send[: p.total_send] = torch.from_numpy(self.o.halo_pack(p.send_idx, x.numpy()))
        reqs = self.halo.exchange_start(p, self.send, self.recv)
        out = np.empty(p.local_n)
        if len(self.irows):  # while the halo is in flight
            out[self.irows] = self.o.spmv(*self.icsr, x.numpy())
        self.halo.exchange_wait(reqs)
        if len(self.brows):
            x_ext = np.concatenate([x.numpy(), self.recv[: p.n_ghost].numpy()])
            out[self.brows] = self.o.spmv(*self.bcsr, x_ext)
        y.copy_(torch.from_numpy(out))

    def dot(self, x, y):
        return self.o.dot(x.numpy(), y.numpy())

    def allreduce_sum(self, v):
        t = torch.tensor([v], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return float(t.item())

    def axpy(self, a, x, y, z):
        z.copy_(torch.from_numpy(self.o.axpy(a, x.numpy(), y.numpy())))

    def axpy2(self, a, x, b, y, z):
        z.copy_(torch.from_numpy(self.o.axpy2(a, x.numpy(), b, y.numpy())))

    def copy(self, src, dst):
        dst.copy_(src)

    def empty_like(self, v):
        return torch.empty_like(v)


def _worker(rank, size, port, case, outdir):
    try:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=rank, world_size=size,
                                timeout=datetime.timedelta(seconds=60))
        from num_b200 import generators as gen
        from num_b200 import halo
        from oracle import oracle
        A = {"lap1d": lambda: gen.laplacian_1d(100), "lap2d": lambda: gen.laplacian_2d(16),
             "lap3d": lambda: gen.laplacian_3d(7)}[case]()
        plan, local = halo.plan_host(A.row_ptr, A.col_idx, A.values, A.nrows, A.ncols, rank, size)
        ops = CpuOps(plan, local, oracle, halo)
        # one halo exchange of a random vector
        x = np.random.default_rng(7).standard_normal(A.nrows)
        xl = torch.tensor(x[plan.row_start:plan.row_end])
        y = torch.empty_like(xl)
        ops.spmv(xl, y)
        ghosts = ops.recv[: plan.n_ghost].numpy().copy()
        # distributed CG, b = ones, x0 = 0
        b = torch.ones(plan.local_n, dtype=torch.float64)
        xs = torch.zeros(plan.local_n, dtype=torch.float64)
        info = halo.cg_distributed(ops, b, xs, tol=1e-10, max_iter=1000)
        np.savez(os.path.join(outdir, f"r{rank}.npz"), y=y.numpy(), ghosts=ghosts,
                 ghost_ids=plan.ghost_ids, xs=xs.numpy(), iters=info["iters"],
                 res=info["residual"], conv=info["converged"], start=plan.row_start,
                 end=plan.row_end)
        dist.barrier()
        dist.destroy_process_group()
    except Exception:
        with open(os.path.join(outdir, f"r{rank}.err"), "w") as f:
            f.write(traceback.format_exc())
        raise


@pytest.mark.timeout(180)
@pytest.mark.parametrize("case,size", [("lap1d", 2), ("lap2d", 2), ("lap3d", 3)])
def test_gloo_halo_and_cg(tmp_path, nmlib, oracle, case, size):
    from num_b200 import generators as gen
    mp.spawn(_worker, args=(size, _free_port(), case, str(tmp_path)), nprocs=size, join=True)
    A = {"lap1d": lambda: gen.laplacian_1d(100), "lap2d": lambda: gen.laplacian_2d(16),
         "lap3d": lambda: gen.laplacian_3d(7)}[case]()
    x = np.random.default_rng(7).standard_normal(A.nrows)
    parts = oracle.partition(A.row_ptr, A.col_idx, A.values, A.nrows, size)
    y_ref = oracle.dist_spmv(parts, x)
    oinfo, ox = oracle.cg_distributed(parts, np.ones(A.nrows), tol=1e-10, max_iter=1000)
    ys, xs = [], []
    for r in range(size):
        d = np.load(tmp_path / f"r{r}.npz")
        assert np.array_equal(d["ghosts"], x[d["ghost_ids"]])  # received halo == owners' values
        ys.append(d["y"])
        xs.append(d["xs"])
        assert int(d["iters"]) == oinfo["iters"] and bool(d["conv"]) == oinfo["converged"]
        if size == 2:  # a+b is the rank-order sum; with 3 ranks gloo's order differs
            assert float(d["res"]) == oinfo["residual"]
        else:
            assert abs(float(d["res"]) - oinfo["residual"]) <= 1e-12
    assert np.array_equal(np.concatenate(ys), y_ref)
    if size == 2:
        assert np.array_equal(np.concatenate(xs), ox)
    else:
        assert np.linalg.norm(np.concatenate(xs) - ox) <= 1e-12 * np.linalg.norm(ox)
