"""Halo pack / unpack and the distributed SpMV at P virtual ranks on one GPU.

Every virtual rank gets its own library handle (its slice, plan and send
indices on the device); the exchange between them is a device-to-device
loopback copy that follows the plans (what NCCL send/recv would move between
GPUs).  Results must equal the oracle's distributed SpMV, which restates the
reference's partition, ghost lists, pack and scatter.
"""
import ctypes as C

import numpy as np
import pytest

from num_b200 import _lib
from num_b200 import generators as gen

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


class VirtualRank:
    def __init__(self, A, r, P):
        from num_b200.halo import HaloPlan
        lib = _lib.load()
        self.h = C.c_void_p()
        _lib.check(lib.nm_dist_create(A.row_ptr.ctypes.data, A.col_idx.ctypes.data,
                                      A.values.ctypes.data, A.nrows, A.ncols, r, P,
                                      C.byref(self.h)))
        self.plan = HaloPlan.from_handle(self.h, rank=r, size=P)
        p = self.plan
        self.x_ext = torch.zeros(p.local_n + p.n_ghost, dtype=torch.float64, device="cuda")
        self.send = torch.full((max(p.total_send, 1),), float("nan"), dtype=torch.float64,
                               device="cuda")
        self.recv = torch.full((max(p.n_ghost, 1),), float("nan"), dtype=torch.float64,
                               device="cuda")
        self.y = torch.full((max(p.local_n, 1),), float("nan"), dtype=torch.float64, device="cuda")

    def __del__(self):
        _lib.load().nm_dist_destroy(self.h)


def dist_spmv_virtual(ranks, x, split=False):
    """split: each rank multiplies its interior rows from x_local before the
    exchange and its boundary rows from x_ext after it (the overlapped
    order); else the whole slice after the exchange."""
    lib = _lib.load()
    s = torch.cuda.current_stream().cuda_stream
    for vr in ranks:  # fill local part + pack (+ interior rows)
        p = vr.plan
        xl = torch.tensor(x[p.row_start:p.row_end], device="cuda")
        vr.x_ext[: p.local_n].copy_(xl)
        _lib.check(lib.nm_halo_pack(vr.h, xl.data_ptr(), vr.send.data_ptr(), s))
        if split:
            _lib.check(lib.nm_dist_spmv_interior(vr.h, xl.data_ptr(), vr.y.data_ptr(), s))
    for vr in ranks:  # loopback exchange: owner q's segment for r -> r's recv buffer
        p = vr.plan
        for q, cnt, off in zip(p.recv_rank, p.recv_count, p.recv_off):
            qp = ranks[q].plan
            k = list(qp.send_rank).index(p.rank)
            so = int(qp.send_off[k])
            assert int(qp.send_count[k]) == int(cnt)
            vr.recv[int(off):int(off) + int(cnt)].copy_(ranks[q].send[so:so + int(cnt)])
    out = []
    for vr in ranks:
        _lib.check(lib.nm_halo_unpack(vr.h, vr.recv.data_ptr(), vr.x_ext.data_ptr(), s))
        if split:
            _lib.check(lib.nm_dist_spmv_boundary(vr.h, vr.x_ext.data_ptr(), vr.y.data_ptr(), s))
        else:
            _lib.check(lib.nm_dist_spmv_local(vr.h, vr.x_ext.data_ptr(), vr.y.data_ptr(), s))
        out.append(vr.y[: vr.plan.local_n].cpu().numpy())
    return np.concatenate(out)


CASES = [("lap1d_200", lambda: gen.laplacian_1d(200), 10),
         ("lap2d_16", lambda: gen.laplacian_2d(16), 11),
         ("lap3d_12", lambda: gen.laplacian_3d(12), 12),
         ("lcg_3000", lambda: gen.lcg_random(3000)[0], 13)]


@pytest.mark.parametrize("P", [1, 2, 3, 4, 7])
@pytest.mark.parametrize("name,make,seed", CASES, ids=[c[0] for c in CASES])
def test_virtual_rank_dist_spmv(kspmv, oracle, P, name, make, seed):
    A = make()
    x = np.random.default_rng(seed).standard_normal(A.nrows)
    ranks = [VirtualRank(A, r, P) for r in range(P)]
    y = dist_spmv_virtual(ranks, x)
    parts = oracle.partition(A.row_ptr, A.col_idx, A.values, A.nrows, P)
    assert np.array_equal(y, oracle.dist_spmv(parts, x))
    # packed send buffers equal the oracle's pack of the same indices
    for vr, part in zip(ranks, parts):
        p = vr.plan
        if p.total_send:
            xl = x[p.row_start:p.row_end]
            assert np.array_equal(vr.send[: p.total_send].cpu().numpy(),
                                  oracle.halo_pack(part["send_idx"], xl))
    ref = A.to_scipy() @ x
    assert np.linalg.norm(y - ref) / np.linalg.norm(ref) < 1e-13


@pytest.mark.parametrize("P", [1, 2, 3, 7])
@pytest.mark.parametrize("name,make,seed", CASES, ids=[c[0] for c in CASES])
def test_virtual_rank_interior_boundary_split(kspmv, oracle, P, name, make, seed):
    # interior rows before the exchange + boundary rows after it == the
    # whole-slice product, bit for bit, and the oracle's distributed SpMV
    A = make()
    x = np.random.default_rng(seed).standard_normal(A.nrows)
    ranks = [VirtualRank(A, r, P) for r in range(P)]
    y_split = dist_spmv_virtual(ranks, x, split=True)
    y_whole = dist_spmv_virtual(ranks, x)
    assert np.array_equal(y_split, y_whole)
    parts = oracle.partition(A.row_ptr, A.col_idx, A.values, A.nrows, P)
    assert np.array_equal(y_split, oracle.dist_spmv(parts, x))
    lib = _lib.load()
    for vr in ranks:
        ni, nb = C.c_int32(), C.c_int32()
        _lib.check(lib.nm_dist_row_split(vr.h, C.byref(ni), C.byref(nb)))
        assert ni.value + nb.value == vr.plan.local_n
        assert (nb.value == 0) == (vr.plan.n_ghost == 0)


def test_virtual_rank_zero_and_basis(kspmv):
    # tests/test_halo_exchange.py:328-415
    N, P = 60, 4
    A = gen.laplacian_1d(N)
    ranks = [VirtualRank(A, r, P) for r in range(P)]
    assert np.array_equal(dist_spmv_virtual(ranks, np.zeros(N)), np.zeros(N))
    dense = A.to_scipy().toarray()
    for col in sorted({0, N // P - 1, N // P, N - 1}):
        e = np.zeros(N)
        e[col] = 1.0
        assert np.array_equal(dist_spmv_virtual(ranks, e), dense[:, col])


def test_virtual_rank_repeated_bit_identical(kspmv):
    A = gen.laplacian_1d(100)
    x = np.random.default_rng(42).standard_normal(100)
    ranks = [VirtualRank(A, r, 3) for r in range(3)]
    ys = [dist_spmv_virtual(ranks, x) for _ in range(5)]
    assert all(np.array_equal(ys[0], y) for y in ys[1:])
