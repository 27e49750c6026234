"""nm_cg_local_static, the CG entry point that allocates nothing, against
nm_cg_local.

Some callers cannot call cudaMalloc when they solve: a process whose device
memory is already claimed by another allocator's pool, or a latency-critical
loop in which cudaMalloc / cudaFree would synchronise the whole device.  They
call nm_cg_local_static, which takes its scratch from a fixed device array in
the library; it must return what nm_cg_local returns.  This file sorts last so
that a run stopping at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from num_b200 import _lib
from num_b200 import generators as gen

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

RTOL = 1e-12  # same tolerance the CG parity tests use for solution agreement


def _solve(name, M, b, x0, tol, max_iter):
    lib = _lib.load()
    x = x0.clone()
    res = _lib.CgResult()
    st = getattr(lib, name)(M._h, b.data_ptr(), x.data_ptr(), float(tol), int(max_iter),
                            C.byref(res), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    _lib.check(st, name)
    return res, x.cpu().numpy()


def _agree(r_s, x_s, r_l, x_l):
    assert r_s.iters == r_l.iters
    assert r_s.converged == r_l.converged
    assert abs(r_s.final_res - r_l.final_res) <= RTOL * abs(r_l.final_res)
    assert np.linalg.norm(x_s - x_l) <= RTOL * np.linalg.norm(x_l)


def _problem(kspmv, A, b):
    M = kspmv.upload_csr(A.row_ptr, A.col_idx, A.values, A.nrows, A.ncols)
    bt = torch.tensor(b, device="cuda")
    x0 = torch.zeros(A.nrows, dtype=torch.float64, device="cuda")
    return M, bt, x0


def test_static_matches_local_two_calls(kspmv, oracle):
    # 256^2 5-point Laplacian, b = A*ones, tol 1e-8: two calls in a row of each.
    A = gen.laplacian_2d(256)
    b = oracle.spmv(A.row_ptr, A.col_idx, A.values, np.ones(A.ncols))
    M, bt, x0 = _problem(kspmv, A, b)
    for _ in range(2):
        r_s, x_s = _solve("nm_cg_local_static", M, bt, x0, 1e-8, 5000)
        r_l, x_l = _solve("nm_cg_local", M, bt, x0, 1e-8, 5000)
        _agree(r_s, x_s, r_l, x_l)
        assert r_s.converged and r_s.iters == 454


def test_static_reuse_across_sizes(kspmv):
    # A different matrix after the first call: the shared scratch keeps the
    # last call's contents, so each call must start from a clean state.
    rng = np.random.default_rng(5)
    for A in (gen.banded_spd(5000, 6, rng), gen.laplacian_3d(30), gen.banded_spd(777, 2, rng)):
        b = rng.standard_normal(A.nrows)
        M, bt, x0 = _problem(kspmv, A, b)
        for _ in range(2):
            r_s, x_s = _solve("nm_cg_local_static", M, bt, x0, 1e-10, 3000)
            r_l, x_l = _solve("nm_cg_local", M, bt, x0, 1e-10, 3000)
            _agree(r_s, x_s, r_l, x_l)
        r_s, _ = _solve("nm_cg_local_static", M, bt, x0, 1e-14, 3)
        r_l, _ = _solve("nm_cg_local", M, bt, x0, 1e-14, 3)
        assert (r_s.iters, r_s.converged) == (r_l.iters, r_l.converged) == (3, 0)


def test_static_rejects_more_rows_than_its_scratch(kspmv):
    A = gen.diagonal(np.ones(262_145))
    M, bt, x0 = _problem(kspmv, A, np.ones(A.nrows))
    with pytest.raises(ValueError, match="exceed the fixed scratch"):
        _solve("nm_cg_local_static", M, bt, x0, 1e-8, 10)


def test_static_leaves_device_free_memory_unchanged(kspmv):
    # The contract itself: once the library's CG code is loaded on the device
    # (one warm-up call), a solve on a matrix it has never seen takes no
    # device memory -- the free-memory figure is the same before and after.
    # nm_cg_local on such a matrix would allocate its workspace (about 2 MB
    # here) and move the figure.
    lib = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    A0 = gen.laplacian_2d(64)
    M0, b0, x0 = _problem(kspmv, A0, np.ones(A0.nrows))
    r0, _ = _solve("nm_cg_local_static", M0, b0, x0, 1e-8, 1000)
    assert r0.converged
    A = gen.laplacian_2d(200)
    M, bt, _ = _problem(kspmv, A, np.ones(A.nrows))
    x = torch.zeros(A.nrows, dtype=torch.float64, device="cuda")
    res = _lib.CgResult()
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        x.zero_()
        st = lib.nm_cg_local_static(M._h, bt.data_ptr(), x.data_ptr(), 1e-8, 5000,
                                    C.byref(res), stream)
        _lib.check(st, "nm_cg_local_static")
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before
    assert res.converged
