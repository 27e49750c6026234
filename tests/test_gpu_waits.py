"""Failure detection on the GPU without a fault: a bounded device wait runs
out.  Every spin-wait of the library's kernels gives up after a limit, sets
the device error word and returns; nm_test_wait_timeout runs those wait
routines where the wait cannot complete (one arrival short, nothing else in
flight) with a short limit.  The checks: the call reports NM_ERR_RUNTIME after
about the limit, nm_check_device_errors reports the timeout once and then is
clear, and a normal solve right after is still correct."""
import ctypes as C

import numpy as np
import pytest

from num_b200 import _lib
from num_b200 import generators as gen

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _c1_solve_ok(kspmv, oracle):
    A = gen.laplacian_2d(256)
    b = oracle.spmv(A.row_ptr, A.col_idx, A.values, np.ones(A.ncols))
    M = kspmv.upload_csr(A.row_ptr, A.col_idx, A.values, A.nrows, A.ncols)
    x = torch.zeros(A.nrows, dtype=torch.float64, device="cuda")
    info = kspmv.cg_solve_local(M, torch.tensor(b, device="cuda"), x, tol=1e-8, max_iter=5000)
    assert info["converged"] and info["iters"] == 454
    assert np.abs(x.cpu().numpy() - 1.0).max() < 1e-6


@pytest.mark.parametrize("kind,ctas", [(0, 1), (1, 1), (1, 16), (1, 64)])
def test_bounded_wait_runs_out(kspmv, oracle, kind, ctas):
    lib = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    assert lib.nm_check_device_errors() == _lib.NM_OK  # start clean
    waited = C.c_double(0.0)
    limit_ms = 20.0
    st = lib.nm_test_wait_timeout(kind, ctas, limit_ms, C.byref(waited), stream)
    assert st == _lib.NM_ERR_RUNTIME, _lib.last_error()
    assert "gave up" in _lib.last_error()
    assert limit_ms <= waited.value < 1000.0  # ended by the limit, not by a hang
    # reported once, then clear
    assert lib.nm_check_device_errors() == _lib.NM_ERR_RUNTIME
    assert "bounded wait" in _lib.last_error()
    assert lib.nm_check_device_errors() == _lib.NM_OK
    # the context is still usable: a normal solve right after is correct
    _c1_solve_ok(kspmv, oracle)
    assert lib.nm_check_device_errors() == _lib.NM_OK


def test_wait_probe_rejects_bad_arguments(kspmv):
    lib = _lib.load()
    s = torch.cuda.current_stream().cuda_stream
    assert lib.nm_test_wait_timeout(2, 1, 10.0, None, s) == _lib.NM_ERR_INVALID
    assert lib.nm_test_wait_timeout(1, 65, 10.0, None, s) == _lib.NM_ERR_INVALID
    assert lib.nm_test_wait_timeout(0, 1, 0.0, None, s) == _lib.NM_ERR_INVALID
    assert lib.nm_test_wait_timeout(0, 1, 5000.0, None, s) == _lib.NM_ERR_INVALID
