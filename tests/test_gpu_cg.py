"""GPU parity of CG, multi-RHS SpMV and the vector ops against the oracle.

CG bar (from the path's specification): iteration counts identical to the
oracle's restatement of cg_solve_local, the same convergence outcome, and the
same relative residual to within reduction-order noise; every known answer of
the reference's tests/test_cg.cpp holds through the drop-in API."""
import ctypes as C
import json

import numpy as np
import pytest

from conftest import GOLDEN
from num_b200 import generators as gen

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _dev(a):
    return torch.tensor(np.asarray(a, np.float64), device="cuda")


def _cg(kspmv, A, b, x0=None, tol=1e-10, max_iter=1000):
    M = kspmv.upload_csr(A.row_ptr, A.col_idx, A.values, A.nrows, A.ncols)
    bt = _dev(b)
    xt = _dev(np.zeros(A.nrows) if x0 is None else x0)
    info = kspmv.cg_solve_local(M, bt, xt, tol=tol, max_iter=max_iter)
    return info, xt.cpu().numpy()


def test_identity(kspmv):
    b = np.arange(1, 51, dtype=np.float64)
    info, x = _cg(kspmv, gen.diagonal(np.ones(50)), b, tol=1e-12, max_iter=200)
    assert info["converged"] and info["iters"] <= 2
    assert np.linalg.norm(x - b) / np.linalg.norm(b) < 1e-10


def test_2x2(kspmv):
    A = gen.Csr(np.array([0, 2, 4], np.int32), np.array([0, 1, 0, 1], np.int32),
                np.array([4.0, 1.0, 1.0, 3.0]), 2, 2)
    info, x = _cg(kspmv, A, [1.0, 2.0], tol=1e-14, max_iter=100)
    ex = np.array([1 / 11, 7 / 11])
    assert info["converged"] and info["iters"] <= 2
    assert np.linalg.norm(x - ex) / np.linalg.norm(ex) < 1e-10


def test_diagonal(kspmv):
    d = np.arange(1, 101, dtype=np.float64)
    info, x = _cg(kspmv, gen.diagonal(d), np.ones(100), tol=1e-12, max_iter=5000)
    assert info["converged"] and np.linalg.norm(x - 1 / d) / np.linalg.norm(1 / d) < 1e-8


def test_laplacian_1d(kspmv):
    info, _ = _cg(kspmv, gen.laplacian_1d(50), np.ones(50), tol=1e-10, max_iter=500)
    assert info["converged"] and info["residual"] < 1e-10 and info["iters"] > 0


def test_zero_rhs(kspmv):
    info, x = _cg(kspmv, gen.laplacian_1d(20), np.zeros(20), tol=1e-10, max_iter=100)
    assert info == {"iters": 0, "residual": 0.0, "converged": True}
    assert np.array_equal(x, np.zeros(20))


def test_manufactured_sin(kspmv):
    N = 500
    xe = np.sin(np.pi * (np.arange(N) + 1.0) / (N + 1.0))
    b = 2.0 * xe
    b[1:] -= xe[:-1]
    b[:-1] -= xe[1:]
    info, x = _cg(kspmv, gen.laplacian_1d(N), b, tol=1e-10, max_iter=2000)
    assert info["converged"] and np.linalg.norm(x - xe) / np.linalg.norm(xe) < 1e-8


@pytest.mark.parametrize("max_iter", [5, 1, 0, -2])
def test_max_iter(kspmv, oracle, max_iter):
    A = gen.laplacian_1d(50)
    info, x = _cg(kspmv, A, np.ones(50), tol=1e-14, max_iter=max_iter)
    oinfo, ox = oracle.cg_local(A.row_ptr, A.col_idx, A.values, np.ones(50), tol=1e-14,
                                max_iter=max_iter)
    assert info["iters"] == oinfo["iters"] == max_iter and not info["converged"]
    assert abs(info["residual"] - oinfo["residual"]) <= 1e-12 * oinfo["residual"]
    assert np.allclose(x, ox, rtol=1e-12, atol=1e-14)


def test_repeated_solves_bit_identical(kspmv):
    A = gen.laplacian_1d(30)
    M = kspmv.upload_csr(A.row_ptr, A.col_idx, A.values, 30, 30)
    b = _dev(np.ones(30))
    sols = []
    for _ in range(3):
        x = torch.zeros(30, dtype=torch.float64, device="cuda")
        kspmv.cg_solve_local(M, b, x, tol=1e-12, max_iter=500)
        sols.append(x.cpu().numpy())
    assert np.array_equal(sols[0], sols[1]) and np.array_equal(sols[0], sols[2])


def test_c1_iteration_parity(kspmv, oracle):
    # 256^2 Laplacian, b = A*ones, x0 = 0, tol 1e-8: 454 iterations, like the
    # oracle and SciPy; true residual < 1e-8.
    probe = json.loads((GOLDEN / "c1_probe.json").read_text())
    A = gen.laplacian_2d(256)
    b = oracle.spmv(A.row_ptr, A.col_idx, A.values, np.ones(A.ncols))
    info, x = _cg(kspmv, A, b, tol=1e-8, max_iter=5000)
    oinfo, ox = oracle.cg_local(A.row_ptr, A.col_idx, A.values, b, tol=1e-8, max_iter=5000)
    assert info["iters"] == oinfo["iters"] == probe["scipy_cg_iters"] == 454
    assert info["converged"]
    assert abs(info["residual"] - oinfo["residual"]) < 1e-6 * oinfo["residual"]
    true_rel = np.linalg.norm(b - A.to_scipy() @ x) / np.linalg.norm(b)
    assert true_rel < 1e-8
    assert np.linalg.norm(x - ox) / np.linalg.norm(ox) < 1e-9


@pytest.mark.parametrize("name", ["laplacian_2d", "laplacian_3d", "random_sparse"])
def test_vs_scipy_cg(kspmv, oracle, name):
    # test_accuracy.py:160-195: solution vs spla.cg(rtol=1e-12), rel < 1e-6
    p = np.load(GOLDEN / "scipy_pins.npz")
    rp, ci, v = p[f"{name}__indptr"], p[f"{name}__indices"], p[f"{name}__data"]
    n = rp.shape[0] - 1
    A = gen.Csr(rp, ci, v, n, n)
    info, x = _cg(kspmv, A, np.ones(n), tol=1e-10, max_iter=5000)
    oinfo, _ = oracle.cg_local(rp, ci, v, np.ones(n), tol=1e-10, max_iter=5000)
    assert info["converged"] and info["iters"] == oinfo["iters"]
    ref = p[f"{name}__cg_x"]
    assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 1e-6


def test_nonzero_initial_guess(kspmv, oracle):
    A = gen.laplacian_3d(20)
    rng = np.random.default_rng(8)
    b, x0 = rng.standard_normal(A.nrows), rng.standard_normal(A.nrows)
    info, x = _cg(kspmv, A, b, x0=x0, tol=1e-9, max_iter=3000)
    oinfo, ox = oracle.cg_local(A.row_ptr, A.col_idx, A.values, b, x0=x0, tol=1e-9, max_iter=3000)
    assert info["iters"] == oinfo["iters"] and info["converged"]
    assert np.linalg.norm(x - ox) / np.linalg.norm(ox) < 1e-8


def test_singular_matrix_runs_to_max_iter(kspmv, oracle):
    # cg_solve_local has no breakdown guard: p.Ap = 0 gives NaN and the loop
    # runs to max_iter, returning converged=False.
    A = gen.Csr(np.arange(5, dtype=np.int32), np.arange(4, dtype=np.int32), np.zeros(4), 4, 4)
    info, _ = _cg(kspmv, A, np.ones(4), max_iter=7)
    oinfo, _ = oracle.cg_local(A.row_ptr, A.col_idx, A.values, np.ones(4), max_iter=7)
    assert info["iters"] == oinfo["iters"] == 7 and not info["converged"]
    assert np.isnan(info["residual"]) and np.isnan(oinfo["residual"])


def test_dist_single_rank_and_guard(kspmv, oracle):
    A = gen.laplacian_2d(40)
    D = kspmv.distribute_csr(A.row_ptr, A.col_idx, A.values, A.nrows, A.ncols)
    assert (D.global_nrows, D.local_row_start, D.local_row_end) == (1600, 0, 1600)
    x = np.random.default_rng(3).standard_normal(A.nrows)
    y = torch.empty(A.nrows, dtype=torch.float64, device="cuda")
    kspmv.dist_spmv(D, _dev(x), y)
    assert np.array_equal(y.cpu().numpy(), oracle.spmv(A.row_ptr, A.col_idx, A.values, x))
    b = np.ones(A.nrows)
    xt = torch.zeros(A.nrows, dtype=torch.float64, device="cuda")
    info = kspmv.cg_solve(D, _dev(b), xt, tol=1e-10, max_iter=1000)
    oinfo, _ = oracle.cg_local(A.row_ptr, A.col_idx, A.values, b, tol=1e-10, max_iter=1000)
    assert info["iters"] == oinfo["iters"] and info["converged"]
    Z = gen.Csr(np.arange(4, dtype=np.int32), np.arange(3, dtype=np.int32), np.zeros(3), 3, 3)
    DZ = kspmv.distribute_csr(Z.row_ptr, Z.col_idx, Z.values, 3, 3)
    with pytest.raises(RuntimeError, match="near zero"):
        kspmv.cg_solve(DZ, _dev(np.ones(3)), torch.zeros(3, dtype=torch.float64, device="cuda"))


# ---- multi-RHS SpMV -------------------------------------------------------------

def test_batch_identity_columns(kspmv):
    # tests/test_spmv_kernel.cpp:134-159
    A = gen.tridiag4()
    M = kspmv.upload_csr(A.row_ptr, A.col_idx, A.values, 4, 4)
    X = _dev(np.eye(4))
    Y = torch.empty(4, 4, dtype=torch.float64, device="cuda")
    kspmv.batch_spmv(M, X, Y)
    assert np.array_equal(Y.cpu().numpy(), A.to_scipy().toarray())


@pytest.mark.parametrize("k", [1, 2, 3, 4, 5, 8, 31, 32, 33, 64, 100, 128, 257, 300])
def test_batch_bit_exact(kspmv, oracle, k):
    A = gen.power_law(5000, seed=k)
    M = kspmv.upload_csr(A.row_ptr, A.col_idx, A.values, A.nrows, A.ncols)
    X = np.random.default_rng(k).standard_normal((A.ncols, k))
    Y = torch.empty(A.nrows, k, dtype=torch.float64, device="cuda")
    kspmv.batch_spmv(M, _dev(X), Y)
    assert np.array_equal(Y.cpu().numpy(), oracle.batch_spmv(A.row_ptr, A.col_idx, A.values, X))


def test_batch_laplacian_k128_bit_exact(kspmv, oracle):
    # 7-nonzero rows, one warp per row, X rows shared by neighbouring rows
    A = gen.laplacian_3d(24)
    M = kspmv.upload_csr(A.row_ptr, A.col_idx, A.values, A.nrows, A.ncols)
    X = np.random.default_rng(128).uniform(-1, 1, (A.ncols, 128))
    Y = torch.empty(A.nrows, 128, dtype=torch.float64, device="cuda")
    for _ in range(2):
        kspmv.batch_spmv(M, _dev(X), Y)
        assert np.array_equal(Y.cpu().numpy(),
                              oracle.batch_spmv(A.row_ptr, A.col_idx, A.values, X))


def test_batch_errors(kspmv):
    A = gen.tridiag4()
    M = kspmv.upload_csr(A.row_ptr, A.col_idx, A.values, 4, 4)
    with pytest.raises(ValueError, match=r"X.shape\[0\]"):
        kspmv.batch_spmv(M, _dev(np.zeros((5, 2))), _dev(np.zeros((4, 2))))
    with pytest.raises(ValueError, match="Y must be"):
        kspmv.batch_spmv(M, _dev(np.zeros((4, 2))), _dev(np.zeros((4, 3))))


# ---- vector ops through the C ABI ----------------------------------------------------

def test_vector_ops_bit_exact(nmlib, kspmv, oracle):
    rng = np.random.default_rng(12)
    n = 1_000_003
    x, y = rng.standard_normal(n), rng.standard_normal(n)
    xt, yt, zt = _dev(x), _dev(y), torch.empty(n, dtype=torch.float64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    assert nmlib.nm_axpy(n, 0.37, xt.data_ptr(), yt.data_ptr(), zt.data_ptr(), s) == 0
    torch.cuda.synchronize()
    assert np.array_equal(zt.cpu().numpy(), oracle.axpy(0.37, x, y))
    assert nmlib.nm_axpy2(n, 0.37, xt.data_ptr(), -1.9, yt.data_ptr(), zt.data_ptr(), s) == 0
    torch.cuda.synchronize()
    assert np.array_equal(zt.cpu().numpy(), oracle.axpy2(0.37, x, -1.9, y))
    # aliasing z == x (as CG's x = alpha*p + x)
    assert nmlib.nm_axpy(n, 2.0, yt.data_ptr(), xt.data_ptr(), xt.data_ptr(), s) == 0
    torch.cuda.synchronize()
    assert np.array_equal(xt.cpu().numpy(), oracle.axpy(2.0, y, x))
    d1, d2 = C.c_double(), C.c_double()
    assert nmlib.nm_dot(n, xt.data_ptr(), yt.data_ptr(), C.byref(d1), s) == 0
    assert nmlib.nm_dot(n, xt.data_ptr(), yt.data_ptr(), C.byref(d2), s) == 0
    xn = xt.cpu().numpy()
    ref = oracle.dot(xn, y)
    assert d1.value == d2.value  # deterministic
    assert abs(d1.value - ref) <= 1e-12 * float(np.abs(xn) @ np.abs(y))
    nrm = C.c_double()
    assert nmlib.nm_norm2(n, yt.data_ptr(), C.byref(nrm), s) == 0
    assert abs(nrm.value - oracle.norm2(y)) < 1e-13 * oracle.norm2(y)
    assert nmlib.nm_fill(n, 2.5, zt.data_ptr(), s) == 0
    assert nmlib.nm_scale(n, -2.0, zt.data_ptr(), s) == 0
    torch.cuda.synchronize()
    assert np.all(zt.cpu().numpy() == -5.0)
    assert nmlib.nm_copy(n, yt.data_ptr(), zt.data_ptr(), s) == 0
    torch.cuda.synchronize()
    assert np.array_equal(zt.cpu().numpy(), y)
    zero = C.c_double(7.0)
    assert nmlib.nm_dot(0, None, None, C.byref(zero), s) == 0 and zero.value == 0.0


def _arrow_spd(n, rng):
    """Row 0 (and column 0) dense, the rest diagonal: row 0 is one block with
    more nonzeros than a tile (the long-row path)."""
    u = 0.01 * rng.uniform(-1, 1, n)
    d = 1.0 + rng.uniform(0, 1, n)
    d[0] = 1.0 + np.abs(u[1:]).sum()
    rp = np.empty(n + 1, np.int32)
    rp[0], rp[1] = 0, n
    rp[2:] = n + 2 * np.arange(1, n, dtype=np.int64)
    ci = np.empty(n + 2 * (n - 1), np.int32)
    v = np.empty(ci.shape[0])
    ci[:n] = np.arange(n)
    v[:n] = np.concatenate([[d[0]], u[1:]])
    ci[n::2], ci[n + 1::2] = 0, np.arange(1, n)
    v[n::2], v[n + 1::2] = u[1:], d[1:]
    return gen.Csr(rp, ci, v, n, n)


# Mode 1 runs the cluster solve where it applies (the 256^2 Laplacian), else
# the TMA-pipelined persistent solve where its grid is co-resident, else the
# resident solve where that applies (rows of <= 8 nonzeros, whole 256-row
# tiles); modes 3 and 4 force the resident and the cluster solve where they
# apply; mode 2 forces the TMA-pipelined one, which runs in its two-barrier form (direction formed
# inside the SpMV) while the SpMV grid fits it -- the 256^2 and 40^3
# Laplacians, the 30,000-row banded system (scattered off-band columns: the
# gather path) and the arrow matrix (a long row) -- and in its three-barrier
# form for the 64^3 Laplacian and the 48^3 variable-coefficient system (grids
# of 444 and 432 CTAs); mode 0 is the CUDA-graph path; the 300,000-row banded
# system takes the graph path in every mode.
@pytest.mark.parametrize("case", ["lap2d_256", "lap3d_40", "banded_30k", "arrow_20k",
                                  "lap3d_64", "varcoef_48", "banded"])
def test_persistent_and_graph_paths_bit_identical(kspmv, nmlib, case):
    # nm_cg_local runs the whole solve in one cooperative launch by default;
    # the three-kernel CUDA-graph path must give the same bits.
    rng = np.random.default_rng(21)
    if case == "lap2d_256":
        A = gen.laplacian_2d(256)
    elif case == "lap3d_40":
        A = gen.laplacian_3d(40)
    elif case == "banded_30k":
        A = gen.banded_spd(30_000, 5, rng)
    elif case == "arrow_20k":
        A = _arrow_spd(20_000, rng)
    elif case == "lap3d_64":
        A = gen.laplacian_3d(64)
    elif case == "varcoef_48":
        A, _ = gen.varcoef_poisson_3d(48, seed=3)
    else:
        A = gen.banded_spd(300_000, 5, rng)
    b = torch.tensor(rng.standard_normal(A.nrows), device="cuda")
    M = kspmv.upload_csr(A.row_ptr, A.col_idx, A.values, A.nrows, A.ncols)
    out = []
    try:
        for persistent in (1, 0, 2, 3, 4, 1):
            nmlib.nm_cg_set_persistent(persistent)
            x = torch.zeros(A.nrows, dtype=torch.float64, device="cuda")
            info = kspmv.cg_solve_local(M, b, x, tol=1e-9, max_iter=3000)
            out.append((info, x.cpu().numpy()))
    finally:
        nmlib.nm_cg_set_persistent(1)
    for info, x in out[1:]:
        assert info == out[0][0]
        assert np.array_equal(x, out[0][1])
    assert out[0][0]["converged"]


@pytest.mark.parametrize("offset", [0, 1])
def test_large_system_graph_path(kspmv, oracle, offset):
    # 600^2 Laplacian (360,000 rows, above the persistent solve's limit, so
    # the CUDA-graph path), x 16-byte aligned or one element off: the same
    # iteration count as the oracle (+-1) and solutions within 1e-9 of it.
    A = gen.laplacian_2d(600)
    b = np.random.default_rng(31).standard_normal(A.nrows)
    M = kspmv.upload_csr(A.row_ptr, A.col_idx, A.values, A.nrows, A.ncols)
    buf = torch.zeros(A.nrows + 1, dtype=torch.float64, device="cuda")
    x = buf[offset:offset + A.nrows]
    info = kspmv.cg_solve_local(M, torch.tensor(b, device="cuda"), x, tol=1e-8, max_iter=5000)
    oinfo, ox = oracle.cg_local(A.row_ptr, A.col_idx, A.values, b, tol=1e-8, max_iter=5000)
    assert info["converged"] and abs(info["iters"] - oinfo["iters"]) <= 1
    xs = x.cpu().numpy()
    assert np.linalg.norm(xs - ox) <= 1e-9 * np.linalg.norm(ox)


def _tridiag(n):
    # 1-D Laplacian: 2 on the diagonal, -1 beside it (3 nonzeros per row)
    rows = np.repeat(np.arange(n), 3)
    cols = (rows + np.tile([-1, 0, 1], n))
    keep = (cols >= 0) & (cols < n)
    rows, cols = rows[keep], cols[keep]
    vals = np.where(rows == cols, 2.0, -1.0)
    rp = np.zeros(n + 1, np.int32)
    np.add.at(rp, rows + 1, 1)
    return gen.Csr(np.cumsum(rp, dtype=np.int32), cols.astype(np.int32), vals, n, n)


def _shifted_laplacian_2d(L, shift):
    # 2-D Laplacian with shift(i) added to the diagonal of row i
    A = gen.laplacian_2d(L)
    v = A.values.copy()
    for i in range(A.nrows):
        for z in range(A.row_ptr[i], A.row_ptr[i + 1]):
            if A.col_idx[z] == i:
                v[z] += shift(i)
    return gen.Csr(A.row_ptr, A.col_idx, v, A.nrows, A.ncols)


@pytest.mark.parametrize("case", ["c1_256sq", "lap3d_32", "lap2d_40", "tridiag_3000",
                                  "intdiag_100", "randdiag_120"])
def test_cluster_solve(kspmv, nmlib, oracle, case):
    # Systems the 16-CTA cluster solve takes (where the device schedules it):
    # the 256^2 Laplacian (5 nonzeros, 1,024 threads x 4 rows: the full
    # cluster), 32^3 (7 nonzeros), 40^2 (a partial last tile) and a 1-D
    # Laplacian (3 nonzeros), whose few distinct values the CTAs hold as
    # dictionary indices; a 100^2 Laplacian with integer diagonals 4..10
    # (floats exactly, more than 4 distinct: held as floats) and a 120^2 one
    # with random diagonals (held as doubles, 512 threads).  The graph path's
    # bits and the oracle's iteration count (454 on the 256^2 system, exactly).
    import ctypes as C
    rng = np.random.default_rng(41)
    A = {"c1_256sq": lambda: gen.laplacian_2d(256), "lap3d_32": lambda: gen.laplacian_3d(32),
         "lap2d_40": lambda: gen.laplacian_2d(40), "tridiag_3000": lambda: _tridiag(3000),
         "intdiag_100": lambda: _shifted_laplacian_2d(100, lambda i: float(i % 7)),
         "randdiag_120": lambda: _shifted_laplacian_2d(120, lambda i: rng.uniform(0, 1))}[case]()
    b = torch.tensor(oracle.spmv(A.row_ptr, A.col_idx, A.values, np.ones(A.ncols)),
                     device="cuda")
    M = kspmv.upload_csr(A.row_ptr, A.col_idx, A.values, A.nrows, A.ncols)
    out = []
    try:
        for mode in (4, 0, 4):
            nmlib.nm_cg_set_persistent(mode)
            x = torch.zeros(A.nrows, dtype=torch.float64, device="cuda")
            info = kspmv.cg_solve_local(M, b, x, tol=1e-8, max_iter=20000)
            path = C.c_int32(-1)
            nmlib.nm_cg_last_path(M._h, C.byref(path))
            out.append((info, x.cpu().numpy(), path.value))
    finally:
        nmlib.nm_cg_set_persistent(1)
    assert out[0][2] in (0, 4) and out[1][2] == 0 and out[2][2] == out[0][2]
    oinfo, _ = oracle.cg_local(A.row_ptr, A.col_idx, A.values, b.cpu().numpy(), tol=1e-8,
                               max_iter=20000)
    for info, x, _ in out:
        assert info["converged"] and info["iters"] == out[1][0]["iters"]
        assert info["residual"] == out[1][0]["residual"]
        assert np.array_equal(x, out[1][1])
    assert abs(out[1][0]["iters"] - oinfo["iters"]) <= 1
    if case == "c1_256sq":
        assert out[1][0]["iters"] == 454
