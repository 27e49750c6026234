"""Pins the CPU oracle before it is trusted as the checker of the device code.

Known answers come from the reference's own tests (read as text; cited per
case) and from SciPy -- the reference's accuracy oracle -- evaluated on the
reference's own generators by tests/golden/make_golden.py.
"""
import json
import math
from fractions import Fraction

import numpy as np
import pytest

from conftest import GOLDEN
from num_b200 import generators as gen


# ---- SpMV known answers: tests/test_spmv_kernel.cpp ---------------------------

def test_tridiag4_spmv(oracle):
    # tests/test_spmv_kernel.cpp:74-89: x=[1,2,3,4] against dense_spmv, |err| < 1e-13
    A = gen.tridiag4()
    y = oracle.spmv(A.row_ptr, A.col_idx, A.values, np.array([1.0, 2.0, 3.0, 4.0]))
    assert np.array_equal(y, [0.0, 0.0, 0.0, 5.0])


def test_identity_spmv(oracle):
    # tests/test_spmv_kernel.cpp:114-130: identity N=100, x=0.1*i, max err < 1e-14
    A = gen.diagonal(np.ones(100))
    x = np.arange(100) * 0.1
    assert np.array_equal(oracle.spmv(A.row_ptr, A.col_idx, A.values, x), x)


def test_batch_identity_columns(oracle):
    # tests/test_spmv_kernel.cpp:134-159: X = I4 gives the columns of A
    A = gen.tridiag4()
    Y = oracle.batch_spmv(A.row_ptr, A.col_idx, A.values, np.eye(4))
    assert np.array_equal(Y, A.to_scipy().toarray())


def test_lcg_random_matches_dense_serial(oracle):
    # tests/test_spmv_kernel.cpp:163-210: LCG matrix (unsorted, repeated
    # columns possible) vs the serial host loop, rel err < 1e-12
    A, x = gen.lcg_random()
    assert A.nnz > 60000 and A.nrows == 10000
    y = oracle.spmv(A.row_ptr, A.col_idx, A.values, x)
    ref = np.zeros(A.nrows)
    for i in range(A.nrows):
        acc = 0.0
        for j in range(A.row_ptr[i], A.row_ptr[i + 1]):
            acc += A.values[j] * x[A.col_idx[j]]
        ref[i] = acc
    assert np.array_equal(y, ref)  # same serial order => identical bits


def test_omp_spmv_bit_identical(oracle):
    A = gen.laplacian_3d(20)
    x = np.random.default_rng(5).uniform(-1, 1, A.ncols)
    assert np.array_equal(oracle.spmv(*A.astuple()[:3], x),
                          oracle.spmv(*A.astuple()[:3], x, threads=True))


# ---- CG known answers: tests/test_cg.cpp ----------------------------------------

def test_cg_identity(oracle):
    # tests/test_cg.cpp:153-181
    A = gen.diagonal(np.ones(50))
    b = np.arange(1, 51, dtype=np.float64)
    info, x = oracle.cg_local(A.row_ptr, A.col_idx, A.values, b, tol=1e-12, max_iter=200)
    assert info["converged"] and info["iters"] <= 2
    assert np.linalg.norm(x - b) / np.linalg.norm(b) < 1e-10


def test_cg_2x2(oracle):
    # tests/test_cg.cpp:185-212: [[4,1],[1,3]] x = [1,2] -> [1/11, 7/11]
    rp = np.array([0, 2, 4], np.int32)
    ci = np.array([0, 1, 0, 1], np.int32)
    v = np.array([4.0, 1.0, 1.0, 3.0])
    info, x = oracle.cg_local(rp, ci, v, np.array([1.0, 2.0]), tol=1e-14, max_iter=100)
    ex = np.array([1 / 11, 7 / 11])
    assert info["converged"] and info["iters"] <= 2
    assert np.linalg.norm(x - ex) / np.linalg.norm(ex) < 1e-10


def test_cg_diagonal(oracle):
    # tests/test_cg.cpp:216-240
    d = np.arange(1, 101, dtype=np.float64)
    A = gen.diagonal(d)
    info, x = oracle.cg_local(A.row_ptr, A.col_idx, A.values, np.ones(100), tol=1e-12, max_iter=5000)
    assert info["converged"]
    assert np.linalg.norm(x - 1 / d) / np.linalg.norm(1 / d) < 1e-8


def test_cg_laplacian_convergence(oracle):
    # tests/test_cg.cpp:244-269
    A = gen.laplacian_1d(50)
    info, _ = oracle.cg_local(A.row_ptr, A.col_idx, A.values, np.ones(50), tol=1e-10, max_iter=500)
    assert info["converged"] and info["residual"] < 1e-10 and info["iters"] > 0


def test_cg_zero_rhs(oracle):
    # tests/test_cg.cpp:273-291: zero iterations, residual exactly 0.0
    A = gen.laplacian_1d(20)
    info, _ = oracle.cg_local(A.row_ptr, A.col_idx, A.values, np.zeros(20), tol=1e-10, max_iter=100)
    assert info == {"iters": 0, "residual": 0.0, "converged": True}


def test_cg_manufactured_sin(oracle):
    # tests/test_cg.cpp:295-326
    N = 500
    A = gen.laplacian_1d(N)
    xe = np.sin(np.pi * (np.arange(N) + 1.0) / (N + 1.0))
    b = 2.0 * xe
    b[1:] -= xe[:-1]
    b[:-1] -= xe[1:]
    info, x = oracle.cg_local(A.row_ptr, A.col_idx, A.values, b, tol=1e-10, max_iter=2000)
    assert info["converged"]
    assert np.linalg.norm(x - xe) / np.linalg.norm(xe) < 1e-8


def test_cg_max_iter(oracle):
    # tests/test_cg.cpp:330-347
    A = gen.laplacian_1d(50)
    info, _ = oracle.cg_local(A.row_ptr, A.col_idx, A.values, np.ones(50), tol=1e-14, max_iter=5)
    assert info["iters"] == 5 and not info["converged"]


def test_cg_repeated_bit_identical(oracle):
    # tests/test_cg.cpp:422-450
    A = gen.laplacian_1d(30)
    xs = [oracle.cg_local(A.row_ptr, A.col_idx, A.values, np.ones(30), tol=1e-12, max_iter=500)[1]
          for _ in range(3)]
    assert np.array_equal(xs[0], xs[1]) and np.array_equal(xs[0], xs[2])


def test_cg_zero_and_negative_max_iter(oracle):
    # cg_solver.hpp:161-195: the loop never runs; iters = max_iter
    A = gen.laplacian_1d(10)
    for m in (0, -3):
        info, x = oracle.cg_local(A.row_ptr, A.col_idx, A.values, np.ones(10), max_iter=m)
        assert info["iters"] == m and not info["converged"]
        assert np.array_equal(x, np.zeros(10))


def test_dist_cg_one_dimensional(oracle):
    # tests/test_cg.cpp:351-418 at 2..5 virtual ranks: true residual < 1e-8
    A = gen.laplacian_1d(100)
    for P in (2, 3, 5):
        parts = oracle.partition(A.row_ptr, A.col_idx, A.values, 100, P)
        info, x = oracle.cg_distributed(parts, np.ones(100), tol=1e-10, max_iter=1000)
        r = np.ones(100) - A.to_scipy() @ x
        assert info["converged"] and np.linalg.norm(r) / 10.0 < 1e-8


def test_dist_cg_breakdown_guard(oracle):
    # cg_solver.hpp:84-85: zero matrix -> p'Ap == 0 raises
    rp = np.array([0, 1, 2], np.int32)
    parts = oracle.partition(rp, np.array([0, 1], np.int32), np.zeros(2), 2, 1)
    with pytest.raises(RuntimeError, match="p'Ap is near zero"):
        oracle.cg_distributed(parts, np.ones(2))


# ---- Partition known answers: tests/test_halo_exchange.py ----------------------------

@pytest.mark.parametrize("P", [1, 2, 3, 4, 5, 8])
def test_row_partition_n127(oracle, P):
    # tests/test_halo_exchange.py:89-143: contiguous, ordered, covers [0,127), max-min <= 1
    r = [oracle.row_range(127, P, k) for k in range(P)]
    assert r[0][0] == 0 and r[-1][1] == 127
    assert all(r[k][1] == r[k + 1][0] for k in range(P - 1))
    sizes = [e - s for s, e in r]
    assert max(sizes) - min(sizes) <= 1


@pytest.mark.parametrize("P", [2, 3, 4])
def test_dist_spmv_ghosts(oracle, P):
    # tests/test_halo_exchange.py:148-271: 1-D N=200 and 2-D 16x16 against SciPy
    for A, seed in ((gen.laplacian_1d(200), 10), (gen.laplacian_2d(16), 11)):
        x = np.random.default_rng(seed).standard_normal(A.nrows)
        parts = oracle.partition(A.row_ptr, A.col_idx, A.values, A.nrows, P)
        y = oracle.dist_spmv(parts, x)
        ref = A.to_scipy() @ x
        assert np.linalg.norm(y - ref) / np.linalg.norm(ref) < 1e-14


def test_dist_spmv_zero_and_basis(oracle):
    # tests/test_halo_exchange.py:328-415: x=0 -> y=0; e_j -> column j
    N, P = 60, 4
    A = gen.laplacian_1d(N)
    parts = oracle.partition(A.row_ptr, A.col_idx, A.values, N, P)
    assert np.array_equal(oracle.dist_spmv(parts, np.zeros(N)), np.zeros(N))
    dense = A.to_scipy().toarray()
    for col in sorted({0, N // P - 1, N // P, N - 1}):
        e = np.zeros(N)
        e[col] = 1.0
        assert np.array_equal(oracle.dist_spmv(parts, e), dense[:, col])


def test_ghost_lists_one_dimensional(oracle):
    # For the 1-D Laplacian rank r needs the last entry of r-1 and the first of r+1.
    parts = oracle.partition(*gen.laplacian_1d(12).astuple()[:3], 12, 3)
    assert parts[1]["recv"] == [(0, [3], 0), (2, [8], 1)]
    assert parts[1]["send"] == [(0, [4]), (2, [7])]
    assert list(parts[1]["send_idx"]) == [0, 3]
    assert parts[0]["recv"] == [(1, [4], 0)] and parts[2]["recv"] == [(1, [7], 0)]


# ---- SciPy pins (the reference's verify_accuracy oracle) -----------------------------

@pytest.fixture(scope="module")
def pins():
    return np.load(GOLDEN / "scipy_pins.npz")


@pytest.mark.parametrize("name", ["laplacian_2d", "laplacian_3d", "random_sparse", "lattice_gauge"])
def test_oracle_spmv_vs_scipy(oracle, pins, name):
    # verify_accuracy.py:67-90 / test_accuracy.py:85-119: rel err < 1e-10
    y = oracle.spmv(pins[f"{name}__indptr"], pins[f"{name}__indices"], pins[f"{name}__data"],
                    pins[f"{name}__x"])
    ref = pins[f"{name}__y"]
    assert np.linalg.norm(y - ref) / np.linalg.norm(ref) < 1e-14


@pytest.mark.parametrize("name", ["laplacian_2d", "laplacian_3d", "random_sparse"])
def test_oracle_cg_vs_scipy(oracle, pins, name):
    # test_accuracy.py:160-195: CG solution vs spla.cg(rtol=1e-12), rel err < 1e-6
    rp, ci, v = pins[f"{name}__indptr"], pins[f"{name}__indices"], pins[f"{name}__data"]
    b = np.ones(rp.shape[0] - 1)
    info, x = oracle.cg_local(rp, ci, v, b, tol=1e-10, max_iter=5000)
    ref = pins[f"{name}__cg_x"]
    assert info["converged"]
    assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 1e-6


def test_oracle_c1_probe(oracle):
    # 256^2 5-point Laplacian: SpMV norm and CG iteration count vs SciPy's.
    probe = json.loads((GOLDEN / "c1_probe.json").read_text())
    A = gen.laplacian_2d(256)
    x = np.random.default_rng(0).uniform(-1.0, 1.0, A.ncols)
    y = oracle.spmv(A.row_ptr, A.col_idx, A.values, x)
    assert abs(np.linalg.norm(y) - probe["spmv_y_norm2"]) < 1e-12 * probe["spmv_y_norm2"]
    b = oracle.spmv(A.row_ptr, A.col_idx, A.values, np.ones(A.ncols))
    info, xs = oracle.cg_local(A.row_ptr, A.col_idx, A.values, b, tol=1e-8, max_iter=5000)
    assert info["converged"] and info["iters"] == probe["scipy_cg_iters"] == 454
    true_rel = np.linalg.norm(b - A.to_scipy() @ xs) / np.linalg.norm(b)
    assert true_rel < 1e-8
    assert abs(true_rel - probe["scipy_cg_true_relres"]) < 1e-3 * probe["scipy_cg_true_relres"]


def test_oracle_pcg_jacobi(oracle):
    A, b = gen.varcoef_poisson_3d(12, seed=3)
    info, x = oracle.pcg_jacobi(A.row_ptr, A.col_idx, A.values, b, tol=1e-10, max_iter=2000)
    r = b - A.to_scipy() @ x
    assert info["converged"] and np.linalg.norm(r) / np.linalg.norm(b) < 1e-9
    info0, _ = oracle.cg_local(A.row_ptr, A.col_idx, A.values, b, tol=1e-10, max_iter=2000)
    assert info["iters"] < info0["iters"]  # the preconditioner helps on variable coefficients


def _fma(a, b, c):
    # exactly rounded a*b + c: exact rational arithmetic, one rounding (int / int
    # true division is correctly rounded in CPython)
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def test_axpy_ops_fma_semantics(oracle):
    rng = np.random.default_rng(3)
    x, y = rng.standard_normal(1000), rng.standard_normal(1000)
    a, b = 0.37, -1.9
    assert np.array_equal(oracle.axpy(a, x, y), [_fma(a, xi, yi) for xi, yi in zip(x, y)])
    assert np.array_equal(oracle.axpy2(a, x, b, y),
                          [_fma(b, yi, a * xi) for xi, yi in zip(x, y)])
