"""Parity at the full sizes of the benchmark workloads, against the oracle.

  C2b  power-law rows, 2,000,000 x 2,000,000 (~32 M nonzeros), FP64 and FP32:
       the kernel the library picks (the warp-gather kernel sums every row
       serially: bit-identical to the serial oracle), the row-block kernel
       (thread rows bit-identical, warp / CTA rows within 1e-12 FP64 or 2e-6
       FP32 of the row's absolute sum), and the autotuner's choice;
  C3   4,096 banded SPD matrices in one launch, FP64 and FP32, every matrix
       bit-identical to the serial oracle (all rows are thread rows);
  C4   the 128^3 variable-coefficient Poisson system through the batched
       engine: FP64 within +-2 iterations of the oracle's Jacobi PCG and
       within 1e-8 of its solution; FP32 / BF16 values with FP64 refinement
       at true FP64 residual <= 1e-10 and within 1e-7 of the oracle solution;
  C5   a served stream of 300 requests of the served distribution arriving by
       a Poisson process at 1,000 req/s: every result at true residual <= 1e-8
       and bit-identical to the same request solved alone.

The 128^3 oracle solve uses the oracle's threaded Jacobi PCG (the serial
recurrence with OpenMP loops: same iteration count, solution within 1e-15 of
the serial one at this size) so the suite stays within minutes.
"""
import numpy as np
import pytest

from num_b200 import generators as gen

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-6


@pytest.fixture(scope="module")
def c2b():
    A = gen.power_law(2_000_000)  # the bench workload: seed 1001
    x = np.random.default_rng(1).uniform(-1.0, 1.0, A.ncols)
    return A, x


def _spmv(kspmv, M, x, precision):
    dt = torch.float64 if precision == "fp64" else torch.float32
    xt = torch.tensor(x, dtype=dt, device="cuda")
    yt = torch.full((M.nrows,), float("nan"), dtype=dt, device="cuda")
    kspmv.spmv(M, xt, yt)
    return yt.cpu().numpy()


def _check(kspmv, M, y, ref, scale, tol):
    assert np.all(np.abs(y - ref) <= tol * scale)
    if kspmv.spmv_kernel(M) == "gather":
        assert np.array_equal(y, ref)  # every row summed serially
    else:
        bins = kspmv.row_blocks(M)[1]
        assert np.array_equal(y[bins == 0], ref[bins == 0])


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_c2b_power_law_2m_full_size(kspmv, oracle, c2b, precision):
    A, x = c2b
    vals = A.values if precision == "fp64" else A.values.astype(np.float32)
    xx = x if precision == "fp64" else x.astype(np.float32)
    ref = oracle.spmv(A.row_ptr, A.col_idx, vals, xx, threads=True)
    scale = oracle.spmv(A.row_ptr, A.col_idx, np.abs(vals), np.abs(xx), threads=True)
    tol = TOL64 if precision == "fp64" else TOL32
    M = kspmv.upload_csr(A.row_ptr, A.col_idx, A.values, A.nrows, A.ncols, precision=precision)
    assert kspmv.spmv_kernel(M) == "gather"
    _check(kspmv, M, _spmv(kspmv, M, xx, precision), ref, scale, tol)
    kspmv.tune(M, kernel="blocks")
    _check(kspmv, M, _spmv(kspmv, M, xx, precision), ref, scale, tol)
    kspmv.autotune(M, x=torch.tensor(xx, device="cuda"), budget_ms=100, cache=False)
    _check(kspmv, M, _spmv(kspmv, M, xx, precision), ref, scale, tol)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_c3_4096_matrices_one_launch(kspmv, oracle, precision):
    mats, xs = gen.banded_batch(4096, seed=2)
    M = kspmv.upload_csr_batched([m.astuple() for m in mats], precision=precision)
    dt = np.float64 if precision == "fp64" else np.float32
    y = _spmv(kspmv, M, np.concatenate(xs).astype(dt), precision)
    ro = M.batch_offsets[0]
    assert ro[-1] == M.nrows == sum(m.nrows for m in mats)
    for k, (A, x) in enumerate(zip(mats, xs)):
        ref = oracle.spmv(A.row_ptr, A.col_idx, A.values.astype(dt), x.astype(dt))
        assert np.array_equal(y[ro[k]:ro[k + 1]], ref), k


@pytest.fixture(scope="module")
def c4(oracle):
    A, b = gen.varcoef_poisson_3d(128, seed=3)
    oracle.set_threads(oracle.num_threads())
    info, x = oracle.cg_omp(A.row_ptr, A.col_idx, A.values, b, tol=1e-10, max_iter=20000,
                            precond=True)
    assert info["converged"] and info["iters"] == 692
    return A, b, info, x


def _true_rel(A, x, b):
    return np.linalg.norm(b - A.to_scipy() @ x) / np.linalg.norm(b)


@pytest.mark.parametrize("precision", ["fp64", "fp32", "bf16"])
def test_c4_128_cubed_engine_vs_oracle(kspmv, c4, precision):
    from num_b200.solver import BatchSolver
    A, b, oinfo, ox = c4
    S = BatchSolver(A.nrows + 4096, A.nnz + 4096, 4, precision=precision)
    (x, info), = S.solve([(A, b)], tol=1e-10, max_iter=20000, chunk=64)
    assert info["converged"]
    rel = _true_rel(A, x, b)
    assert rel < 1e-10
    err = np.linalg.norm(x - ox) / np.linalg.norm(ox)
    if precision == "fp64":
        assert abs(info["iters"] - oinfo["iters"]) <= 2
        assert err < 1e-8
    else:
        assert info["outer"] >= 2
        assert err < 1e-7, err


def test_c5_poisson_stream_alone_equals_mixed(kspmv):
    from num_b200 import serve
    from num_b200.solver import BatchSolver, arena_for
    reqs = serve.make_requests(300, rate=1000.0, seed=4)
    rows, nnz = arena_for(16e9, nnz_per_row=5.0, precision="fp32")
    S = BatchSolver(rows, nnz, 1024, precision="fp32")
    got = {}
    stats, _ = serve.serve(reqs, S, tol=1e-8, chunk=16,
                           check=lambda i, x, info: got.__setitem__(i, (x, info)))
    assert stats["completed"] == len(reqs) and len(got) == len(reqs)
    assert stats["p99_ms"] >= stats["p50_ms"] > 0
    del S
    alone = BatchSolver(rows, nnz, 8, precision="fp32")
    for i, (t, A, b, kind) in enumerate(reqs):
        x, info = got[i]
        assert info["converged"] and _true_rel(A, x, b) < 1e-8, kind
        (xa, ia), = alone.solve([(A, b)], tol=1e-8, chunk=16)
        assert ia["iters"] == info["iters"] and np.array_equal(xa, x), (i, kind)
