"""The batched / mixed-precision solver engine (nm_solver_*).

Bars: every system reaches its tolerance on the TRUE residual |b - A x| / |b|
computed here in FP64; FP64 mode matches the oracle's Jacobi-PCG iteration
count to within the refinement wrapper's rescaling (+-2) and its solution; the
FP32 / BF16 modes' solutions are compared with the FP64 oracle solution (the
error is bounded by cond(A) x tol); and every system's result is bit-identical
whether it is solved alone or inside a mixed batch (per-system reductions run
in a fixed order over that system's own blocks).
"""
import numpy as np
import pytest

from num_b200 import generators as gen

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _solver(precision, rows=2_000_000, nnz=20_000_000, systems=512, **kw):
    from num_b200.solver import BatchSolver
    return BatchSolver(rows, nnz, systems, precision=precision, **kw)


def _true_rel(A, x, b):
    r = b - A.to_scipy() @ x
    return np.linalg.norm(r) / np.linalg.norm(b)


def test_fp64_matches_oracle_pcg(kspmv, oracle):
    A, b = gen.varcoef_poisson_3d(24, seed=3)
    S = _solver("fp64")
    (x, info), = S.solve([(A, b)], tol=1e-10, max_iter=5000)
    oinfo, ox = oracle.pcg_jacobi(A.row_ptr, A.col_idx, A.values, b, tol=1e-10, max_iter=5000)
    assert info["converged"] and oinfo["converged"]
    assert abs(info["iters"] - oinfo["iters"]) <= 2
    assert _true_rel(A, x, b) < 1e-10
    assert np.linalg.norm(x - ox) / np.linalg.norm(ox) < 1e-8


@pytest.mark.parametrize("precision", ["fp32", "bf16"])
def test_mixed_precision_refinement(kspmv, oracle, precision):
    # 3-D variable-coefficient Poisson (face coefficients exp(N(0,1))):
    # inner Jacobi-PCG in FP32 (values FP32 / BF16), FP64 refinement to 1e-10.
    A, b = gen.varcoef_poisson_3d(24, seed=3)
    S = _solver(precision)
    (x, info), = S.solve([(A, b)], tol=1e-10, max_iter=20000)
    assert info["converged"] and info["outer"] >= 2
    rel = _true_rel(A, x, b)
    assert rel < 1e-10 and abs(rel - info["residual"]) < 1e-3 * 1e-10
    _, ox = oracle.pcg_jacobi(A.row_ptr, A.col_idx, A.values, b, tol=1e-12, max_iter=20000)
    assert np.linalg.norm(x - ox) / np.linalg.norm(ox) < 1e-7


def test_laplacian_bf16_values_exact(kspmv):
    # 5-point Laplacian values (4, -1) are exact in BF16.
    A = gen.laplacian_2d(96)
    b = np.random.default_rng(4).standard_normal(A.nrows)
    S = _solver("bf16")
    (x, info), = S.solve([(A, b)], tol=1e-8, max_iter=20000)
    assert info["converged"] and _true_rel(A, x, b) < 1e-8


def _mix(seed=2, count=40):
    rng = np.random.default_rng(seed)
    mats, _ = gen.banded_batch(count, seed=seed)
    systems = [(A, rng.standard_normal(A.nrows)) for A in mats]
    for side in (17, 40, 63):
        A = gen.laplacian_2d(side)
        systems.append((A, rng.standard_normal(A.nrows)))
    systems.append((gen.laplacian_3d(20), rng.standard_normal(8000)))
    return systems


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_batch_alone_equals_mixed(kspmv, precision):
    systems = _mix()
    S = _solver(precision)
    mixed = S.solve(systems, tol=1e-8, max_iter=20000, chunk=6)
    for (A, b), (x, info) in zip(systems, mixed):
        assert info["converged"], info
        assert _true_rel(A, x, b) < 1e-8
    for k in (0, 7, len(systems) - 1, len(systems) - 3):
        A, b = systems[k]
        S1 = _solver(precision)
        (xa, ia), = S1.solve([(A, b)], tol=1e-8, max_iter=20000, chunk=5)
        xm, im = mixed[k]
        assert ia["iters"] == im["iters"] and ia["outer"] == im["outer"]
        assert np.array_equal(xa, xm)  # same bits alone and in the mix


def test_admission_by_free_memory(kspmv):
    # Arena of 10,000 rows: a 6,400-row system fits, a second one does not
    # until the first is taken; slots are reused.
    S = _solver("fp32", rows=10_000, nnz=60_000, systems=4)
    A = gen.laplacian_2d(80)
    b = np.ones(A.nrows)
    s1 = S.admit(A, b, tol=1e-8)
    assert s1 is not None
    assert S.admit(A, b, tol=1e-8) is None           # no room
    small = gen.laplacian_2d(20)
    s2 = S.admit(small, np.ones(400), tol=1e-8)      # a small one still fits
    assert s2 is not None
    while S.active:
        S.step(16)
    x1, i1 = S.take(s1)
    assert i1["converged"] and _true_rel(A, x1, b) < 1e-8
    s3 = S.admit(A, b, tol=1e-8)                     # room again
    assert s3 is not None
    while S.active:
        S.step(16)
    x3, i3 = S.take(s3)
    assert np.array_equal(x1, x3)
    S.take(s2)


def test_zero_rhs_and_iteration_cap(kspmv):
    S = _solver("fp32")
    A = gen.laplacian_2d(30)
    (x, info), = S.solve([(A, np.zeros(A.nrows))], tol=1e-8)
    assert info["converged"] and info["iters"] == 0 and np.array_equal(x, np.zeros(A.nrows))
    (x, info), = S.solve([(A, np.ones(A.nrows))], tol=1e-14, max_iter=7, chunk=3)
    assert not info["converged"] and info["iters"] <= 7 + 3


def test_many_small_systems(kspmv, oracle):
    # 256 banded SPD systems (n 32..4096) in one batch, FP32 + refinement.
    mats, xs = gen.banded_batch(256, seed=9)
    rng = np.random.default_rng(1)
    systems = [(A, rng.standard_normal(A.nrows)) for A in mats]
    S = _solver("fp32")
    out = S.solve(systems, tol=1e-8, max_iter=5000, chunk=8)
    for (A, b), (x, info) in zip(systems, out):
        assert info["converged"] and _true_rel(A, x, b) < 1e-8


def test_admit_many_fifo_and_invalid(kspmv):
    # Batch admission stops at the first system that does not fit (FIFO); an
    # invalid system is refused with ValueError and leaves no slot behind.
    S = _solver("fp32", rows=10_000, nnz=60_000, systems=8)
    A = gen.laplacian_2d(60)                        # 3,600 rows each
    small = gen.laplacian_2d(10)
    got = S.admit_many([(A, np.ones(3600)), (A, np.ones(3600)), (A, np.ones(3600)),
                        (small, np.ones(100))], tol=1e-8)
    assert len(got) == 2                            # the third does not fit; the fourth waits
    bad = gen.laplacian_2d(10)
    ci = bad.col_idx.copy()
    ci[5] = 100                                     # outside [0, 100)
    with pytest.raises(ValueError):
        S.admit_many([((bad.row_ptr, ci, bad.values, 100), np.ones(100))], tol=1e-8)
    assert S.info()["free_slots"] == 6
    while S.active:
        S.step(16)
    xs = [S.take(s) for s in got]
    for x, info in xs:
        assert info["converged"] and _true_rel(A, x, np.ones(3600)) < 1e-8
    assert np.array_equal(xs[0][0], xs[1][0])


def test_resolve_and_solution(kspmv):
    # A solved system re-solved in place (same b) repeats its bits; with a new
    # b it converges to the new solution; solution() reads x without freeing.
    S = _solver("fp32", rows=100_000, nnz=600_000, systems=4)
    A = gen.laplacian_2d(64)
    rng = np.random.default_rng(11)
    b1, b2 = rng.standard_normal(A.nrows), rng.standard_normal(A.nrows)
    s = S.admit(A, b1, tol=1e-9)
    while S.active:
        S.step(8)
    x1 = S.solution(s)
    i1 = S.status(s)
    S.resolve(s)
    while S.active:
        S.step(8)
    assert np.array_equal(S.solution(s), x1) and S.status(s)["iters"] == i1["iters"]
    S.resolve(s, b=b2)
    while S.active:
        S.step(8)
    x2, i2 = S.take(s)
    assert i2["converged"] and _true_rel(A, x2, b2) < 1e-9


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_large_system_scalar_path(kspmv, oracle, precision):
    # A 512^2 Laplacian has more than 512 row blocks, so its alpha / beta are
    # reduced by one CTA per system instead of in every tile CTA: it must
    # still converge on the true residual, match the FP64 oracle's iteration
    # count in FP64 mode, and give the same bits alone and beside small ones.
    A = gen.laplacian_2d(512)
    b = np.random.default_rng(12).standard_normal(A.nrows)
    S = _solver(precision, rows=1_000_000, nnz=6_000_000, systems=16)
    (x, info), = S.solve([(A, b)], tol=1e-8, max_iter=20000, chunk=16)
    assert info["converged"] and _true_rel(A, x, b) < 1e-8
    if precision == "fp64":
        oinfo, _ = oracle.pcg_jacobi(A.row_ptr, A.col_idx, A.values, b, tol=1e-8,
                                     max_iter=20000)
        assert abs(info["iters"] - oinfo["iters"]) <= 2
    rng = np.random.default_rng(13)
    mix = [(gen.laplacian_2d(s), None) for s in (20, 33)]
    mix = [(M, rng.standard_normal(M.nrows)) for M, _ in mix]
    S2 = _solver(precision, rows=1_000_000, nnz=6_000_000, systems=16)
    out = S2.solve([mix[0], (A, b), mix[1]], tol=1e-8, max_iter=20000, chunk=16)
    assert out[1][1]["iters"] == info["iters"] and np.array_equal(out[1][0], x)


def test_served_stream_results_equal_alone(kspmv):
    # Continuous batching end to end: 24 requests (2-D Laplacians and banded
    # SPD systems) arriving by a Poisson process at 400 req/s are served with
    # admissions overlapping running steps; every result reaches the tolerance
    # on its true residual and carries the same bits as the same system solved
    # alone on a fresh solver.
    from num_b200 import serve
    from num_b200.solver import BatchSolver
    reqs = serve.make_requests(24, rate=400.0, seed=7, side_range=(16, 160),
                               banded_range=(64, 8192))
    S = BatchSolver(4_000_000, 30_000_000, 64, precision="fp32")
    got = {}
    stats, rec = serve.serve(reqs, S, tol=1e-8, chunk=16,
                             check=lambda i, x, info: got.__setitem__(i, (x, info)))
    assert stats["completed"] == len(reqs) and len(got) == len(reqs)
    assert stats["p99_ms"] >= stats["p50_ms"] > 0
    for i, (t, A, b, kind) in enumerate(reqs):
        x, info = got[i]
        assert info["converged"] and _true_rel(A, x, b) < 1e-8, kind
        alone = BatchSolver(4_000_000, 30_000_000, 4, precision="fp32")
        (xa, ia), = alone.solve([(A, b)], tol=1e-8, chunk=16)
        assert ia["iters"] == info["iters"] and np.array_equal(xa, x), kind


def test_take_many_matches_take(kspmv):
    # Batch retirement returns the same solutions and infos as one-by-one
    # take(), frees the slots and rejects a slot given twice.
    mats, _ = gen.banded_batch(12, seed=5)
    rng = np.random.default_rng(6)
    systems = [(A, rng.standard_normal(A.nrows)) for A in mats]
    S1 = _solver("fp32", rows=200_000, nnz=2_000_000, systems=16)
    S2 = _solver("fp32", rows=200_000, nnz=2_000_000, systems=16)
    s1 = [S1.admit(A, b, tol=1e-9) for A, b in systems]
    s2 = [S2.admit(A, b, tol=1e-9) for A, b in systems]
    while S1.active or S2.active:
        if S1.active:
            S1.step(16)
        if S2.active:
            S2.step(16)
    one = [S1.take(s) for s in s1]
    with pytest.raises(ValueError):
        S2.take_many([s2[0], s2[0]])
    many = S2.take_many(s2)
    for (xa, ia), (xb, ib) in zip(one, many):
        assert ia == ib and np.array_equal(xa, xb)
    assert S2.info()["free_slots"] == 16


@pytest.mark.parametrize("precision", ["fp64", "fp32", "bf16"])
def test_persistent_step_equals_graph_step(kspmv, nmlib, precision):
    # The step loop in one cooperative launch (grid barriers between the SpMV,
    # update and p-update phases) and the CUDA-graph loop of kernels give the
    # same bits and iteration counts, for a mix of small banded systems and a
    # large Laplacian (more than 512 row blocks: its alpha / beta reduced by
    # bs_alpha / bs_beta on the graph path, in-CTA on the persistent one).
    mats, _ = gen.banded_batch(24, seed=8)
    rng = np.random.default_rng(9)
    systems = [(A, rng.standard_normal(A.nrows)) for A in mats]
    L = gen.laplacian_2d(400)
    systems.insert(7, (L, rng.standard_normal(L.nrows)))
    out = []
    try:
        for mode in (0, 1, 0):
            nmlib.nm_solver_set_persistent(mode)
            S = _solver(precision, rows=1_000_000, nnz=6_000_000, systems=64)
            out.append(S.solve(systems, tol=1e-9, max_iter=20000, chunk=16))
            del S
    finally:
        nmlib.nm_solver_set_persistent(0)
    for run in out[1:]:
        for (xa, ia), (xb, ib) in zip(out[0], run):
            assert ia == ib and np.array_equal(xa, xb)
    for (A, b), (x, info) in zip(systems, out[0]):
        assert info["converged"] and _true_rel(A, x, b) < 1e-9
