"""GPU parity of the SpMV kernels against the CPU oracle (through the drop-in
module, i.e. the C ABI).  Bar: rows reduced by one thread sum in CSR order and
must be bit-identical to the oracle's serial loop; warp / CTA rows differ only
in reduction order and must agree to 1e-12 relative (FP64)."""
import ctypes as C
import json

import numpy as np
import pytest

from conftest import GOLDEN
from num_b200 import generators as gen

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL64 = 1e-12   # FP64: relative, reduction order differs
TOL32 = 2e-6    # FP32 accumulate: relative to the row's absolute sum


def _run(kspmv, A, x, precision="fp64", kk=True, tuning=None):
    M = kspmv.upload_csr(A.row_ptr, A.col_idx, A.values, A.nrows, A.ncols, precision=precision)
    if tuning:
        kspmv.tune(M, **tuning)
    dt = torch.float64 if precision == "fp64" else torch.float32
    xt = torch.tensor(x, dtype=dt, device="cuda")
    yt = torch.full((A.nrows,), float("nan"), dtype=dt, device="cuda")
    kspmv.spmv(M, xt, yt, kokkoskernels=kk)
    return yt.cpu().numpy(), M


def _check64(oracle, A, x, y, bins=None):
    ref = oracle.spmv(A.row_ptr, A.col_idx, A.values, x)
    scale = oracle.spmv(A.row_ptr, A.col_idx, np.abs(A.values), np.abs(x))
    err = np.abs(y - ref)
    assert np.all(err <= TOL64 * np.maximum(scale, 1e-300)), float((err / np.maximum(scale, 1e-300)).max())
    if bins is not None:
        thread_rows = bins == 0
        assert np.array_equal(y[thread_rows], ref[thread_rows])
    return ref


@pytest.mark.parametrize("kk", [True, False])
def test_tridiag4_known_answer(kspmv, kk):
    # tests/test_spmv_kernel.cpp:74-110 (custom and KokkosKernels backends)
    y, _ = _run(kspmv, gen.tridiag4(), np.array([1.0, 2.0, 3.0, 4.0]), kk=kk)
    assert np.array_equal(y, [0.0, 0.0, 0.0, 5.0])


def test_identity_known_answer(kspmv):
    # tests/test_spmv_kernel.cpp:114-130
    x = np.arange(100) * 0.1
    y, _ = _run(kspmv, gen.diagonal(np.ones(100)), x)
    assert np.array_equal(y, x)


def test_lcg_random(kspmv, oracle):
    # tests/test_spmv_kernel.cpp:163-210 (unsorted columns, possible repeats)
    A, x = gen.lcg_random()
    y, M = _run(kspmv, A, x)
    _, bins = kspmv.row_blocks(M)
    ref = _check64(oracle, A, x, y, bins)
    assert np.abs(y - ref).max() / np.abs(ref).max() < 1e-12


def test_c1_laplacian_2d_bit_exact(kspmv, oracle):
    # 256^2 5-point Laplacian, x ~ U[-1,1] (default_rng(0)): every row is
    # thread-reduced, so the whole vector equals the serial oracle.
    probe = json.loads((GOLDEN / "c1_probe.json").read_text())
    A = gen.laplacian_2d(256)
    x = np.random.default_rng(0).uniform(-1.0, 1.0, A.ncols)
    y, _ = _run(kspmv, A, x)
    assert np.array_equal(y, oracle.spmv(A.row_ptr, A.col_idx, A.values, x))
    assert abs(np.linalg.norm(y) - probe["spmv_y_norm2"]) < 1e-12 * probe["spmv_y_norm2"]


@pytest.mark.parametrize("name", ["laplacian_2d", "laplacian_3d", "random_sparse", "lattice_gauge"])
def test_reference_matrices_vs_scipy(kspmv, oracle, name):
    # verify_accuracy.py:67-90: rel err vs SciPy < 1e-10 (we hold 1e-12)
    p = np.load(GOLDEN / "scipy_pins.npz")
    A = gen.Csr(p[f"{name}__indptr"], p[f"{name}__indices"], p[f"{name}__data"],
                p[f"{name}__indptr"].shape[0] - 1, p[f"{name}__indptr"].shape[0] - 1)
    x = p[f"{name}__x"]
    y, M = _run(kspmv, A, x)
    ref = p[f"{name}__y"]
    assert np.linalg.norm(y - ref) / np.linalg.norm(ref) < TOL64
    _check64(oracle, A, x, y, kspmv.row_blocks(M)[1])


# the row-block kernel (scattered columns would get the warp-gather kernel)
@pytest.mark.parametrize("tuning", [{"kernel": "blocks"},
                                    {"tile": 1024, "short_max": 8, "kernel": "blocks"},
                                    {"tile": 4096, "max_rows": 128, "short_max": 64,
                                     "kernel": "blocks"},
                                    {"grid_mult": 2, "kernel": "blocks"}])
def test_power_law_all_bins(kspmv, oracle, tuning):
    A = gen.power_law(200_000, seed=5)
    x = np.random.default_rng(1).uniform(-1, 1, A.ncols)
    y, M = _run(kspmv, A, x, tuning=tuning)
    blk, bins = kspmv.row_blocks(M)
    t = kspmv.tuning(M)  # effective tuning, read only
    oblk, obins = oracle.row_blocks(A.row_ptr, t["tile"], t["max_rows"], t["short_max"])
    assert np.array_equal(blk, oblk) and np.array_equal(bins, obins)  # device copy == oracle
    assert (bins == 1).any()
    _check64(oracle, A, x, y, bins)


# ---- warp-gather kernel (scattered columns) ------------------------------------

def test_gather_kernel_chosen_and_bit_exact(kspmv, oracle):
    # power-law rows over 200,000 columns: no block has x windows, so spmv
    # runs the warp-gather kernel, which sums every row serially
    A = gen.power_law(200_000, seed=11)
    x = np.random.default_rng(11).uniform(-1, 1, A.ncols)
    y, M = _run(kspmv, A, x)
    assert kspmv.spmv_kernel(M) == "gather" and kspmv.tuning(M)["kernel"] == "auto"
    assert np.array_equal(y, oracle.spmv(A.row_ptr, A.col_idx, A.values, x))
    y2, M2 = _run(kspmv, A, x, tuning={"kernel": "blocks"})
    assert kspmv.spmv_kernel(M2) == "blocks"
    _check64(oracle, A, x, y2, kspmv.row_blocks(M2)[1])


def _scattered(nrows, lens_from, seed, ncols=1_000_000):
    rng = np.random.default_rng(seed)
    lens = rng.choice(lens_from, nrows)
    lens[:: 7] = 0
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ci = np.concatenate([np.sort(rng.choice(ncols, l, replace=False)) if l else
                         np.empty(0, np.int64) for l in lens]).astype(np.int32)
    return gen.Csr(rp, ci, rng.standard_normal(rp[-1]), nrows, ncols), rng


@pytest.mark.parametrize("nrows", [1, 31, 32, 33, 100, 1000])
def test_gather_ragged_groups_and_empty_rows(kspmv, oracle, nrows):
    # row groups cut at 32 rows, rows of 0 ... 4096 nonzeros over a million columns
    A, rng = _scattered(nrows, [0, 1, 5, 40, 193, 300, 4096], nrows)
    x = rng.uniform(-1, 1, A.ncols)
    y, M = _run(kspmv, A, x)
    if A.nnz:
        assert kspmv.spmv_kernel(M) == "gather"
    assert np.array_equal(y, oracle.spmv(A.row_ptr, A.col_idx, A.values, x))
    assert np.all(y[np.diff(A.row_ptr) == 0] == 0.0)


def test_gather_long_row_falls_back_and_forced(kspmv, oracle):
    # a row longer than 4096 nonzeros keeps the row-block kernel under "auto";
    # forced, the warp-gather kernel still sums it serially
    A, rng = _scattered(200, [3, 17, 64, 5000], 5)
    x = rng.uniform(-1, 1, A.ncols)
    y, M = _run(kspmv, A, x)
    assert kspmv.spmv_kernel(M) == "blocks"
    _check64(oracle, A, x, y, kspmv.row_blocks(M)[1])
    yg, Mg = _run(kspmv, A, x, tuning={"kernel": "gather"})
    assert kspmv.spmv_kernel(Mg) == "gather"
    assert np.array_equal(yg, oracle.spmv(A.row_ptr, A.col_idx, A.values, x))


def test_gather_fp32_and_bf16_every_row_bit_exact(kspmv, oracle):
    A = gen.power_law(100_000, seed=13)
    x = np.random.default_rng(13).uniform(-1, 1, A.ncols).astype(np.float32)
    y32, M = _run(kspmv, A, x, precision="fp32")
    assert kspmv.spmv_kernel(M) == "gather"
    assert np.array_equal(y32, oracle.spmv(A.row_ptr, A.col_idx, A.values.astype(np.float32), x))
    yb, Mb = _run(kspmv, A, x, precision="bf16")
    from num_b200.kokkos_spmv import _values_for
    bits, _ = _values_for(A.values, "bf16")
    vb = (bits.astype(np.uint32) << 16).view(np.float32)
    assert kspmv.spmv_kernel(Mb) == "gather"
    assert np.array_equal(yb, oracle.spmv(A.row_ptr, A.col_idx, vb, x))


@pytest.mark.parametrize("precision", ["fp64", "fp32", "bf16"])
@pytest.mark.parametrize("case", ["power_law", "random_sparse", "ragged"])
def test_sliced_kernel_every_row_bit_exact(kspmv, oracle, precision, case):
    # The sliced gather kernel (rows sorted by length, column-major 32-row
    # slices, lane per row) sums every row serially in CSR order: bit-identical
    # to the serial oracle for rows of any length, in every precision; empty
    # rows give 0 and the permuted rows land in their own places.
    if case == "power_law":
        A = gen.power_law(150_000, seed=17)
        x = np.random.default_rng(17).uniform(-1, 1, A.ncols)
    elif case == "random_sparse":
        A = gen.get_matrix("random_sparse", 30_000)
        x = np.random.default_rng(18).uniform(-1, 1, A.ncols)
    else:
        A, rng = _scattered(70_001, [0, 1, 3, 9, 40, 200], 19, ncols=300_000)
        x = rng.uniform(-1, 1, A.ncols)
    vals = A.values
    if precision == "fp32":
        vals, x = A.values.astype(np.float32), x.astype(np.float32)
    elif precision == "bf16":
        from num_b200.kokkos_spmv import _values_for
        bits, _ = _values_for(A.values, "bf16")
        vals, x = (bits.astype(np.uint32) << 16).view(np.float32), x.astype(np.float32)
    y, M = _run(kspmv, A, x, precision=precision, tuning={"kernel": "sliced"})
    assert kspmv.spmv_kernel(M) == "sliced"
    assert np.array_equal(y, oracle.spmv(A.row_ptr, A.col_idx, vals, x))
    assert np.all(y[np.diff(A.row_ptr) == 0] == 0.0)


def test_tune_kernel_argument_errors(kspmv):
    A = gen.tridiag4()
    M = kspmv.upload_csr(*A.astuple())
    with pytest.raises(ValueError):
        kspmv.tune(M, kernel="fastest")
    with pytest.raises(ValueError, match="kernel"):
        kspmv.tune(M, kernel=7)
    assert kspmv.tune(M, kernel="gather")["kernel"] == "gather"
    assert kspmv.tune(M)["kernel"] == "gather"  # None keeps it
    assert kspmv.tune(M, kernel="auto")["kernel"] == "auto"


def test_ragged_long_and_empty_rows(kspmv, oracle):
    rng = np.random.default_rng(9)
    lens = np.array([0, 0, 9000, 1, 2047, 2048, 2049, 0, 33, 32, 31, 4097, 3, 20000, 0, 5] * 8)
    n = lens.shape[0]
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ci = np.concatenate([np.sort(rng.choice(50_000, l, replace=False)) if l else
                         np.empty(0, np.int64) for l in lens]).astype(np.int32)
    A = gen.Csr(rp, ci, rng.standard_normal(rp[-1]), n, 50_000)
    x = rng.uniform(-1, 1, 50_000)
    y, M = _run(kspmv, A, x)
    bins = kspmv.row_blocks(M)[1]
    assert (bins == 2).any() and (bins == 1).any() and (bins == 0).any()
    _check64(oracle, A, x, y, bins)
    assert np.all(y[lens == 0] == 0.0)


def test_rectangular_and_all_empty(kspmv, oracle):
    rng = np.random.default_rng(4)
    A = gen.Csr(np.zeros(11, np.int32), np.empty(0, np.int32), np.empty(0), 10, 3)
    y, _ = _run(kspmv, A, np.ones(3))
    assert np.array_equal(y, np.zeros(10))
    rp = np.arange(0, 3 * 501, 3, dtype=np.int32)
    ci = rng.integers(0, 7, rp[-1]).astype(np.int32)  # wide-short rectangular, repeats
    A = gen.Csr(rp, ci, rng.standard_normal(rp[-1]), 500, 7)
    x = rng.standard_normal(7)
    y, _ = _run(kspmv, A, x)
    assert np.array_equal(y, oracle.spmv(rp, ci, A.values, x))


def test_c2a_full_size(kspmv, oracle):
    # 3-D 7-point Laplacian 160^3 (4,096,000 rows, 28,518,400 nonzeros), x ~ U[-1,1]
    # (seed 1): bit-identical to the serial oracle (all rows are thread-reduced),
    # and A * ones equals the exact row sums.
    A = gen.laplacian_3d(160)
    x = np.random.default_rng(1).uniform(-1, 1, A.ncols)
    y, M = _run(kspmv, A, x)
    assert np.array_equal(y, oracle.spmv(A.row_ptr, A.col_idx, A.values, x, threads=True))
    xt = torch.ones(A.ncols, dtype=torch.float64, device="cuda")
    yt = torch.empty(A.nrows, dtype=torch.float64, device="cuda")
    kspmv.spmv(M, xt, yt)
    rowsum = np.add.reduceat(A.values, A.row_ptr[:-1])
    assert np.array_equal(yt.cpu().numpy(), rowsum)


def test_fp32_and_bf16(kspmv, oracle):
    A = gen.power_law(100_000, seed=3)
    x = np.random.default_rng(2).uniform(-1, 1, A.ncols).astype(np.float32)
    y32, M = _run(kspmv, A, x, precision="fp32")
    bins = kspmv.row_blocks(M)[1]
    ref = oracle.spmv(A.row_ptr, A.col_idx, A.values.astype(np.float32), x)
    scale = oracle.spmv(A.row_ptr, A.col_idx, np.abs(A.values).astype(np.float32), np.abs(x))
    assert np.array_equal(y32[bins == 0], ref[bins == 0])
    assert np.all(np.abs(y32 - ref) <= TOL32 * scale)
    # bf16 values: the oracle runs FP32 on the bf16-rounded values
    yb, Mb = _run(kspmv, A, x, precision="bf16")
    from num_b200.kokkos_spmv import _values_for
    bits, _ = _values_for(A.values, "bf16")
    vb = (bits.astype(np.uint32) << 16).view(np.float32)
    refb = oracle.spmv(A.row_ptr, A.col_idx, vb, x)
    assert np.array_equal(yb[bins == 0], refb[bins == 0])
    assert np.all(np.abs(yb - refb) <= TOL32 * scale)


def test_batched_many_matrices(kspmv, oracle):
    mats, xs = gen.banded_batch(96, seed=2)
    M = kspmv.upload_csr_batched([m.astuple() for m in mats])
    assert M.nrows == sum(m.nrows for m in mats) and M.nnz == sum(m.nnz for m in mats)
    xt = torch.tensor(np.concatenate(xs), device="cuda")
    yt = torch.empty(M.nrows, dtype=torch.float64, device="cuda")
    kspmv.spmv(M, xt, yt)
    y = yt.cpu().numpy()
    ro = M.batch_offsets[0]
    for k, (A, x) in enumerate(zip(mats, xs)):
        assert np.array_equal(y[ro[k]:ro[k + 1]], oracle.spmv(A.row_ptr, A.col_idx, A.values, x))


def test_argument_errors(kspmv):
    A = gen.tridiag4()
    M = kspmv.upload_csr(A.row_ptr, A.col_idx, A.values, 4, 4)
    good = torch.zeros(4, dtype=torch.float64, device="cuda")
    assert repr(M) == "<CrsMatrix nrows=4 ncols=4 nnz=10>"
    with pytest.raises(ValueError, match="x length"):
        kspmv.spmv(M, torch.zeros(5, dtype=torch.float64, device="cuda"), good)
    with pytest.raises(ValueError, match="y length"):
        kspmv.spmv(M, good, torch.zeros(3, dtype=torch.float64, device="cuda"))
    with pytest.raises(TypeError):
        kspmv.spmv(M, torch.zeros(4, dtype=torch.float32, device="cuda"), good)
    with pytest.raises(TypeError):
        kspmv.spmv(M, torch.zeros(4, dtype=torch.float64), good)
    with pytest.raises(ValueError, match="contiguous"):
        kspmv.spmv(M, torch.zeros(8, dtype=torch.float64, device="cuda")[::2], good)


@pytest.mark.parametrize("tile,stages", [(1024, 2), (1024, 3), (2048, 2), (2048, 3), (4096, 2)])
@pytest.mark.parametrize("aligned", [True, False])
def test_staged_x_windows_and_fallback(kspmv, oracle, tile, stages, aligned):
    # Stencil blocks stage their x windows (TMA) when x is 16-byte aligned; an
    # x that starts 8 bytes into an allocation must take the gather path.
    # Both must equal the serial oracle bit for bit (all rows thread-reduced).
    A = gen.laplacian_3d(48)
    x = np.random.default_rng(tile + stages).uniform(-1, 1, A.ncols)
    M = kspmv.upload_csr(A.row_ptr, A.col_idx, A.values, A.nrows, A.ncols)
    kspmv.tune(M, tile=tile, stages=stages)
    buf = torch.zeros(A.ncols + 1, dtype=torch.float64, device="cuda")
    xt = buf[1:] if not aligned else buf[:-1]
    xt.copy_(torch.tensor(x))
    assert (xt.data_ptr() % 16 == 0) == aligned
    yt = torch.full((A.nrows,), float("nan"), dtype=torch.float64, device="cuda")
    kspmv.spmv(M, xt, yt)
    assert np.array_equal(yt.cpu().numpy(), oracle.spmv(A.row_ptr, A.col_idx, A.values, x))


@pytest.mark.parametrize("tile", [1024, 2048])
def test_staged_x_ragged_columns(kspmv, oracle, tile):
    # Rows whose columns fall in a few narrow bands (staged) mixed with rows of
    # random columns (too many windows: gathered), odd ncols (the last block's
    # windows would pass the end of x, so it must gather), FP64 and FP32.
    rng = np.random.default_rng(tile)
    n, ncols = 20_000, 20_003
    rows = []
    for i in range(n):
        if (i // 300) % 2 == 0:
            base = [i, (i * 7) % (ncols - 40), ncols - 1 - (i % 37)]
            c = np.unique(np.concatenate([b + np.arange(-3, 4) for b in base]))
            c = c[(c >= 0) & (c < ncols)]
        else:
            c = np.unique(rng.integers(0, ncols, rng.integers(1, 12)))
        rows.append(c)
    rp = np.concatenate([[0], np.cumsum([len(c) for c in rows])]).astype(np.int32)
    ci = np.concatenate(rows).astype(np.int32)
    A = gen.Csr(rp, ci, rng.standard_normal(rp[-1]), n, ncols)
    x = rng.uniform(-1, 1, ncols)
    y, M = _run(kspmv, A, x, tuning={"tile": tile})
    _check64(oracle, A, x, y, kspmv.row_blocks(M)[1])
    y32, _ = _run(kspmv, A, x.astype(np.float32), precision="fp32", tuning={"tile": tile})
    ref32 = oracle.spmv(A.row_ptr, A.col_idx, A.values.astype(np.float32), x.astype(np.float32))
    scale = oracle.spmv(A.row_ptr, A.col_idx, np.abs(A.values).astype(np.float32),
                        np.abs(x).astype(np.float32))
    assert np.all(np.abs(y32 - ref32) <= TOL32 * scale)


def test_autotune_installs_a_valid_tuning(kspmv, oracle, tmp_path, monkeypatch):
    # The autotuner times every candidate, installs the fastest, and the
    # product under the chosen partition keeps the bar (rows of <= 32
    # nonzeros stay thread-per-row: bit-exact).  A second call hits the cache.
    monkeypatch.setenv("NUM_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    kspmv._TUNE_CACHE.clear()
    A = gen.power_law(200_000, seed=1001)
    x = np.random.default_rng(1).uniform(-1, 1, A.ncols)
    M = kspmv.upload_csr(A.row_ptr, A.col_idx, A.values, A.nrows, A.ncols)
    res = kspmv.autotune(M, budget_ms=50)
    assert not res["cached"] and len(res["trials"]) >= 20
    assert res["tile"] in (1024, 2048, 4096) and res["short_max"] in (32, 64)
    assert res["stages"] in (2, 3, 4) and res["grid_mult"] in (0, 1, 2)
    assert res["us"] == min(t["us"] for t in res["trials"])
    assert {"blocks", "gather"} <= {t["kernel"] for t in res["trials"]} <= \
        {"blocks", "gather", "sliced"}
    assert {k: res[k] for k in ("tile", "short_max", "stages", "grid_mult", "kernel")} == \
        {k: kspmv.tuning(M)[k] for k in ("tile", "short_max", "stages", "grid_mult", "kernel")}
    xt = torch.tensor(x, device="cuda")
    yt = torch.full((A.nrows,), float("nan"), dtype=torch.float64, device="cuda")
    kspmv.spmv(M, xt, yt)
    _, bins = kspmv.row_blocks(M)
    _check64(oracle, A, x, yt.cpu().numpy(), bins)
    assert json.loads((tmp_path / "tune.json").read_text())
    kspmv._TUNE_CACHE.clear()
    again = kspmv.autotune(M, budget_ms=50)
    assert again["cached"] and again["tile"] == res["tile"] and again["stages"] == res["stages"]
    assert again["kernel"] == res["kernel"]
