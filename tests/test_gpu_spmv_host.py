"""nm_spmv_host (kokkos_spmv.spmv_host): y = A x with x and y in host memory,
x copied in as pieces and the row blocks run in chunks whose rows of y are
copied out while later chunks compute.  Bar: the same bits as nm_spmv on
device buffers (the same kernel over the same row blocks), and the serial
oracle's bits where every row is thread-reduced (the stencil Laplacians)."""
import numpy as np
import pytest

from num_b200 import generators as gen

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _dt(precision):
    return torch.float64 if precision == "fp64" else torch.float32


def _upload(kspmv, A, precision="fp64"):
    return kspmv.upload_csr(A.row_ptr, A.col_idx, A.values, A.nrows, A.ncols,
                            precision=precision)


def _device_y(kspmv, M, x, precision="fp64"):
    xt = torch.tensor(x, dtype=_dt(precision), device="cuda")
    yt = torch.full((M.nrows,), float("nan"), dtype=_dt(precision), device="cuda")
    kspmv.spmv(M, xt, yt)
    return yt.cpu().numpy()


def _host_y(kspmv, M, x, precision="fp64", pinned=True):
    xh = torch.tensor(x, dtype=_dt(precision))
    yh = torch.full((M.nrows,), float("nan"), dtype=_dt(precision))
    if pinned:
        xh, yh = xh.pin_memory(), yh.pin_memory()
    kspmv.spmv_host(M, xh, yh)
    return yh.numpy().copy()


def _shifted_band(nrows, ncols, seed, reverse=False):
    """Row i references the columns next to c(i) = i * ncols // nrows (or
    ncols - 1 - c(i) when reverse: the first rows read the end of x)."""
    rng = np.random.default_rng(seed)
    c = np.arange(nrows, dtype=np.int64) * ncols // nrows
    if reverse:
        c = ncols - 1 - c
    cols = c[:, None] + np.array([-1, 0, 1])[None, :]
    valid = (cols >= 0) & (cols < ncols)
    rp = np.zeros(nrows + 1, np.int32)
    np.cumsum(valid.sum(1), out=rp[1:])
    ci = cols[valid].astype(np.int32)
    return gen.Csr(rp, ci, rng.standard_normal(ci.size), nrows, ncols)


@pytest.mark.parametrize("pinned", [True, False])
def test_laplacian_3d_chunked_bit_exact(kspmv, oracle, pinned):
    # 100^3 (1,000,000 rows, 8 MB of x and of y): four x pieces, four row chunks
    A = gen.laplacian_3d(100)
    M = _upload(kspmv, A)
    for seed in (1, 2):  # the handle's buffers are reused by the second call
        x = np.random.default_rng(seed).uniform(-1, 1, A.ncols)
        y = _host_y(kspmv, M, x, pinned=pinned)
        assert np.array_equal(y, _device_y(kspmv, M, x))
        assert np.array_equal(y, oracle.spmv(A.row_ptr, A.col_idx, A.values, x, threads=True))


def test_laplacian_2d_numpy_arrays(kspmv, oracle):
    A = gen.laplacian_2d(1024)
    M = _upload(kspmv, A)
    x = np.random.default_rng(3).uniform(-1, 1, A.ncols)
    y = np.full(A.nrows, np.nan)
    kspmv.spmv_host(M, x, y)
    assert np.array_equal(y, oracle.spmv(A.row_ptr, A.col_idx, A.values, x, threads=True))


@pytest.mark.parametrize("precision", ["fp32", "bf16"])
def test_low_precision_values(kspmv, precision):
    A = gen.laplacian_3d(100)
    M = _upload(kspmv, A, precision)
    x = np.random.default_rng(4).uniform(-1, 1, A.ncols).astype(np.float32)
    assert np.array_equal(_host_y(kspmv, M, x, precision), _device_y(kspmv, M, x, precision))


@pytest.mark.parametrize("nrows,ncols,reverse", [(1_000_000, 1_000_000, True),
                                                 (1_200_000, 600_000, False),
                                                 (600_000, 1_200_000, True)])
def test_shifted_and_reversed_bands(kspmv, oracle, nrows, ncols, reverse):
    # reversed: the first row chunk waits for the last x piece; rectangular:
    # x pieces and row chunks fall at different places
    A = _shifted_band(nrows, ncols, 5, reverse)
    M = _upload(kspmv, A)
    x = np.random.default_rng(6).standard_normal(ncols)
    y = _host_y(kspmv, M, x)
    assert np.array_equal(y, _device_y(kspmv, M, x))
    assert np.array_equal(y, oracle.spmv(A.row_ptr, A.col_idx, A.values, x, threads=True))


@pytest.mark.parametrize("name", ["power_law", "c1"])
def test_one_chunk_forms(kspmv, name):
    # scattered columns (the warp-gather kernel) and a small matrix: one copy
    # in, one SpMV, one copy out
    A = gen.power_law(300_000, seed=7) if name == "power_law" else gen.laplacian_2d(256)
    M = _upload(kspmv, A)
    x = np.random.default_rng(8).uniform(-1, 1, A.ncols)
    assert np.array_equal(_host_y(kspmv, M, x), _device_y(kspmv, M, x))


def test_retuned_partition(kspmv):
    # a new row-block partition makes a new split of the chunks
    A = gen.laplacian_3d(100)
    M = _upload(kspmv, A)
    x = np.random.default_rng(9).uniform(-1, 1, A.ncols)
    y0 = _host_y(kspmv, M, x)
    kspmv.tune(M, tile=1024, stages=3)
    y1 = _host_y(kspmv, M, x)
    assert np.array_equal(y1, _device_y(kspmv, M, x))
    assert np.array_equal(y0, y1)


def test_empty_rows_and_rectangular_small(kspmv, oracle):
    A = gen.Csr(np.zeros(11, np.int32), np.empty(0, np.int32), np.empty(0), 10, 3)
    M = _upload(kspmv, A)
    y = np.full(10, np.nan)
    kspmv.spmv_host(M, np.ones(3), y)
    assert np.array_equal(y, np.zeros(10))


def test_argument_errors(kspmv):
    A = gen.laplacian_2d(16)
    M = _upload(kspmv, A)
    x, y = np.ones(A.ncols), np.empty(A.nrows)
    with pytest.raises(ValueError):
        kspmv.spmv_host(M, np.ones(A.ncols + 1), y)
    with pytest.raises(ValueError):
        kspmv.spmv_host(M, x, np.empty(A.nrows - 1))
    with pytest.raises(TypeError):
        kspmv.spmv_host(M, x.astype(np.float32), y)
    with pytest.raises(TypeError):
        kspmv.spmv_host(M, torch.ones(A.ncols, dtype=torch.float64, device="cuda"), y)
    with pytest.raises(ValueError):
        kspmv.spmv_host(M, x, np.empty(2 * A.nrows)[::2])
