"""On-device assembly of the stencil Laplacians (kokkos_spmv.laplacian, C ABI
nm_csr_laplacian) against the host generators, which are pinned to the
reference's python/matrix_generators.py (make_laplacian_2d :16-37,
make_laplacian_3d_fast :68-80) by the golden fixtures.  Bar: bit-identical
row_ptr, col_idx and values, and the same partition, so SpMV results are
bit-identical too."""
import numpy as np
import pytest

from num_b200 import generators as gen

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _host(dim, L):
    return gen.laplacian_2d(L) if dim == 2 else gen.laplacian_3d(L)


@pytest.mark.parametrize("dim,L", [(2, 1), (2, 2), (2, 3), (2, 17), (2, 256),
                                   (3, 1), (3, 2), (3, 5), (3, 31), (3, 64)])
def test_laplacian_arrays_match_host(kspmv, dim, L):
    A = _host(dim, L)
    M = kspmv.laplacian(dim, L)
    assert (M.nrows, M.ncols, M.nnz) == (A.nrows, A.ncols, A.nnz)
    rp, ci, v = kspmv.download_csr(M)
    assert np.array_equal(rp, A.row_ptr)
    assert np.array_equal(ci, A.col_idx)
    assert np.array_equal(v, A.values)


@pytest.mark.parametrize("precision", ["fp32", "bf16"])
def test_laplacian_low_precision_values_match_upload(kspmv, precision):
    A = gen.laplacian_3d(20)
    M = kspmv.laplacian(3, 20, precision=precision)
    U = kspmv.upload_csr(*A.astuple(), precision=precision)
    assert M.precision == precision
    for a, b in zip(kspmv.download_csr(M), kspmv.download_csr(U)):
        assert a.dtype == b.dtype and np.array_equal(a, b)


def test_laplacian_160_cubed_matches_host_and_spmv(kspmv):
    # The 160^3 Laplacian (n = 4,096,000, nnz = 28,518,400), full size.
    A = gen.laplacian_3d(160)
    M = kspmv.laplacian(3, 160)
    assert M.nnz == 28_518_400
    rp, ci, v = kspmv.download_csr(M)
    assert np.array_equal(rp, A.row_ptr)
    assert np.array_equal(ci, A.col_idx)
    assert np.array_equal(v, A.values)
    U = kspmv.upload_csr(*A.astuple())
    bm, _ = kspmv.row_blocks(M)
    bu, _ = kspmv.row_blocks(U)
    assert np.array_equal(bm, bu)
    x = torch.empty(A.ncols, dtype=torch.float64, device="cuda").uniform_(-1, 1)
    ym = torch.empty(A.nrows, dtype=torch.float64, device="cuda")
    yu = torch.empty_like(ym)
    kspmv.spmv(M, x, ym)
    kspmv.spmv(U, x, yu)
    assert torch.equal(ym, yu)


def test_laplacian_cg_matches_uploaded(kspmv):
    # 256^2 (the 2-D CG workload): same iterations and bits as the uploaded copy.
    A = gen.laplacian_2d(256)
    M = kspmv.laplacian(2, 256)
    U = kspmv.upload_csr(*A.astuple())
    b = torch.tensor(A.to_scipy() @ np.ones(A.nrows), device="cuda")
    xm = torch.zeros(A.nrows, dtype=torch.float64, device="cuda")
    xu = torch.zeros_like(xm)
    rm = kspmv.cg_solve_local(M, b, xm, tol=1e-8, max_iter=2000)
    ru = kspmv.cg_solve_local(U, b, xu, tol=1e-8, max_iter=2000)
    assert rm == ru and rm["iters"] == 454
    assert torch.equal(xm, xu)


def test_download_round_trip_of_uploaded(kspmv):
    A = gen.power_law(5000, seed=7)
    U = kspmv.upload_csr(*A.astuple())
    rp, ci, v = kspmv.download_csr(U)
    assert np.array_equal(rp, A.row_ptr) and np.array_equal(ci, A.col_idx)
    assert np.array_equal(v, A.values)

