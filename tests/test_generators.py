"""The workload generators: identical to the reference's generators where it
has them (hashes recorded from the reference by tests/golden/make_golden.py),
and the stated properties of the synthetic workloads otherwise."""
import hashlib
import json

import numpy as np
import pytest

from conftest import GOLDEN
from num_b200 import generators as gen


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


REF = json.loads((GOLDEN / "ref_generators.json").read_text())


def _build(key):
    """The generator call a fixture key names (the reference's function of the
    same name with the same arguments: size, then mass / nnz_per_row / m,
    then a default_rng seed, then symmetric=False)."""
    if key.startswith("laplacian_"):
        kind, L = key.rsplit("_", 1)
        return (gen.laplacian_2d if kind == "laplacian_2d" else gen.laplacian_3d)(int(L))
    head, _, rest = key.partition("_")[2].partition("_")
    name = {"gauge": "lattice_gauge", "sparse": "random_sparse", "law": "power_law"}[head]
    parts = rest.split("_")
    size = int(parts[0])
    if len(parts) == 1:
        return gen.get_matrix(name, size * size if name == "lattice_gauge" else size)
    rng = np.random.default_rng(int(parts[2].replace("seed", "")))
    if name == "lattice_gauge":
        return gen.lattice_gauge(size, float(parts[1].replace("mass", "")), rng)
    if name == "random_sparse":
        return gen.random_sparse(size, int(parts[1].replace("nnz", "")), rng,
                                 symmetric="nonsym" not in parts)
    return gen.ba_laplacian(size, int(parts[1].replace("m", "")), rng)


@pytest.mark.parametrize("key", sorted(REF))
def test_matches_reference_generators(key):
    A = _build(key)
    ref = REF[key]
    assert A.nnz == ref["nnz"]
    assert sha(A.row_ptr) == ref["indptr"]
    assert sha(A.col_idx) == ref["indices"]
    assert sha(A.values) == ref["data"]


def test_power_law_properties():
    A = gen.power_law(200_000, seed=11)
    lens = np.diff(A.row_ptr)
    assert lens.min() >= 1 and lens.max() <= 2048
    assert 14.0 < lens.mean() < 18.0
    for i in np.random.default_rng(0).integers(0, A.nrows, 2000):
        c = A.col_idx[A.row_ptr[i]:A.row_ptr[i + 1]]
        assert np.all(np.diff(c) > 0)  # ascending, no repeats
    assert abs(A.values.mean()) < 0.01 and abs(A.values.std() - 1) < 0.01


def test_banded_batch_properties():
    mats, xs = gen.banded_batch(64, seed=2)
    for A, x in zip(mats, xs):
        assert 32 <= A.nrows <= 4096 and x.shape == (A.nrows,)
        S = A.to_scipy()
        assert (S - S.T).nnz == 0                       # symmetric
        d = S.diagonal()
        off = np.asarray(abs(S).sum(axis=1)).ravel() - np.abs(d)
        assert np.allclose(d, 1.05 * off)                # diagonal = 1.05 x row sum
        assert np.all(S.data[S.indices != np.repeat(np.arange(A.nrows), np.diff(A.row_ptr))] <= 0)
        for i in range(0, A.nrows, 7):
            assert np.all(np.diff(A.col_idx[A.row_ptr[i]:A.row_ptr[i + 1]]) > 0)


def test_varcoef_poisson_properties():
    A, b = gen.varcoef_poisson_3d(16, seed=3)
    n = 16 ** 3
    assert A.nrows == n and A.nnz == 7 * n - 6 * 16 * 16 and b.shape == (n,)
    S = A.to_scipy()
    assert abs(S - S.T).max() == 0
    off = np.asarray(abs(S).sum(axis=1)).ravel() - S.diagonal()
    # weakly diagonally dominant everywhere (equality inside), strictly at the
    # Dirichlet boundary, irreducible => SPD
    assert np.all(S.diagonal() >= off * (1 - 1e-15)) and np.any(S.diagonal() > off * 1.01)


def test_c4_nnz_matches_stencil_count():
    # 128^3: n = 2,097,152 and 7n - 6*128^2 = 14,581,760 nonzeros
    L = 128
    assert 7 * L ** 3 - 6 * L * L == 14_581_760


def test_spmv_bytes_formula():
    # 3-D 160^3 FP64: 424.14 MB per SpMV
    A_nnz, n = 28_518_400, 4_096_000
    assert gen.spmv_bytes(A_nnz, n, n) == 12 * A_nnz + 4 * (n + 1) + 16 * n
    assert abs(gen.spmv_bytes(A_nnz, n, n) / 1e6 - 424.14) < 0.01


def test_get_matrix_registry_sizes():
    # the reference registry's N -> size mapping (python/matrix_generators.py:234-241)
    assert gen.get_matrix("laplacian_2d", 1000).nrows == 31 * 31
    assert gen.get_matrix("laplacian_3d", 1000).nrows == 1000
    assert gen.get_matrix("lattice_gauge", 1000).nrows == 31 * 31
    assert gen.get_matrix("random_sparse", 1000).nrows == 1000
    assert gen.get_matrix("power_law", 300).nrows == 300
    with pytest.raises(ValueError, match="Unknown matrix"):
        gen.get_matrix("dense", 10)


@pytest.mark.parametrize("name", ["lattice_gauge", "random_sparse", "power_law"])
def test_family_symmetric_sorted(name):
    A = gen.get_matrix(name, 900)
    S = A.to_scipy()
    assert abs(S - S.T).max() == 0
    for i in range(A.nrows):
        assert np.all(np.diff(A.col_idx[A.row_ptr[i]:A.row_ptr[i + 1]]) > 0)
    # diagonally dominant with a positive diagonal (SPD, or PSD for the graph)
    d = S.diagonal()
    off = np.asarray(abs(S).sum(axis=1)).ravel() - np.abs(d)
    assert np.all(d > 0) and np.all(d >= off * (1 - 1e-12))
