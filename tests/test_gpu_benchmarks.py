"""The reference-interface benchmark harness on the GPU: the drop-in
backends produce rows, and the CG row matches SciPy's iteration count."""
import pytest

from num_b200 import benchmarks as B

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_spmv_backends_and_batch(kspmv, tmp_path):
    rows = B.run_spmv(["--N", "100000", "--backend", "kokkos", "kokkos_custom", "--batch", "8",
                       "--repeat", "5", "--out", str(tmp_path)])
    assert [r["backend"] for r in rows] == ["kokkos_kk_1gpu", "kokkos_custom_1gpu",
                                            "kokkos_batch_k8"]
    assert all(r["elapsed_us"] > 0 and r["bw_GB_s"] > 0 for r in rows)
    assert rows[-1]["k"] == 8 and len(list(tmp_path.glob("spmv_*.csv"))) == 1


def test_cg_matches_scipy_iterations(kspmv, tmp_path):
    rows = B.run_cg(["--N", "4096", "--matrix", "laplacian_2d", "--backend", "scipy", "kokkos",
                     "--out", str(tmp_path)])
    by = {r["backend"]: r for r in rows}
    assert by["kspmv_cg_1gpu"]["converged"] and by["scipy_cg"]["converged"]
    assert abs(by["kspmv_cg_1gpu"]["iters"] - by["scipy_cg"]["iters"]) <= 1
    assert by["kspmv_cg_1gpu"]["residual"] < 1e-8
