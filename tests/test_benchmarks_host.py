"""The benchmark harness with the reference scripts' interface
(num_b200.benchmarks): sizing, metric formulas and CSV layout, on the CPU
(scipy backends only)."""
import csv

import pytest

from num_b200 import benchmarks as B


def test_registry_sizing_follows_the_reference():
    # matrix_generators.py:234-241: L = int(N**0.5) / round(N**(1/3)), N rows otherwise
    assert B.get_matrix("laplacian_2d", 100_000).nrows == 316 * 316
    assert B.get_matrix("laplacian_3d", 1_000_000).nrows == 100 ** 3
    assert B.get_matrix("lattice_gauge", 100_000).nrows == 316 * 316
    assert B.get_matrix("random_sparse", 3000).nrows == 3000
    assert B.get_matrix("power_law", 1000).nrows == 1000
    with pytest.raises(ValueError, match="Unknown matrix"):
        B.get_matrix("dense", 1000)


def test_spmv_metrics_formula():
    # benchmark_spmv.py:108-114
    m = B.spmv_metrics(1e-3, N=1000, nnz=5000, k=4)
    assert m["elapsed_us"] == pytest.approx(1000.0)
    assert m["bw_GB_s"] == pytest.approx((5000 * 12 + 4 * 1000 * 8 + 1000 * 8) / 1e-3 / 1e9)
    assert m["gflops"] == pytest.approx(2 * 5000 * 4 / 1e-3 / 1e9)


def test_spmv_scipy_rows_and_csv(tmp_path, capsys):
    rows = B.run_spmv(["--N", "4096", "--matrix", "laplacian_2d", "--backend", "scipy", "jax",
                       "--repeat", "3", "--out", str(tmp_path)])
    assert [r["backend"] for r in rows] == ["scipy_cpu"]
    r = rows[0]
    assert r["N"] == 4096 and r["nnz"] == 5 * 4096 - 4 * 64
    assert r["bw_GB_s"] == pytest.approx((12 * r["nnz"] + 16 * r["N"]) / (r["elapsed_us"] * 1e-6) / 1e9)
    files = list(tmp_path.glob("spmv_*.csv"))
    assert len(files) == 1
    with open(files[0]) as f:
        got = list(csv.DictReader(f))
    assert list(got[0].keys()) == ["backend", "N", "nnz", "elapsed_us", "bw_GB_s", "gflops"]
    assert "[SKIP] jax_1gpu" in capsys.readouterr().err


def test_cg_scipy_row(tmp_path):
    rows = B.run_cg(["--N", "4096", "--matrix", "laplacian_2d", "--backend", "scipy",
                     "--out", str(tmp_path)])
    r = rows[0]
    assert r["backend"] == "scipy_cg" and r["converged"] and r["iters"] > 0
    assert r["residual"] < 1e-8
    with open(next(tmp_path.glob("cg_*.csv"))) as f:
        assert list(csv.DictReader(f))[0]["backend"] == "scipy_cg"


@pytest.mark.parametrize("name", ["lattice_gauge", "random_sparse", "power_law"])
def test_spmv_scipy_rows_on_the_rest_of_the_registry(tmp_path, name):
    # the reference's own invocation, e.g. benchmark_spmv.py --matrix random_sparse
    rows = B.run_spmv(["--N", "2500", "--matrix", name, "--backend", "scipy", "--repeat", "3",
                       "--out", str(tmp_path)])
    assert rows[0]["backend"] == "scipy_cpu" and rows[0]["nnz"] > rows[0]["N"]


def test_cli_usage():
    assert B.main([]) == 2
    with pytest.raises(SystemExit):
        B.main(["spmv", "--matrix", "dense"])
