"""bench.py's host side without a GPU: the reference arm's JSON line, the CPU
baseline's solution output, and the algorithmic byte counts."""
import importlib.util
import json
import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_reference_arm_line_for_cg_c1():
    # The driver's reference arm: the oracle port timed on the host cores,
    # one JSON line with the same metric, unit and config keys as our arm's.
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload",
                          "cg_c1", "--steps", "2", "--warmup", "3"], cwd=ROOT,
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "solves/s"
    assert line["higher_is_better"] is True and line["value"] > 0
    cfg = line["config"]
    assert cfg["name"] == "cg_c1" and cfg["nrows"] == 65536 and cfg["nnz"] == 326656
    assert cfg["tol"] == 1e-8
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0


def test_cpu_baseline_cg_hands_back_the_solution():
    # The C4 line compares the engine's solution with the oracle's Jacobi-PCG
    # one; the CPU leg returns that solution when it times full solves.
    from num_b200 import generators as gen
    bench = _bench()
    A, b = gen.varcoef_poisson_3d(12, seed=3)
    got = {}
    cb = bench.cpu_baseline_cg(A, b, 1e-10, budget_s=0.5, precond=True, full_iters=60, out=got)
    assert cb["unit"] == "solves/s" and cb["value"] > 0
    x = got["x"]
    assert np.linalg.norm(A.to_scipy() @ x - b) <= 1e-9 * np.linalg.norm(b)


def test_algorithmic_byte_counts():
    bench = _bench()
    assert bench.vec_bytes(10) == 640                  # axpy 24n + axpy2 24n + dot 16n
    assert bench.halo_bytes(3, 2) == 3 * 20 + 2 * 16   # pack 20 B per value, unpack 16
