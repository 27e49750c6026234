"""Regenerate the golden fixtures of tests/golden/ from the reference itself.

Run in a checkout that has the reference project next to it:

    python tests/golden/make_golden.py /path/to/reference

It imports the reference's python/matrix_generators.py (its fixture source) and
evaluates the reference's accuracy oracle, SciPy (python/verify_accuracy.py:
53-54 `A @ x`; tests/test_accuracy.py:172 `spla.cg(A, b, rtol=1e-12)`), on
small instances.  Outputs:

  ref_generators.json  sha256 of (indptr, indices, data) of the reference's
                       make_laplacian_2d / make_laplacian_3d_fast /
                       make_lattice_gauge / make_random_sparse / make_power_law
                       (default seeds, and one case each with a caller's
                       generator and non-default parameters)
  scipy_pins.npz       small reference matrices with x, SciPy y = A @ x, and
                       SciPy CG solutions for b = ones
  c1_probe.json        the 256x256 5-point Laplacian workload: ||A x||_2 for
                       x ~ U[-1, 1] (default_rng(0)), and SciPy's CG
                       iteration count / true residual at rtol 1e-8
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np
import scipy.sparse.linalg as spla

OUT = Path(__file__).resolve().parent


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main(ref_root: str) -> None:
    sys.path.insert(0, str(Path(ref_root) / "python"))
    import matrix_generators as mg  # the reference's generators

    gens = {}
    for L in (16, 64, 256):
        A = mg.make_laplacian_2d(L)
        gens[f"laplacian_2d_{L}"] = {
            "indptr": sha(A.indptr.astype(np.int32)), "indices": sha(A.indices.astype(np.int32)),
            "data": sha(A.data.astype(np.float64)), "nnz": int(A.nnz)}
    for L in (10, 40, 64):
        A = mg.make_laplacian_3d_fast(L)
        gens[f"laplacian_3d_{L}"] = {
            "indptr": sha(A.indptr.astype(np.int32)), "indices": sha(A.indices.astype(np.int32)),
            "data": sha(A.data.astype(np.float64)), "nnz": int(A.nnz)}
    def put(key, A):
        A = A.tocsr()
        gens[key] = {
            "indptr": sha(A.indptr.astype(np.int32)), "indices": sha(A.indices.astype(np.int32)),
            "data": sha(A.data.astype(np.float64)), "nnz": int(A.nnz)}

    for L in (2, 3, 8, 100):
        put(f"lattice_gauge_{L}", mg.make_lattice_gauge(L))
    put("lattice_gauge_20_mass0.5_seed3", mg.make_lattice_gauge(20, 0.5, np.random.default_rng(3)))
    for N in (1, 5, 300, 10000):
        put(f"random_sparse_{N}", mg.make_random_sparse(N))
    put("random_sparse_500_nnz4_seed7_nonsym",
        mg.make_random_sparse(500, 4, np.random.default_rng(7), symmetric=False))
    for N in (5, 500, 3000):
        put(f"power_law_{N}", mg.make_power_law(N))
    put("power_law_800_m5_seed9", mg.make_power_law(800, 5, np.random.default_rng(9)))
    (OUT / "ref_generators.json").write_text(json.dumps(gens, indent=1) + "\n")

    pins = {}
    cases = [("laplacian_2d", 1024), ("laplacian_3d", 1000), ("random_sparse", 300),
             ("lattice_gauge", 1024)]
    for name, N in cases:
        A = mg.get_matrix(name, N).tocsr()
        A.sort_indices()
        x = np.random.default_rng(0).standard_normal(A.shape[1])
        y = np.asarray(A @ x, dtype=np.float64)
        b = np.ones(A.shape[0])
        xs, info = spla.cg(A, b, rtol=1e-12, maxiter=5000)
        pins[f"{name}__indptr"] = A.indptr.astype(np.int32)
        pins[f"{name}__indices"] = A.indices.astype(np.int32)
        pins[f"{name}__data"] = A.data.astype(np.float64)
        pins[f"{name}__x"] = x
        pins[f"{name}__y"] = y
        pins[f"{name}__cg_x"] = xs
        pins[f"{name}__cg_info"] = np.array([info])
    np.savez_compressed(OUT / "scipy_pins.npz", **pins)

    A = mg.make_laplacian_2d(256)
    x = np.random.default_rng(0).uniform(-1.0, 1.0, A.shape[1])
    y = A @ x
    b = A @ np.ones(A.shape[0])
    it = [0]
    xs, info = spla.cg(A, b, rtol=1e-8, maxiter=5000, callback=lambda _: it.__setitem__(0, it[0] + 1))
    probe = {
        "n": int(A.shape[0]), "nnz": int(A.nnz),
        "spmv_y_norm2": float(np.linalg.norm(y)),
        "spmv_y_sha256": sha(np.asarray(y, np.float64)),
        "scipy_cg_iters": it[0], "scipy_cg_info": int(info),
        "scipy_cg_true_relres": float(np.linalg.norm(b - A @ xs) / np.linalg.norm(b)),
    }
    (OUT / "c1_probe.json").write_text(json.dumps(probe, indent=1) + "\n")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "../reference")
