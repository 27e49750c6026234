"""Deterministic CSR generators for the benchmark workloads and the reference's
test matrices.  Host-side numpy; every function returns int32 row_ptr / col_idx
(columns ascending within a row) and float64 values.

Reference counterparts (python/matrix_generators.py of w-jiwonchoi/num):
  laplacian_2d  <- make_laplacian_2d (:16-37), identical arrays
  laplacian_3d  <- make_laplacian_3d_fast (:68-80), identical arrays
The remaining generators define the synthetic workloads of this library
(power-law rows, many banded SPD systems, variable-coefficient Poisson) and
the known-answer matrices of the reference's C++ tests.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


@dataclass
class Csr:
    row_ptr: np.ndarray   # int32[n+1]
    col_idx: np.ndarray   # int32[nnz]
    values: np.ndarray    # float64[nnz]
    nrows: int
    ncols: int

    @property
    def nnz(self) -> int:
        return int(self.row_ptr[self.nrows])

    def astuple(self):
        return self.row_ptr, self.col_idx, self.values, self.nrows, self.ncols

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.values, self.col_idx, self.row_ptr),
                             shape=(self.nrows, self.ncols))


def _from_candidates(cols: np.ndarray, vals: np.ndarray, valid: np.ndarray, n: int,
                     ncols: int | None = None) -> Csr:
    """Rows given as fixed-width candidate lists (already in ascending column
    order) with a validity mask."""
    counts = valid.sum(axis=1)
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(counts, out=rp[1:])
    ci = cols[valid].astype(np.int32)
    v = vals[valid].astype(np.float64)
    return Csr(rp.astype(np.int32), ci, v, n, n if ncols is None else ncols)


def laplacian_2d(L: int) -> Csr:
    """5-point Laplacian (4 / -1) on an L x L grid, row-major, Dirichlet."""
    n = L * L
    i = np.arange(n, dtype=np.int64)
    x, y = i % L, i // L
    cols = np.stack([i - L, i - 1, i, i + 1, i + L], axis=1)
    valid = np.stack([y > 0, x > 0, np.ones(n, bool), x < L - 1, y < L - 1], axis=1)
    vals = np.broadcast_to(np.array([-1.0, -1.0, 4.0, -1.0, -1.0]), (n, 5))
    return _from_candidates(cols, vals, valid, n)


def laplacian_3d(L: int) -> Csr:
    """7-point Laplacian (6 / -1) on an L^3 grid (x fastest), Dirichlet."""
    n = L * L * L
    i = np.arange(n, dtype=np.int64)
    x, y, z = i % L, (i // L) % L, i // (L * L)
    LL = L * L
    cols = np.stack([i - LL, i - L, i - 1, i, i + 1, i + L, i + LL], axis=1)
    valid = np.stack([z > 0, y > 0, x > 0, np.ones(n, bool), x < L - 1, y < L - 1, z < L - 1],
                     axis=1)
    vals = np.broadcast_to(np.array([-1.0, -1.0, -1.0, 6.0, -1.0, -1.0, -1.0]), (n, 7))
    return _from_candidates(cols, vals, valid, n)


def laplacian_1d(N: int) -> Csr:
    """Tridiagonal [-1, 2, -1] (tests/test_cg.cpp:76-95)."""
    i = np.arange(N, dtype=np.int64)
    cols = np.stack([i - 1, i, i + 1], axis=1)
    valid = np.stack([i > 0, np.ones(N, bool), i < N - 1], axis=1)
    vals = np.broadcast_to(np.array([-1.0, 2.0, -1.0]), (N, 3))
    return _from_candidates(cols, vals, valid, N)


def diagonal(d) -> Csr:
    d = np.asarray(d, np.float64)
    n = d.shape[0]
    return Csr(np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32), d.copy(), n, n)


def tridiag4() -> Csr:
    """The 4x4 [-1, 2, -1] matrix of tests/test_spmv_kernel.cpp:65-70."""
    return Csr(np.array([0, 2, 5, 8, 10], np.int32),
               np.array([0, 1, 0, 1, 2, 1, 2, 3, 2, 3], np.int32),
               np.array([2, -1, -1, 2, -1, -1, 2, -1, -1, 2], np.float64), 4, 4)


def lcg_random(N: int = 10000, nnz_per_row: int = 7):
    """The seeded LCG matrix and x of tests/test_spmv_kernel.cpp:163-195
    (seed 42, seed = seed*1664525 + 1013904223 mod 2^32; diagonal first, then
    random off-diagonals in draw order, so columns are unsorted and may repeat)."""
    seed = 42
    mask = 0xFFFFFFFF

    def lcg():
        nonlocal seed
        seed = (seed * 1664525 + 1013904223) & mask
        return seed

    x = np.array([(lcg() % 1000) * 0.001 - 0.5 for _ in range(N)], np.float64)
    rp = [0]
    ci: list[int] = []
    vals: list[float] = []
    for i in range(N):
        ci.append(i)
        vals.append(float(nnz_per_row))
        for _ in range(1, nnz_per_row):
            j = lcg() % N
            if j != i:
                ci.append(j)
                vals.append(-1.0)
        rp.append(len(ci))
    return Csr(np.array(rp, np.int32), np.array(ci, np.int32), np.array(vals), N, N), x


def power_law(n: int = 2_000_000, mean: float = 16.0, sigma: float = 1.2, max_len: int = 2048,
              seed: int = 1001) -> Csr:
    """Random matrix with lognormal row lengths (distribution mean `mean`,
    log-space sigma `sigma`, rounded, clipped to [1, max_len]); columns uniform
    without repeats within a row, ascending; values N(0, 1)."""
    rng = np.random.default_rng(seed)
    mu = math.log(mean) - sigma * sigma / 2.0
    lens = np.clip(np.rint(rng.lognormal(mu, sigma, n)), 1, max_len).astype(np.int64)
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(lens, out=rp[1:])
    nnz = int(rp[-1])
    row = np.repeat(np.arange(n, dtype=np.int64), lens)
    col = rng.integers(0, n, size=nnz, dtype=np.int64)
    for _ in range(64):
        key = row * n + col
        order = np.argsort(key, kind="stable")
        key = key[order]
        col = col[order]
        dup = np.zeros(nnz, bool)
        dup[1:] = key[1:] == key[:-1]
        nd = int(dup.sum())
        if nd == 0:
            break
        col[dup] = rng.integers(0, n, size=nd, dtype=np.int64)
    else:  # pragma: no cover - needs astronomically bad luck
        raise RuntimeError("power_law: could not remove repeated columns")
    vals = rng.standard_normal(nnz)
    return Csr(rp.astype(np.int32), col.astype(np.int32), vals, n, n)


def banded_spd(n: int, hb: int, rng: np.random.Generator, offband: int = 2) -> Csr:
    """Symmetric banded matrix: half-bandwidth hb, `offband` random entries per
    row outside the band (mirrored), off-diagonals U[-1, 0], diagonal 1.05 x
    the row's absolute off-diagonal sum (strictly diagonally dominant => SPD)."""
    i = np.arange(n, dtype=np.int64)
    # band pairs (i, i+d), d = 1..hb
    ba = np.concatenate([np.arange(n - d, dtype=np.int64) for d in range(1, hb + 1) if d < n])
    bb = np.concatenate([np.arange(d, n, dtype=np.int64) for d in range(1, hb + 1) if d < n])
    # off-band draws: uniform over the columns outside [i-hb, i+hb]
    lo = np.maximum(i - hb, 0)
    hi = np.minimum(i + hb, n - 1)
    cand = n - (hi - lo + 1)
    rows_o = np.repeat(i, offband)
    cand_o = np.repeat(cand, offband)
    u = np.floor(rng.random(rows_o.shape[0]) * np.maximum(cand_o, 1)).astype(np.int64)
    lo_o = np.repeat(lo, offband)
    width_o = np.repeat(hi - lo + 1, offband)
    j = np.where(u < lo_o, u, u + width_o)
    keep = cand_o > 0
    oa = np.minimum(rows_o, j)[keep]
    ob = np.maximum(rows_o, j)[keep]
    okey = np.unique(oa * n + ob)
    oa, ob = okey // n, okey % n
    pa = np.concatenate([ba, oa])
    pb = np.concatenate([bb, ob])
    pv = rng.uniform(-1.0, 0.0, pa.shape[0])
    diag = np.zeros(n)
    np.add.at(diag, pa, np.abs(pv))
    np.add.at(diag, pb, np.abs(pv))
    diag *= 1.05
    r = np.concatenate([pa, pb, i])
    c = np.concatenate([pb, pa, i])
    v = np.concatenate([pv, pv, diag])
    order = np.lexsort((c, r))
    r, c, v = r[order], c[order], v[order]
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(r, minlength=n), out=rp[1:])
    return Csr(rp.astype(np.int32), c.astype(np.int32), v, n, n)


def banded_batch(count: int = 4096, nmin: int = 32, nmax: int = 4096, seed: int = 2):
    """`count` banded SPD matrices, n log-uniform in [nmin, nmax], half-bandwidth
    uniform in {1..8}; returns (list of Csr, list of x ~ U[-1, 1])."""
    rng = np.random.default_rng(seed)
    xrng = np.random.default_rng(seed + 100)
    mats, xs = [], []
    for _ in range(count):
        n = int(round(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
        hb = int(rng.integers(1, 9))
        mats.append(banded_spd(n, hb, rng))
        xs.append(xrng.uniform(-1.0, 1.0, n))
    return mats, xs


def varcoef_poisson_3d(L: int = 128, seed: int = 3):
    """7-point variable-coefficient Poisson on an L^3 grid: every cell face f
    (boundary faces included) carries c_f = exp(g_f), g_f ~ N(0, 1) i.i.d.,
    drawn x-faces, then y-faces, then z-faces; A_ij = -c_f for the face
    between cells i and j, A_ii = sum of the cell's six face coefficients
    (Dirichlet boundary), so A is SPD.  Returns (Csr, b ~ N(0, 1))."""
    rng = np.random.default_rng(seed)
    cx = np.exp(rng.standard_normal((L, L, L + 1)))   # [z, y, x-face]
    cy = np.exp(rng.standard_normal((L, L + 1, L)))   # [z, y-face, x]
    cz = np.exp(rng.standard_normal((L + 1, L, L)))   # [z-face, y, x]
    b = rng.standard_normal(L * L * L)
    n = L * L * L
    i = np.arange(n, dtype=np.int64)
    x, y, z = i % L, (i // L) % L, i // (L * L)
    LL = L * L
    w_xm = cx[z, y, x]
    w_xp = cx[z, y, x + 1]
    w_ym = cy[z, y, x]
    w_yp = cy[z, y + 1, x]
    w_zm = cz[z, y, x]
    w_zp = cz[z + 1, y, x]
    diag = w_xm + w_xp + w_ym + w_yp + w_zm + w_zp
    cols = np.stack([i - LL, i - L, i - 1, i, i + 1, i + L, i + LL], axis=1)
    vals = np.stack([-w_zm, -w_ym, -w_xm, diag, -w_xp, -w_yp, -w_zp], axis=1)
    valid = np.stack([z > 0, y > 0, x > 0, np.ones(n, bool), x < L - 1, y < L - 1, z < L - 1],
                     axis=1)
    return _from_candidates(cols, vals, valid, n), b


def spmv_bytes(nnz: int, nrows: int, ncols: int, val_bytes: int = 8, vec_bytes: int = 8,
               k: int = 1) -> int:
    """Algorithmic HBM bytes of one CSR SpMV: values + int32 col_idx, int32
    row_ptr, x read once, y written once (k right-hand sides)."""
    return (val_bytes + 4) * nnz + 4 * (nrows + 1) + vec_bytes * k * (ncols + nrows)
