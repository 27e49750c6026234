"""Deterministic CSR generators for the benchmark workloads and the reference's
test matrices.  Host-side numpy; every function returns int32 row_ptr / col_idx
(columns ascending within a row) and float64 values.

Reference counterparts (python/matrix_generators.py of w-jiwonchoi/num), each
producing the same arrays as the reference function followed by SciPy's CSR
canonicalisation (columns ascending, repeated entries summed):
  laplacian_2d   <- make_laplacian_2d (:16-37)
  laplacian_3d   <- make_laplacian_3d_fast (:68-80)
  lattice_gauge  <- make_lattice_gauge (:85-139), same numpy random stream
  random_sparse  <- make_random_sparse (:144-170), same numpy random stream
  ba_laplacian   <- make_power_law (:175-229), same numpy random stream
  get_matrix     <- get_matrix / MATRIX_REGISTRY (:234-260)
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


# ---- the rest of the reference's generator family -------------------------------------

def _canonical(rows, cols, vals, n: int, ncols: int | None = None, drop_zeros: bool = False) -> Csr:
    """COO triplets -> CSR, columns ascending within a row, repeated (row, col)
    entries summed (the canonical form SciPy's COO -> CSR conversion gives;
    bit-exact for up to two repeats of an entry, where the order of the sum
    cannot matter).  drop_zeros removes entries whose value is exactly zero,
    as SciPy's sparse + / - do."""
    r = np.asarray(rows, np.int64)
    c = np.asarray(cols, np.int64)
    v = np.asarray(vals, np.float64)
    order = np.lexsort((c, r))
    r, c, v = r[order], c[order], v[order]
    if r.size:
        first = np.ones(r.size, bool)
        first[1:] = (r[1:] != r[:-1]) | (c[1:] != c[:-1])
        seg = np.cumsum(first) - 1
        out = np.zeros(int(first.sum()), np.float64)
        # sequential sums in the stored order: one pass per repeat depth
        pos = np.arange(r.size) - np.flatnonzero(first)[seg]
        for d in range(int(pos.max()) + 1):
            m = pos == d
            out[seg[m]] = out[seg[m]] + v[m] if d else v[m]
        r, c, v = r[first], c[first], out
    if drop_zeros:
        keep = v != 0.0
        r, c, v = r[keep], c[keep], v[keep]
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(r, minlength=n), out=rp[1:])
    return Csr(rp.astype(np.int32), c.astype(np.int32), v, n, n if ncols is None else ncols)


def _row_sums(A: Csr, absolute: bool = False) -> np.ndarray:
    """Row sums formed the way SciPy's CSR sum(axis=1) forms them: one
    np.add.reduceat over the stored values of the non-empty rows (numpy adds
    a row's first value to the pairwise sum of the rest), 0 for empty rows --
    so the diagonals built from them carry the same bits."""
    rp = A.row_ptr.astype(np.int64)
    v = np.abs(A.values) if absolute else A.values
    out = np.zeros(A.nrows)
    rows = np.flatnonzero(np.diff(rp))
    if rows.size:
        out[rows] = np.add.reduceat(v, rp[rows])
    return out


def _coo(A: Csr):
    rows = np.repeat(np.arange(A.nrows, dtype=np.int64), np.diff(A.row_ptr.astype(np.int64)))
    return rows, A.col_idx.astype(np.int64), A.values


def lattice_gauge(L: int, mass: float = 0.1, rng: np.random.Generator | None = None) -> Csr:
    """Scalar 2-D lattice-gauge (Dirac-like) operator on an L x L torus
    (make_lattice_gauge, python/matrix_generators.py:85-139): random U(1)
    phases phi_x, phi_y ~ U[0, 2 pi) per site (drawn in that order, (y, x)
    layout, default_rng(42)); site i = y L + x couples to itself with 4 + mass
    and to its four periodic neighbours with -Re(e^{+-i phi}) / 2 (the +x / +y
    hop uses the site's own link, -x / -y the neighbour's); the result is
    symmetrised as (A + A^T) / 2.  n = L^2, 5 nonzeros per row for L >= 3.
    Bit-exact with the reference for L >= 2."""
    if rng is None:
        rng = np.random.default_rng(42)
    n = L * L
    phi_x = rng.uniform(0, 2 * np.pi, (L, L))
    phi_y = rng.uniform(0, 2 * np.pi, (L, L))
    i = np.arange(n, dtype=np.int64)
    x, y = i % L, i // L
    xp, xm, yp, ym = (x + 1) % L, (x - 1) % L, (y + 1) % L, (y - 1) % L
    hop = lambda phi, s: -0.5 * np.exp(s * 1j * phi).real  # noqa: E731
    # per site in the reference's append order: self, +x, -x, +y, -y
    cols = np.stack([i, y * L + xp, y * L + xm, yp * L + x, ym * L + x], axis=1)
    vals = np.stack([np.full(n, 4.0 + mass), hop(phi_x[y, x], 1), hop(phi_x[y, xm], -1),
                     hop(phi_y[y, x], 1), hop(phi_y[ym, x], -1)], axis=1)
    A = _canonical(np.repeat(i, 5), cols.ravel(), vals.ravel(), n)
    r, c, v = _coo(A)
    S = _canonical(np.concatenate([r, c]), np.concatenate([c, r]), np.concatenate([v, v]), n,
                   drop_zeros=True)
    S.values = 0.5 * S.values
    return S


def random_sparse(N: int, nnz_per_row: int = 10, rng: np.random.Generator | None = None,
                  symmetric: bool = True) -> Csr:
    """Random diagonally dominant SPD matrix (make_random_sparse,
    python/matrix_generators.py:144-170): row i draws min(nnz_per_row - 1, i)
    distinct columns j < i (Generator.choice without replacement) and one
    value v ~ U[0.1, 1) per column, in that order, from default_rng(0); entry
    -v at (i, j) and, when symmetric, at (j, i); the diagonal is the row's
    absolute sum + 1."""
    if rng is None:
        rng = np.random.default_rng(0)
    rows, cols, vals = [], [], []
    for i in range(N):
        n_off = min(nnz_per_row - 1, i)
        if n_off > 0:
            js = rng.choice(i, size=n_off, replace=False)
            vs = rng.uniform(0.1, 1.0, size=n_off)  # the same draws as n_off scalar calls
            rows.append(np.full(n_off, i, np.int64))
            cols.append(np.asarray(js, np.int64))
            vals.append(-vs)
    r = np.concatenate(rows) if rows else np.zeros(0, np.int64)
    c = np.concatenate(cols) if cols else np.zeros(0, np.int64)
    v = np.concatenate(vals) if vals else np.zeros(0)
    if symmetric:
        r, c, v = np.concatenate([r, c]), np.concatenate([c, r]), np.concatenate([v, v])
    A = _canonical(r, c, v, N)
    d = _row_sums(A, absolute=True) + 1.0
    ar, ac, av = _coo(A)
    i = np.arange(N, dtype=np.int64)
    return _canonical(np.concatenate([ar, i]), np.concatenate([ac, i]), np.concatenate([av, d]),
                      N, drop_zeros=True)


def ba_laplacian(N: int, m: int = 3, rng: np.random.Generator | None = None) -> Csr:
    """Barabasi-Albert preferential-attachment graph as an SPD matrix
    (make_power_law, python/matrix_generators.py:175-229): a clique on the
    first min(m + 1, N) nodes, then every later node attaches to min(m, node)
    distinct earlier nodes drawn with probability degree / total degree
    (Generator.choice without replacement, default_rng(1)); the matrix is
    diag(degree) - A with A_uv = -1 on every edge, i.e. degrees on the diagonal
    and +1 per edge.  O(N^2) host work, like the reference."""
    if rng is None:
        rng = np.random.default_rng(1)
    degrees = np.zeros(N, dtype=np.int64)
    us: list = []
    vs: list = []
    seed = min(m + 1, N)
    for a in range(seed):
        for b in range(a):
            us.append(a)
            vs.append(b)
            degrees[a] += 1
            degrees[b] += 1
    for node in range(seed, N):
        deg_sum = degrees[:node].sum()
        if deg_sum == 0:
            targets = rng.choice(node, size=min(m, node), replace=False)
        else:
            p = degrees[:node] / deg_sum
            targets = rng.choice(node, size=min(m, node), replace=False, p=p)
        for t in targets:
            us.append(node)
            vs.append(int(t))
            degrees[node] += 1
            degrees[t] += 1
    u = np.asarray(us, np.int64)
    v = np.asarray(vs, np.int64)
    A = _canonical(np.concatenate([u, v]), np.concatenate([v, u]), np.full(2 * u.size, -1.0), N)
    d = _row_sums(A, absolute=True)
    ar, ac, av = _coo(A)
    i = np.arange(N, dtype=np.int64)
    return _canonical(np.concatenate([i, ar]), np.concatenate([i, ac]), np.concatenate([d, -av]),
                      N, drop_zeros=True)


MATRICES = ("laplacian_2d", "laplacian_3d", "lattice_gauge", "random_sparse", "power_law")


def get_matrix(name: str, N: int) -> Csr:
    """The reference's registry (python/matrix_generators.py:234-260): N is
    the approximate row count -- L = int(N ** 0.5) for the 2-D grids,
    round(N ** (1/3)) for the 3-D one, N itself for the random and graph
    matrices."""
    if name == "laplacian_2d":
        return laplacian_2d(int(N ** 0.5))
    if name == "laplacian_3d":
        return laplacian_3d(int(round(N ** (1.0 / 3.0))))
    if name == "lattice_gauge":
        return lattice_gauge(int(N ** 0.5))
    if name == "random_sparse":
        return random_sparse(N)
    if name == "power_law":
        return ba_laplacian(N)
    raise ValueError(f"Unknown matrix '{name}'. Choose from: {list(MATRICES)}")
