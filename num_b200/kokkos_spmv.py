"""Drop-in replacement for the reference's `kokkos_spmv` Python module
(w-jiwonchoi/num, src/bindings.cpp:38-294), backed by the num_b200 CUDA
library for B200 through its C ABI (include/num_b200.h).

    from num_b200 import kokkos_spmv as kspmv
    kspmv.init(0)
    A = kspmv.upload_csr(indptr_i32, indices_i32, data_f64, n, n)
    kspmv.spmv(A, x, y)                      # x, y: torch CUDA float64
    info = kspmv.cg_solve_local(A, b, x, tol=1e-10, max_iter=1000)

Same names, argument meanings, defaults and exception types as the reference
binding.  Every call is synchronous with respect to torch's current CUDA
stream (the reference fences after each kernel); device arrays are borrowed
zero-copy and written in place.  Device arrays are torch CUDA tensors or any
object exporting DLPack / __cuda_array_interface__.

Additions beyond the reference surface are keyword-only or separate names:
`upload_csr(..., precision="fp32"|"bf16")`, `upload_csr_batched`, `tune`,
`tuning`, `autotune`, `row_blocks`.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._arrays import device_array, host_array, stream_of

try:
    import torch
except ImportError:  # pragma: no cover
    torch = None

__all__ = [
    "init", "finalize", "rank", "size", "barrier", "CrsMatrix", "DistCrsMatrix", "upload_csr",
    "upload_csr_batched", "distribute_csr", "spmv", "spmv_host", "batch_spmv", "dist_spmv",
    "cg_solve", "cg_solve_local", "tune", "tuning", "autotune", "row_blocks", "laplacian",
    "download_csr", "spmv_kernel",
]

_PRECISIONS = {"fp64": _lib.NM_F64, "fp32": _lib.NM_F32, "bf16": _lib.NM_BF16}
# nm_tuning.kernel: the plain SpMV kernel (auto, the row-block pipeline, the warp gather)
_KERNELS = {"auto": 1, "blocks": 2, "gather": 3, "sliced": 4}


def _dist():
    if torch is not None and torch.distributed.is_available() and torch.distributed.is_initialized():
        return torch.distributed
    return None


# ---- init / MPI-style helpers (src/bindings.cpp:53-76) ----------------------

def init(device_id: int = 0):
    """Select the CUDA device and create its context.  Returns (rank, size).

    Safe to call multiple times.  One process per GPU: pass
    device_id = rank % n_gpu.  rank/size come from torch.distributed when a
    process group is initialised, else (0, 1)."""
    lib = _lib.load()
    r, s = C.c_int32(0), C.c_int32(1)
    _lib.check(lib.nm_init(int(device_id), C.byref(r), C.byref(s)), "init")
    if torch is not None:
        torch.cuda.set_device(int(device_id))
    return rank(), size()


def finalize() -> None:
    """Release cached library workspaces (optional)."""
    _lib.check(_lib.load().nm_finalize(), "finalize")


def rank() -> int:
    d = _dist()
    return d.get_rank() if d else 0


def size() -> int:
    d = _dist()
    return d.get_world_size() if d else 1


def barrier() -> None:
    """Barrier over the process group (no-op with one process)."""
    d = _dist()
    if d:
        d.barrier()


# ---- matrix handles (src/bindings.cpp:79-94) ---------------------------------

class CrsMatrix:
    """Opaque handle to a device-side CSR matrix."""

    __slots__ = ("_h", "_nrows", "_ncols", "_nnz", "_dtype", "_batch", "__weakref__")

    def __init__(self, handle: int, batch=None):
        self._h = C.c_void_p(handle)
        nr, nc, nz, dt, nb = (C.c_int32() for _ in range(5))
        _lib.check(_lib.load().nm_csr_info(self._h, C.byref(nr), C.byref(nc), C.byref(nz),
                                           C.byref(dt), C.byref(nb)))
        self._nrows, self._ncols, self._nnz, self._dtype = nr.value, nc.value, nz.value, dt.value
        self._batch = batch

    @property
    def nrows(self) -> int:
        return self._nrows

    @property
    def ncols(self) -> int:
        return self._ncols

    @property
    def nnz(self) -> int:
        return self._nnz

    @property
    def precision(self) -> str:
        return {v: k for k, v in _PRECISIONS.items()}[self._dtype]

    @property
    def batch_offsets(self):
        """(row offsets, column offsets) of a many-matrix handle, else None."""
        return self._batch

    def __repr__(self) -> str:
        return f"<CrsMatrix nrows={self._nrows} ncols={self._ncols} nnz={self._nnz}>"

    def __del__(self):
        h = getattr(self, "_h", None)
        try:
            if h is not None and h.value and _lib._lib is not None:
                _lib._lib.nm_csr_destroy(h)
        except (AttributeError, TypeError):  # interpreter shutdown
            pass
        self._h = None


class DistCrsMatrix:
    """Opaque handle to this rank's slice of a row-distributed CSR matrix."""

    def __init__(self, handle: int):
        self._h = C.c_void_p(handle)
        vals = [C.c_int32() for _ in range(7)]
        _lib.check(_lib.load().nm_dist_info(self._h, *map(C.byref, vals)))
        (self._global_nrows, self._row_start, self._row_end, self.n_ghost, self.total_send,
         self.n_send_nbrs, self.n_recv_nbrs) = (v.value for v in vals)
        self._plan = None

    @property
    def global_nrows(self) -> int:
        return self._global_nrows

    @property
    def local_row_start(self) -> int:
        return self._row_start

    @property
    def local_row_end(self) -> int:
        return self._row_end

    def plan(self):
        """The halo exchange plan (num_b200.halo.HaloPlan) of this rank."""
        if self._plan is None:
            from .halo import HaloPlan
            self._plan = HaloPlan.from_handle(self._h, self)
        return self._plan

    def __repr__(self) -> str:
        return (f"<DistCrsMatrix global_nrows={self._global_nrows} "
                f"rows=[{self._row_start}, {self._row_end}) ghosts={self.n_ghost}>")

    def __del__(self):
        h = getattr(self, "_h", None)
        try:
            if h is not None and h.value and _lib._lib is not None:
                _lib._lib.nm_dist_destroy(h)
        except (AttributeError, TypeError):  # interpreter shutdown
            pass
        self._h = None


# ---- upload / distribute (src/bindings.cpp:97-148) -----------------------------

def _values_for(values: np.ndarray, precision: str):
    if precision not in _PRECISIONS:
        raise ValueError(f"precision must be one of {sorted(_PRECISIONS)}, got {precision!r}")
    if precision == "fp64":
        return values, _lib.NM_F64
    if precision == "fp32":
        return values.astype(np.float32), _lib.NM_F32
    # bf16: round-to-nearest-even of the float32 value, stored as uint16 bits.
    f = values.astype(np.float32).view(np.uint32).astype(np.uint64)
    rounded = ((f + 0x7FFF + ((f >> 16) & 1)) >> 16).astype(np.uint16)
    return rounded, _lib.NM_BF16


def _check_csr_lengths(rowptr, colind, values, nrows, who):
    if nrows <= 0:
        raise ValueError("CrsMatrixHandle: non-positive dimensions")
    if rowptr.shape[0] < nrows + 1:
        raise ValueError(f"{who}: rowptr length {rowptr.shape[0]} < nrows+1 = {nrows + 1}")
    nnz = int(rowptr[nrows])
    if colind.shape[0] < nnz or values.shape[0] < nnz:
        raise ValueError(f"{who}: colind/values shorter than nnz = rowptr[nrows] = {nnz}")


def upload_csr(rowptr, colind, values, nrows: int, ncols: int, *, precision: str = "fp64"):
    """Upload a CSR matrix from host NumPy arrays to the GPU.

    rowptr int32[nrows+1], colind int32[nnz], values float64[nnz].  Returns a
    CrsMatrix.  `precision` (addition) stores the values as fp32 or bf16."""
    rowptr = host_array(rowptr, np.int32, "rowptr")
    colind = host_array(colind, np.int32, "colind")
    values = host_array(values, np.float64, "values")
    nrows, ncols = int(nrows), int(ncols)
    if nrows <= 0 or ncols <= 0:
        raise ValueError("CrsMatrixHandle: non-positive dimensions")
    _check_csr_lengths(rowptr, colind, values, nrows, "upload_csr")
    vals, dt = _values_for(values, precision)
    out = C.c_void_p()
    _lib.check(_lib.load().nm_csr_create(rowptr.ctypes.data, colind.ctypes.data, vals.ctypes.data,
                                         dt, nrows, ncols, C.byref(out)), "upload_csr")
    return CrsMatrix(out.value)


def laplacian(dim: int, L: int, *, precision: str = "fp64") -> CrsMatrix:
    """The Dirichlet Laplacian on an L^dim grid (dim 2: 5-point, 4 / -1;
    dim 3: 7-point, 6 / -1; x fastest) assembled on the GPU (addition).

    Same matrix as upload_csr of the reference generators
    make_laplacian_2d(L) / make_laplacian_3d_fast(L)
    (python/matrix_generators.py:16-37, :68-80), without the host build and
    the host-to-device copy."""
    if precision not in _PRECISIONS:
        raise ValueError(f"precision must be one of {sorted(_PRECISIONS)}, got {precision!r}")
    out = C.c_void_p()
    _lib.check(_lib.load().nm_csr_laplacian(int(dim), int(L), _PRECISIONS[precision],
                                            C.byref(out)), "laplacian")
    return CrsMatrix(out.value)


def download_csr(A: CrsMatrix):
    """(rowptr int32, colind int32, values) copied back from the device
    (addition); values in the stored precision (bf16 as uint16 bits)."""
    dt = {_lib.NM_F64: np.float64, _lib.NM_F32: np.float32, _lib.NM_BF16: np.uint16}[A._dtype]
    rp = np.empty(A.nrows + 1, np.int32)
    ci = np.empty(max(A.nnz, 1), np.int32)
    v = np.empty(max(A.nnz, 1), dt)
    _lib.check(_lib.load().nm_csr_export(A._h, rp.ctypes.data, ci.ctypes.data, v.ctypes.data),
               "download_csr")
    return rp, ci[: A.nnz], v[: A.nnz]


def upload_csr_batched(matrices, *, precision: str = "fp64"):
    """Upload many independent CSR matrices as one block-diagonal device matrix
    (addition).  `matrices` is a sequence of (rowptr, colind, values, nrows,
    ncols); spmv on the result multiplies every matrix in one launch, with x
    and y the per-matrix vectors concatenated in order."""
    mats = list(matrices)
    if not mats:
        raise ValueError("upload_csr_batched: no matrices")
    nr = np.empty(len(mats), np.int32)
    nc = np.empty(len(mats), np.int32)
    rps, cis, vls = [], [], []
    for m, (rp, ci, v, n, k) in enumerate(mats):
        rp = host_array(rp, np.int32, f"rowptr[{m}]")
        ci = host_array(ci, np.int32, f"colind[{m}]")
        v = host_array(v, np.float64, f"values[{m}]")
        _check_csr_lengths(rp, ci, v, int(n), f"upload_csr_batched[{m}]")
        nz = int(rp[int(n)])
        nr[m], nc[m] = int(n), int(k)
        rps.append(rp[: int(n) + 1])
        cis.append(ci[:nz])
        vls.append(v[:nz])
    rp_all = np.ascontiguousarray(np.concatenate(rps))
    ci_all = np.ascontiguousarray(np.concatenate(cis))
    v_all, dt = _values_for(np.ascontiguousarray(np.concatenate(vls)), precision)
    out = C.c_void_p()
    _lib.check(_lib.load().nm_csr_create_batched(len(mats), nr.ctypes.data, nc.ctypes.data,
                                                 rp_all.ctypes.data, ci_all.ctypes.data,
                                                 v_all.ctypes.data, dt, C.byref(out)),
               "upload_csr_batched")
    row_off = np.concatenate([[0], np.cumsum(nr.astype(np.int64))])
    col_off = np.concatenate([[0], np.cumsum(nc.astype(np.int64))])
    return CrsMatrix(out.value, batch=(row_off, col_off))


def distribute_csr(rowptr, colind, values, global_nrows: int, global_ncols: int):
    """Partition a CSR matrix across the process group by rows; this rank
    receives its local submatrix (columns remapped to [own | ghost]) and the
    cached halo plan.  With one process the slice is the whole matrix."""
    rowptr = host_array(rowptr, np.int32, "rowptr")
    colind = host_array(colind, np.int32, "colind")
    values = host_array(values, np.float64, "values")
    n, ncols = int(global_nrows), int(global_ncols)
    if n <= 0 or ncols <= 0:
        raise ValueError("CrsMatrixHandle: non-positive dimensions")
    _check_csr_lengths(rowptr, colind, values, n, "distribute_csr")
    out = C.c_void_p()
    _lib.check(_lib.load().nm_dist_create(rowptr.ctypes.data, colind.ctypes.data,
                                          values.ctypes.data, n, ncols, rank(), size(),
                                          C.byref(out)), "distribute_csr")
    return DistCrsMatrix(out.value)


# ---- compute (src/bindings.cpp:150-290) ----------------------------------------

def _vec_dtype(A: CrsMatrix) -> str:
    return "float64" if A._dtype == _lib.NM_F64 else "float32"


def spmv(A: CrsMatrix, x, y, kokkoskernels: bool = True, *, async_: bool = False) -> None:
    """Single-GPU SpMV: y = A @ x (in place into y).

    `kokkoskernels` is accepted for compatibility; both settings run the
    kernel chosen for A (spmv_kernel: the row-block pipeline or, for
    scattered columns, the warp-gather kernel; the reference's two backends
    compute the same product).  fp32/bf16 matrices take float32 x and y."""
    dt = _vec_dtype(A)
    xt = device_array(x, dt, "x")
    yt = device_array(y, dt, "y")
    if xt.shape[0] != A.ncols:
        raise ValueError("spmv: x length != A.ncols")
    if yt.shape[0] != A.nrows:
        raise ValueError("spmv: y length != A.nrows")
    s = stream_of(yt)
    lib = _lib.load()
    _lib.check(lib.nm_spmv(A._h, xt.data_ptr(), yt.data_ptr(), s), "spmv")
    if not async_:
        torch.cuda.current_stream(yt.device).synchronize()
        _lib.check(lib.nm_check_device_errors(), "spmv")


def spmv_host(A: CrsMatrix, x, y) -> None:
    """y = A @ x with x and y in host memory (numpy arrays or CPU tensors;
    float64 for fp64 matrices, float32 for fp32/bf16 ones), through the C
    ABI's nm_spmv_host: x is copied in and y out around the SpMV, the row
    blocks in chunks so that the two copies overlap, and the call returns when
    y is written.  Page-locked arrays (torch `pin_memory()`) let the copies
    run at the full link rate.  y must be contiguous and writable.  Addition:
    the reference's spmv takes device arrays only."""
    dt = _vec_dtype(A)
    xa = host_array(x, dt, "x")
    if isinstance(y, np.ndarray):
        if not (y.flags.c_contiguous and y.flags.writeable):
            raise ValueError("spmv_host: y must be a contiguous, writable array")
    elif torch is not None and isinstance(y, torch.Tensor):
        if y.device.type == "cpu" and not y.is_contiguous():
            raise ValueError("spmv_host: y must be contiguous")
    ya = host_array(y, dt, "y")
    if xa.shape[0] != A.ncols:
        raise ValueError("spmv_host: x length != A.ncols")
    if ya.shape[0] != A.nrows:
        raise ValueError("spmv_host: y length != A.nrows")
    lib = _lib.load()
    s = torch.cuda.current_stream().cuda_stream
    _lib.check(lib.nm_spmv_host(A._h, xa.ctypes.data, ya.ctypes.data, s), "spmv_host")
    _lib.check(lib.nm_check_device_errors(), "spmv_host")


def batch_spmv(A: CrsMatrix, X, Y, *, async_: bool = False) -> None:
    """Batch SpMV: Y = A @ X with X of shape (ncols, k), Y (nrows, k), C order."""
    Xt = device_array(X, "float64", "X", ndim=2)
    Yt = device_array(Y, "float64", "Y", ndim=2)
    k = Xt.shape[1]
    if Xt.shape[0] != A.ncols:
        raise ValueError("batch_spmv: X.shape[0] != A.ncols")
    if Yt.shape[0] != A.nrows or Yt.shape[1] != k:
        raise ValueError("batch_spmv: Y must be (A.nrows, k)")
    if A._dtype != _lib.NM_F64:
        raise TypeError("batch_spmv: float64 matrices only")
    s = stream_of(Yt)
    _lib.check(_lib.load().nm_batch_spmv(A._h, Xt.data_ptr(), Yt.data_ptr(), k, s), "batch_spmv")
    if not async_:
        torch.cuda.current_stream(Yt.device).synchronize()


def dist_spmv(A_dist: DistCrsMatrix, x_local, y_local) -> None:
    """Distributed SpMV: y_local = A_dist @ x_global, with the halo packed and
    unpacked on the GPU and exchanged over torch.distributed."""
    from . import halo
    halo.dist_spmv(A_dist, x_local, y_local)


def _cg_dict(res: _lib.CgResult) -> dict:
    return {"iters": int(res.iters), "residual": float(res.final_res),
            "converged": bool(res.converged)}


def cg_solve_local(A: CrsMatrix, b, x, tol: float = 1e-10, max_iter: int = 1000) -> dict:
    """Single-GPU CG solver (no MPI).  x is the initial guess and is
    overwritten with the solution.  Returns {'iters', 'residual', 'converged'}."""
    bt = device_array(b, "float64", "b")
    xt = device_array(x, "float64", "x")
    if A._dtype != _lib.NM_F64:
        raise TypeError("cg_solve_local: float64 matrices only")
    if bt.shape[0] != A.nrows or xt.shape[0] != A.ncols:
        raise ValueError("cg_solve_local: b / x length does not match A")
    res = _lib.CgResult()
    _lib.check(_lib.load().nm_cg_local(A._h, bt.data_ptr(), xt.data_ptr(), float(tol),
                                       int(max_iter), C.byref(res), stream_of(xt)),
               "cg_solve_local")
    return _cg_dict(res)


def cg_solve(A_dist: DistCrsMatrix, b, x, tol: float = 1e-10, max_iter: int = 1000) -> dict:
    """Distributed Conjugate Gradient solver for A x = b (A SPD).  x is the
    initial guess and is overwritten.  Raises RuntimeError when p'Ap is near
    zero, as the reference does."""
    from . import halo
    return halo.cg_solve(A_dist, b, x, tol, max_iter)


# ---- additions -----------------------------------------------------------------

def tuning(A: CrsMatrix) -> dict:
    """The row-block partition parameters of A and its plain-SpMV kernel."""
    out = _lib.Tuning()
    _lib.check(_lib.load().nm_csr_get_tuning(A._h, C.byref(out)))
    names = {v: k for k, v in _KERNELS.items()}
    return {"tile": out.tile, "max_rows": out.max_rows, "short_max": out.short_max,
            "grid_mult": out.grid_mult, "stages": out.stages, "kernel": names[out.kernel]}


def spmv_kernel(A: CrsMatrix) -> str:
    """The kernel spmv runs on A: "blocks" (row-block pipeline) or "gather"
    (warp per 32 rows, for scattered columns)."""
    k = C.c_int32()
    _lib.check(_lib.load().nm_csr_spmv_kernel(A._h, C.byref(k)))
    return {v: n for n, v in _KERNELS.items()}[k.value]


def tune(A: CrsMatrix, tile: int = 0, max_rows: int = 0, short_max: int = 0,
         grid_mult: int = -1, stages: int = 0, kernel=None) -> dict:
    """Set the row-block partition parameters of A (tile / max_rows /
    short_max / stages <= 0 and grid_mult < 0 keep the current value;
    grid_mult 0 is the automatic grid) and its plain-SpMV kernel ("auto",
    "blocks" or "gather"; None keeps it), and return the effective ones."""
    if kernel is None:
        k = 0
    elif isinstance(kernel, str):
        if kernel not in _KERNELS:
            raise ValueError(f"kernel must be one of {sorted(_KERNELS)}, got {kernel!r}")
        k = _KERNELS[kernel]
    else:
        k = int(kernel)
    t = _lib.Tuning(int(tile), int(max_rows), int(short_max), int(grid_mult), int(stages), k)
    _lib.check(_lib.load().nm_csr_set_tuning(A._h, C.byref(t)), "tune")
    return tuning(A)


_TUNE_CACHE: dict = {}


def _tune_key(A: CrsMatrix) -> str:
    # shape, precision and the histogram of per-row reduction bins under the
    # default partition: matrices with the same key get the same tuning
    _, bins = row_blocks(A)
    h = np.bincount(bins.astype(np.int64), minlength=3)
    return f"{A.nrows}x{A.ncols}:{A.nnz}:{A.precision}:{h[0]}/{h[1]}/{h[2]}"


def autotune(A: CrsMatrix, x=None, budget_ms: float = 200.0, cache: bool = True) -> dict:
    """Choose A's SpMV partition and launch shape by timing candidates on the
    device (nm_csr_autotune: tile 1024/2048/4096, short_max 32/64, stages
    2/3/4, grid_mult 0/1/2 of the row-block kernel, and the warp-gather
    kernel) and install the fastest.  `x` (optional) is the
    vector to time with, else U[-1, 1].  Results are cached per matrix
    signature in-process and, when NUM_B200_TUNE_CACHE names a JSON file,
    across processes.  Returns the installed tuning plus 'us' (its SpMV time)
    and 'trials' (every candidate timed; empty on a cache hit)."""
    import json
    import os
    path = os.environ.get("NUM_B200_TUNE_CACHE")
    tune(A, tile=2048, max_rows=256, short_max=32, grid_mult=0, stages=2,
         kernel="auto")  # key on defaults
    key = _tune_key(A)
    if cache:
        if not _TUNE_CACHE and path and os.path.exists(path):
            try:
                with open(path) as f:
                    _TUNE_CACHE.update(json.load(f))
            except (OSError, ValueError):
                pass
        hit = _TUNE_CACHE.get(key)
        if hit:
            t = tune(A, **{k: hit[k] for k in ("tile", "max_rows", "short_max", "grid_mult",
                                                "stages")}, kernel=hit.get("kernel", "auto"))
            return {**t, "us": hit.get("us"), "trials": [], "cached": True}
    dt = torch.float64 if A.precision == "fp64" else torch.float32
    dev = torch.device("cuda", torch.cuda.current_device())
    if x is None:
        g = torch.Generator(device=dev).manual_seed(1)
        xt = torch.rand(A.ncols, dtype=dt, device=dev, generator=g) * 2 - 1
    else:
        xt = device_array(x, "float64" if dt == torch.float64 else "float32", "x")
    y = torch.empty(A.nrows, dtype=dt, device=dev)
    cap = 64
    trials = (_lib.TuneTrial * cap)()
    best = _lib.Tuning()
    nt = C.c_int32(0)
    s = stream_of(y)
    _lib.check(_lib.load().nm_csr_autotune(A._h, xt.data_ptr(), y.data_ptr(), s,
                                           float(budget_ms), C.byref(best), trials, cap,
                                           C.byref(nt)), "autotune")
    out = []
    for t in trials[: min(cap, nt.value)]:
        out.append({"tile": t.tuning.tile, "short_max": t.tuning.short_max,
                    "stages": t.tuning.stages, "grid_mult": t.tuning.grid_mult,
                    "kernel": {v: k for k, v in _KERNELS.items()}[t.tuning.kernel],
                    "us": round(float(t.us), 3)})
    res = tuning(A)
    us = min(o["us"] for o in out) if out else None
    if cache:
        _TUNE_CACHE[key] = {**res, "us": us}
        if path:
            try:
                with open(path, "w") as f:
                    json.dump(_TUNE_CACHE, f, indent=1, sort_keys=True)
            except OSError:
                pass
    return {**res, "us": us, "trials": out, "cached": False}


def row_blocks(A: CrsMatrix):
    """(blk, bins): the device row-block boundaries and per-row reduction bins
    (0 thread, 1 warp, 2 CTA)."""
    nb = C.c_int32()
    lib = _lib.load()
    _lib.check(lib.nm_csr_info(A._h, None, None, None, None, C.byref(nb)))
    blk = np.empty(nb.value + 1, np.int32)
    bins = np.empty(A.nrows, np.int8)
    _lib.check(lib.nm_csr_row_blocks(A._h, blk.ctypes.data, blk.shape[0], bins.ctypes.data))
    return blk, bins
