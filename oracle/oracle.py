"""Python face of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Loads oracle/liboracle.so (oracle.c, built by oracle/Makefile) and adds the
pieces of the reference that are host-side index work, restated in Python for
P virtual ranks in one process:

  partition / ghost map / send lists   src/dist_spmv.hpp:38-99,
                                       src/halo_exchange.hpp:38-130, :154-191
  cg_solve_distributed                 src/cg_solver.hpp:38-125

Only the tests, __graft_entry__.smoke() and bench.py's CPU-baseline /
reference arms use this module, as the checker or as the timed CPU stand-in
for the reference (whose Kokkos-OpenMP build cannot be built in this image).
The num_b200 package never imports it.
"""
from __future__ import annotations

import ctypes as C
import math
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"

_lib = None

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int32)


class _CgRes(C.Structure):
    _fields_ = [("iters", C.c_int), ("final_res", C.c_double), ("converged", C.c_int)]


def build() -> Path:
    """Compile liboracle.so with its Makefile (if missing or stale)."""
    src = HERE / "oracle.c"
    if not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB))
        vp = C.c_void_p
        sig = {
            "or_spmv_f64": [C.c_int, vp, vp, vp, vp, vp],
            "or_spmv_f64_omp": [C.c_int, vp, vp, vp, vp, vp],
            "or_spmv_f32": [C.c_int, vp, vp, vp, vp, vp],
            "or_spmv_f32_omp": [C.c_int, vp, vp, vp, vp, vp],
            "or_batch_spmv_f64": [C.c_int, C.c_int, vp, vp, vp, vp, vp],
            "or_axpy": [C.c_int, C.c_double, vp, vp, vp],
            "or_axpy2": [C.c_int, C.c_double, vp, C.c_double, vp, vp],
            "or_scale": [C.c_int, C.c_double, vp],
            "or_cg_local": [C.c_int, vp, vp, vp, vp, vp, C.c_double, C.c_int, C.POINTER(_CgRes)],
            "or_pcg_jacobi": [C.c_int, vp, vp, vp, vp, vp, C.c_double, C.c_int, C.POINTER(_CgRes)],
            "or_cg_omp": [C.c_int, vp, vp, vp, vp, vp, C.c_double, C.c_int, C.c_int,
                          C.POINTER(_CgRes)],
            "or_jacobi_dinv": [C.c_int, vp, vp, vp, vp],
            "or_row_blocks": [C.c_int, vp, C.c_int, C.c_int, C.c_int, vp, C.c_int, vp],
            "or_halo_pack": [C.c_int, vp, vp, vp],
            "or_halo_scatter": [C.c_int, C.c_int, vp, vp],
            "or_set_num_threads": [C.c_int],
        }
        for name, args in sig.items():
            getattr(L, name).argtypes = args
            getattr(L, name).restype = None
        L.or_dot.argtypes = [C.c_int, vp, vp]
        L.or_dot.restype = C.c_double
        L.or_norm2.argtypes = [C.c_int, vp]
        L.or_norm2.restype = C.c_double
        L.or_num_threads.argtypes = []
        L.or_num_threads.restype = C.c_int
        L.or_row_blocks.restype = C.c_int
        _lib = L
    return _lib


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def _p(a):
    return a.ctypes.data


# ---- SpMV / vector ops ----------------------------------------------------------

def spmv(row_ptr, col_idx, values, x, *, threads: bool = False) -> np.ndarray:
    """y = A x in serial CSR row order (FP64, or FP32 if values are float32)."""
    rp = _c(row_ptr, np.int32)
    ci = _c(col_idx, np.int32)
    n = rp.shape[0] - 1
    if np.asarray(values).dtype == np.float32:
        v, xx = _c(values, np.float32), _c(x, np.float32)
        y = np.empty(n, np.float32)
        fn = lib().or_spmv_f32_omp if threads else lib().or_spmv_f32
    else:
        v, xx = _c(values, np.float64), _c(x, np.float64)
        y = np.empty(n, np.float64)
        fn = lib().or_spmv_f64_omp if threads else lib().or_spmv_f64
    fn(n, _p(rp), _p(ci), _p(v), _p(xx), _p(y))
    return y


def batch_spmv(row_ptr, col_idx, values, X) -> np.ndarray:
    rp, ci, v = _c(row_ptr, np.int32), _c(col_idx, np.int32), _c(values, np.float64)
    X = _c(X, np.float64)
    n, k = rp.shape[0] - 1, X.shape[1]
    Y = np.empty((n, k), np.float64)
    lib().or_batch_spmv_f64(n, k, _p(rp), _p(ci), _p(v), _p(X), _p(Y))
    return Y


def axpy(alpha, x, y) -> np.ndarray:
    x, y = _c(x, np.float64), _c(y, np.float64)
    z = np.empty_like(x)
    lib().or_axpy(x.shape[0], alpha, _p(x), _p(y), _p(z))
    return z


def axpy2(alpha, x, beta, y) -> np.ndarray:
    x, y = _c(x, np.float64), _c(y, np.float64)
    z = np.empty_like(x)
    lib().or_axpy2(x.shape[0], alpha, _p(x), beta, _p(y), _p(z))
    return z


def dot(x, y) -> float:
    x, y = _c(x, np.float64), _c(y, np.float64)
    return lib().or_dot(x.shape[0], _p(x), _p(y))


def norm2(x) -> float:
    x = _c(x, np.float64)
    return lib().or_norm2(x.shape[0], _p(x))


def cg_local(row_ptr, col_idx, values, b, x0=None, tol=1e-10, max_iter=1000):
    """cg_solve_local (src/cg_solver.hpp:133-196).  Returns (dict, x)."""
    rp, ci, v = _c(row_ptr, np.int32), _c(col_idx, np.int32), _c(values, np.float64)
    b = _c(b, np.float64)
    n = rp.shape[0] - 1
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
    res = _CgRes()
    lib().or_cg_local(n, _p(rp), _p(ci), _p(v), _p(b), _p(x), float(tol), int(max_iter),
                      C.byref(res))
    return {"iters": res.iters, "residual": res.final_res, "converged": bool(res.converged)}, x


def pcg_jacobi(row_ptr, col_idx, values, b, x0=None, tol=1e-10, max_iter=1000):
    rp, ci, v = _c(row_ptr, np.int32), _c(col_idx, np.int32), _c(values, np.float64)
    b = _c(b, np.float64)
    n = rp.shape[0] - 1
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
    res = _CgRes()
    lib().or_pcg_jacobi(n, _p(rp), _p(ci), _p(v), _p(b), _p(x), float(tol), int(max_iter),
                        C.byref(res))
    return {"iters": res.iters, "residual": res.final_res, "converged": bool(res.converged)}, x


def cg_omp(row_ptr, col_idx, values, b, x0=None, tol=1e-10, max_iter=1000, precond=False):
    """Threaded CG / Jacobi-PCG (timed CPU baseline, not a parity reference)."""
    rp, ci, v = _c(row_ptr, np.int32), _c(col_idx, np.int32), _c(values, np.float64)
    b = _c(b, np.float64)
    n = rp.shape[0] - 1
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
    res = _CgRes()
    lib().or_cg_omp(n, _p(rp), _p(ci), _p(v), _p(b), _p(x), float(tol), int(max_iter),
                    int(bool(precond)), C.byref(res))
    return {"iters": res.iters, "residual": res.final_res, "converged": bool(res.converged)}, x


def row_blocks(row_ptr, tile=2048, max_rows=256, short_max=32):
    """CPU restatement of the device row-block partition -> (blk, bins)."""
    rp = _c(row_ptr, np.int32)
    n = rp.shape[0] - 1
    blk = np.empty(n + 2, np.int32)
    bins = np.empty(max(n, 1), np.int8)
    nb = lib().or_row_blocks(n, _p(rp), tile, max_rows, short_max, _p(blk), blk.shape[0],
                             _p(bins))
    assert nb >= 0
    return blk[: nb + 1].copy(), bins[:n].copy()


def halo_pack(send_idx, x_local) -> np.ndarray:
    idx, x = _c(send_idx, np.int32), _c(x_local, np.float64)
    buf = np.empty(idx.shape[0], np.float64)
    lib().or_halo_pack(idx.shape[0], _p(idx), _p(x), _p(buf))
    return buf


def set_threads(n: int) -> None:
    lib().or_set_num_threads(int(n))


def num_threads() -> int:
    return lib().or_num_threads()


# ---- distributed index work for P virtual ranks ---------------------------------------

def row_range(n: int, size: int, rank: int):
    """Even block-row split (src/dist_spmv.hpp:39-43)."""
    base, extra = n // size, n % size
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def partition(row_ptr, col_idx, values, n: int, size: int):
    """distribute_csr + build_ghost_map + build_send_indices for every rank of
    `size` (pure Python loops; small matrices).  Returns a list of dicts with
    the local CSR (remapped columns), recv list [(rank, ids, offset)], send
    list [(rank, ids)], total_ghost and the flat LOCAL send index array."""
    rp = [int(v) for v in row_ptr]
    ci = [int(v) for v in col_idx]
    ranges = [row_range(n, size, r) for r in range(size)]

    def owner_of(col):  # src/halo_exchange.hpp:54-59
        for r, (s, e) in enumerate(ranges):
            if s <= col < e:
                return r
        raise RuntimeError(f"build_ghost_map: column index {col} is out of the global row range")

    # what each rank receives from each owner: sorted sets (:62-72)
    recv_cols = []
    for r, (s, e) in enumerate(ranges):
        want = {}
        for i in range(s, e):
            for j in range(rp[i], rp[i + 1]):
                c = ci[j]
                if c < s or c >= e:
                    want.setdefault(owner_of(c), set()).add(c)
        recv_cols.append({o: sorted(ids) for o, ids in want.items()})

    out = []
    for r, (s, e) in enumerate(ranges):
        recv, send, off = [], [], 0
        for q in range(size):  # :108-127
            if q == r:
                continue
            ids = recv_cols[r].get(q, [])
            if ids:
                recv.append((q, list(ids), off))
                off += len(ids)
            sent = recv_cols[q].get(r, [])
            if sent:
                send.append((q, list(sent)))
        pos = {}
        for q, ids, o in recv:
            for k, g in enumerate(ids):
                pos[g] = o + k
        ln = e - s
        z0 = rp[s]
        lrp = [rp[s + i] - z0 for i in range(ln + 1)]
        lci = []
        for j in range(rp[s], rp[e]):  # src/dist_spmv.hpp:69-81
            c = ci[j]
            lci.append(c - s if s <= c < e else ln + pos[c])
        send_idx = [g - s for _, ids in send for g in ids]  # build_send_indices
        out.append({
            "rank": r, "row_start": s, "row_end": e, "total_ghost": off,
            "recv": recv, "send": send, "send_idx": np.array(send_idx, np.int32),
            "row_ptr": np.array(lrp, np.int32), "col_idx": np.array(lci, np.int32),
            "values": np.asarray(values[rp[s]:rp[e]], np.float64),
        })
    return out


def dist_spmv(parts, x_global) -> np.ndarray:
    """distributed_spmv over all virtual ranks, exchange by loopback."""
    size = len(parts)
    xl = [np.asarray(x_global[p["row_start"]:p["row_end"]], np.float64) for p in parts]
    bufs = {}
    for p in parts:  # pack (src/halo_exchange.hpp:228-233), then "send"
        packed = halo_pack(p["send_idx"], xl[p["rank"]])
        off = 0
        for q, ids in p["send"]:
            bufs[(p["rank"], q)] = packed[off:off + len(ids)]
            off += len(ids)
    ys = []
    for p in parts:
        ln = p["row_end"] - p["row_start"]
        x_ext = np.zeros(ln + p["total_ghost"])
        x_ext[:ln] = xl[p["rank"]]
        for q, ids, o in p["recv"]:  # scatter (:289-298)
            x_ext[ln + o: ln + o + len(ids)] = bufs[(q, p["rank"])]
        ys.append(spmv(p["row_ptr"], p["col_idx"], p["values"], x_ext))
    assert size == len(ys)
    return np.concatenate(ys)


def cg_distributed(parts, b_global, tol=1e-10, max_iter=1000):
    """cg_solve_distributed (src/cg_solver.hpp:38-125) over P virtual ranks;
    global dots sum the ranks' serial local dots in rank order."""
    sl = [slice(p["row_start"], p["row_end"]) for p in parts]
    n = len(b_global)
    b = np.asarray(b_global, np.float64)
    x = np.zeros(n)

    def gdot(u, v):
        return float(sum(dot(u[s], v[s]) for s in sl))

    Ap = dist_spmv(parts, x)
    r = axpy(-1.0, Ap, b)
    p = r.copy()
    bn = math.sqrt(gdot(b, b))
    if bn == 0.0:
        bn = 1.0
    rr = gdot(r, r)
    if math.sqrt(rr) / bn < tol:
        return {"iters": 0, "residual": math.sqrt(rr) / bn, "converged": True}, x
    for it in range(max_iter):
        Ap = dist_spmv(parts, p)
        pAp = gdot(p, Ap)
        if abs(pAp) < 1e-300:
            raise RuntimeError("CG: p'Ap is near zero — A may not be SPD")
        alpha = rr / pAp
        x = axpy(alpha, p, x)
        r = axpy(-alpha, Ap, r)
        rr_new = gdot(r, r)
        rel = math.sqrt(rr_new) / bn
        if rel < tol:
            return {"iters": it + 1, "residual": rel, "converged": True}, x
        beta = rr_new / rr
        rr = rr_new
        p = axpy2(1.0, r, beta, p)
    return {"iters": max_iter, "residual": math.sqrt(gdot(r, r)) / bn, "converged": False}, x
