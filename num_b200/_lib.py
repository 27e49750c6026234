"""ctypes binding of libnum_b200.so (C ABI in include/num_b200.h).

Loading fails loudly: there is no CPU fallback.  If the shared library has not
been built, build it with `python -m num_b200.build`.
"""
from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libnum_b200.so"

NM_OK, NM_ERR_INVALID, NM_ERR_TYPE, NM_ERR_RUNTIME, NM_ERR_CUDA, NM_ERR_NOMEM = range(6)
NM_F64, NM_F32, NM_BF16 = 0, 1, 2

i32 = C.c_int32
i64 = C.c_int64
dbl = C.c_double
vp = C.c_void_p
P_i32 = C.POINTER(C.c_int32)
P_i8 = C.POINTER(C.c_int8)


class CgResult(C.Structure):
    _fields_ = [("iters", C.c_int32), ("final_res", C.c_double), ("converged", C.c_int32)]


class SolverOpts(C.Structure):
    _fields_ = [("inner", C.c_int32), ("precond", C.c_int32), ("inner_rtol", C.c_double),
                ("max_outer", C.c_int32), ("cont_window", C.c_double)]


class Tuning(C.Structure):
    _fields_ = [("tile", C.c_int32), ("max_rows", C.c_int32), ("short_max", C.c_int32),
                ("grid_mult", C.c_int32), ("stages", C.c_int32), ("kernel", C.c_int32)]


class SolverCounters(C.Structure):
    _fields_ = [(n, C.c_int64) for n in ("steps", "list_uploads", "graph_captures",
                                         "graph_instantiations", "outer_launches",
                                         "inner_iterations")] + \
               [(n, C.c_double) for n in ("s_lists", "s_outer", "s_capture", "s_run", "s_scan",
                                          "s_admit_prep", "s_admit_commit", "s_device",
                                          "last_step_ms")] + \
               [("last_step_iters", C.c_int64)]


class TuneTrial(C.Structure):
    _fields_ = [("tuning", Tuning), ("us", C.c_float)]


# name -> (argtypes); every function returns int (nm_status) unless noted.
_SIGNATURES = {
    "nm_last_error": ([], C.c_char_p),
    "nm_version": ([], C.c_char_p),
    "nm_init": ([C.c_int, P_i32, P_i32], C.c_int),
    "nm_finalize": ([], C.c_int),
    "nm_check_device_errors": ([], C.c_int),
    "nm_test_wait_timeout": ([i32, i32, dbl, C.POINTER(dbl), vp], C.c_int),
    "nm_csr_create": ([vp, vp, vp, C.c_int, i32, i32, C.POINTER(vp)], C.c_int),
    "nm_csr_create_batched": ([i32, vp, vp, vp, vp, vp, C.c_int, C.POINTER(vp)], C.c_int),
    "nm_csr_destroy": ([vp], C.c_int),
    "nm_csr_laplacian": ([i32, i32, C.c_int, C.POINTER(vp)], C.c_int),
    "nm_csr_spmv_kernel": ([vp, P_i32], C.c_int),
    "nm_csr_export": ([vp, vp, vp, vp], C.c_int),
    "nm_csr_info": ([vp, P_i32, P_i32, P_i32, P_i32, P_i32], C.c_int),
    "nm_csr_set_tuning": ([vp, C.POINTER(Tuning)], C.c_int),
    "nm_csr_get_tuning": ([vp, C.POINTER(Tuning)], C.c_int),
    "nm_cg_set_persistent": ([i32], C.c_int),
    "nm_cg_last_path": ([vp, P_i32], C.c_int),
    "nm_csr_autotune": ([vp, vp, vp, vp, C.c_double, C.POINTER(Tuning), vp, i32, P_i32], C.c_int),
    "nm_csr_row_blocks": ([vp, vp, i32, vp], C.c_int),
    "nm_row_blocks_host": ([vp, i32, C.POINTER(Tuning), vp, i32, vp, P_i32], C.c_int),
    "nm_spmv": ([vp, vp, vp, vp], C.c_int),
    "nm_spmv_host": ([vp, vp, vp, vp], C.c_int),
    "nm_batch_spmv": ([vp, vp, vp, i32, vp], C.c_int),
    "nm_axpy": ([i64, dbl, vp, vp, vp, vp], C.c_int),
    "nm_axpy2": ([i64, dbl, vp, dbl, vp, vp, vp], C.c_int),
    "nm_dot": ([i64, vp, vp, C.POINTER(dbl), vp], C.c_int),
    "nm_norm2": ([i64, vp, C.POINTER(dbl), vp], C.c_int),
    "nm_copy": ([i64, vp, vp, vp], C.c_int),
    "nm_fill": ([i64, dbl, vp, vp], C.c_int),
    "nm_scale": ([i64, dbl, vp, vp], C.c_int),
    "nm_cg_local": ([vp, vp, vp, dbl, i32, C.POINTER(CgResult), vp], C.c_int),
    "nm_cg_local_static": ([vp, vp, vp, dbl, i32, C.POINTER(CgResult), vp], C.c_int),
    "nm_solver_create": ([i64, i64, i32, C.POINTER(SolverOpts), C.POINTER(vp)], C.c_int),
    "nm_solver_destroy": ([vp], C.c_int),
    "nm_solver_set_persistent": ([i32], C.c_int),
    "nm_solver_admit": ([vp, vp, vp, vp, i32, vp, vp, dbl, i32, P_i32], C.c_int),
    "nm_solver_admit_batch": ([vp, i32, vp, vp, vp, vp, vp, dbl, i32, P_i32, P_i32], C.c_int),
    "nm_solver_step": ([vp, i32, P_i32], C.c_int),
    "nm_solver_step_begin": ([vp, i32], C.c_int),
    "nm_solver_take_batch": ([vp, i32, vp, vp], C.c_int),
    "nm_solver_resolve": ([vp, i32, vp, vp], C.c_int),
    "nm_solver_stream": ([vp, C.POINTER(vp)], C.c_int),
    "nm_solver_solution": ([vp, i32, vp], C.c_int),
    "nm_solver_step_end": ([vp, P_i32], C.c_int),
    "nm_solver_counters_get": ([vp, vp], C.c_int),
    "nm_solver_status": ([vp, i32, P_i32, C.POINTER(CgResult), P_i32], C.c_int),
    "nm_solver_take": ([vp, i32, vp], C.c_int),
    "nm_solver_info": ([vp, C.POINTER(i64), C.POINTER(i64), P_i32, P_i32], C.c_int),
    "nm_dist_create": ([vp, vp, vp, i32, i32, i32, i32, C.POINTER(vp)], C.c_int),
    "nm_dist_destroy": ([vp], C.c_int),
    "nm_dist_plan": ([vp, vp, vp, i32, i32, i32, i32, C.POINTER(vp)], C.c_int),
    "nm_dist_local_host": ([vp, P_i32, vp, vp, vp], C.c_int),
    "nm_dist_info": ([vp, P_i32, P_i32, P_i32, P_i32, P_i32, P_i32, P_i32], C.c_int),
    "nm_dist_send_plan": ([vp, vp, vp, vp, vp], C.c_int),
    "nm_dist_recv_plan": ([vp, vp, vp, vp, vp], C.c_int),
    "nm_dist_local": ([vp, C.POINTER(vp)], C.c_int),
    "nm_halo_pack": ([vp, vp, vp, vp], C.c_int),
    "nm_halo_unpack": ([vp, vp, vp, vp], C.c_int),
    "nm_dist_spmv_local": ([vp, vp, vp, vp], C.c_int),
    "nm_dist_spmv_interior": ([vp, vp, vp, vp], C.c_int),
    "nm_dist_spmv_boundary": ([vp, vp, vp, vp], C.c_int),
    "nm_dist_row_split": ([vp, P_i32, P_i32], C.c_int),
    "nm_dist_cg_single": ([vp, vp, vp, dbl, i32, C.POINTER(CgResult), vp], C.c_int),
}

_lock = threading.Lock()
_lib = None


class NativeLibraryMissing(RuntimeError):
    """The CUDA library is not built; there is deliberately no fallback."""


def load() -> C.CDLL:
    """Load libnum_b200.so once and attach the C signatures."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not LIB_PATH.exists():
            raise NativeLibraryMissing(
                f"{LIB_PATH} is missing: build the CUDA library with `python -m num_b200.build`")
        lib = C.CDLL(str(LIB_PATH))
        for name, (args, res) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _lib = lib
        return lib


def exported_symbols() -> list[str]:
    return list(_SIGNATURES)


def last_error() -> str:
    return load().nm_last_error().decode(errors="replace")


def check(status: int, what: str = "") -> None:
    """Map an nm_status to the exception types of the reference binding."""
    if status == NM_OK:
        return
    msg = last_error() or what or f"status {status}"
    if status == NM_ERR_INVALID:
        raise ValueError(msg)
    if status == NM_ERR_TYPE:
        raise TypeError(msg)
    if status == NM_ERR_NOMEM:
        raise MemoryError(msg)
    raise RuntimeError(msg)
