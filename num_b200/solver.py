"""Batched, mixed-precision, continuously batched PCG solves (the library's
nm_solver_* entry points).  No counterpart in the reference, whose CG solves one
system at a time in FP64 without a preconditioner (src/cg_solver.hpp:133-196).

    S = BatchSolver(max_rows=..., max_nnz=..., precision="fp32")   # or "bf16", "fp64"
    slot = S.admit(A, b, tol=1e-8)            # None: no room in the arena right now
    while S.active:
        S.step(8)                             # refinement steps + 8 lockstep iterations
    x, info = S.take(slot)

precision "fp64": plain FP64 Jacobi-PCG; "fp32" / "bf16": matrix values in FP32
/ BF16, Krylov vectors and accumulation in FP32, FP64 iterative refinement (the
true residual b - A x, the correction x += d and the stopping test in FP64).
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import _lib

_PREC = {"fp64": _lib.NM_F64, "fp32": _lib.NM_F32, "bf16": _lib.NM_BF16}

PHASE_REFINE, PHASE_ITERATE, PHASE_DONE = 1, 2, 3


def arena_bytes(max_rows: int, max_nnz: int, precision: str = "fp32") -> int:
    """Device bytes a solver with these capacities allocates."""
    t = 8 if precision == "fp64" else 4
    v = {"fp64": 0, "fp32": 4, "bf16": 2}[precision]
    return (max_rows + 16) * (4 + 3 * 8 + 6 * t) + (max_nnz + 16) * (4 + 8 + v)


def arena_for(budget_bytes: int, nnz_per_row: float = 8.0, precision: str = "fp32"):
    """(max_rows, max_nnz) that fill `budget_bytes` for matrices with about
    nnz_per_row nonzeros per row."""
    per_row = arena_bytes(1, 0, precision) + nnz_per_row * (arena_bytes(0, 1, precision))
    rows = int(budget_bytes // per_row)
    rows = min(rows, 2**31 - 8192)
    return rows, min(int(rows * nnz_per_row), 2**31 - 8192)


class BatchSolver:
    def __init__(self, max_rows: int, max_nnz: int, max_systems: int = 4096,
                 precision: str = "fp32", precond: str = "jacobi", inner_rtol: float = 1e-3,
                 max_outer: int = 30, device: int = 0, cont_window: float = 2.0):
        import torch
        torch.cuda.set_device(device)
        if precision not in _PREC:
            raise ValueError(f"precision must be one of {sorted(_PREC)}")
        self.lib = _lib.load()
        _lib.check(self.lib.nm_init(device, None, None), "init")
        opts = _lib.SolverOpts(_PREC[precision], 1 if precond == "jacobi" else 0,
                               float(inner_rtol), int(max_outer), float(cont_window))
        h = C.c_void_p()
        _lib.check(self.lib.nm_solver_create(int(max_rows), int(max_nnz), int(max_systems),
                                             C.byref(opts), C.byref(h)), "nm_solver_create")
        self._h = h
        self.precision = precision
        self.n = {}          # slot -> rows
        self.active = set()  # slots not yet finished
        self.seconds = {"admit": 0.0, "step": 0.0, "take": 0.0}  # host wall time per call kind
        self.rows_admitted = 0  # rows of all systems admitted so far

    def __del__(self):
        h = getattr(self, "_h", None)
        try:
            if h is not None and h.value and _lib._lib is not None:
                _lib._lib.nm_solver_destroy(h)
        except (AttributeError, TypeError):  # interpreter shutdown
            pass
        self._h = None

    def admit(self, A, b, x0=None, tol: float = 1e-8, max_iter: int = 10000):
        """Admit A x = b (A: generators.Csr or (row_ptr, col_idx, values, n)).
        Returns the slot, or None when the arena or the slot table is full."""
        rp, ci, v, n = (A.row_ptr, A.col_idx, A.values, A.nrows) if hasattr(A, "row_ptr") else A
        rp = np.ascontiguousarray(rp, np.int32)
        ci = np.ascontiguousarray(ci, np.int32)
        v = np.ascontiguousarray(v, np.float64)
        b = np.ascontiguousarray(b, np.float64)
        x0p = None
        if x0 is not None:
            x0 = np.ascontiguousarray(x0, np.float64)
            x0p = x0.ctypes.data
        if b.shape[0] != n:
            raise ValueError("admit: b length != n")
        slot = C.c_int32(-1)
        t0 = time.perf_counter()
        st = self.lib.nm_solver_admit(self._h, rp.ctypes.data, ci.ctypes.data, v.ctypes.data,
                                      int(n), b.ctypes.data, x0p, float(tol), int(max_iter),
                                      C.byref(slot))
        self.seconds["admit"] += time.perf_counter() - t0
        if st == _lib.NM_ERR_NOMEM:
            return None
        _lib.check(st, "admit")
        self.n[slot.value] = int(n)
        self.active.add(slot.value)
        self.rows_admitted += int(n)
        return slot.value

    def admit_many(self, systems, tol: float = 1e-8, max_iter: int = 10000):
        """Admit [(A, b)] in order, preparing them in parallel on the host,
        until one does not fit.  Returns the slots of the admitted prefix."""
        k = len(systems)
        if k == 0:
            return []
        keep = []
        rp_p = (C.c_void_p * k)()
        ci_p = (C.c_void_p * k)()
        v_p = (C.c_void_p * k)()
        b_p = (C.c_void_p * k)()
        ns = (C.c_int32 * k)()
        for i, (A, b) in enumerate(systems):
            rp, ci, v, n = (A.row_ptr, A.col_idx, A.values, A.nrows) if hasattr(A, "row_ptr") else A
            arrs = (np.ascontiguousarray(rp, np.int32), np.ascontiguousarray(ci, np.int32),
                    np.ascontiguousarray(v, np.float64), np.ascontiguousarray(b, np.float64))
            if arrs[3].shape[0] != n:
                raise ValueError("admit_many: b length != n")
            keep.append(arrs)
            rp_p[i], ci_p[i], v_p[i], b_p[i] = (a.ctypes.data for a in arrs)
            ns[i] = int(n)
        slots = (C.c_int32 * k)()
        got = C.c_int32(0)
        t0 = time.perf_counter()
        st = self.lib.nm_solver_admit_batch(self._h, k, rp_p, ci_p, v_p, ns, b_p, float(tol),
                                            int(max_iter), slots, C.byref(got))
        self.seconds["admit"] += time.perf_counter() - t0
        out = list(slots[: got.value])
        for i, s in enumerate(out):
            self.n[s] = int(ns[i])
            self.active.add(s)
            self.rows_admitted += int(ns[i])
        _lib.check(st, "admit_many")
        return out

    def step(self, iters: int = 8):
        """Refinement steps + up to `iters` inner iterations (a multiple of 8;
        the device stops early once no system iterates);
        returns the slots that finished in this step."""
        self.step_begin(iters)
        return self.step_end()

    def step_begin(self, iters: int = 8):
        """Enqueue a step and return at once; admit() / admit_many() may run
        before step_end() (their host work overlaps the device)."""
        t0 = time.perf_counter()
        _lib.check(self.lib.nm_solver_step_begin(self._h, int(iters)), "step")
        self.seconds["step"] += time.perf_counter() - t0

    def step_end(self):
        """Wait for the step; returns the slots that finished in it."""
        nd = C.c_int32(0)
        t0 = time.perf_counter()
        _lib.check(self.lib.nm_solver_step_end(self._h, C.byref(nd)), "step")
        self.seconds["step"] += time.perf_counter() - t0
        done = []
        if nd.value:
            for s in list(self.active):
                if self.status(s)["phase"] == PHASE_DONE:
                    done.append(s)
                    self.active.discard(s)
        return done

    def status(self, slot: int) -> dict:
        ph, outer = C.c_int32(), C.c_int32()
        res = _lib.CgResult()
        _lib.check(self.lib.nm_solver_status(self._h, int(slot), C.byref(ph), C.byref(res),
                                             C.byref(outer)), "status")
        return {"phase": ph.value, "iters": res.iters, "residual": res.final_res,
                "converged": bool(res.converged), "outer": outer.value}

    def take(self, slot: int):
        """(x, info) of a finished (or abandoned) system; frees its slot."""
        t0 = time.perf_counter()
        info = self.status(slot)
        x = np.empty(self.n[slot], np.float64)
        _lib.check(self.lib.nm_solver_take(self._h, int(slot), x.ctypes.data), "take")
        self.seconds["take"] += time.perf_counter() - t0
        self.n.pop(slot, None)
        self.active.discard(slot)
        return x, info

    def resolve(self, slot: int, b=None, x0=None) -> None:
        """Solve the admitted system in `slot` again: new b (None keeps it),
        x0 (None: zero); it rejoins at the next step."""
        bp = x0p = None
        if b is not None:
            b = np.ascontiguousarray(b, np.float64)
            if b.shape[0] != self.n[slot]:
                raise ValueError("resolve: b length != n")
            bp = b.ctypes.data
        if x0 is not None:
            x0 = np.ascontiguousarray(x0, np.float64)
            if x0.shape[0] != self.n[slot]:
                raise ValueError("resolve: x0 length != n")
            x0p = x0.ctypes.data
        _lib.check(self.lib.nm_solver_resolve(self._h, int(slot), bp, x0p), "resolve")
        self.active.add(slot)

    def solution(self, slot: int) -> np.ndarray:
        """Copy of a system's current x (the slot stays admitted)."""
        x = np.empty(self.n[slot], np.float64)
        _lib.check(self.lib.nm_solver_solution(self._h, int(slot), x.ctypes.data), "solution")
        return x

    def stream(self) -> int:
        """cudaStream_t of the solver's steps (an integer handle)."""
        h = C.c_void_p()
        _lib.check(self.lib.nm_solver_stream(self._h, C.byref(h)), "stream")
        return h.value or 0

    def counters(self) -> dict:
        """Engine counters (nm_solver_counters_get)."""
        c = _lib.SolverCounters()
        _lib.check(self.lib.nm_solver_counters_get(self._h, C.byref(c)), "counters")
        return {n: getattr(c, n) for n, _ in c._fields_}

    def take_many(self, slots):
        """take() for several slots with one device synchronisation; returns
        [(x, info)] in the order of `slots`."""
        slots = list(slots)
        if not slots:
            return []
        t0 = time.perf_counter()
        infos = [self.status(s) for s in slots]
        xs = [np.empty(self.n[s], np.float64) for s in slots]
        k = len(slots)
        arr = (C.c_int32 * k)(*slots)
        ptrs = (C.c_void_p * k)(*[x.ctypes.data for x in xs])
        _lib.check(self.lib.nm_solver_take_batch(self._h, k, arr, ptrs), "take_many")
        self.seconds["take"] += time.perf_counter() - t0
        for s in slots:
            self.n.pop(s, None)
            self.active.discard(s)
        return list(zip(xs, infos))

    def info(self) -> dict:
        fr, fz = C.c_int64(), C.c_int64()
        a, fs = C.c_int32(), C.c_int32()
        _lib.check(self.lib.nm_solver_info(self._h, C.byref(fr), C.byref(fz), C.byref(a),
                                           C.byref(fs)), "info")
        return {"free_rows": fr.value, "free_nnz": fz.value, "active": a.value,
                "free_slots": fs.value}

    def solve(self, systems, tol: float = 1e-8, max_iter: int = 10000, chunk: int = 8):
        """Solve every (A, b) of `systems`, admitting as the arena allows;
        returns [(x, info)] in input order."""
        systems = list(systems)
        out = [None] * len(systems)
        owner = {}
        nxt = 0

        def admit():
            nonlocal nxt
            got = self.admit_many(systems[nxt:nxt + 1024], tol=tol, max_iter=max_iter)
            for s in got:
                owner[s] = nxt
                nxt += 1
            return got

        while nxt < len(systems) or self.active:
            if not self.active:
                if not admit():
                    raise MemoryError("solve: a system does not fit the empty arena")
            self.step_begin(chunk)
            if nxt < len(systems):
                admit()  # host preparation overlaps the step
            done = self.step_end()
            for s, r in zip(done, self.take_many(done)):
                out[owner.pop(s)] = r
        return out
