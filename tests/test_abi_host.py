"""The C-ABI library on the host (no GPU): it loads, exports every entry point
include/num_b200.h declares, and its host-side index work -- the row-block
partition and the distributed partition / halo plan -- is bit-exact with the
oracle's restatement of the reference."""
import ctypes as C
import re

import numpy as np
import pytest

from conftest import ROOT
from num_b200 import generators as gen


def header_symbols():
    text = (ROOT / "include" / "num_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(nm_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_header_symbol(nmlib):
    syms = header_symbols()
    assert len(syms) >= 30
    for s in syms:
        assert hasattr(nmlib, s), f"libnum_b200.so does not export {s}"


def test_ctypes_table_covers_header(nmlib):
    from num_b200 import _lib
    assert sorted(_lib.exported_symbols()) == header_symbols()


def test_version_and_no_error(nmlib):
    assert b"sm_100a" in nmlib.nm_version()
    assert nmlib.nm_last_error() == b""


def _host_blocks(nmlib, rp, tile=0, max_rows=0, short_max=0):
    from num_b200 import _lib
    n = rp.shape[0] - 1
    blk = np.empty(n + 2, np.int32)
    bins = np.empty(max(n, 1), np.int8)
    nb = C.c_int32()
    t = _lib.Tuning(tile, max_rows, short_max, 0, 0)
    _lib.check(nmlib.nm_row_blocks_host(rp.ctypes.data, n, C.byref(t), blk.ctypes.data,
                                        blk.shape[0], bins.ctypes.data, C.byref(nb)))
    return blk[: nb.value + 1], bins[:n]


def _matrices():
    yield "lap2d_64", gen.laplacian_2d(64).row_ptr
    yield "lap3d_24", gen.laplacian_3d(24).row_ptr
    yield "power_law_20k", gen.power_law(20000, seed=7).row_ptr
    yield "lcg_random", gen.lcg_random(2000)[0].row_ptr
    lens = np.array([0, 0, 5000, 1, 2047, 2048, 2049, 0, 33, 32, 31, 4097, 3] * 40)
    yield "ragged_long", np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    yield "single_row", np.array([0, 7], np.int32)
    yield "empty_rows", np.zeros(300, np.int32)


@pytest.mark.parametrize("name,rp", list(_matrices()), ids=[m[0] for m in _matrices()])
@pytest.mark.parametrize("tile,max_rows,short_max", [(2048, 256, 32), (1024, 128, 8),
                                                     (4096, 256, 64)])
def test_row_blocks_bit_exact(nmlib, oracle, name, rp, tile, max_rows, short_max):
    blk, bins = _host_blocks(nmlib, rp, tile, max_rows, short_max)
    oblk, obins = oracle.row_blocks(rp, tile, max_rows, short_max)
    assert np.array_equal(blk, oblk)
    assert np.array_equal(bins, obins)
    # structural invariants of the partition
    assert blk[0] == 0 and blk[-1] == rp.shape[0] - 1 and np.all(np.diff(blk) > 0)
    nz = rp[blk[1:]] - rp[blk[:-1]]
    rows = np.diff(blk)
    assert np.all((nz <= tile) | (rows == 1)) and np.all(rows <= max_rows)


def test_row_blocks_defaults(nmlib, oracle):
    rp = gen.laplacian_3d(16).row_ptr
    blk, _ = _host_blocks(nmlib, rp)
    assert np.array_equal(blk, oracle.row_blocks(rp)[0])


def _plans():
    yield "lap1d_12_P3", gen.laplacian_1d(12), 3
    yield "lap1d_127_P4", gen.laplacian_1d(127), 4
    yield "lap2d_16_P3", gen.laplacian_2d(16), 3
    yield "lap3d_8_P5", gen.laplacian_3d(8), 5
    yield "lcg_500_P4", gen.lcg_random(500)[0], 4
    yield "lap1d_5_P8", gen.laplacian_1d(5), 8  # more ranks than rows


@pytest.mark.parametrize("name,A,P", list(_plans()), ids=[p[0] for p in _plans()])
def test_dist_plan_bit_exact(nmlib, oracle, name, A, P):
    from num_b200.halo import plan_host
    parts = oracle.partition(A.row_ptr, A.col_idx, A.values, A.nrows, P)
    for r in range(P):
        plan, (lrp, lci, lv) = plan_host(A.row_ptr, A.col_idx, A.values, A.nrows, A.ncols, r, P)
        o = parts[r]
        assert (plan.row_start, plan.row_end) == (o["row_start"], o["row_end"])
        assert plan.n_ghost == o["total_ghost"]
        assert [(int(q), list(map(int, plan.ghost_ids[off:off + c])), int(off))
                for q, c, off in zip(plan.recv_rank, plan.recv_count, plan.recv_off)] == o["recv"]
        got_send = [(int(q), [int(v) + plan.row_start for v in plan.send_idx[off:off + c]])
                    for q, c, off in zip(plan.send_rank, plan.send_count, plan.send_off)]
        assert got_send == o["send"]
        assert np.array_equal(plan.send_idx, o["send_idx"])
        assert np.array_equal(lrp, o["row_ptr"])
        assert np.array_equal(lci, o["col_idx"])
        assert np.array_equal(lv, o["values"])


@pytest.mark.parametrize("name,A,P", list(_plans()), ids=[p[0] for p in _plans()])
def test_dist_row_split_counts(nmlib, name, A, P):
    """Interior rows (every column owned) and boundary rows (a ghost column)
    of each rank's slice, counted on a host-only plan."""
    from num_b200.halo import plan_host
    for r in range(P):
        plan, (lrp, lci, _) = plan_host(A.row_ptr, A.col_idx, A.values, A.nrows, A.ncols, r, P)
        h = C.c_void_p()
        from num_b200._lib import check as _lib_check
        _lib_check(nmlib.nm_dist_plan(A.row_ptr.ctypes.data, A.col_idx.ctypes.data,
                                      A.values.ctypes.data, A.nrows, A.ncols, r, P, C.byref(h)))
        ni, nb = C.c_int32(), C.c_int32()
        try:
            _lib_check(nmlib.nm_dist_row_split(h, C.byref(ni), C.byref(nb)))
        finally:
            nmlib.nm_dist_destroy(h)
        n = plan.row_end - plan.row_start
        ghost = np.array([bool((lci[lrp[i]:lrp[i + 1]] >= n).any()) for i in range(n)], bool)
        assert (ni.value, nb.value) == (int((~ghost).sum()), int(ghost.sum()))


def test_dist_plan_rejects_out_of_range_column(nmlib):
    from num_b200.halo import plan_host
    # Row 1 (owned by rank 1 of 2) names column 5 of a 2-row matrix; rank 1's
    # ghost scan raises, as build_ghost_map does (src/halo_exchange.hpp:54-59).
    rp = np.array([0, 1, 2], np.int32)
    with pytest.raises(RuntimeError, match="out of the global row range"):
        plan_host(rp, np.array([0, 5], np.int32), np.ones(2), 2, 6, 1, 2)


def test_create_validation_errors_before_device_work(nmlib):
    """Invalid CSR input is rejected on the host with the reference's error
    types, before any device call (so this runs without a GPU)."""
    from num_b200 import _lib
    out = C.c_void_p()
    rp = np.array([0, 1, 2], np.int32)
    ci = np.array([0, 3], np.int32)
    v = np.ones(2)
    st = nmlib.nm_csr_create(rp.ctypes.data, ci.ctypes.data, v.ctypes.data, 0, 2, 2, C.byref(out))
    assert st == _lib.NM_ERR_INVALID and b"outside" in nmlib.nm_last_error()
    st = nmlib.nm_csr_create(rp.ctypes.data, ci.ctypes.data, v.ctypes.data, 0, 0, 2, C.byref(out))
    assert st == _lib.NM_ERR_INVALID and b"non-positive" in nmlib.nm_last_error()
    st = nmlib.nm_csr_create(rp.ctypes.data, ci.ctypes.data, v.ctypes.data, 9, 2, 4, C.byref(out))
    assert st == _lib.NM_ERR_TYPE
    bad = np.array([0, 2, 1], np.int32)
    st = nmlib.nm_csr_create(bad.ctypes.data, ci.ctypes.data, v.ctypes.data, 0, 2, 4, C.byref(out))
    assert st == _lib.NM_ERR_INVALID and b"decreases" in nmlib.nm_last_error()
    with pytest.raises(ValueError, match="decreases"):
        _lib.check(st)


@pytest.mark.parametrize("dim,L,what", [(4, 8, b"dim must be"), (2, 0, b"non-positive"),
                                        (3, -1, b"non-positive"), (3, 700, b"int32 offset"),
                                        (2, 50000, b"int32 row")])
def test_laplacian_rejects_bad_sizes_before_device_work(nmlib, dim, L, what):
    """nm_csr_laplacian checks dim and L (rows and nonzeros within the int32
    offsets: 700^3 gives 2.4e9 nonzeros) on the host."""
    from num_b200 import _lib
    out = C.c_void_p()
    assert nmlib.nm_csr_laplacian(dim, L, 0, C.byref(out)) == _lib.NM_ERR_INVALID
    assert what in nmlib.nm_last_error() and not out.value
    assert nmlib.nm_csr_laplacian(3, 4, 9, C.byref(out)) == _lib.NM_ERR_TYPE


def test_python_module_errors_on_host(nmlib):
    """upload_csr argument checking mirrors the nanobind signature: wrong
    dtype -> TypeError, non-positive dims / short arrays -> ValueError."""
    from num_b200 import kokkos_spmv as k
    A = gen.tridiag4()
    with pytest.raises(TypeError):
        k.upload_csr(A.row_ptr.astype(np.int64), A.col_idx, A.values, 4, 4)
    with pytest.raises(TypeError):
        k.upload_csr(A.row_ptr, A.col_idx, A.values.astype(np.float32), 4, 4)
    with pytest.raises(ValueError, match="non-positive"):
        k.upload_csr(A.row_ptr, A.col_idx, A.values, 0, 4)
    with pytest.raises(ValueError):
        k.upload_csr(A.row_ptr, A.col_idx[:5], A.values, 4, 4)
    with pytest.raises(ValueError, match="outside"):
        k.upload_csr(A.row_ptr, A.col_idx, A.values, 4, 3)  # column 3 >= ncols


def test_tune_kernel_names_checked_on_host(nmlib):
    """kokkos_spmv.tune(kernel=...) validates the name before any device call;
    the names map to nm_tuning.kernel as the header defines them."""
    from num_b200 import kokkos_spmv as k
    with pytest.raises(ValueError, match="kernel must be one of"):
        k.tune(None, kernel="fastest")
    assert k._KERNELS == {"auto": 1, "blocks": 2, "gather": 3, "sliced": 4}
    t = C.c_int32()
    st = nmlib.nm_csr_spmv_kernel(None, C.byref(t))
    from num_b200 import _lib
    assert st == _lib.NM_ERR_INVALID



def test_spmv_host_null_arguments_rejected_on_host(nmlib):
    """nm_spmv_host checks its pointers before any device call."""
    from num_b200 import _lib
    y = np.empty(4)
    assert nmlib.nm_spmv_host(None, y.ctypes.data, y.ctypes.data, None) == _lib.NM_ERR_INVALID
    assert b"NULL" in nmlib.nm_last_error()
