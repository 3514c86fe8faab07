"""ipr_gemv_query_noalloc: the GEMV query for callers that cannot allocate.

A process whose framework has reserved all free device memory for its own
pool, or a request path that cannot take the device-wide synchronisation of
cudaMalloc, cannot use gpu_gemv_query, which allocates device copies of the
query row and the result on every call.  ipr_gemv_query_noalloc stages both in
a fixed device array inside the library instead.  This test drives it through
the C ABI and checks that it returns exactly what gpu_gemv_query returns, on
two calls in a row with different queries (the second call must not see
anything left over from the first).  The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DB_ROWS, DB_COLS = 2048, 16384  # the 10k-record (config 0) first dimension
Q0, Q1 = 268369921, 249561089


def _query(seed):
    rng = np.random.default_rng(seed)
    lo = rng.integers(0, Q0, DB_ROWS, dtype=np.uint64)
    hi = rng.integers(0, Q1, DB_ROWS, dtype=np.uint64)
    return np.ascontiguousarray(lo | (hi << np.uint64(32)))


def _with_alloc(lib, orc, d_db, a):
    """the existing entry point (allocates its staging buffers per call)"""
    p = orc.params()
    c = np.zeros(DB_COLS, dtype=np.uint64)
    u64 = ctypes.c_uint64
    lib.gpu_init_memory_pool()
    lib.gpu_gemv_query(ctypes.c_void_p(c.ctypes.data), ctypes.c_void_p(a.ctypes.data), ctypes.c_void_p(d_db),
                       ctypes.c_int(DB_ROWS), ctypes.c_int(DB_COLS), u64(Q0), u64(Q1), u64(p.barrett_cr1[0]),
                       u64(p.barrett_cr1[1]), u64(p.mod0_inv_mod1), u64(p.mod1_inv_mod0), u64(Q0 * Q1),
                       u64(p.cr0_mod), u64(p.cr1_mod))
    return c


def _no_alloc(lib, d_db, a):
    c = np.zeros(DB_COLS, dtype=np.uint64)
    f = lib.ipr_gemv_query_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    st = f(c.ctypes.data, a.ctypes.data, d_db, DB_ROWS, DB_COLS)
    assert st == 0, lib.ipr_last_error()
    return c


def test_noalloc_gemv_matches_allocating_entry_point(pkg, orc):
    import torch
    torch.cuda.set_device(0)
    rng = np.random.default_rng(99)
    db = rng.integers(0, 65535, DB_ROWS * DB_COLS, dtype=np.uint16)  # encoded values are < 65535
    d_db = torch.from_numpy(db.view(np.int16)).cuda()
    for seed in (1, 2):  # two calls in a row share the library's array
        a = _query(seed)
        got = _no_alloc(pkg.lib, d_db.data_ptr(), a)
        want = _with_alloc(pkg.lib, orc, d_db.data_ptr(), a)
        assert np.array_equal(got, want)  # integer results: exact
        assert int(got.max()) < Q0 * Q1


def test_noalloc_rejects_oversize_shapes(pkg):
    f = pkg.lib.ipr_gemv_query_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    buf = np.zeros(16, dtype=np.uint64)
    st = f(buf.ctypes.data, buf.ctypes.data, buf.ctypes.data, 131072, 16)  # rejected before any device work
    assert st == -1
    pkg.lib.ipr_last_error.restype = ctypes.c_char_p
    assert b"65536" in pkg.lib.ipr_last_error()
