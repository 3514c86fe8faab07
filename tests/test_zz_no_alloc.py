"""ipr_gemv_query_noalloc: the GEMV query for callers that cannot allocate.

A process whose framework has reserved all free device memory for its own
pool, or a request path that cannot take the device-wide synchronisation of
cudaMalloc, cannot use gpu_gemv_query, which allocates device copies of the
query row and the result on every call.  ipr_gemv_query_noalloc stages both in
a fixed device array inside the library instead.  These tests drive it through
the C ABI and check:

* its results equal the oracle's GEMV (exact integers) at the 10k-record
  first dimension (2048 x 16384), at a 8192-row shape, and at both limits of
  the array (65,536 rows; 1,048,576 columns), on two calls in a row with
  different queries, so the second call cannot lean on the first's contents;
* they also equal what the allocating entry point gpu_gemv_query returns;
* after a first call, further calls leave the device's free memory unchanged
  (no allocation hides in the call);
* an unreduced query row and an oversize shape are refused before any device work.

The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

Q0, Q1 = 268369921, 249561089
IPR_E_ARGS = -1


def _query(seed, rows):
    rng = np.random.default_rng(seed)
    lo = rng.integers(0, Q0, rows, dtype=np.uint64)
    hi = rng.integers(0, Q1, rows, dtype=np.uint64)
    return np.ascontiguousarray(lo | (hi << np.uint64(32)))


def _db(seed, rows, cols):
    rng = np.random.default_rng(seed)
    return rng.integers(0, 65535, rows * cols, dtype=np.uint16)  # encoded DB values are < 65535


def _fn(lib):
    f = lib.ipr_gemv_query_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    return f


def _no_alloc(lib, d_db, a, rows, cols):
    c = np.zeros(cols, dtype=np.uint64)
    st = _fn(lib)(c.ctypes.data, a.ctypes.data, d_db, rows, cols)
    assert st == 0, lib.ipr_last_error()
    return c


def _with_alloc(lib, orc, d_db, a, rows, cols):
    """the existing entry point (allocates its staging buffers per call)"""
    p = orc.params()
    c = np.zeros(cols, dtype=np.uint64)
    u64 = ctypes.c_uint64
    lib.gpu_init_memory_pool()
    lib.gpu_gemv_query(ctypes.c_void_p(c.ctypes.data), ctypes.c_void_p(a.ctypes.data), ctypes.c_void_p(d_db),
                       ctypes.c_int(rows), ctypes.c_int(cols), u64(Q0), u64(Q1), u64(p.barrett_cr1[0]),
                       u64(p.barrett_cr1[1]), u64(p.mod0_inv_mod1), u64(p.mod1_inv_mod0), u64(Q0 * Q1),
                       u64(p.cr0_mod), u64(p.cr1_mod))
    return c


@pytest.mark.parametrize("rows,cols", [(2048, 16384), (8192, 8192), (65536, 16), (256, 1 << 20)])
def test_noalloc_gemv_matches_oracle(pkg, orc, rows, cols):
    import torch
    torch.cuda.set_device(0)
    db = _db(rows + cols, rows, cols)
    d_db = torch.from_numpy(db.view(np.int16)).cuda()
    for seed in (1, 2):  # two calls in a row share the library's array
        a = _query(seed, rows)
        got = _no_alloc(pkg.lib, d_db.data_ptr(), a, rows, cols)
        assert np.array_equal(got, orc.gemv_db(db, rows, a))  # integer results: exact
        if rows * cols <= 2048 * 16384:
            assert np.array_equal(got, _with_alloc(pkg.lib, orc, d_db.data_ptr(), a, rows, cols))
    del d_db
    torch.cuda.empty_cache()


def test_noalloc_calls_leave_free_memory_unchanged(pkg):
    import torch
    torch.cuda.set_device(0)
    rows, cols = 2048, 16384
    d_db = torch.from_numpy(_db(5, rows, cols).view(np.int16)).cuda()
    torch.cuda.synchronize()
    _no_alloc(pkg.lib, d_db.data_ptr(), _query(10, rows), rows, cols)  # first call: per-device set-up
    free0, _ = torch.cuda.mem_get_info()
    for seed in range(11, 16):
        _no_alloc(pkg.lib, d_db.data_ptr(), _query(seed, rows), rows, cols)
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_rejects_bad_arguments(pkg):
    f = _fn(pkg.lib)
    pkg.lib.ipr_last_error.restype = ctypes.c_char_p
    buf = np.zeros(256, dtype=np.uint64)
    assert f(buf.ctypes.data, buf.ctypes.data, buf.ctypes.data, 131072, 16) == IPR_E_ARGS  # above the maximum
    assert b"65536" in pkg.lib.ipr_last_error()
    bad = _query(3, 256)
    bad[7] = np.uint64(Q0)  # limb 0 equal to q0: not reduced
    assert f(buf.ctypes.data, bad.ctypes.data, buf.ctypes.data, 256, 16) == IPR_E_ARGS
    assert b"not reduced" in pkg.lib.ipr_last_error()
