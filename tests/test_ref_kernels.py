"""Pins the oracle's GEMV, rotation and packing steps to the reference's own
CUDA kernels (native/cuda/gemv_kernel.cu, rotation_kernel.cu,
packing_online_kernel.cu of rkdud007/inspire-rs), compiled unmodified into
oracle/_ref/ by `make -C oracle ref`.  Skipped where that build is absent.
The reference is called through its own extern "C" entry points."""
import ctypes
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 2048


@pytest.fixture(scope="module")
def ref(orc):
    if not os.path.exists(orc.REF_LIB):
        pytest.skip("reference kernels not built (make -C oracle ref)")
    lib = ctypes.CDLL(orc.REF_LIB)
    lib.gpu_packing_online_get_d_y_all.restype = ctypes.c_void_p
    lib.gpu_packing_online_get_d_y_bar_all.restype = ctypes.c_void_p
    return lib


@pytest.fixture(scope="module")
def sdb(orc):
    return orc.SynthDB(2048, 4, 2, 2, seed=2026)


def test_reference_gemv_equals_oracle(ref, orc, sdb):
    vp, i32, u64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64
    d_db = ctypes.c_void_p()
    ref.gpu_gemv_upload_db(vp(sdb.db.ctypes.data), ctypes.byref(d_db), ctypes.c_size_t(sdb.db.nbytes))
    assert d_db.value
    p = orc.params()
    for s in (1, 2):
        q = orc.synth_query(s, sdb.db_rows, 1)
        _, _, rows, _ = orc.parse_query(q, sdb.db_rows)
        a = np.ascontiguousarray(rows[0])
        c = np.zeros(sdb.db_cols, dtype=np.uint64)
        ref.gpu_gemv_query(vp(c.ctypes.data), vp(a.ctypes.data), d_db, i32(sdb.db_rows), i32(sdb.db_cols),
                           u64(orc.Q0), u64(orc.Q1), u64(p.barrett_cr1[0]), u64(p.barrett_cr1[1]),
                           u64(p.mod0_inv_mod1), u64(p.mod1_inv_mod0), u64(orc.Q), u64(p.cr0_mod), u64(p.cr1_mod))
        assert np.array_equal(c, orc.gemv(sdb, a))
    ref.gpu_gemv_free_db(d_db)


def test_reference_rotation_and_packing_equal_oracle(ref, orc, sdb):
    vp, i32, u64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64
    tables = np.stack([orc.automorph_table(t) for t in range(1, 4096, 2)]).astype(np.uint32)
    gen = np.array([orc.gen_pow(i) for i in range(1023)], dtype=np.uint32)
    ref.gpu_rotation_upload_tables(vp(tables.ctypes.data), vp(gen.ctypes.data), i32(2048), i32(1023), i32(2048))
    ref.gpu_packing_online_upload_precomp(vp(sdb.bold_t.ctypes.data), vp(sdb.bold_t_bar.ctypes.data),
                                          vp(sdb.bold_t_hat.ctypes.data), i32(sdb.instances), i32(3069), i32(3),
                                          i32(2048))
    ref.gpu_packing_online_ensure_key_buffers(i32(3069), i32(3), i32(2048))
    p = orc.params()
    for s in (3, 4):
        q = orc.synth_query(s, sdb.db_rows, 1)
        y, z, _, _ = orc.parse_query(q, sdb.db_rows)
        dya, dyb = ref.gpu_packing_online_get_d_y_all(), ref.gpu_packing_online_get_d_y_bar_all()
        ref.gpu_rotation_expand_keys(vp(dya), vp(dyb), vp(y.ctypes.data), i32(1023), i32(3), i32(2048))
        ref.gpu_packing_online_upload_z_body(vp(z.ctypes.data), i32(3), i32(2048))
        out = np.zeros(sdb.instances * 2 * N, dtype=np.uint64)
        ref.gpu_packing_online_compute(vp(out.ctypes.data), i32(sdb.instances), i32(1023), i32(3), i32(2048),
                                       i32(128), u64(orc.Q0), u64(orc.Q1), u64(p.barrett_cr1[0]),
                                       u64(p.barrett_cr1[1]))
        assert np.array_equal(out.reshape(sdb.instances, 2, N), orc.packing_sum(sdb, y, z))
    ref.gpu_packing_online_free()
