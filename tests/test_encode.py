"""Setup-time DB layout and encode: KeywordCuckooTable::to_raw_db
(src/pir/keyword/cuckoo.rs:314-353) and gpu_encode_db
(native/cuda/encode_kernel.cu:18-228, 264-386).

CPU: the oracle's restatements against direct NumPy statements of the same
definitions (big-endian byte pairs into column-major u16; for two polynomials
the interpolation is ((a0 + a1) / 2, (a0 - a1) / 2) mod 65535) and against the
linearity every encode must have.  GPU: the device kernels equal the oracle for
every interpolation degree the plans produce (1 .. 32), the reference's own
encode kernel (compiled from its sources into oracle/_ref) equals the oracle,
and a server built from the raw DB answers like one built from the encoded DB.
"""
import ctypes
import os

import numpy as np
import pytest

N = 2048
P = 65535
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libinspire_ref_kernels.so")


def _table(rng, num_buckets, entry_size, fill=0.8):
    entries = rng.integers(0, 256, (num_buckets, entry_size), dtype=np.uint8)
    occupied = (rng.random(num_buckets) < fill).astype(np.uint8)
    return entries, occupied


def test_oracle_raw_db_matches_definition(orc):
    rng = np.random.default_rng(1)
    db_rows, per, es = 16, 3, 10
    ise = es // 2
    num_buckets = db_rows * per - 2  # the last two slots of the table do not exist
    db_cols = 2048
    entries, occupied = _table(rng, num_buckets, es)
    got = orc.raw_db(entries, occupied, es, db_rows, db_cols, per).reshape(db_cols, db_rows)
    want = np.zeros((db_cols, db_rows), dtype=np.uint16)
    for item in range(per):
        for row in range(db_rows):
            b = row * per + item
            if b >= num_buckets or not occupied[b]:
                continue
            for j in range(ise):
                want[item * ise + j, row] = (int(entries[b, 2 * j]) << 8) | int(entries[b, 2 * j + 1])
    assert np.array_equal(got, want)


def test_oracle_encode_two_points_closed_form(orc):
    rng = np.random.default_rng(2)
    db_rows = 16
    raw = rng.integers(0, P + 1, (2 * N, db_rows), dtype=np.uint16)  # 65535 (= 0 mod p) included
    raw[0, 0] = P
    enc = orc.encode_db(raw.reshape(-1), db_rows, 2 * N, 2).reshape(2 * N, db_rows)
    a0, a1 = raw[:N].astype(np.int64) % P, raw[N:].astype(np.int64) % P
    half = pow(2, -1, P)
    assert np.array_equal(enc[:N], ((a0 + a1) * half) % P)
    assert np.array_equal(enc[N:], ((a0 - a1) * half) % P)


@pytest.mark.parametrize("interp", [1, 4, 32])
def test_oracle_encode_is_linear(orc, interp):
    rng = np.random.default_rng(interp)
    db_rows, cols = 16, interp * N
    a = rng.integers(0, P, cols * db_rows, dtype=np.int64)
    b = rng.integers(0, P, cols * db_rows, dtype=np.int64)
    ea = orc.encode_db(a.astype(np.uint16), db_rows, cols, interp).astype(np.int64)
    eb = orc.encode_db(b.astype(np.uint16), db_rows, cols, interp).astype(np.int64)
    eab = orc.encode_db(((a + b) % P).astype(np.uint16), db_rows, cols, interp).astype(np.int64)
    assert np.array_equal(eab, (ea + eb) % P)
    assert eab.max() < P


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.gpu
@pytest.mark.parametrize("interp,c,db_rows", [(1, 2, 32), (2, 1, 32), (4, 2, 64), (8, 1, 256), (16, 1, 32),
                                              (32, 1, 32), (32, 2, 96)])
def test_device_encode_matches_oracle(pkg, orc, interp, c, db_rows):
    import torch
    rng = np.random.default_rng(100 + interp + c)
    cols = interp * N * c
    raw = rng.integers(0, P + 1, cols * db_rows, dtype=np.uint16)
    want = orc.encode_db(raw, db_rows, cols, interp)
    d_in = _dev(raw.view(np.int16))
    d_out = torch.zeros_like(d_in)
    pkg.encode_db(d_in.data_ptr(), d_out.data_ptr(), db_rows, cols, interp)
    torch.cuda.synchronize()
    assert np.array_equal(d_out.cpu().numpy().view(np.uint16), want)


@pytest.mark.gpu
def test_device_raw_db_matches_oracle(pkg, orc):
    import torch
    rng = np.random.default_rng(7)
    db_rows, per, es = 96, 5, 1216
    num_buckets = db_rows * per - 3
    db_cols = 4 * N
    entries, occupied = _table(rng, num_buckets, es)
    want = orc.raw_db(entries, occupied, es, db_rows, db_cols, per)
    d_e, d_o = _dev(entries), _dev(occupied)
    d_raw = torch.full((db_rows * db_cols,), 7, dtype=torch.int16, device="cuda")  # cleared by the call
    pkg.cuckoo_to_raw_db(d_e.data_ptr(), d_o.data_ptr(), num_buckets, es, db_rows, db_cols, per, d_raw.data_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(d_raw.cpu().numpy().view(np.uint16), want)


@pytest.mark.gpu
def test_reference_encode_kernel_matches_oracle(orc):
    """the reference's own gpu_encode_db_from_host, built from its sources, pins the oracle"""
    if not os.path.exists(REF_LIB):
        pytest.skip("reference kernels not built (make -C oracle ref)")
    from cuda.bindings import runtime as rt
    lib = ctypes.CDLL(REF_LIB)
    lib.gpu_encode_db_from_host.argtypes = [ctypes.c_void_p, ctypes.c_void_p] + [ctypes.c_int] * 5 + \
        [ctypes.c_uint32, ctypes.c_uint32]
    lib.gpu_encode_get_device_db.restype = ctypes.c_void_p
    for interp, c, db_rows in ((8, 1, 32), (32, 1, 32)):  # its tiled gather needs rows in 32s
        rng = np.random.default_rng(interp)
        cols = interp * N * c
        raw = rng.integers(0, P, cols * db_rows, dtype=np.uint16)
        inv = pow(interp, -1, P)
        lib.gpu_encode_db_from_host(raw.ctypes.data, None, db_rows, cols, interp, N, c, P, inv)
        ptr = lib.gpu_encode_get_device_db()
        assert ptr
        got = np.zeros_like(raw)
        err, = rt.cudaMemcpy(got.ctypes.data, ptr, got.nbytes, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
        assert err == rt.cudaError_t.cudaSuccess
        assert np.array_equal(got, orc.encode_db(raw, db_rows, cols, interp))


@pytest.mark.gpu
def test_server_from_raw_answers_like_encoded(pkg, orc):
    instances, interp = 4, 2
    plan = pkg.Plan(num_items=32768, entry_size=1216, item_size_bits=9728, dim0=2048, db_rows=2048,
                    db_cols=instances * N, instances=instances, interp=interp, c=2, peak_bytes=0)
    sdb = orc.SynthDB(plan.db_rows, instances, interp, 2, seed=71)
    rng = np.random.default_rng(71)
    raw = rng.integers(0, P + 1, plan.db_rows * plan.db_cols, dtype=np.uint16)
    enc = orc.encode_db(raw, plan.db_rows, plan.db_cols, interp)
    q = orc.synth_query(5, plan.db_rows, 2)
    with pkg.KeywordServer.from_raw(plan, raw, sdb.a_hat, sdb.bold_t, sdb.bold_t_bar, sdb.bold_t_hat) as a, \
            pkg.KeywordServer.from_encoded(plan, enc, sdb.a_hat, sdb.bold_t, sdb.bold_t_bar, sdb.bold_t_hat) as b:
        ra = a.respond_to_serialized_query(q)
        assert ra == b.respond_to_serialized_query(q)
        sdb.db[:] = enc  # the oracle answers over the encoded DB
        assert ra == orc.respond(sdb, q)
        assert a.respond_batch([q, q]) == [ra, ra]


@pytest.mark.gpu
def test_compat_encode_fold_and_swap(pkg, orc):
    """gpu_encode_db_from_host_fold / gpu_encode_get_device_db_fold / gpu_encode_swap_primary
    (encode_kernel.cu:452-516): a second DB is encoded into the secondary slot while the
    primary stays as it was; the swap promotes it"""
    from cuda.bindings import runtime as rt
    lib = pkg.lib
    sig = [ctypes.c_void_p] + [ctypes.c_int] * 5 + [ctypes.c_uint32, ctypes.c_uint32]
    lib.gpu_encode_db_from_host.argtypes = [ctypes.c_void_p] + sig
    lib.gpu_encode_db_from_host_fold.argtypes = sig
    lib.gpu_encode_get_device_db.restype = ctypes.c_void_p
    lib.gpu_encode_get_device_db_fold.restype = ctypes.c_void_p
    db_rows, interp, c = 64, 8, 2
    cols = interp * N * c
    inv = pow(interp, -1, P)
    rng = np.random.default_rng(19)
    a = rng.integers(0, P, cols * db_rows, dtype=np.uint16)
    b = rng.integers(0, P, cols * db_rows, dtype=np.uint16)

    def dev(ptr):
        got = np.zeros_like(a)
        err, = rt.cudaMemcpy(got.ctypes.data, ptr, got.nbytes, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
        assert err == rt.cudaError_t.cudaSuccess
        return got

    lib.gpu_encode_db_from_host(a.ctypes.data, None, db_rows, cols, interp, N, c, P, inv)
    primary = lib.gpu_encode_get_device_db()
    lib.gpu_encode_db_from_host_fold(b.ctypes.data, db_rows, cols, interp, N, c, P, inv)
    second = lib.gpu_encode_get_device_db_fold()
    assert primary and second and primary != second
    assert lib.gpu_encode_get_device_db() == primary
    assert np.array_equal(dev(primary), orc.encode_db(a, db_rows, cols, interp))
    assert np.array_equal(dev(second), orc.encode_db(b, db_rows, cols, interp))
    lib.gpu_encode_swap_primary()
    assert lib.gpu_encode_get_device_db() == second and not lib.gpu_encode_get_device_db_fold()
    assert np.array_equal(dev(second), orc.encode_db(b, db_rows, cols, interp))
    lib.gpu_encode_free_device_db()
    assert not lib.gpu_encode_get_device_db()
