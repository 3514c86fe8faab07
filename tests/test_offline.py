"""Offline precomputation: PirServer::perform_offline_precomputation_simplepir
(src/pir/server/engine.rs:677-1042) -> a_hat, bold_t, bold_t_bar, bold_t_hat.

CPU: the device's algorithm — the packing sums of full_packing_with_preprocessing_offline
(packing.rs:2627-2679) as one NTT over j per slot followed by a slot gather — equals the
oracle's brute-force restatement of the reference's loops on a full instance.  GPU:
ipr_offline_precompute equals the oracle's whole pipeline bit for bit (one and two
row polynomials, one and several instances per pass).
"""
import numpy as np
import pytest

N = 2048


def test_packing_sum_as_ntt_then_gather(orc):
    """r_all[i][z] = N^-1 E[tau_{5^i}(z)][z], r_bar_all[i][z] = N^-1 E[tau_{-5^i}(z)][z],
    E[s] = NTT over j of (a_j[s])_j"""
    rng = np.random.default_rng(5)
    db = rng.integers(0, 65535, N * N, dtype=np.uint16)
    a = orc.prep_pack(db, N, 0, orc.hint_query(1))
    r, rb = orc.pack_r(a)
    E = np.stack([orc.ntt_forward(np.concatenate([a[:, 0, s], a[:, 1, s]])).reshape(2, N) for s in range(N)])
    z = np.arange(N)
    for li, q in enumerate((orc.Q0, orc.Q1)):
        ninv = pow(N, -1, q)
        El = E[:, li, :].astype(object)
        for i in (0, 1, 2, 511, 1000, 1023):
            g = int(orc.gen_pow(i))
            got = (El[orc.automorph_table(g).astype(np.int64), z] * ninv) % q
            gotb = (El[orc.automorph_table(2 * N - g).astype(np.int64), z] * ninv) % q
            assert np.array_equal(got.astype(np.uint64), r[i, li]), (i, li)
            assert np.array_equal(gotb.astype(np.uint64), rb[i, li]), (i, li)


def test_offline_keys_are_rotations_of_the_masks(orc):
    wm, vm, wa, wb = orc.offline_keys()
    assert wm.shape == (3, 2, N) and (wm[:, 0] < orc.Q0).all() and (wm[:, 1] < orc.Q1).all()
    assert not np.array_equal(wm, vm)
    for i in (0, 7, 1022):
        g = int(orc.gen_pow(i))
        t, tb = orc.automorph_table(g).astype(np.int64), orc.automorph_table(2 * N - g).astype(np.int64)
        assert np.array_equal(wa[i], wm[:, :, t]) and np.array_equal(wb[i], wm[:, :, tb])
    assert np.array_equal(wa[0], wm)  # gen_pows[0] = 1


def _device_precompute(pkg, db, db_rows, instances, scratch=0):
    import torch
    d_db = torch.from_numpy(db.view(np.int16)).cuda()
    a_hat = torch.zeros(instances * N, dtype=torch.int64, device="cuda")
    bt = torch.zeros(instances * 3069 * N, dtype=torch.int64, device="cuda")
    btb = torch.zeros_like(bt)
    bth = torch.zeros(instances * 3 * N, dtype=torch.int64, device="cuda")
    pkg.offline_precompute(d_db.data_ptr(), db_rows, instances, a_hat.data_ptr(), bt.data_ptr(), btb.data_ptr(),
                           bth.data_ptr(), scratch)
    torch.cuda.synchronize()
    out = [x.cpu().numpy().view(np.uint64) for x in (a_hat, bt, btb, bth)]
    return (out[0].reshape(instances, N), out[1].reshape(instances, 3069, N), out[2].reshape(instances, 3069, N),
            out[3].reshape(instances, 3, N))


@pytest.mark.gpu
@pytest.mark.parametrize("db_rows,instances,scratch", [(N, 2, 0), (2 * N, 1, 0), (N, 2, 1)])
def test_device_offline_matches_oracle(pkg, orc, db_rows, instances, scratch):
    """scratch=1 forces one instance per pass"""
    rng = np.random.default_rng(db_rows + instances + scratch)
    db = rng.integers(0, 65535, instances * N * db_rows, dtype=np.uint16)
    want = orc.offline_precompute(db, db_rows, instances)
    got = _device_precompute(pkg, db, db_rows, instances, scratch)
    for name, w, g in zip(("a_hat", "bold_t", "bold_t_bar", "bold_t_hat"), want, got):
        assert np.array_equal(w, g), name


def _oracle_db(orc, plan, db, pre, stash=()):
    sdb = orc.SynthDB.__new__(orc.SynthDB)
    sdb.db_rows, sdb.instances, sdb.interp, sdb.c, sdb.seed = plan.db_rows, plan.instances, plan.interp, plan.c, 0
    sdb.db_cols = plan.db_cols
    sdb.db = np.ascontiguousarray(db, dtype=np.uint16)
    sdb.a_hat, sdb.bold_t, sdb.bold_t_bar, sdb.bold_t_hat = (np.ascontiguousarray(x).reshape(-1) for x in pre)
    sdb.stash = [bytes(s) for s in stash]
    sdb._stash_buf = np.frombuffer(b"".join(sdb.stash) or b"\0", dtype=np.uint8).copy()
    return sdb


@pytest.mark.gpu
def test_server_setup_from_raw_db_answers_like_the_oracle(pkg, orc):
    """KeywordServer::setup on the device: raw DB -> encode -> offline precomputation -> respond"""
    instances, interp = 2, 2
    plan = pkg.Plan(num_items=32768, entry_size=1216, item_size_bits=9728, dim0=2048, db_rows=N,
                    db_cols=instances * N, instances=instances, interp=interp, c=1, peak_bytes=0)
    rng = np.random.default_rng(12)
    raw = rng.integers(0, 65536, plan.db_rows * plan.db_cols, dtype=np.uint16)
    enc = orc.encode_db(raw, plan.db_rows, plan.db_cols, interp)
    pre = orc.offline_precompute(enc, plan.db_rows, instances)
    stash = [bytes([5]) * 1216]
    sdb = _oracle_db(orc, plan, enc, pre, stash)
    q = orc.synth_query(3, plan.db_rows, 2)
    with pkg.KeywordServer.setup(plan, raw, raw=True, stash=stash) as srv:
        got = srv.respond_to_serialized_query(q)
        assert got == orc.respond(sdb, q)
        assert srv.respond_batch([q, q]) == [got, got]


def _ref_lib():
    import ctypes
    import os
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                        "libinspire_ref_offline.so")
    if not os.path.exists(path):
        pytest.skip("reference offline kernels not built (make -C oracle ref)")
    return ctypes.CDLL(path)


@pytest.mark.gpu
def test_reference_offline_kernels_match_oracle(orc):
    """the reference's own GPU kernels for the offline steps (hint_kernel.cu, prep_pack_kernel.cu,
    packing_kernel.cu, collapse_kernel.cu, built from its sources) pin the oracle's restatement:
    a_ct_tilde, the packing sums after the automorphisms, and the collapse outputs"""
    import ctypes
    from cuda.bindings import runtime as rt
    lib = _ref_lib()
    u64, i32, u32, vp = ctypes.c_uint64, ctypes.c_int, ctypes.c_uint32, ctypes.c_void_p
    P = orc.params()
    tables = np.ctypeslib.as_array(P.ntt).reshape(-1).astype(np.uint64).copy()  # [2][4][N]
    rng = np.random.default_rng(77)
    db_rows, inst = N, 1
    db = rng.integers(0, 65535, inst * N * db_rows, dtype=np.uint16)
    query = orc.hint_query(1)

    def d2h(dst, ptr):
        err, = rt.cudaMemcpy(dst.ctypes.data, ptr, dst.nbytes, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
        assert err == rt.cudaError_t.cudaSuccess

    def h2d(ptr, src):
        err, = rt.cudaMemcpy(ptr, src.ctypes.data, src.nbytes, rt.cudaMemcpyKind.cudaMemcpyHostToDevice)
        assert err == rt.cudaError_t.cudaSuccess

    # hint + prep_pack (engine.rs:749-792)
    lib.gpu_hint_upload_tables.argtypes = [vp, i32]
    lib.gpu_hint_upload_query_ffi.argtypes = [vp, i32, i32]
    lib.gpu_hint_compute_from_host.argtypes = [vp, vp, i32, i32, i32, u32, u32, u64, u64, u64, u64, u64, u64, u64]
    lib.gpu_hint_get_device_output.restype = vp
    lib.gpu_hint_get_ntt_tables.restype = vp
    lib.gpu_prep_pack_compute.argtypes = [vp, vp, i32, u32, u32, u64]
    lib.gpu_prep_pack_get_output.restype = vp
    lib.gpu_hint_upload_tables(tables.ctypes.data, N)
    q64 = np.ascontiguousarray(query, dtype=np.uint64)
    lib.gpu_hint_upload_query_ffi(q64.ctypes.data, 1, N)
    hint = np.zeros(inst * N * N, dtype=np.uint64)
    lib.gpu_hint_compute_from_host(db.ctypes.data, hint.ctypes.data, db_rows, 1, inst * N, P.q[0], P.q[1],
                                   P.barrett_cr1[0], P.barrett_cr1[1], P.mod0_inv_mod1, P.mod1_inv_mod0, P.modulus,
                                   P.cr0_mod, P.cr1_mod)
    lib.gpu_prep_pack_compute(lib.gpu_hint_get_device_output(), lib.gpu_hint_get_ntt_tables(), inst * N,
                              P.q[0], P.q[1], P.modulus)
    a_ref = np.zeros(inst * N * 2 * N, dtype=np.uint64)
    d2h(a_ref, lib.gpu_prep_pack_get_output())
    a_or = orc.prep_pack(db, db_rows, 0, query)
    assert np.array_equal(a_ref.reshape(N, 2, N), a_or)

    # packing sums (gpu_packing_precomp) + the automorphisms the reference applies on the CPU
    r_or, rb_or = orc.pack_r(a_or)
    mono = np.zeros((2 * N, 2 * N), dtype=np.uint64)
    for e in range(N):
        raw = np.zeros(N, dtype=np.uint64)
        raw[e] = 1
        mono[e] = orc.to_ntt(raw)
        mono[N + e] = np.where(mono[e] == 0, 0, np.concatenate([np.full(N, orc.Q0), np.full(N, orc.Q1)]) - mono[e])
    half = N // 2
    idx = np.zeros((half, N), dtype=np.int32)
    idxb = np.zeros((half, N), dtype=np.int32)
    j = np.arange(N, dtype=np.int64)
    for i in range(half):
        gp = int(orc.gen_pow((N - i) % N))
        ind = (j * gp) % (2 * N)
        indb = (2 * N - (j * gp) % (2 * N)) % (2 * N)
        idx[i] = np.where(ind < N, ind, N + ind % N)
        idxb[i] = np.where(indb < N, indb, N + indb % N)
    inv_raw = np.zeros(N, dtype=np.uint64)
    inv_raw[0] = pow(N, -1, orc.Q)
    mod_inv = orc.to_ntt(inv_raw)
    lib.gpu_packing_precomp.argtypes = [vp, vp, vp, vp, vp, vp, vp, i32, i32, i32, i32, u64, u64, u64, u64]
    r_ref = np.zeros(half * 2 * N, dtype=np.uint64)
    rb_ref = np.zeros(half * 2 * N, dtype=np.uint64)
    a_flat = np.ascontiguousarray(a_or.reshape(-1))
    lib.gpu_packing_precomp(mono.ctypes.data, a_flat.ctypes.data, idx.ctypes.data, idxb.ctypes.data,
                            mod_inv.ctypes.data, r_ref.ctypes.data, rb_ref.ctypes.data, half, N, N, 2, P.q[0],
                            P.q[1], P.barrett_cr1[0], P.barrett_cr1[1])
    r_ref, rb_ref = r_ref.reshape(half, 2, N), rb_ref.reshape(half, 2, N)
    for i in (0, 1, 500, 1023):
        g = int(orc.gen_pow(i))
        t, tb = orc.automorph_table(g).astype(np.int64), orc.automorph_table(2 * N - g).astype(np.int64)
        assert np.array_equal(r_ref[i][:, t], r_or[i]), i
        assert np.array_equal(rb_ref[i][:, tb], rb_or[i]), i

    # collapse (gpu_collapse_setup / gpu_collapse_run, collapse_kernel.cu)
    _, vm, wa, wb = orc.offline_keys()
    want = orc.collapse(r_or, rb_or, wa, wb, vm)
    lib.gpu_collapse_alloc_r.argtypes = [i32, i32, i32]
    lib.gpu_collapse_get_r_all_col.argtypes = [i32, i32, i32]
    lib.gpu_collapse_get_r_all_col.restype = vp
    lib.gpu_collapse_get_r_bar_all_col.argtypes = [i32, i32, i32]
    lib.gpu_collapse_get_r_bar_all_col.restype = vp
    lib.gpu_collapse_setup.argtypes = [vp, vp, vp, vp, i32, i32, i32, i32]
    lib.gpu_collapse_run.argtypes = [i32, i32, i32, i32, u32, u32, u64, u64, u64, u64, u64, u64, u64]
    lib.gpu_collapse_download_a_hat.argtypes = [vp, i32]
    for name in ("gpu_collapse_get_bold_t", "gpu_collapse_get_bold_t_bar", "gpu_collapse_get_bold_t_hat"):
        getattr(lib, name).restype = vp
    lib.gpu_collapse_alloc_r(1, half, 2 * N)
    h2d(lib.gpu_collapse_get_r_all_col(0, half, 2 * N), np.ascontiguousarray(r_or))
    h2d(lib.gpu_collapse_get_r_bar_all_col(0, half, 2 * N), np.ascontiguousarray(rb_or))
    wa_f, wb_f, vm_f = (np.ascontiguousarray(x).reshape(-1) for x in (wa, wb, vm))
    lib.gpu_collapse_setup(wa_f.ctypes.data, wb_f.ctypes.data, vm_f.ctypes.data, tables.ctypes.data, 1, half, 3,
                           2 * N)
    lib.gpu_collapse_run(1, half, 3, 19, P.q[0], P.q[1], P.barrett_cr1[0], P.barrett_cr1[1], P.mod0_inv_mod1,
                         P.mod1_inv_mod0, P.modulus, P.cr0_mod, P.cr1_mod)
    a_hat = np.zeros(N, dtype=np.uint64)
    lib.gpu_collapse_download_a_hat(a_hat.ctypes.data, 1)
    bt = np.zeros(3069 * N, dtype=np.uint64)
    btb = np.zeros(3069 * N, dtype=np.uint64)
    bth = np.zeros(3 * N, dtype=np.uint64)
    d2h(bt, lib.gpu_collapse_get_bold_t())
    d2h(btb, lib.gpu_collapse_get_bold_t_bar())
    d2h(bth, lib.gpu_collapse_get_bold_t_hat())
    for name, w, g in zip(("a_hat", "bold_t", "bold_t_bar", "bold_t_hat"), want,
                          (a_hat, bt.reshape(3069, N), btb.reshape(3069, N), bth.reshape(3, N))):
        assert np.array_equal(w, g), name


def _random_condensed(rng, rows):
    lo = rng.integers(0, orc_q()[0], (rows, N), dtype=np.uint64)
    hi = rng.integers(0, orc_q()[1], (rows, N), dtype=np.uint64)
    return lo | (hi << np.uint64(32))


def orc_q():
    return 268369921, 249561089


@pytest.mark.gpu
def test_inspiring_pack_matches_oracle(pkg, orc):
    """packing_fully_online for two sets of 2048 LWEs (uniform mod q, seeded) with random keys"""
    import torch
    rng = np.random.default_rng(31)
    sets = 2
    lwe = rng.integers(0, orc.Q, (sets, N + 1, N), dtype=np.uint64)
    y = _random_condensed(rng, 3)
    z = _random_condensed(rng, 3)
    want = [orc.inspiring_pack(lwe[c], y, z) for c in range(sets)]
    d_lwe = torch.from_numpy(lwe.view(np.int64)).cuda()
    d_y = torch.from_numpy(y.view(np.int64)).cuda()
    d_z = torch.from_numpy(z.view(np.int64)).cuda()
    d_out = torch.zeros((sets, 2, N), dtype=torch.int64, device="cuda")
    with pkg.InspiringPacker(max_sets=sets) as pk:
        for n in (sets, 1):  # both sets together, then the first alone
            d_out.zero_()
            pk.pack(n, d_lwe.data_ptr(), d_y.data_ptr(), d_z.data_ptr(), d_out.data_ptr())
            torch.cuda.synchronize()
            got = d_out.cpu().numpy().view(np.uint64)
            for c in range(n):
                assert np.array_equal(got[c], want[c]), (n, c)
