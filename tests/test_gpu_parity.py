"""Parity of the sm_100a respond() path with the oracle, through the C ABI.

Every comparison is bit-exact (integer arithmetic).  Server state comes from
the seeded synthetic generator that the device (ipr_server_create_synthetic)
and the oracle (SynthDB) share, or from host arrays (ipr_server_create).
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 2048


def _plan(pkg, instances, interp, db_rows=2048, c=None):
    c = instances // interp if c is None else c
    return pkg.Plan(num_items=max(db_rows, 32768), entry_size=1216, item_size_bits=9728, dim0=db_rows,
                    db_rows=db_rows, db_cols=instances * N, instances=instances, interp=interp, c=c, peak_bytes=0)


@pytest.fixture(scope="module")
def cfg0(pkg, orc):
    """config-0 shape: 10k ML-KEM-768 records -> db 2048 x 16384, 8 instances, interp 8, c 1"""
    plan = pkg.plan_from_shape(10_000, 32, 1184)
    assert (plan.instances, plan.interp, plan.c) == (8, 8, 1)
    srv = pkg.KeywordServer.synthetic(plan, seed=7)
    sdb = orc.SynthDB(plan.db_rows, plan.instances, plan.interp, plan.c, seed=7)
    yield plan, srv, sdb
    srv.close()


@pytest.mark.parametrize("qseed", [1, 2026])
def test_respond_config0_bit_exact(cfg0, orc, qseed):
    plan, srv, sdb = cfg0
    q = orc.synth_query(qseed, plan.db_rows, 2)
    assert len(q) == 286_721
    got = srv.respond_to_serialized_query(q)
    want = orc.respond(sdb, q)
    assert len(got) == len(want) == 4 + 2 * (4 + 12288) + 4
    assert got == want


@pytest.mark.parametrize("nq", [0, 1, 3])
def test_respond_query_counts(cfg0, orc, nq):
    plan, srv, sdb = cfg0
    q = orc.synth_query(100 + nq, plan.db_rows, nq)
    assert srv.respond_to_serialized_query(q) == orc.respond(sdb, q)


def test_respond_repeatable_and_interleaved(cfg0, orc):
    plan, srv, sdb = cfg0
    qa, qb = orc.synth_query(31, plan.db_rows, 2), orc.synth_query(32, plan.db_rows, 2)
    ra = srv.respond_to_serialized_query(qa)
    rb = srv.respond_to_serialized_query(qb)
    assert srv.respond_to_serialized_query(qa) == ra
    assert ra != rb
    assert rb == orc.respond(sdb, qb)


@pytest.mark.parametrize("instances,interp", [(8, 2), (6, 1), (4, 4), (16, 8)])
def test_respond_other_shapes(pkg, orc, instances, interp):
    plan = _plan(pkg, instances, interp)
    with pkg.KeywordServer.synthetic(plan, seed=instances * 10 + interp) as srv:
        sdb = orc.SynthDB(plan.db_rows, instances, interp, plan.c, seed=instances * 10 + interp)
        q = orc.synth_query(5, plan.db_rows, 2)
        assert srv.respond_to_serialized_query(q) == orc.respond(sdb, q)


def test_respond_wider_first_dimension(pkg, orc):
    plan = _plan(pkg, 2, 2, db_rows=8192)
    with pkg.KeywordServer.synthetic(plan, seed=3) as srv:
        sdb = orc.SynthDB(plan.db_rows, 2, 2, 1, seed=3)
        q = orc.synth_query(9, plan.db_rows, 2)
        assert srv.respond_to_serialized_query(q) == orc.respond(sdb, q)


@pytest.mark.parametrize("tensor", [0, 1])
@pytest.mark.parametrize("nq", [1, 2, 3])
def test_first_dimension_paths(cfg0, pkg, orc, tensor, nq):
    """tcgen05 byte-plane GEMM and the CUDA-core GEMV give the oracle's bytes"""
    plan, srv, sdb = cfg0
    srv.set_option(pkg.KeywordServer.OPT_TENSOR_GEMV, tensor)
    try:
        q = orc.synth_query(40 + nq, plan.db_rows, nq)
        assert srv.respond_to_serialized_query(q) == orc.respond(sdb, q)
    finally:
        srv.set_option(pkg.KeywordServer.OPT_TENSOR_GEMV, 1)


@pytest.mark.parametrize("regs", [0, 1, 2, 3, 4, 5])
@pytest.mark.parametrize("instances,interp", [(8, 8), (8, 1), (6, 2)])
def test_fold_kernels(pkg, orc, regs, instances, interp):
    """the four fold forms (shared-memory NTTs, register NTTs after a separate INTT + CRT
    pass, register NTTs with that pass fused in on two chains or one chain per CTA) give the
    oracle's bytes, for one, eight and three fold groups (an odd count leaves the two-chain
    form's second team of a CTA idle)"""
    plan = _plan(pkg, instances, interp)
    with pkg.KeywordServer.synthetic(plan, seed=50 + instances + interp) as srv:
        srv.set_option(pkg.KeywordServer.OPT_FOLD_REGISTER_NTT, regs)
        sdb = orc.SynthDB(plan.db_rows, instances, interp, plan.c, seed=50 + instances + interp)
        for nq in (1, 2, 3):
            q = orc.synth_query(60 + nq, plan.db_rows, nq)
            assert srv.respond_to_serialized_query(q) == orc.respond(sdb, q)


@pytest.mark.parametrize("form", [0, 1, 2, 3, 4, 5, 6])
def test_u64_gemv_forms(cfg0, pkg, orc, form):
    """the CUDA-core GEMV forms (8 / 4 / 2 DB columns per warp in registers, 8 columns staged
    through a shared-memory ring, products on the FP64 pipe, limbs split between the integer
    and FP64 pipes) give the oracle's bytes"""
    plan, srv, sdb = cfg0
    srv.set_option(pkg.KeywordServer.OPT_TENSOR_GEMV, 0)
    srv.set_option(pkg.KeywordServer.OPT_GEMV_FORM, form)
    try:
        for nq in (1, 2, 3):
            q = orc.synth_query(70 + nq + form, plan.db_rows, nq)
            assert srv.respond_to_serialized_query(q) == orc.respond(sdb, q)
    finally:
        srv.set_option(pkg.KeywordServer.OPT_GEMV_FORM, 6)
        srv.set_option(pkg.KeywordServer.OPT_TENSOR_GEMV, 1)


@pytest.mark.parametrize("db_rows", [4096, 16384, 32768])
def test_fp64_gemv_forms_at_their_row_limit(pkg, orc, db_rows):
    """the FP64-pipe GEMV forms at their row limits, where a lane's partial sum of full-range
    products can come within a factor 2 of 2^53: form 5 at 4,096 rows (above it, form 4), form 4
    at 16,384, and past both (32,768 rows, run as form 0); form 6, which flushes its double sums
    every 256 rows, at all three"""
    plan = _plan(pkg, 2, 2, db_rows=db_rows)
    with pkg.KeywordServer.synthetic(plan, seed=23) as srv:
        sdb = orc.SynthDB(plan.db_rows, 2, 2, 1, seed=23)
        q = orc.synth_query(6, plan.db_rows, 2)
        want = orc.respond(sdb, q)
        srv.set_option(pkg.KeywordServer.OPT_TENSOR_GEMV, 0)
        for form in (4, 5, 6):
            srv.set_option(pkg.KeywordServer.OPT_GEMV_FORM, form)
            assert srv.respond_to_serialized_query(q) == want


def test_first_dimension_tensor_wide_rows(pkg, orc):
    plan = _plan(pkg, 2, 2, db_rows=16384)
    with pkg.KeywordServer.synthetic(plan, seed=21) as srv:
        sdb = orc.SynthDB(plan.db_rows, 2, 2, 1, seed=21)
        q = orc.synth_query(4, plan.db_rows, 2)
        want = orc.respond(sdb, q)
        assert srv.respond_to_serialized_query(q) == want
        srv.set_option(pkg.KeywordServer.OPT_TENSOR_GEMV, 0)
        assert srv.respond_to_serialized_query(q) == want


def test_from_encoded_with_stash(pkg, orc):
    plan = _plan(pkg, 4, 2)
    stash = [bytes([i]) * 1216 for i in range(3)]
    sdb = orc.SynthDB(plan.db_rows, 4, 2, 2, seed=44, stash=stash)
    with pkg.KeywordServer.from_encoded(plan, sdb.db, sdb.a_hat, sdb.bold_t, sdb.bold_t_bar, sdb.bold_t_hat,
                                        stash=stash, num_records=1234) as srv:
        q = orc.synth_query(8, plan.db_rows, 2)
        got = srv.respond_to_serialized_query(q)
        assert got == orc.respond(sdb, q)
        r = pkg.deserialize_keyword_response(got)
        assert r.stash_entries == stash and len(r.responses) == 2
        pp = srv.public_params()
        assert pp["keyword_pir"]["num_records"] == 1234 and pp["item_size_bits"] == 1216 * 8


def test_respond_payload_api(cfg0, pkg, orc):
    plan, srv, sdb = cfg0
    q = orc.synth_query(77, plan.db_rows, 2)
    y, z, rows, gsw = orc.parse_query(q, plan.db_rows)
    payload = pkg.KeywordQueryPayload(y.reshape(3, N), z.reshape(3, N), [(rows[i], gsw[i]) for i in range(2)])
    r = srv.respond(payload)
    want = pkg.deserialize_keyword_response(orc.respond(sdb, q))
    assert r.responses == want.responses


def test_malformed_queries(cfg0, pkg, orc):
    plan, srv, _ = cfg0
    q = orc.synth_query(1, plan.db_rows, 2)
    with pytest.raises(pkg.IprError) as e:
        srv.respond_to_serialized_query(q[:-10])
    assert e.value.status == -5
    with pytest.raises(pkg.IprError) as e:
        srv.respond_to_serialized_query(b"")
    assert e.value.status == -5
    # trailing bytes are ignored, as in the reference
    assert srv.respond_to_serialized_query(q + b"\0" * 5) == srv.respond_to_serialized_query(q)


def test_response_capacity_error(cfg0, pkg, orc):
    plan, srv, _ = cfg0
    q = orc.synth_query(1, plan.db_rows, 2)
    qa = (ctypes.c_uint8 * len(q)).from_buffer_copy(q)
    out = (ctypes.c_uint8 * 100)()
    n = ctypes.c_size_t()
    st = pkg.lib.ipr_server_respond(srv._h, qa, len(q), out, 100, ctypes.byref(n))
    assert st == -6 and n.value == srv.response_bytes(2)


def test_respond_device_and_profiling(cfg0, orc):
    import torch
    plan, srv, sdb = cfg0
    q = orc.synth_query(55, plan.db_rows, 2)
    dq = torch.frombuffer(bytearray(q), dtype=torch.uint8).cuda()
    rb = srv.response_bytes(2)
    dout = torch.zeros(rb, dtype=torch.uint8, device="cuda")
    srv.set_profiling(True)
    n = srv.respond_device(dq.data_ptr(), len(q), dout.data_ptr(), rb)
    srv.sync()
    times, calls = srv.stage_times()
    srv.set_profiling(False)
    assert n == rb and calls == 1 and times["pack"] > 0
    assert bytes(dout.cpu().numpy()) == orc.respond(sdb, q)


def test_step_gemv_matches_oracle(cfg0, pkg, orc):
    """first-dimension GEMV through the reference-named entry point gpu_gemv_query"""
    import torch
    plan, srv, sdb = cfg0
    lib = pkg.lib
    q = orc.synth_query(3, plan.db_rows, 1)
    _, _, rows, _ = orc.parse_query(q, plan.db_rows)
    a = np.ascontiguousarray(rows[0])
    ddb = torch.from_numpy(sdb.db.view(np.int16)).cuda()
    c = np.zeros(plan.db_cols, dtype=np.uint64)
    p = orc.params()
    lib.gpu_init_memory_pool()
    lib.gpu_gemv_query(ctypes.c_void_p(c.ctypes.data), ctypes.c_void_p(a.ctypes.data), ctypes.c_void_p(ddb.data_ptr()),
                       ctypes.c_int(plan.db_rows), ctypes.c_int(plan.db_cols), ctypes.c_uint64(orc.Q0),
                       ctypes.c_uint64(orc.Q1), ctypes.c_uint64(p.barrett_cr1[0]), ctypes.c_uint64(p.barrett_cr1[1]),
                       ctypes.c_uint64(p.mod0_inv_mod1), ctypes.c_uint64(p.mod1_inv_mod0), ctypes.c_uint64(orc.Q),
                       ctypes.c_uint64(p.cr0_mod), ctypes.c_uint64(p.cr1_mod))
    assert np.array_equal(c, orc.gemv(sdb, a))


def _d2h(ptr, nbytes):
    """copy device memory the library owns into a host array (cuda-python runtime API)"""
    from cuda.bindings import runtime as cudart
    out = np.zeros(nbytes // 8, dtype=np.uint64)
    err, = cudart.cudaMemcpy(out.ctypes.data, ptr, nbytes, cudart.cudaMemcpyKind.cudaMemcpyDeviceToHost)
    assert int(err) == 0, err
    return out


def test_compat_rotation_and_packing(cfg0, orc):
    """gpu_rotation_expand_keys + gpu_packing_online_compute (reference-named entry points)"""
    lib = __import__("inspire_rs_b200").lib
    plan, srv, sdb = cfg0
    q = orc.synth_query(12, plan.db_rows, 1)
    y, z, _, _ = orc.parse_query(q, plan.db_rows)
    tables = np.stack([orc.automorph_table(t) for t in range(1, 4096, 2)]).astype(np.uint32)
    gen = np.array([orc.gen_pow(i) for i in range(1023)], dtype=np.uint32)
    vp, i32 = ctypes.c_void_p, ctypes.c_int
    lib.gpu_init_memory_pool()
    lib.gpu_rotation_upload_tables(vp(tables.ctypes.data), vp(gen.ctypes.data), i32(2048), i32(1023), i32(2048))
    lib.gpu_packing_online_ensure_key_buffers(i32(3069), i32(3), i32(2048))
    lib.gpu_packing_online_get_d_y_all.restype = ctypes.c_void_p
    lib.gpu_packing_online_get_d_y_bar_all.restype = ctypes.c_void_p
    dya, dyb = lib.gpu_packing_online_get_d_y_all(), lib.gpu_packing_online_get_d_y_bar_all()
    lib.gpu_rotation_expand_keys(vp(dya), vp(dyb), vp(y.ctypes.data), i32(1023), i32(3), i32(2048))
    lib.gpu_packing_online_upload_z_body(vp(z.ctypes.data), i32(3), i32(2048))
    lib.gpu_packing_online_upload_precomp(vp(sdb.bold_t.ctypes.data), vp(sdb.bold_t_bar.ctypes.data),
                                          vp(sdb.bold_t_hat.ctypes.data), i32(sdb.instances), i32(3069), i32(3),
                                          i32(2048))
    out = np.zeros(sdb.instances * 2 * N, dtype=np.uint64)
    p = orc.params()
    lib.gpu_packing_online_compute(vp(out.ctypes.data), i32(sdb.instances), i32(1023), i32(3), i32(2048), i32(128),
                                   ctypes.c_uint64(orc.Q0), ctypes.c_uint64(orc.Q1),
                                   ctypes.c_uint64(p.barrett_cr1[0]), ctypes.c_uint64(p.barrett_cr1[1]))
    ya, yb = orc.rotations(y)
    assert np.array_equal(_d2h(dya, 3069 * N * 8), ya)
    assert np.array_equal(_d2h(dyb, 3069 * N * 8), yb)
    assert np.array_equal(out.reshape(sdb.instances, 2, N), orc.packing_sum(sdb, y, z))
    lib.gpu_packing_online_free()
    lib.gpu_rotation_free()


# ---------------------------------------------------------------------------
# batched respond: tensor-core packing of many clients at once
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("B", [2, 3, 8, 17])
def test_respond_batch_bit_exact(cfg0, orc, B):
    plan, srv, sdb = cfg0
    qs = [orc.synth_query(1000 + 7 * B + i, plan.db_rows, 2) for i in range(B)]
    got = srv.respond_batch(qs)
    assert len(got) == B
    for q, g in zip(qs, got):
        assert g == orc.respond(sdb, q)


def test_respond_batch_matches_single(cfg0, orc):
    plan, srv, sdb = cfg0
    qs = [orc.synth_query(2000 + i, plan.db_rows, 2) for i in range(5)]
    single = [srv.respond_to_serialized_query(q) for q in qs]
    assert srv.respond_batch(qs) == single


def test_respond_batch_mixed_query_counts(cfg0, orc):
    plan, srv, sdb = cfg0
    qs = [orc.synth_query(3000, plan.db_rows, 2), orc.synth_query(3001, plan.db_rows, 1),
          orc.synth_query(3002, plan.db_rows, 2), orc.synth_query(3003, plan.db_rows, 3)]
    got = srv.respond_batch(qs)
    for q, g in zip(qs, got):
        assert g == orc.respond(sdb, q)


@pytest.mark.parametrize("instances,interp", [(8, 2), (40, 8)])
def test_respond_batch_other_shapes(pkg, orc, instances, interp):
    plan = _plan(pkg, instances, interp)
    stash = [b"\x07" * 100, b"\x09" * 100]
    sdb = orc.SynthDB(plan.db_rows, instances, interp, plan.c, seed=90 + instances, stash=stash)
    with pkg.KeywordServer.from_encoded(plan, sdb.db, sdb.a_hat, sdb.bold_t, sdb.bold_t_bar, sdb.bold_t_hat,
                                        stash=stash) as srv:
        qs = [orc.synth_query(4000 + i, plan.db_rows, 2) for i in range(6)]
        got = srv.respond_batch(qs)
        for q, g in zip(qs, got):
            assert g == orc.respond(sdb, q)


@pytest.mark.parametrize("form", [1, 2, 3, 4, 5])
def test_respond_batch_fold_forms(pkg, orc, form):
    """the batch path's fold forms give the oracle's bytes at an odd fold-group count (40 / 8 = 5)
    with 9 payloads = 18 queries, 90 chains"""
    plan = _plan(pkg, 40, 8)
    sdb = orc.SynthDB(plan.db_rows, 40, 8, plan.c, seed=95)
    with pkg.KeywordServer.synthetic(plan, seed=95) as srv:
        srv.set_option(pkg.KeywordServer.OPT_FOLD_REGISTER_NTT, form)
        qs = [orc.synth_query(4500 + 11 * form + i, plan.db_rows, 2) for i in range(9)]
        got = srv.respond_batch(qs)
        for q, g in zip(qs, got):
            assert g == orc.respond(sdb, q)
        # the scaled RGSW bodies of one batch do not leak into the next
        assert srv.respond_batch(qs[:3]) == got[:3]


def test_respond_batch_device_entry(cfg0, orc):
    import torch
    plan, srv, sdb = cfg0
    qs = [orc.synth_query(5000 + i, plan.db_rows, 2) for i in range(4)]
    dq = torch.frombuffer(bytearray(b"".join(qs)), dtype=torch.uint8).cuda()
    rb = srv.response_bytes(2)
    dout = torch.zeros(4 * rb, dtype=torch.uint8, device="cuda")
    srv.respond_batch_device(4, dq.data_ptr(), dout.data_ptr())
    srv.sync()
    host = bytes(dout.cpu().numpy())
    for i, q in enumerate(qs):
        assert host[i * rb:(i + 1) * rb] == orc.respond(sdb, q)


@pytest.mark.parametrize("pair", [0, 1])
@pytest.mark.parametrize("B", [1, 5, 32, 64])
def test_packing_gemm_forms(cfg0, pkg, orc, pair, B):
    """the CTA-pair (M = 256 over two SMs) and one-CTA packing GEMMs give the oracle's bytes
    for client counts across the tile widths (N = 16 .. 256)"""
    import torch
    plan, srv, sdb = cfg0
    qs = [orc.synth_query(6000 + 97 * B + i, plan.db_rows, 2) for i in range(B)]
    srv.set_option(pkg.KeywordServer.OPT_PACK_CTA_PAIR, pair)
    try:
        if B > 1:
            got = srv.respond_batch(qs)
        else:  # a one-payload batch through the device entry
            dq = torch.frombuffer(bytearray(qs[0]), dtype=torch.uint8).cuda()
            dout = torch.zeros(srv.response_bytes(2), dtype=torch.uint8, device="cuda")
            srv.respond_batch_device(1, dq.data_ptr(), dout.data_ptr())
            srv.sync()
            got = [bytes(dout.cpu().numpy())]
    finally:
        srv.set_option(pkg.KeywordServer.OPT_PACK_CTA_PAIR, 2)
    for i in sorted({0, B // 2, B - 1}):
        assert got[i] == orc.respond(sdb, qs[i])
    if B > 1:
        assert got == [srv.respond_to_serialized_query(q) for q in qs]


@pytest.mark.gpu
def test_every_batch_configuration_is_exact_and_autotune_keeps_one(cfg0, pkg, orc):
    """the autotuner's candidates (packing GEMM on one CTA, a CTA pair or pairs from 48 payloads
    up; first-dimension GEMM tile 256 or 128) all answer bit-exactly; autotune times them at 64
    and 16 payloads and leaves the one with the least time per payload over both sizes set"""
    plan, srv, sdb = cfg0
    qs = [orc.synth_query(600 + i, plan.db_rows, 2) for i in range(64)]
    want = [orc.respond(sdb, q) for q in qs[:3]] + [orc.respond(sdb, qs[63])]
    for pair in (0, 1, 2):
        for tile in (0, 128):
            srv.set_option(pkg.KeywordServer.OPT_PACK_CTA_PAIR, pair)
            srv.set_option(pkg.KeywordServer.OPT_GEMV_TILE, tile)
            got = srv.respond_batch(qs)
            assert got[:3] + [got[63]] == want, (pair, tile)
    res = srv.autotune(64, 2)
    assert res["small_payloads"] == 16
    score = [c["ms"] / 64 + c["ms_small"] / 16 for c in res["candidates"]]
    assert len(score) == 6 and all(c["ms"] > 0 and c["ms_small"] > 0 for c in res["candidates"])
    chosen = res["chosen"]
    assert chosen["ms"] / 64 + chosen["ms_small"] / 16 == min(score)
    assert {c["pack_cta_pair"] for c in res["candidates"]} == {0, 1, 2}
    got = srv.respond_batch(qs)
    assert got[:3] + [got[63]] == want
    assert srv.respond_to_serialized_query(qs[1]) == want[1]
    srv.set_option(pkg.KeywordServer.OPT_PACK_CTA_PAIR, 2)  # back to the defaults for later tests
    srv.set_option(pkg.KeywordServer.OPT_GEMV_TILE, 0)
