"""The reference's offline-precomputation FFI on this library (compat_offline.cu), called
side by side with the reference's own kernels (hint_kernel.cu, prep_pack_kernel.cu,
packing_kernel.cu, collapse_kernel.cu, built from their sources into oracle/_ref):
same symbol, same arguments, same outputs, bit for bit.

CPU: every symbol the reference's Rust crate declares for these steps
(src/pir/gpu/hint.rs, prep_pack.rs, packing.rs, collapse.rs) is exported.
"""
import ctypes
import os

import numpy as np
import pytest

N = 2048
CC = 2 * N
HALF = N // 2
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_OFFLINE = os.path.join(ROOT, "oracle", "_ref", "libinspire_ref_offline.so")
u64, i32, u32, vp = ctypes.c_uint64, ctypes.c_int, ctypes.c_uint32, ctypes.c_void_p

# (name, restype, argtypes) of the functions this file calls, as both libraries define them
SIGS = {
    "gpu_hint_upload_tables": (None, [vp, i32]),
    "gpu_hint_upload_query_ffi": (None, [vp, i32, i32]),
    "gpu_hint_compute_from_host": (None, [vp, vp, i32, i32, i32, u32, u32, u64, u64, u64, u64, u64, u64, u64]),
    "gpu_hint_get_device_output": (vp, []),
    "gpu_hint_get_ntt_tables": (vp, []),
    "gpu_hint_free": (None, []),
    "gpu_prep_pack_compute": (None, [vp, vp, i32, u32, u32, u64]),
    "gpu_prep_pack_get_output": (vp, []),
    "gpu_prep_pack_free": (None, []),
    "gpu_packing_setup": (None, [vp, vp, vp, vp, i32, i32, i32, i32, u64, u64, u64, u64]),
    "gpu_packing_precomp_fast": (None, [vp, vp, vp]),
    "gpu_packing_precomp_fast_device_no_d2h": (None, [vp]),
    "gpu_packing_get_s_r_out": (vp, []),
    "gpu_packing_get_s_r_bar_out": (vp, []),
    "gpu_packing_teardown": (None, []),
    "gpu_collapse_alloc_r": (None, [i32, i32, i32]),
    "gpu_collapse_automorph_column": (None, [vp, vp, i32, i32, i32, i32, i32, vp, vp, i32]),
    "gpu_collapse_setup": (None, [vp, vp, vp, vp, i32, i32, i32, i32]),
    "gpu_collapse_run": (None, [i32, i32, i32, i32, u32, u32, u64, u64, u64, u64, u64, u64, u64]),
    "gpu_collapse_download_a_hat": (None, [vp, i32]),
    "gpu_collapse_get_bold_t": (vp, []),
    "gpu_collapse_get_bold_t_bar": (vp, []),
    "gpu_collapse_get_bold_t_hat": (vp, []),
    "gpu_collapse_get_r_all": (vp, []),
    "gpu_collapse_free_all": (None, []),
}


def _bind(lib):
    for name, (res, args) in SIGS.items():
        f = getattr(lib, name)
        f.restype, f.argtypes = res, args
    return lib


def test_every_reference_offline_symbol_is_exported(pkg):
    """every offline FFI function the crate declares (src/pir/gpu/{hint,prep_pack,packing,
    collapse}.rs extern "C" blocks, listed in SIGS) is exported"""
    missing = [n for n in sorted(SIGS) if not hasattr(pkg.lib, n)]
    assert not missing, missing


def _libs(pkg):
    if not os.path.exists(REF_OFFLINE):
        pytest.skip("reference offline kernels not built (make -C oracle ref)")
    return _bind(pkg.lib), _bind(ctypes.CDLL(REF_OFFLINE))


def _d2h(ptr, n):
    from cuda.bindings import runtime as rt
    out = np.zeros(n, dtype=np.uint64)
    err, = rt.cudaMemcpy(out.ctypes.data, ptr, out.nbytes, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
    assert err == rt.cudaError_t.cudaSuccess
    return out


def _h2d(ptr, arr):
    from cuda.bindings import runtime as rt
    err, = rt.cudaMemcpy(ptr, arr.ctypes.data, arr.nbytes, rt.cudaMemcpyKind.cudaMemcpyHostToDevice)
    assert err == rt.cudaError_t.cudaSuccess


def _dev(arr):
    from cuda.bindings import runtime as rt
    err, p = rt.cudaMalloc(arr.nbytes)
    assert err == rt.cudaError_t.cudaSuccess
    _h2d(p, arr)
    return p


def _free(p):
    from cuda.bindings import runtime as rt
    rt.cudaFree(p)


@pytest.mark.gpu
@pytest.mark.parametrize("db_rows,cols", [(N, 2 * N), (2 * N, N)])
def test_hint_and_prep_pack_match_reference(pkg, orc, db_rows, cols):
    ours, ref = _libs(pkg)
    P = orc.params()
    tables = np.ctypeslib.as_array(P.ntt).reshape(-1).astype(np.uint64).copy()
    polys = db_rows // N
    query = np.ascontiguousarray(orc.hint_query(polys), dtype=np.uint64)
    db = np.random.default_rng(db_rows + cols).integers(0, 65535, cols * db_rows, dtype=np.uint16)
    got = []
    for lib in (ours, ref):
        lib.gpu_hint_upload_tables(tables.ctypes.data, N)
        lib.gpu_hint_upload_query_ffi(query.ctypes.data, polys, N)
        hint = np.zeros(cols * N, dtype=np.uint64)
        lib.gpu_hint_compute_from_host(db.ctypes.data, hint.ctypes.data, db_rows, polys, cols, P.q[0], P.q[1],
                                       P.barrett_cr1[0], P.barrett_cr1[1], P.mod0_inv_mod1, P.mod1_inv_mod0,
                                       P.modulus, P.cr0_mod, P.cr1_mod)
        lib.gpu_prep_pack_compute(lib.gpu_hint_get_device_output(), lib.gpu_hint_get_ntt_tables(), cols, P.q[0],
                                  P.q[1], P.modulus)
        got.append((hint, _d2h(lib.gpu_prep_pack_get_output(), cols * CC)))
        lib.gpu_prep_pack_free()
        lib.gpu_hint_free()
    assert np.array_equal(got[0][0], got[1][0]), "hint"
    assert np.array_equal(got[0][1], got[1][1]), "prep_pack"
    # the prepacked polynomials of the first instance equal the oracle's a_ct_tilde
    assert np.array_equal(got[0][1][:N * CC].reshape(N, 2, N), orc.prep_pack(db, db_rows, 0, query))


def _packing_tables(orc):
    mono = np.zeros((2 * N, CC), dtype=np.uint64)
    for e in range(N):
        raw = np.zeros(N, dtype=np.uint64)
        raw[e] = 1
        mono[e] = orc.to_ntt(raw)
        qv = np.concatenate([np.full(N, orc.Q0), np.full(N, orc.Q1)]).astype(np.uint64)
        mono[N + e] = np.where(mono[e] == 0, 0, qv - mono[e])
    idx = np.zeros((HALF, N), dtype=np.int32)
    idxb = np.zeros((HALF, N), dtype=np.int32)
    j = np.arange(N, dtype=np.int64)
    for i in range(HALF):
        gp = int(orc.gen_pow((N - i) % N))
        ind = (j * gp) % (2 * N)
        indb = (2 * N - ind) % (2 * N)
        idx[i] = np.where(ind < N, ind, N + ind % N)
        idxb[i] = np.where(indb < N, indb, N + indb % N)
    inv_raw = np.zeros(N, dtype=np.uint64)
    inv_raw[0] = pow(N, -1, orc.Q)
    return mono, idx, idxb, orc.to_ntt(inv_raw)


@pytest.mark.gpu
@pytest.mark.parametrize("canonical", [True, False])
def test_packing_precomp_matches_reference(pkg, orc, canonical):
    """canonical tables take the NTT-over-j path, altered ones (mod_inv doubled) the direct sums"""
    ours, ref = _libs(pkg)
    P = orc.params()
    mono, idx, idxb, mod_inv = _packing_tables(orc)
    if not canonical:
        mod_inv = np.concatenate([(mod_inv[:N] * 2) % orc.Q0, (mod_inv[N:] * 2) % orc.Q1]).astype(np.uint64)
    a_ct = np.random.default_rng(9).integers(0, orc.Q0, (N, CC), dtype=np.uint64)
    a_ct[:, N:] %= orc.Q1
    outs = []
    for lib in (ours, ref):
        lib.gpu_packing_setup(mono.ctypes.data, idx.ctypes.data, idxb.ctypes.data, mod_inv.ctypes.data, HALF, N, N,
                              2, P.q[0], P.q[1], P.barrett_cr1[0], P.barrett_cr1[1])
        r = np.zeros(HALF * CC, dtype=np.uint64)
        rb = np.zeros(HALF * CC, dtype=np.uint64)
        lib.gpu_packing_precomp_fast(a_ct.ctypes.data, r.ctypes.data, rb.ctypes.data)
        lib.gpu_packing_teardown()
        outs.append((r, rb))
    assert np.array_equal(outs[0][0], outs[1][0]), "r"
    assert np.array_equal(outs[0][1], outs[1][1]), "r_bar"


@pytest.mark.gpu
def test_collapse_matches_reference(pkg, orc):
    """gpu_packing_setup -> precomp_fast_device_no_d2h -> collapse automorphism -> setup -> run,
    the sequence of engine.rs:849-922, on one column group"""
    ours, ref = _libs(pkg)
    P = orc.params()
    tables = np.ctypeslib.as_array(P.ntt).reshape(-1).astype(np.uint64).copy()
    mono, idx, idxb, mod_inv = _packing_tables(orc)
    a_ct = np.ascontiguousarray(orc.prep_pack(np.random.default_rng(4).integers(0, 65535, N * N, dtype=np.uint16),
                                              N, 0, orc.hint_query(1)).reshape(N, CC))
    _, vm, wa, wb = orc.offline_keys()
    wa, wb, vm = (np.ascontiguousarray(x, dtype=np.uint64).reshape(-1) for x in (wa, wb, vm))
    auto = np.stack([orc.automorph_table(2 * t + 1) for t in range(N)]).astype(np.uint32)
    gen = np.array([orc.gen_pow(i) for i in range(HALF)], dtype=np.uint32)
    d_auto, d_gen, d_act = _dev(auto), _dev(gen), _dev(a_ct)
    outs = []
    try:
        for lib in (ours, ref):
            lib.gpu_packing_setup(mono.ctypes.data, idx.ctypes.data, idxb.ctypes.data, mod_inv.ctypes.data, HALF, N,
                                  N, 2, P.q[0], P.q[1], P.barrett_cr1[0], P.barrett_cr1[1])
            lib.gpu_collapse_alloc_r(1, HALF, CC)
            lib.gpu_packing_precomp_fast_device_no_d2h(d_act)
            lib.gpu_collapse_automorph_column(lib.gpu_packing_get_s_r_out(), lib.gpu_packing_get_s_r_bar_out(), 0,
                                              HALF, CC, N, 2, d_auto, d_gen, N)
            r_all = _d2h(lib.gpu_collapse_get_r_all(), HALF * CC)
            lib.gpu_collapse_setup(wa.ctypes.data, wb.ctypes.data, vm.ctypes.data, tables.ctypes.data, 1, HALF, 3, CC)
            lib.gpu_collapse_run(1, HALF, 3, 19, P.q[0], P.q[1], P.barrett_cr1[0], P.barrett_cr1[1], P.mod0_inv_mod1,
                                 P.mod1_inv_mod0, P.modulus, P.cr0_mod, P.cr1_mod)
            a_hat = np.zeros(N, dtype=np.uint64)
            lib.gpu_collapse_download_a_hat(a_hat.ctypes.data, 1)
            outs.append((r_all, a_hat, _d2h(lib.gpu_collapse_get_bold_t(), 3069 * N),
                         _d2h(lib.gpu_collapse_get_bold_t_bar(), 3069 * N), _d2h(lib.gpu_collapse_get_bold_t_hat(), 3 * N)))
            lib.gpu_collapse_free_all()
            lib.gpu_packing_teardown()
    finally:
        for p in (d_auto, d_gen, d_act):
            _free(p)
    for name, a, b in zip(("r_all", "a_hat", "bold_t", "bold_t_bar", "bold_t_hat"), outs[0], outs[1]):
        assert np.array_equal(a, b), name
    # the same column through the library's own offline path
    r, rb = orc.pack_r(a_ct.reshape(N, 2, N))
    assert np.array_equal(outs[0][0].reshape(HALF, 2, N), r)
