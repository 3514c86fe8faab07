"""ctypes bindings of the CPU oracle (liboracle.so).  TEST INFRASTRUCTURE ONLY.

Imported by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
reference legs as the checker; the product package never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libinspire_ref_kernels.so")

N = 2048
NINNER = 3069
Q0, Q1 = 268369921, 249561089
Q = Q0 * Q1
RESULT_BYTES = 12288


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


if not os.path.exists(LIB):
    build()
_lib = ctypes.CDLL(LIB)

_u64 = ctypes.c_uint64
_p = ctypes.c_void_p
_sz = ctypes.c_size_t


class Params(ctypes.Structure):
    _fields_ = [("q", _u64 * 2), ("modulus", _u64), ("barrett_cr0", _u64 * 2), ("barrett_cr1", _u64 * 2),
                ("cr0_mod", _u64), ("cr1_mod", _u64), ("mod0_inv_mod1", _u64), ("mod1_inv_mod0", _u64),
                ("modulus_log2", _u64), ("root", _u64 * 2), ("ntt", ((_u64 * N) * 4) * 2)]


class CPlan(ctypes.Structure):
    _fields_ = [(n, _u64) for n in ("num_items", "entry_size", "item_size_bits", "dim0", "db_rows", "db_cols",
                                   "instances", "interp", "c", "peak_bytes")]


class OracleDB(ctypes.Structure):
    _fields_ = [("db_rows", _u64), ("db_cols", _u64), ("num_outputs", _u64), ("interp", _u64), ("c", _u64),
                ("db", _p), ("a_hat", _p), ("bold_t", _p), ("bold_t_bar", _p), ("bold_t_hat", _p),
                ("stash", _p), ("stash_count", _u64), ("stash_entry_bytes", _u64)]


def _sig(name, res, *args):
    f = getattr(_lib, name)
    f.restype = res
    f.argtypes = list(args)
    return f


_params_init = _sig("ipr_params_init", None, ctypes.POINTER(Params))
get_barrett_crs_c = _sig("ipr_get_barrett_crs", None, _u64, ctypes.POINTER(_u64), ctypes.POINTER(_u64))
barrett_raw_u64 = _sig("ipr_barrett_raw_u64", _u64, _u64, _u64, _u64)
barrett_reduction_u128_raw = _sig("ipr_barrett_reduction_u128_raw", _u64, _u64, _u64, _u64, _u64, _u64)
div2_uint_mod = _sig("ipr_div2_uint_mod", _u64, _u64, _u64)
invert_uint_mod = _sig("ipr_invert_uint_mod", _u64, _u64, _u64)
rescale = _sig("ipr_rescale", _u64, _u64, _u64, _u64)
_crt = _sig("ipr_crt_compose", _u64, ctypes.POINTER(Params), _u64, _u64)
_ntt_f = _sig("ipr_ntt_forward", None, ctypes.POINTER(Params), _p)
_ntt_i = _sig("ipr_ntt_inverse", None, ctypes.POINTER(Params), _p)
_to_ntt = _sig("ipr_to_ntt", None, ctypes.POINTER(Params), _p, _p)
_from_ntt = _sig("ipr_from_ntt", None, ctypes.POINTER(Params), _p, _p)
_gadget = _sig("ipr_gadget_invert_2", None, ctypes.POINTER(Params), _p, _p)
_gadget_g = _sig("ipr_gadget_invert_general", None, ctypes.POINTER(Params), _p, ctypes.c_uint, ctypes.c_uint, _p)
_auto_poly = _sig("ipr_automorph_poly", None, ctypes.POINTER(Params), _p, _p, _u64)
_auto_table = _sig("ipr_automorph_table", None, _u64, _p)
_auto_bf = _sig("ipr_automorph_table_bruteforce", ctypes.c_int, ctypes.POINTER(Params), _u64, _p, _u64)
gen_pow = _sig("ipr_gen_pow", _u64, ctypes.c_uint)
_read_bits = _sig("ipr_read_bits", _u64, _p, _sz, ctypes.c_uint)
_write_bits = _sig("ipr_write_bits", None, _p, _u64, _sz, ctypes.c_uint)
_chacha_rfc = _sig("ipr_chacha20_rfc8439_block", None, _p, ctypes.c_uint32, _p, _p)
_rgsw_row0 = _sig("ipr_rgsw_row0", None, ctypes.POINTER(Params), _p)
_plan = _sig("ipr_plan_from_shape", ctypes.c_int, _u64, _u64, _u64, _u64, _u64, ctypes.POINTER(CPlan))
_gemv = _sig("ipr_oracle_gemv", None, ctypes.POINTER(Params), ctypes.POINTER(OracleDB), _p, _p)
_rot = _sig("ipr_oracle_rotations", None, _p, _p, _p)
_pack = _sig("ipr_oracle_packing_sum", None, ctypes.POINTER(Params), ctypes.POINTER(OracleDB), _p, _p, _p)
_post = _sig("ipr_oracle_postprocess", None, ctypes.POINTER(Params), ctypes.POINTER(OracleDB), _p, _p, _p)
_fold = _sig("ipr_oracle_fold", None, ctypes.POINTER(Params), ctypes.POINTER(OracleDB), _p, _p, _p, _p)
_switch = _sig("ipr_oracle_switch", None, ctypes.POINTER(Params), _p, _p)
query_bytes = _sig("ipr_query_bytes", _sz, _u64, ctypes.c_uint)
_parse = _sig("ipr_oracle_parse_query", ctypes.c_int, _p, _sz, _u64, ctypes.POINTER(ctypes.c_uint), _p, _p, _p, _p,
              ctypes.c_uint)
_resp_bytes = _sig("ipr_response_bytes", _sz, ctypes.POINTER(OracleDB), ctypes.c_uint)
_respond = _sig("ipr_oracle_respond", ctypes.c_int, ctypes.POINTER(Params), ctypes.POINTER(OracleDB), _p, _sz, _p, _sz,
                ctypes.POINTER(_sz))
synth = _sig("ipr_synth", _u64, _u64, _u64, _u64)
_synth_db = _sig("ipr_synth_db", None, _u64, _u64, _u64, _p)
_synth_pre = _sig("ipr_synth_precomp", None, _u64, _u64, _p, _p, _p, _p)
_synth_shard = _sig("ipr_synth_shard", None, _u64, _u64, _u64, _u64, _p, _p, _p, _p, _p)
_raw_db = _sig("ipr_oracle_raw_db", None, _p, _p, _u64, _u64, _u64, _u64, _u64, _p)
_encode_db = _sig("ipr_oracle_encode_db", ctypes.c_int, _p, _p, _u64, _u64, _u64)
_synth_q = _sig("ipr_synth_query", ctypes.c_int, _u64, _u64, ctypes.c_uint, _p, _sz, ctypes.POINTER(_sz))
threads = _sig("ipr_oracle_threads", ctypes.c_int)
_random_raw = _sig("ipr_oracle_random_raw", None, ctypes.POINTER(Params), _p, _u64, _p)
_rescale_many = _sig("ipr_oracle_rescale_many", None, _p, _u64, _u64, _u64, _p)
_chacha_blocks = _sig("ipr_oracle_chacha_blocks", None, _p, _u64, _u64, _u64, _p)


_PARAMS = None


def params() -> Params:
    global _PARAMS
    if _PARAMS is None:
        _PARAMS = Params()
        _params_init(ctypes.byref(_PARAMS))
    return _PARAMS


def _ptr(a: np.ndarray) -> int:
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def get_barrett_crs(m: int):
    a, b = _u64(), _u64()
    get_barrett_crs_c(m, ctypes.byref(a), ctypes.byref(b))
    return a.value, b.value


def ntt_tables() -> np.ndarray:
    return np.ctypeslib.as_array(params().ntt).reshape(2, 4, N).copy()


def crt_compose(x: int, y: int) -> int:
    return _crt(ctypes.byref(params()), x, y)


def ntt_forward(limbs: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(limbs, dtype=np.uint64).copy()
    _ntt_f(ctypes.byref(params()), _ptr(a))
    return a


def ntt_inverse(limbs: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(limbs, dtype=np.uint64).copy()
    _ntt_i(ctypes.byref(params()), _ptr(a))
    return a


def to_ntt(raw: np.ndarray) -> np.ndarray:
    r = np.ascontiguousarray(raw, dtype=np.uint64)
    out = np.zeros(2 * N, dtype=np.uint64)
    _to_ntt(ctypes.byref(params()), _ptr(r), _ptr(out))
    return out


def from_ntt(ntt: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(ntt, dtype=np.uint64)
    out = np.zeros(N, dtype=np.uint64)
    _from_ntt(ctypes.byref(params()), _ptr(a), _ptr(out))
    return out


def gadget_invert_2(rows2: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(rows2, dtype=np.uint64).reshape(2 * N)
    out = np.zeros(6 * N, dtype=np.uint64)
    _gadget(ctypes.byref(params()), _ptr(a), _ptr(out))
    return out.reshape(6, N)


def gadget_invert_general(rows: np.ndarray, num_elems: int) -> np.ndarray:
    a = np.ascontiguousarray(rows, dtype=np.uint64)
    r = a.size // N
    out = np.zeros(r * num_elems * N, dtype=np.uint64)
    _gadget_g(ctypes.byref(params()), _ptr(a), r, num_elems, _ptr(out))
    return out.reshape(r * num_elems, N)


def automorph_poly(a: np.ndarray, t: int) -> np.ndarray:
    x = np.ascontiguousarray(a, dtype=np.uint64)
    out = np.zeros(N, dtype=np.uint64)
    _auto_poly(ctypes.byref(params()), _ptr(x), _ptr(out), t)
    return out


def automorph_table(t: int) -> np.ndarray:
    out = np.zeros(N, dtype=np.uint32)
    _auto_table(t, _ptr(out))
    return out


def automorph_table_bruteforce(t: int, seed: int = 1):
    out = np.zeros(N, dtype=np.uint32)
    bad = _auto_bf(ctypes.byref(params()), t, _ptr(out), seed)
    return None if bad else out


def read_bits(buf: np.ndarray, off: int, n: int) -> int:
    return _read_bits(_ptr(buf), off, n)


def write_bits(buf: np.ndarray, val: int, off: int, n: int):
    _write_bits(_ptr(buf), val, off, n)


def chacha20_rfc8439_block(key: bytes, counter: int, nonce: bytes) -> bytes:
    k = np.frombuffer(key, dtype="<u4").copy()
    n = np.frombuffer(nonce, dtype="<u4").copy()
    out = np.zeros(16, dtype=np.uint32)
    _chacha_rfc(_ptr(k), counter, _ptr(n), _ptr(out))
    return out.astype("<u4").tobytes()


def random_raw(seed: bytes, count: int) -> np.ndarray:
    """PolyMatrixRaw::random_rng (poly.rs:211-231): `count` ChaCha20Rng u64 draws mod q"""
    sd = np.frombuffer(bytes(seed), dtype=np.uint8).copy()
    assert sd.size == 32
    out = np.zeros(count, dtype=np.uint64)
    _random_raw(ctypes.byref(params()), _ptr(sd), count, _ptr(out))
    return out


def chacha_blocks(seed: bytes, stream: int, first: int, count: int) -> np.ndarray:
    """ChaCha20 blocks [count][16] u32 of (seed, stream) from block counter `first`"""
    sd = np.frombuffer(bytes(seed), dtype=np.uint8).copy()
    assert sd.size == 32
    out = np.zeros(count * 16, dtype=np.uint32)
    _chacha_blocks(_ptr(sd), stream, first, count, _ptr(out))
    return out.reshape(count, 16)


def rescale_many(vals: np.ndarray, inp_mod: int, out_mod: int) -> np.ndarray:
    """rescale (arith.rs:436-452) of every element"""
    v = np.ascontiguousarray(vals, dtype=np.uint64)
    out = np.zeros(v.size, dtype=np.uint64)
    _rescale_many(_ptr(v), v.size, inp_mod, out_mod, _ptr(out))
    return out.reshape(v.shape)


def rgsw_row0() -> np.ndarray:
    out = np.zeros(2 * N, dtype=np.uint64)
    _rgsw_row0(ctypes.byref(params()), _ptr(out))
    return out


def plan_from_shape(records, key_size, value_size, buckets=0, dim0=0):
    p = CPlan()
    st = _plan(records, key_size, value_size, buckets or 0, dim0 or 0, ctypes.byref(p))
    if st:
        return None
    return {f: getattr(p, f) for f, _ in CPlan._fields_}


class SynthDB:
    """Seeded synthetic server state (same generator as the device's
    ipr_server_create_synthetic) held in host memory for the oracle."""

    def __init__(self, db_rows, instances, interp, c, seed, stash=()):
        self.db_rows, self.instances, self.interp, self.c, self.seed = db_rows, instances, interp, c, seed
        self.db_cols = instances * N
        self.db = np.zeros(self.db_cols * db_rows, dtype=np.uint16)
        _synth_db(seed, db_rows, self.db_cols, _ptr(self.db))
        self.a_hat = np.zeros(instances * N, dtype=np.uint64)
        self.bold_t = np.zeros(instances * NINNER * N, dtype=np.uint64)
        self.bold_t_bar = np.zeros(instances * NINNER * N, dtype=np.uint64)
        self.bold_t_hat = np.zeros(instances * 3 * N, dtype=np.uint64)
        _synth_pre(seed, instances, _ptr(self.a_hat), _ptr(self.bold_t), _ptr(self.bold_t_bar),
                   _ptr(self.bold_t_hat))
        self.stash = [bytes(s) for s in stash]
        self._stash_buf = np.frombuffer(b"".join(self.stash) or b"\0", dtype=np.uint8).copy()

    @classmethod
    def shard_of(cls, db_rows, first_instance, instances, interp, c, seed, stash=()):
        """the state of instances [first_instance, first_instance + instances) of a synthetic
        server with `seed`, generated alone (same element indices as the whole server)"""
        sub = cls.__new__(cls)
        sub.db_rows, sub.instances, sub.interp, sub.c, sub.seed = db_rows, instances, interp, c, seed
        sub.db_cols = instances * N
        sub.db = np.zeros(sub.db_cols * db_rows, dtype=np.uint16)
        sub.a_hat = np.zeros(instances * N, dtype=np.uint64)
        sub.bold_t = np.zeros(instances * NINNER * N, dtype=np.uint64)
        sub.bold_t_bar = np.zeros(instances * NINNER * N, dtype=np.uint64)
        sub.bold_t_hat = np.zeros(instances * 3 * N, dtype=np.uint64)
        _synth_shard(seed, db_rows, first_instance, instances, _ptr(sub.db), _ptr(sub.a_hat), _ptr(sub.bold_t),
                     _ptr(sub.bold_t_bar), _ptr(sub.bold_t_hat))
        sub.stash = [bytes(s) for s in stash]
        sub._stash_buf = np.frombuffer(b"".join(sub.stash) or b"\0", dtype=np.uint8).copy()
        return sub

    def shard(self, first_instance: int, instances: int, interp: int, c: int) -> "SynthDB":
        """the state of fold groups starting at `first_instance` (views into this state)"""
        sub = SynthDB.__new__(SynthDB)
        sub.db_rows, sub.instances, sub.interp, sub.c, sub.seed = self.db_rows, instances, interp, c, self.seed
        sub.db_cols = instances * N
        f, n = first_instance, instances
        sub.db = self.db[f * N * self.db_rows:(f + n) * N * self.db_rows]
        sub.a_hat = self.a_hat[f * N:(f + n) * N]
        sub.bold_t = self.bold_t[f * NINNER * N:(f + n) * NINNER * N]
        sub.bold_t_bar = self.bold_t_bar[f * NINNER * N:(f + n) * NINNER * N]
        sub.bold_t_hat = self.bold_t_hat[f * 3 * N:(f + n) * 3 * N]
        sub.stash, sub._stash_buf = self.stash, self._stash_buf
        return sub

    def c_struct(self) -> OracleDB:
        d = OracleDB()
        d.db_rows, d.db_cols, d.num_outputs, d.interp, d.c = (self.db_rows, self.db_cols, self.instances,
                                                              self.interp, self.c)
        d.db, d.a_hat = _ptr(self.db), _ptr(self.a_hat)
        d.bold_t, d.bold_t_bar, d.bold_t_hat = _ptr(self.bold_t), _ptr(self.bold_t_bar), _ptr(self.bold_t_hat)
        d.stash = _ptr(self._stash_buf)
        d.stash_count = len(self.stash)
        d.stash_entry_bytes = len(self.stash[0]) if self.stash else 0
        return d


def synth_query(seed: int, db_rows: int, nq: int = 2) -> bytes:
    cap = query_bytes(db_rows, nq)
    buf = np.zeros(cap, dtype=np.uint8)
    n = _sz()
    assert _synth_q(seed, db_rows, nq, _ptr(buf), cap, ctypes.byref(n)) == 0
    return buf[:n.value].tobytes()


def respond(sdb: SynthDB, query: bytes) -> bytes:
    d = sdb.c_struct()
    q = np.frombuffer(query, dtype=np.uint8).copy()
    nq = query[0]
    cap = _resp_bytes(ctypes.byref(d), nq)
    out = np.zeros(cap, dtype=np.uint8)
    n = _sz()
    st = _respond(ctypes.byref(params()), ctypes.byref(d), _ptr(q), len(query), _ptr(out), cap, ctypes.byref(n))
    if st:
        raise ValueError(f"oracle respond status {st}")
    return out[:n.value].tobytes()


def parse_query(query: bytes, db_rows: int):
    q = np.frombuffer(query, dtype=np.uint8).copy()
    nq = query[0]
    y = np.zeros(3 * N, dtype=np.uint64)
    z = np.zeros(3 * N, dtype=np.uint64)
    rows = np.zeros(max(nq, 1) * db_rows, dtype=np.uint64)
    gsw = np.zeros(max(nq, 1) * 12 * N, dtype=np.uint64)
    got = ctypes.c_uint()
    st = _parse(_ptr(q), len(query), db_rows, ctypes.byref(got), _ptr(y), _ptr(z), _ptr(rows), _ptr(gsw), 255)
    if st:
        raise ValueError(f"parse status {st}")
    return y, z, rows.reshape(max(nq, 1), db_rows), gsw.reshape(max(nq, 1), 6, 2, N)


def gemv(sdb: SynthDB, a: np.ndarray) -> np.ndarray:
    d = sdb.c_struct()
    av = np.ascontiguousarray(a, dtype=np.uint64)
    c = np.zeros(sdb.db_cols, dtype=np.uint64)
    _gemv(ctypes.byref(params()), ctypes.byref(d), _ptr(av), _ptr(c))
    return c


def gemv_db(db: np.ndarray, db_rows: int, a: np.ndarray) -> np.ndarray:
    """the first-dimension GEMV (ipr_oracle_gemv) over a bare column-major u16 DB
    [db_cols][db_rows] and one condensed query row, without a server state around it"""
    dbv = np.ascontiguousarray(db, dtype=np.uint16)
    assert dbv.size % db_rows == 0
    d = OracleDB()
    d.db_rows, d.db_cols, d.num_outputs, d.interp, d.c = db_rows, dbv.size // db_rows, 0, 1, 0
    d.db = _ptr(dbv)
    av = np.ascontiguousarray(a, dtype=np.uint64)
    assert av.size == db_rows
    c = np.zeros(d.db_cols, dtype=np.uint64)
    _gemv(ctypes.byref(params()), ctypes.byref(d), _ptr(av), _ptr(c))
    return c


def rotations(y_body: np.ndarray):
    y = np.ascontiguousarray(y_body, dtype=np.uint64)
    ya = np.zeros(NINNER * N, dtype=np.uint64)
    yb = np.zeros(NINNER * N, dtype=np.uint64)
    _rot(_ptr(y), _ptr(ya), _ptr(yb))
    return ya, yb


def packing_sum(sdb: SynthDB, y_body, z_body) -> np.ndarray:
    d = sdb.c_struct()
    y = np.ascontiguousarray(y_body, dtype=np.uint64)
    z = np.ascontiguousarray(z_body, dtype=np.uint64)
    S = np.zeros(sdb.instances * 2 * N, dtype=np.uint64)
    _pack(ctypes.byref(params()), ctypes.byref(d), _ptr(y), _ptr(z), _ptr(S))
    return S.reshape(sdb.instances, 2, N)


def postprocess(sdb: SynthDB, S, b_values) -> np.ndarray:
    d = sdb.c_struct()
    s = np.ascontiguousarray(S, dtype=np.uint64)
    b = np.ascontiguousarray(b_values, dtype=np.uint64)
    out = np.zeros(sdb.instances * 2 * N, dtype=np.uint64)
    _post(ctypes.byref(params()), ctypes.byref(d), _ptr(s), _ptr(b), _ptr(out))
    return out.reshape(sdb.instances, 2, N)


def fold(sdb: SynthDB, gsw_body, packed) -> np.ndarray:
    d = sdb.c_struct()
    row0 = rgsw_row0()
    g = np.ascontiguousarray(gsw_body, dtype=np.uint64)
    p = np.ascontiguousarray(packed, dtype=np.uint64)
    out = np.zeros(sdb.c * 2 * N, dtype=np.uint64)
    _fold(ctypes.byref(params()), ctypes.byref(d), _ptr(row0), _ptr(g), _ptr(p), _ptr(out))
    return out.reshape(sdb.c, 2, N)


def switch(result) -> bytes:
    r = np.ascontiguousarray(result, dtype=np.uint64)
    out = np.zeros(RESULT_BYTES, dtype=np.uint8)
    _switch(ctypes.byref(params()), _ptr(r), _ptr(out))
    return out.tobytes()


def raw_db(entries: np.ndarray, occupied: np.ndarray, entry_size: int, db_rows: int, db_cols: int,
           per: int) -> np.ndarray:
    """KeywordCuckooTable::to_raw_db: column-major u16 [db_cols][db_rows]"""
    e = np.ascontiguousarray(entries, dtype=np.uint8)
    o = np.ascontiguousarray(occupied, dtype=np.uint8)
    out = np.zeros(db_rows * db_cols, dtype=np.uint16)
    _raw_db(_ptr(e), _ptr(o), o.size, entry_size, db_rows, db_cols, per, _ptr(out))
    return out


def encode_db(raw: np.ndarray, db_rows: int, db_cols: int, interp: int) -> np.ndarray:
    """gpu_encode_db: the interpolation encode of a column-major raw DB"""
    r = np.ascontiguousarray(raw, dtype=np.uint16)
    out = np.zeros(db_rows * db_cols, dtype=np.uint16)
    st = _encode_db(_ptr(r), _ptr(out), db_rows, db_cols, interp)
    if st:
        raise ValueError(f"oracle encode status {st}")
    return out


# --- offline precomputation (ipr_offline.c) ---------------------------------
_hint_query = _sig("ipr_oracle_hint_query", None, ctypes.POINTER(Params), ctypes.c_uint, _p)
_prep_pack = _sig("ipr_oracle_prep_pack", None, ctypes.POINTER(Params), _p, _u64, _u64, _p, _p)
_offline_keys = _sig("ipr_oracle_offline_keys", None, ctypes.POINTER(Params), _p, _p, _p, _p)
_pack_r = _sig("ipr_oracle_pack_r", None, ctypes.POINTER(Params), _p, _p, _p)
_collapse = _sig("ipr_oracle_collapse", None, ctypes.POINTER(Params), _p, _p, _p, _p, _p, _p, _p, _p, _p)


def hint_query(polys: int) -> np.ndarray:
    """generate_pseudorandom_query(SEED_0): [polys][2][N] NTT"""
    out = np.zeros(polys * 2 * N, dtype=np.uint64)
    _hint_query(ctypes.byref(params()), polys, _ptr(out))
    return out.reshape(polys, 2, N)


def prep_pack(db: np.ndarray, db_rows: int, inst: int, query: np.ndarray) -> np.ndarray:
    """a_ct_tilde of instance `inst`: [2048][2][N] NTT"""
    d = np.ascontiguousarray(db, dtype=np.uint16)
    q = np.ascontiguousarray(query, dtype=np.uint64)
    out = np.zeros(N * 2 * N, dtype=np.uint64)
    _prep_pack(ctypes.byref(params()), _ptr(d), db_rows, inst, _ptr(q), _ptr(out))
    return out.reshape(N, 2, N)


def offline_keys():
    """OfflinePackingKeys::init_full(W_SEED, V_SEED): w_mask, v_mask [3][2][N];
    w_all, w_bar_all [1023][3][2][N]"""
    wm = np.zeros(3 * 2 * N, dtype=np.uint64)
    vm = np.zeros(3 * 2 * N, dtype=np.uint64)
    wa = np.zeros(1023 * 3 * 2 * N, dtype=np.uint64)
    wb = np.zeros(1023 * 3 * 2 * N, dtype=np.uint64)
    _offline_keys(ctypes.byref(params()), _ptr(wm), _ptr(vm), _ptr(wa), _ptr(wb))
    return wm.reshape(3, 2, N), vm.reshape(3, 2, N), wa.reshape(1023, 3, 2, N), wb.reshape(1023, 3, 2, N)


def pack_r(a_ct: np.ndarray):
    """brute-force packing sums of one instance: r_all, r_bar_all [1024][2][N]"""
    a = np.ascontiguousarray(a_ct, dtype=np.uint64)
    r = np.zeros(1024 * 2 * N, dtype=np.uint64)
    rb = np.zeros(1024 * 2 * N, dtype=np.uint64)
    _pack_r(ctypes.byref(params()), _ptr(a), _ptr(r), _ptr(rb))
    return r.reshape(1024, 2, N), rb.reshape(1024, 2, N)


def collapse(r_all: np.ndarray, r_bar_all: np.ndarray, w_all, w_bar_all, v_mask):
    """1023-step collapse of one instance: a_hat [N], bold_t / bold_t_bar [3069][N] condensed,
    bold_t_hat [3][N] condensed (r_all, r_bar_all are copied, not modified)"""
    r = np.ascontiguousarray(r_all, dtype=np.uint64).copy()
    rb = np.ascontiguousarray(r_bar_all, dtype=np.uint64).copy()
    wa, wb, vm = (np.ascontiguousarray(x, dtype=np.uint64) for x in (w_all, w_bar_all, v_mask))
    a_hat = np.zeros(N, dtype=np.uint64)
    bt = np.zeros(NINNER * N, dtype=np.uint64)
    btb = np.zeros(NINNER * N, dtype=np.uint64)
    bth = np.zeros(3 * N, dtype=np.uint64)
    _collapse(ctypes.byref(params()), _ptr(r), _ptr(rb), _ptr(wa), _ptr(wb), _ptr(vm), _ptr(a_hat), _ptr(bt),
              _ptr(btb), _ptr(bth))
    return a_hat, bt.reshape(NINNER, N), btb.reshape(NINNER, N), bth.reshape(3, N)


def offline_precompute(db: np.ndarray, db_rows: int, instances: int):
    """the whole offline precomputation for `instances` packing outputs:
    a_hat [inst][N], bold_t / bold_t_bar [inst][3069][N], bold_t_hat [inst][3][N]"""
    q = hint_query(db_rows // N)
    _, vm, wa, wb = offline_keys()
    a_hat = np.zeros((instances, N), dtype=np.uint64)
    bt = np.zeros((instances, NINNER, N), dtype=np.uint64)
    btb = np.zeros((instances, NINNER, N), dtype=np.uint64)
    bth = np.zeros((instances, 3, N), dtype=np.uint64)
    for i in range(instances):
        r, rb = pack_r(prep_pack(db, db_rows, i, q))
        a_hat[i], bt[i], btb[i], bth[i] = collapse(r, rb, wa, wb, vm)
    return a_hat, bt, btb, bth


_prep_pack_lwes = _sig("ipr_oracle_prep_pack_lwes", None, ctypes.POINTER(Params), _p, _p)


def prep_pack_lwes(lwe: np.ndarray) -> np.ndarray:
    """prep_pack_lwes: lwe [N+1][N] (rows = a-vector coefficients, last row = b) -> a_ct [N][2][N]"""
    l = np.ascontiguousarray(lwe, dtype=np.uint64)
    assert l.size == (N + 1) * N
    out = np.zeros(N * 2 * N, dtype=np.uint64)
    _prep_pack_lwes(ctypes.byref(params()), _ptr(l), _ptr(out))
    return out.reshape(N, 2, N)


def inspiring_pack(lwe: np.ndarray, y_body: np.ndarray, z_body: np.ndarray) -> np.ndarray:
    """packing_fully_online (packing.rs:3122-3162) for 2048 LWEs: the offline precomputation of
    full_packing_with_preprocessing_offline (r / r_bar sums, 1023-step collapse) on their
    a-vectors, then full_packing_with_preprocessing_online (packing.rs:2941-3021) with the
    packing keys (y_body, z_body condensed [3][N]) and the b row -> RLWE [2][N] raw
    (row 1 = b + sum, not reduced)"""
    lwe = np.ascontiguousarray(lwe, dtype=np.uint64).reshape(N + 1, N)
    r, rb = pack_r(prep_pack_lwes(lwe))
    _, vm, wa, wb = offline_keys()
    a_hat, bt, btb, bth = collapse(r, rb, wa, wb, vm)
    sdb = SynthDB.__new__(SynthDB)
    sdb.db_rows, sdb.instances, sdb.interp, sdb.c, sdb.seed, sdb.db_cols = N, 1, 1, 1, 0, N
    sdb.db = np.zeros(N * N, dtype=np.uint16)
    sdb.a_hat, sdb.bold_t, sdb.bold_t_bar, sdb.bold_t_hat = (np.ascontiguousarray(x).reshape(-1)
                                                               for x in (a_hat, bt, btb, bth))
    sdb.stash, sdb._stash_buf = [], np.zeros(1, dtype=np.uint8)
    S = packing_sum(sdb, y_body, z_body)
    return postprocess(sdb, S, lwe[N])[0]


# --- dataset generation (ipr_dataset.c): FIPS 202 / FIPS 203 / rand seeds ------------------
_sha3_256 = _sig("ipr_sha3_256", None, _p, _sz, _p)
_sha3_512 = _sig("ipr_sha3_512", None, _p, _sz, _p)
_shake128 = _sig("ipr_shake128", None, _p, _sz, _p, _sz)
_shake256 = _sig("ipr_shake256", None, _p, _sz, _p, _sz)
_mlkem_ek = _sig("ipr_mlkem_ek", None, ctypes.c_int, _p, _p)
_seed_u64 = _sig("ipr_seed_from_u64", None, _u64, _p)
_record = _sig("ipr_dataset_record", None, ctypes.c_int, _u64, _u64, _p)

KEM_K = {"ml-kem-512": 2, "ml-kem-768": 3, "ml-kem-1024": 4}


def _bufp(b: bytes):
    a = np.frombuffer(bytes(b) or b"\0", dtype=np.uint8).copy()
    return a, _ptr(a)


def sha3_256(m: bytes) -> bytes:
    a, p = _bufp(m)
    out = np.zeros(32, dtype=np.uint8)
    _sha3_256(p, len(m), _ptr(out))
    return out.tobytes()


def sha3_512(m: bytes) -> bytes:
    a, p = _bufp(m)
    out = np.zeros(64, dtype=np.uint8)
    _sha3_512(p, len(m), _ptr(out))
    return out.tobytes()


def shake128(m: bytes, n: int) -> bytes:
    a, p = _bufp(m)
    out = np.zeros(max(n, 1), dtype=np.uint8)
    _shake128(p, len(m), _ptr(out), n)
    return out[:n].tobytes()


def shake256(m: bytes, n: int) -> bytes:
    a, p = _bufp(m)
    out = np.zeros(max(n, 1), dtype=np.uint8)
    _shake256(p, len(m), _ptr(out), n)
    return out[:n].tobytes()


def mlkem_ek(kem: str, d: bytes) -> bytes:
    """FIPS 203 K-PKE.KeyGen(d) encapsulation key (ML-KEM.KeyGen_internal's ek)"""
    k = KEM_K[kem]
    a, p = _bufp(d[:32])
    out = np.zeros(384 * k + 32, dtype=np.uint8)
    _mlkem_ek(k, p, _ptr(out))
    return out.tobytes()


def seed_from_u64(seed: int) -> bytes:
    out = np.zeros(32, dtype=np.uint8)
    _seed_u64(seed, _ptr(out))
    return out.tobytes()


def dataset_record(kem: str, seed: int, idx: int):
    """(id, public key) of record idx of DatasetGenerator(kem).with_seed(seed)"""
    k = KEM_K[kem]
    out = np.zeros(32 + 384 * k + 32, dtype=np.uint8)
    _record(k, seed, idx, _ptr(out))
    return out[:32].tobytes(), out[32:].tobytes()
