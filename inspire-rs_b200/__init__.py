"""inspire-rs_b200 — B200-native respond() path of the InsPIRe keyword-PIR server.

Python mirror of the reference's server interface (rkdud007/inspire-rs,
src/pir/server/keyword.rs): ``KeywordServer`` with ``public_params()``,
``respond(payload)`` and ``respond_to_serialized_query(bytes)``, plus the shape
plan of ``KeywordServerSetupPlan::from_shape`` (keyword.rs:145-233).  All work
runs in ``libipr_b200.so`` (sm_100a CUDA behind the C ABI in
``include/ipr_b200.h``); there is no CPU fallback.  Importing the package on a
machine without the built library raises ``ImportError``.
"""
from __future__ import annotations

import ctypes
import json
import os
from dataclasses import dataclass
from typing import List, Optional, Sequence

__all__ = [
    "IprError", "Plan", "KeywordServer", "plan_from_shape", "query_bytes", "lib",
    "KeywordQueryPayload", "KeywordResponsePayload", "serialize_keyword_query",
    "deserialize_keyword_response", "POLY_LEN", "RESULT_BYTES", "KeywordService", "ServiceStats",
    "shard_plan", "merge_responses", "ShardedKeywordServer", "ntt_batch", "automorph_batch", "encode_db",
    "cuckoo_to_raw_db", "state_file_plan", "offline_precompute", "InspiringPacker",
    "DatasetGenerator", "Dataset", "DatasetRecord", "derive_public_key_id", "public_key_matches_id",
    "build_cuckoo_table", "setup_keyword_server", "BOUNDS_CHECK", "bounds_checked_build", "bounds_report",
    "debug_check_extent", "debug_cut_fold_extent",
]

POLY_LEN = 2048
RESULT_BYTES = 12288
STAGES = ("parse", "gemv", "pack", "post", "fold")

_HERE = os.path.dirname(os.path.abspath(__file__))
# IPR_B200_BOUNDS_CHECK=1 selects the bounds-checked debug build (`make -C inspire-rs_b200 debug`)
BOUNDS_CHECK = os.environ.get("IPR_B200_BOUNDS_CHECK", "0") == "1"
_LIB_NAME = "libipr_b200_dbg.so" if BOUNDS_CHECK else "libipr_b200.so"
_LIB_PATH = os.path.join(_HERE, _LIB_NAME)

if not os.path.exists(_LIB_PATH):
    raise ImportError(
        f"{_LIB_NAME} not built at {_LIB_PATH}; run `make -C inspire-rs_b200`"
        + (" debug" if BOUNDS_CHECK else "") + " (the respond() path has no CPU fallback)")
lib = ctypes.CDLL(_LIB_PATH)

_u64, _i32, _sz = ctypes.c_uint64, ctypes.c_int, ctypes.c_size_t
_u8p = ctypes.POINTER(ctypes.c_uint8)
_vp = ctypes.c_void_p


class _Plan(ctypes.Structure):
    _fields_ = [(n, _u64) for n in (
        "num_items", "entry_size", "item_size_bits", "dim0", "db_rows", "db_cols",
        "instances", "interp", "c", "peak_bytes")]


class _ServerData(ctypes.Structure):
    _fields_ = [("db", _vp), ("a_hat", _vp), ("bold_t", _vp), ("bold_t_bar", _vp),
                ("bold_t_hat", _vp), ("stash", _vp), ("stash_count", _u64),
                ("stash_entry_bytes", _u64), ("key_size", _u64), ("value_size", _u64),
                ("num_records", _u64), ("cuckoo_seed", ctypes.c_uint8 * 16)]


def _sig(name, restype, *argtypes):
    f = getattr(lib, name)
    f.restype = restype
    f.argtypes = list(argtypes)
    return f


_plan_from_shape = _sig("ipr_plan_from_shape", _i32, _u64, _u64, _u64, _u64, _u64, ctypes.POINTER(_Plan))
_query_bytes = _sig("ipr_query_bytes", _u64, _u64, ctypes.c_uint)
_create = _sig("ipr_server_create", _i32, _i32, ctypes.POINTER(_Plan), ctypes.POINTER(_ServerData), ctypes.POINTER(_vp))
_create_synth = _sig("ipr_server_create_synthetic", _i32, _i32, ctypes.POINTER(_Plan), _u64, ctypes.POINTER(_vp))
_create_synth_shard = _sig("ipr_server_create_synthetic_shard", _i32, _i32, ctypes.c_void_p, _i32, _i32, _u64,
                           ctypes.POINTER(_vp))
_destroy = _sig("ipr_server_destroy", None, _vp)
_pp_json = _sig("ipr_server_public_params_json", _i32, _vp, ctypes.c_char_p, _sz, ctypes.POINTER(_sz))
_srv_qbytes = _sig("ipr_server_query_bytes", _u64, _vp, ctypes.c_uint)
_srv_rbytes = _sig("ipr_server_response_bytes", _u64, _vp, ctypes.c_uint)
_hbm = _sig("ipr_server_hbm_bytes", _i32, _vp, ctypes.POINTER(_u64))
_respond = _sig("ipr_server_respond", _i32, _vp, _u8p, _sz, _u8p, _sz, ctypes.POINTER(_sz))
_respond_dev = _sig("ipr_server_respond_device", _i32, _vp, _vp, _sz, _vp, _sz, ctypes.POINTER(_sz))
_stream = _sig("ipr_server_stream", _i32, _vp, ctypes.POINTER(_vp))
_respond_batch = _sig("ipr_server_respond_batch", _i32, _vp, _i32, ctypes.POINTER(_u8p), ctypes.POINTER(_sz),
                      ctypes.POINTER(_u8p), ctypes.POINTER(_sz), ctypes.POINTER(_sz), ctypes.POINTER(_i32))
_prepare_batch = _sig("ipr_server_prepare_batch", _i32, _vp, _i32)
_respond_batch_dev = _sig("ipr_server_respond_batch_device", _i32, _vp, _i32, _vp, _vp)
_sync = _sig("ipr_server_sync", _i32, _vp)
_set_prof = _sig("ipr_server_set_profiling", _i32, _vp, _i32)
_set_opt = _sig("ipr_server_set_option", _i32, _vp, _i32, ctypes.c_int64)
_stage_times = _sig("ipr_server_stage_times", _i32, _vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_u64))
_last_error = _sig("ipr_last_error", ctypes.c_char_p)


class _AutotuneResult(ctypes.Structure):
    _fields_ = [("candidates", _i32), ("pack_cta_pair", _i32 * 8), ("gemv_tile", _i32 * 8),
                ("ms", ctypes.c_double * 8), ("chosen", _i32), ("small_payloads", _i32),
                ("ms_small", ctypes.c_double * 8)]


_autotune = _sig("ipr_server_autotune", _i32, _vp, _i32, _i32, ctypes.POINTER(_AutotuneResult))


class _ServiceConfig(ctypes.Structure):
    _fields_ = [("max_batch", _i32), ("max_pending", _i32), ("hbm_budget_bytes", _u64)]


class _ServiceStats(ctypes.Structure):
    _fields_ = [("submitted", _u64), ("completed", _u64), ("rejected", _u64), ("failed", _u64),
                ("batches", _u64), ("batched_payloads", _u64), ("pending", _u64), ("in_flight", _u64),
                ("max_batch", _i32), ("hbm_bytes", _u64), ("p50_us", ctypes.c_double),
                ("p99_us", ctypes.c_double), ("mean_us", ctypes.c_double), ("max_us", ctypes.c_double),
                ("latency_samples", _u64), ("batch_ms_mean", ctypes.c_double), ("batch_ms_max", ctypes.c_double),
                ("queue_ms_mean", ctypes.c_double), ("queue_ms_max", ctypes.c_double)]


_plan_shard = _sig("ipr_plan_shard", _i32, ctypes.POINTER(_Plan), _i32, _i32, ctypes.POINTER(_Plan),
                   ctypes.POINTER(_u64))
_merge = _sig("ipr_response_merge", _i32, ctypes.POINTER(_u8p), ctypes.POINTER(_sz), _i32, _u8p, _sz,
              ctypes.POINTER(_sz))
_ntt_batch = _sig("ipr_ntt_batch", _i32, _i32, _vp, _u64, _i32, _i32, _vp)
_automorph_batch = _sig("ipr_automorph_batch", _i32, _i32, _vp, _u64, _vp, _i32, _vp, _vp)
_setup = _sig("ipr_server_setup", _i32, _i32, ctypes.POINTER(_Plan), ctypes.POINTER(_ServerData), _i32,
              ctypes.POINTER(_vp))
_create_raw = _sig("ipr_server_create_from_raw", _i32, _i32, ctypes.POINTER(_Plan), ctypes.POINTER(_ServerData),
                   ctypes.POINTER(_vp))
_encode = _sig("ipr_encode_db", _i32, _i32, _vp, _vp, _u64, _u64, _u64, _vp)
_raw_db = _sig("ipr_cuckoo_to_raw_db", _i32, _i32, _vp, _vp, _u64, _u64, _u64, _u64, _u64, _vp, _vp)
_wait_selftest = _sig("ipr_selftest_bounded_wait", _i32, _i32, ctypes.c_uint32)
_bounds_build = _sig("ipr_bounds_checked_build", _i32)
_bounds_report = _sig("ipr_bounds_report", _i32, ctypes.c_char_p, _sz)
_dbg_extent = _sig("ipr_debug_check_extent", _i32, _vp, _u64)
_dbg_cut = _sig("ipr_debug_cut_fold_extent", _i32, ctypes.c_int64)
_offline = _sig("ipr_offline_precompute", _i32, _i32, _vp, _u64, _u64, _vp, _vp, _vp, _vp, _u64, _vp)
_insp_create = _sig("ipr_inspiring_create", _i32, _i32, _i32, ctypes.POINTER(_vp))
_insp_pack = _sig("ipr_inspiring_pack", _i32, _vp, _i32, _vp, _vp, _vp, _vp, _vp)
_insp_destroy = _sig("ipr_inspiring_destroy", None, _vp)
_save = _sig("ipr_server_save", _i32, _vp, ctypes.c_char_p)
_load = _sig("ipr_server_load", _i32, _i32, ctypes.c_char_p, ctypes.POINTER(_vp))
_state_plan = _sig("ipr_state_file_plan", _i32, ctypes.c_char_p, ctypes.POINTER(_Plan))
_svc_create = _sig("ipr_service_create", _i32, ctypes.POINTER(_vp), _i32, ctypes.POINTER(_ServiceConfig),
                   ctypes.POINTER(_vp))
_svc_submit = _sig("ipr_service_submit", _i32, _vp, _i32, _u8p, _sz, ctypes.POINTER(_u64))
_svc_add_db = _sig("ipr_service_add_database", _i32, _vp, _vp, ctypes.POINTER(_i32))
_svc_submit_batch = _sig("ipr_service_submit_batch", _i32, _vp, _i32, _i32, ctypes.POINTER(_u8p),
                         ctypes.POINTER(_sz), ctypes.POINTER(_u64))
_svc_poll = _sig("ipr_service_poll", _i32, _vp, _u64, _u8p, _sz, ctypes.POINTER(_sz))
_svc_wait = _sig("ipr_service_wait", _i32, _vp, _u64, _i32, _u8p, _sz, ctypes.POINTER(_sz))
_svc_stats = _sig("ipr_service_get_stats", _i32, _vp, ctypes.POINTER(_ServiceStats))
_svc_reset = _sig("ipr_service_reset_stats", _i32, _vp)
_svc_diagnose = _sig("ipr_service_diagnose", _i32, _vp, ctypes.c_char_p, _sz)


class _ServiceBatch(ctypes.Structure):
    _fields_ = [("db", _i32), ("payloads", _i32), ("launch_ms", ctypes.c_double), ("start_ms", ctypes.c_double),
                ("ready_ms", ctypes.c_double), ("queue_ms_max", ctypes.c_double)]


_svc_log = _sig("ipr_service_batch_log", _i32, _vp, ctypes.POINTER(_ServiceBatch), _i32, ctypes.POINTER(_i32))
_svc_destroy = _sig("ipr_service_destroy", None, _vp)
_version = _sig("ipr_version", ctypes.c_char_p)

STATUS = {0: "IPR_OK", 1: "IPR_PENDING", -1: "IPR_E_ARGS", -2: "IPR_E_OOM", -3: "IPR_E_CUDA",
          -4: "IPR_E_TIMEOUT", -5: "IPR_E_FORMAT", -6: "IPR_E_SPACE", -7: "IPR_E_STATE", -8: "IPR_E_BUSY",
          -9: "IPR_E_IO"}
IPR_PENDING = 1
IPR_E_BUSY = -8


class IprError(RuntimeError):
    def __init__(self, status: int, where: str):
        msg = (_last_error() or b"").decode(errors="replace")
        super().__init__(f"{where}: {STATUS.get(status, status)}: {msg}")
        self.status = status


def _check(st: int, where: str):
    if st != 0:
        raise IprError(st, where)


@dataclass(frozen=True)
class Plan:
    """KeywordServerSetupPlan (keyword.rs:91-102) plus the GPU memory estimate."""
    num_items: int
    entry_size: int
    item_size_bits: int
    dim0: int
    db_rows: int
    db_cols: int
    instances: int
    interp: int
    c: int
    peak_bytes: int

    def _c(self) -> _Plan:
        return _Plan(*[getattr(self, f) for f, _ in _Plan._fields_])

    @property
    def query_bytes(self) -> int:
        return query_bytes(self.db_rows, 2)


_fail_alloc = _sig("ipr_debug_fail_allocation", _i32, ctypes.c_int64)


def fail_allocation_after(n: int):
    """test hook: the next n server device allocations succeed, the one after fails (IPR_E_OOM);
    n < 0 switches the hook off"""
    _check(_fail_alloc(n), "ipr_debug_fail_allocation")


def bounds_checked_build() -> bool:
    """ipr_bounds_checked_build: True for the bounds-checked debug library"""
    return bool(_bounds_build())


def bounds_report():
    """ipr_bounds_report: (number of failed checks since the last report, their lines); the
    debug build synchronises the current device first, the release build reports (0, "")"""
    buf = ctypes.create_string_buffer(1 << 13)
    n = _bounds_report(buf, len(buf))
    return int(n), buf.value.decode()


def debug_check_extent(d_ptr: int, nbytes: int) -> int:
    """ipr_debug_check_extent (debug build): the launch-argument range check on
    [d_ptr, d_ptr + nbytes); IPR_OK inside one allocation, IPR_E_ARGS outside"""
    return int(_dbg_extent(d_ptr, nbytes))


def debug_cut_fold_extent(words: int) -> int:
    """ipr_debug_cut_fold_extent (debug build): later fold launches believe their packing
    output buffer is `words` words shorter, so the fold's own index checks trip; 0 restores"""
    return int(_dbg_cut(words))


def selftest_bounded_wait(limit_us: int = 20_000, device: int = 0) -> int:
    """ipr_selftest_bounded_wait: the status of a bounded mbarrier wait that nobody
    satisfies, given up after limit_us microseconds (IPR_E_TIMEOUT = -4 when the failure
    is detected; IPR_E_ARGS for a limit outside 1 .. 1,000,000)"""
    return int(_wait_selftest(device, limit_us))


def offline_precompute(d_db: int, db_rows: int, instances: int, d_a_hat: int, d_bold_t: int, d_bold_t_bar: int,
                       d_bold_t_hat: int, scratch_bytes: int = 0, device: int = 0, stream: int = 0):
    """ipr_offline_precompute on device pointers: the encoded DB [instances*2048][db_rows] u16
    -> a_hat [inst][2048], bold_t / bold_t_bar [inst][3069][2048], bold_t_hat [inst][3][2048]
    (u64; the setup outputs of perform_offline_precomputation_simplepir)"""
    _check(_offline(device, d_db, db_rows, instances, d_a_hat, d_bold_t, d_bold_t_bar, d_bold_t_hat, scratch_bytes,
                    stream or None), "ipr_offline_precompute")


class InspiringPacker:
    """packing_fully_online on the GPU (ipr_inspiring_*): packs sets of 2048 LWE ciphertexts
    (device arrays [sets][2049][2048] u64) into RLWE ciphertexts [sets][2][2048]"""

    def __init__(self, max_sets: int = 1, device: int = 0):
        h = _vp()
        _check(_insp_create(device, max_sets, ctypes.byref(h)), "ipr_inspiring_create")
        self._h, self.max_sets, self.device = h, max_sets, device

    def pack(self, sets: int, d_lwe: int, d_y_body: int, d_z_body: int, d_out: int, stream: int = 0):
        _check(_insp_pack(self._h, sets, d_lwe, d_y_body, d_z_body, d_out, stream or None), "ipr_inspiring_pack")

    def close(self):
        if self._h and self._h.value:
            _insp_destroy(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def state_file_plan(path: str) -> Plan:
    """the plan recorded in a server state file's header (reads the header only)"""
    p = _Plan()
    _check(_state_plan(os.fsencode(path), ctypes.byref(p)), "ipr_state_file_plan")
    return Plan(*[getattr(p, f) for f, _ in _Plan._fields_])


def plan_from_shape(record_count: int, key_size: int, value_size: int,
                    buckets: Optional[int] = None, dim0: Optional[int] = None) -> Plan:
    """KeywordServerSetupPlan::from_shape (keyword.rs:145-233); raises on the
    shapes the reference rejects (e.g. buckets < records, keyword.rs:171-180)."""
    p = _Plan()
    _check(_plan_from_shape(record_count, key_size, value_size, buckets or 0, dim0 or 0, ctypes.byref(p)),
           "plan_from_shape")
    return Plan(*[getattr(p, f) for f, _ in _Plan._fields_])


def query_bytes(db_rows: int, num_queries: int = 2) -> int:
    return int(_query_bytes(db_rows, num_queries))


# ---------------------------------------------------------------------------
# wire payloads (src/protocol/wire.rs:522-538, 542-615, 708-759)
# ---------------------------------------------------------------------------
@dataclass
class KeywordQueryPayload:
    """Decoded form of a keyword query.  y_body/z_body: 3 x 2048 condensed u64
    (lo32 = mod q0, hi32 = mod q1); queries: list of (packed_query_row
    [db_rows] condensed, ct_gsw_body 6 x (2 x 2048) limb-major residues)."""
    y_body: Sequence[Sequence[int]]
    z_body: Sequence[Sequence[int]]
    queries: List[tuple]


@dataclass
class KeywordResponsePayload:
    responses: List[bytes]
    stash_entries: List[bytes]


def serialize_keyword_query(p: KeywordQueryPayload) -> bytes:
    """serialize_keyword_query (wire.rs:542-615): 1 count byte, then 56-bit
    fields (crt0 | crt1 << 28) LSB-first from bit 8."""
    import numpy as np
    m28 = (1 << 28) - 1
    vals = []
    for i in range(3):
        yz = np.empty(2 * POLY_LEN, dtype=np.uint64)
        yz[0::2] = np.asarray(p.y_body[i], dtype=np.uint64)
        yz[1::2] = np.asarray(p.z_body[i], dtype=np.uint64)
        vals.append((yz & np.uint64(m28)) | ((yz >> np.uint64(32)) << np.uint64(28)))
    for row, gsw in p.queries:
        r = np.asarray(row, dtype=np.uint64)
        vals.append((r & np.uint64(m28)) | ((r >> np.uint64(32)) << np.uint64(28)))
        g = np.asarray(gsw, dtype=np.uint64).reshape(6, 2, POLY_LEN)
        vals.append(((g[:, 0, :] & np.uint64(m28)) | (g[:, 1, :] << np.uint64(28))).reshape(-1))
    allv = np.concatenate(vals).astype("<u8")
    by = allv.view(np.uint8).reshape(-1, 8)[:, :7].reshape(-1)
    return bytes([len(p.queries)]) + by.tobytes()


def deserialize_keyword_response(data: bytes) -> KeywordResponsePayload:
    """deserialize_keyword_response (wire.rs:729-759)."""
    off = 0

    def u32():
        nonlocal off
        v = int.from_bytes(data[off:off + 4], "little")
        off += 4
        return v
    responses = []
    for _ in range(u32()):
        n = u32()
        responses.append(bytes(data[off:off + n]))
        off += n
    stash = []
    for _ in range(u32()):
        n = u32()
        stash.append(bytes(data[off:off + n]))
        off += n
    return KeywordResponsePayload(responses, stash)


# ---------------------------------------------------------------------------
# server
# ---------------------------------------------------------------------------
class KeywordServer:
    """Device-resident keyword server (KeywordServer<u16>, keyword.rs:49-63).

    Build with ``KeywordServer.from_encoded`` (encoded DB + InspiRING
    precomputation arrays, the state the reference's setup leaves on the GPU)
    or ``KeywordServer.synthetic`` (seeded synthetic state of the same shapes).
    """

    def __init__(self, handle: int, plan: Plan, device: int):
        self._h = _vp(handle)
        self.plan = plan
        self.device = device

    @classmethod
    def from_raw(cls, plan: Plan, raw_db, a_hat, bold_t, bold_t_bar, bold_t_hat, **kw) -> "KeywordServer":
        """as from_encoded, with the RAW database (to_raw_db layout), encoded on the device"""
        return cls.from_encoded(plan, raw_db, a_hat, bold_t, bold_t_bar, bold_t_hat, _raw=True, **kw)

    @classmethod
    def from_encoded(cls, plan: Plan, db, a_hat, bold_t, bold_t_bar, bold_t_hat, stash=(),
                     key_size: int = 32, value_size: Optional[int] = None, num_records: int = 0,
                     cuckoo_seed: bytes = bytes(16), device: int = 0, _raw: bool = False) -> "KeywordServer":
        import numpy as np
        arrs = {
            "db": np.ascontiguousarray(db, dtype=np.uint16),
            "a_hat": np.ascontiguousarray(a_hat, dtype=np.uint64),
            "bold_t": np.ascontiguousarray(bold_t, dtype=np.uint64),
            "bold_t_bar": np.ascontiguousarray(bold_t_bar, dtype=np.uint64),
            "bold_t_hat": np.ascontiguousarray(bold_t_hat, dtype=np.uint64),
        }
        n, ninner = plan.instances, 3069
        want = {"db": plan.db_rows * plan.db_cols, "a_hat": n * POLY_LEN, "bold_t": n * ninner * POLY_LEN,
                "bold_t_bar": n * ninner * POLY_LEN, "bold_t_hat": n * 3 * POLY_LEN}
        for k, v in arrs.items():
            if v.size != want[k]:
                raise ValueError(f"{k} has {v.size} elements, plan needs {want[k]}")
        stash = [bytes(s) for s in stash]
        entry = len(stash[0]) if stash else 0
        if any(len(s) != entry for s in stash):
            raise ValueError("stash entries must have equal length")
        stash_buf = np.frombuffer(b"".join(stash), dtype=np.uint8) if stash else None
        d = _ServerData()
        for k, v in arrs.items():
            setattr(d, k, v.ctypes.data)
        d.stash = stash_buf.ctypes.data if stash_buf is not None else None
        d.stash_count, d.stash_entry_bytes = len(stash), entry
        d.key_size = key_size
        d.value_size = plan.entry_size - key_size if value_size is None else value_size
        d.num_records = num_records
        d.cuckoo_seed[:] = list(cuckoo_seed[:16].ljust(16, b"\0"))
        h = _vp()
        pc = plan._c()
        fn, name = (_create_raw, "ipr_server_create_from_raw") if _raw else (_create, "ipr_server_create")
        _check(fn(device, ctypes.byref(pc), ctypes.byref(d), ctypes.byref(h)), name)
        return cls(h.value, plan, device)

    @classmethod
    def setup(cls, plan: Plan, db, raw: bool = False, stash=(), key_size: int = 32,
              value_size: Optional[int] = None, num_records: int = 0, cuckoo_seed: bytes = bytes(16),
              device: int = 0) -> "KeywordServer":
        """KeywordServer::setup on the GPU: from the DB alone (raw to_raw_db layout when `raw`,
        else encoded), running the encode and the offline precomputation on the device"""
        import numpy as np
        d8 = np.ascontiguousarray(db, dtype=np.uint16)
        if d8.size != plan.db_rows * plan.db_cols:
            raise ValueError(f"db has {d8.size} elements, plan needs {plan.db_rows * plan.db_cols}")
        stash = [bytes(s) for s in stash]
        entry = len(stash[0]) if stash else 0
        if any(len(s) != entry for s in stash):
            raise ValueError("stash entries must have equal length")
        stash_buf = np.frombuffer(b"".join(stash), dtype=np.uint8) if stash else None
        d = _ServerData()
        d.db = d8.ctypes.data
        d.stash = stash_buf.ctypes.data if stash_buf is not None else None
        d.stash_count, d.stash_entry_bytes = len(stash), entry
        d.key_size = key_size
        d.value_size = plan.entry_size - key_size if value_size is None else value_size
        d.num_records = num_records
        d.cuckoo_seed[:] = list(cuckoo_seed[:16].ljust(16, b"\0"))
        h = _vp()
        pc = plan._c()
        _check(_setup(device, ctypes.byref(pc), ctypes.byref(d), 1 if raw else 0, ctypes.byref(h)), "ipr_server_setup")
        return cls(h.value, plan, device)

    @classmethod
    def synthetic(cls, plan: Plan, seed: int = 7, device: int = 0) -> "KeywordServer":
        h = _vp()
        pc = plan._c()
        _check(_create_synth(device, ctypes.byref(pc), seed, ctypes.byref(h)), "ipr_server_create_synthetic")
        return cls(h.value, plan, device)

    @classmethod
    def synthetic_shard(cls, full: Plan, num_shards: int, shard: int, seed: int = 7,
                        device: int = 0) -> "KeywordServer":
        """shard `shard` of `num_shards` (fold groups, ipr_plan_shard) of synthetic(full, seed),
        generated alone on the device: the shards' merged responses are the full server's"""
        h = _vp()
        pc = full._c()
        _check(_create_synth_shard(device, ctypes.byref(pc), num_shards, shard, seed, ctypes.byref(h)),
               "ipr_server_create_synthetic_shard")
        return cls(h.value, shard_plan(full, num_shards, shard)[0], device)

    @classmethod
    def load(cls, path: str, device: int = 0) -> "KeywordServer":
        """rebuild a server from a state file written by ``save`` (no setup rerun)"""
        plan = state_file_plan(path)
        h = _vp()
        _check(_load(device, os.fsencode(path), ctypes.byref(h)), "ipr_server_load")
        return cls(h.value, plan, device)

    def save(self, path: str):
        """write the setup outputs this server was built from to a state file
        (format: ipr_server_save in include/ipr_b200.h)"""
        _check(_save(self._h, os.fsencode(path)), "ipr_server_save")

    def close(self):
        if self._h and self._h.value:
            _destroy(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # --- reference API -------------------------------------------------
    def public_params(self) -> dict:
        """KeywordServer::public_params (keyword.rs:511-532) as the serde JSON dict."""
        n = _sz()
        _pp_json(self._h, None, 0, ctypes.byref(n))
        buf = ctypes.create_string_buffer(n.value + 1)
        _check(_pp_json(self._h, buf, n.value + 1, ctypes.byref(n)), "public_params")
        return json.loads(buf.value.decode())

    def respond_to_serialized_query(self, query: bytes) -> bytes:
        """keyword.rs:636-640: serialized query payload -> serialized response."""
        q = (ctypes.c_uint8 * len(query)).from_buffer_copy(query)
        nq = query[0] if query else 0
        cap = int(_srv_rbytes(self._h, nq))
        out = (ctypes.c_uint8 * cap)()
        n = _sz()
        _check(_respond(self._h, q, len(query), out, cap, ctypes.byref(n)), "respond")
        return bytes(out)[:n.value]

    def respond(self, payload: KeywordQueryPayload) -> KeywordResponsePayload:
        """KeywordServer::respond (keyword.rs:534-628)."""
        return deserialize_keyword_response(self.respond_to_serialized_query(serialize_keyword_query(payload)))

    def respond_batch(self, queries: Sequence[bytes]) -> List[bytes]:
        """Answer many serialized payloads in one call (ipr_server_respond_batch);
        two-query payloads share the tensor-core batch path.  Raises on the
        first failing payload."""
        n = len(queries)
        if n == 0:
            return []
        qbufs = [(ctypes.c_uint8 * len(q)).from_buffer_copy(q) for q in queries]
        caps = [int(_srv_rbytes(self._h, q[0] if q else 0)) for q in queries]
        obufs = [(ctypes.c_uint8 * c)() for c in caps]
        qp = (_u8p * n)(*[ctypes.cast(b, _u8p) for b in qbufs])
        op = (_u8p * n)(*[ctypes.cast(b, _u8p) for b in obufs])
        lens = (_sz * n)(*[len(q) for q in queries])
        capa = (_sz * n)(*caps)
        olen = (_sz * n)()
        sts = (_i32 * n)()
        st = _respond_batch(self._h, n, qp, lens, op, capa, olen, sts)
        for i in range(n):
            if sts[i]:
                raise IprError(sts[i], f"respond_batch[{i}]")
        _check(st, "respond_batch")
        return [bytes(obufs[i])[:olen[i]] for i in range(n)]

    def prepare_batch(self, max_payloads: int = 64):
        _check(_prepare_batch(self._h, max_payloads), "prepare_batch")

    def respond_batch_device(self, n: int, d_queries_ptr: int, d_out_ptr: int):
        """n two-query payloads back to back in device memory -> responses back to back (async)."""
        _check(_respond_batch_dev(self._h, n, _vp(d_queries_ptr), _vp(d_out_ptr)), "respond_batch_device")

    # --- device-level helpers (bench / serving) ---------------------------
    def respond_device(self, d_query_ptr: int, length: int, d_out_ptr: int, cap: int) -> int:
        n = _sz()
        _check(_respond_dev(self._h, _vp(d_query_ptr), length, _vp(d_out_ptr), cap, ctypes.byref(n)),
               "respond_device")
        return n.value

    def autotune(self, payloads: int = 64, reps: int = 3) -> dict:
        """ipr_server_autotune: time the batch path's candidate configurations on synthetic
        batches of `payloads` and of payloads // 4 and keep the one with the least device time
        per payload over both sizes (every candidate gives identical responses)"""
        r = _AutotuneResult()
        _check(_autotune(self._h, payloads, reps, ctypes.byref(r)), "ipr_server_autotune")
        cands = [{"pack_cta_pair": r.pack_cta_pair[i], "gemv_tile": r.gemv_tile[i], "ms": r.ms[i],
                  "ms_small": r.ms_small[i] if r.small_payloads else None}
                 for i in range(r.candidates)]
        return {"candidates": cands, "chosen": cands[r.chosen], "small_payloads": r.small_payloads}

    def stream_handle(self) -> int:
        s = _vp()
        _check(_stream(self._h, ctypes.byref(s)), "stream")
        return s.value or 0

    def sync(self):
        _check(_sync(self._h), "sync")

    OPT_TENSOR_GEMV = 1
    OPT_FOLD_REGISTER_NTT = 2
    OPT_PACK_CTA_PAIR = 3
    OPT_GEMV_TILE = 4
    OPT_GEMV_FORM = 5

    def set_option(self, option: int, value: int):
        """ipr_server_set_option: e.g. OPT_TENSOR_GEMV 0/1 selects the CUDA-core or
        tensor-core first-dimension GEMV (identical results)."""
        _check(_set_opt(self._h, option, value), "set_option")

    def set_profiling(self, on: bool):
        _check(_set_prof(self._h, 1 if on else 0), "set_profiling")

    def stage_times(self):
        arr = (ctypes.c_double * len(STAGES))()
        calls = _u64()
        _check(_stage_times(self._h, arr, ctypes.byref(calls)), "stage_times")
        return dict(zip(STAGES, list(arr))), calls.value

    def query_bytes(self, num_queries: int = 2) -> int:
        return int(_srv_qbytes(self._h, num_queries))

    def response_bytes(self, num_queries: int = 2) -> int:
        return int(_srv_rbytes(self._h, num_queries))

    def hbm_bytes(self) -> int:
        v = _u64()
        _check(_hbm(self._h, ctypes.byref(v)), "hbm_bytes")
        return v.value


def version() -> str:
    return _version().decode()


@dataclass(frozen=True)
class ServiceStats:
    submitted: int
    completed: int
    rejected: int
    failed: int
    batches: int
    batched_payloads: int
    pending: int
    in_flight: int
    max_batch: int
    hbm_bytes: int
    p50_us: float
    p99_us: float
    mean_us: float
    max_us: float
    latency_samples: int
    batch_ms_mean: float
    batch_ms_max: float
    queue_ms_mean: float
    queue_ms_max: float


class KeywordService:
    """Continuous-batching serving loop over one or more KeywordServers
    (ipr_service_*): ``submit`` queues a serialized payload for database
    ``db`` and returns a ticket; ``wait`` / ``poll`` return the serialized
    response, byte-identical to ``KeywordServer.respond_to_serialized_query``.
    The servers must stay open while the service runs."""

    def __init__(self, servers: Sequence["KeywordServer"], max_batch: int = 64, max_pending: int = 0,
                 hbm_budget_bytes: int = 0, autotune: bool = False):
        self._servers = list(servers)
        if autotune:  # each database's batch path set to its fastest exact configuration first
            for srv in self._servers:
                srv.prepare_batch(max_batch)
                srv.autotune(max_batch)
        arr = (_vp * len(self._servers))(*[s._h.value for s in self._servers])
        cfg = _ServiceConfig(max_batch, max_pending, hbm_budget_bytes)
        self._h = _vp()
        _check(_svc_create(arr, len(self._servers), ctypes.byref(cfg), ctypes.byref(self._h)), "service_create")
        self._cap = max(s.response_bytes(2) for s in self._servers)

    def add_database(self, server: "KeywordServer") -> int:
        """ipr_service_add_database: serve one more database (admitted under what is left of
        the HBM budget); returns its index for submit"""
        db = _i32()
        _check(_svc_add_db(self._h, server._h, ctypes.byref(db)), "service_add_database")
        self._servers.append(server)
        self._cap = max(self._cap, server.response_bytes(2))
        return db.value

    def submit(self, db: int, query: bytes) -> int:
        t = _u64()
        query = bytes(query)
        ptr = ctypes.cast(ctypes.c_char_p(query), _u8p)  # no copy: the service copies on submit
        _check(_svc_submit(self._h, db, ptr, len(query), ctypes.byref(t)), "service_submit")
        return t.value

    def submit_many(self, db: int, queries: Sequence[bytes]) -> List[int]:
        """ipr_service_submit_batch: all payloads queued at once (all or none)"""
        n = len(queries)
        qs = [bytes(q) for q in queries]
        ptrs = (_u8p * n)(*[ctypes.cast(ctypes.c_char_p(q), _u8p) for q in qs])
        lens = (_sz * n)(*[len(q) for q in qs])
        out = (_u64 * n)()
        _check(_svc_submit_batch(self._h, db, n, ptrs, lens, out), "service_submit_batch")
        return list(out)

    def _buffer(self, cap: int):
        """a per-thread result buffer, reused across calls (no allocation or zeroing per result)"""
        import threading
        tl = self.__dict__.setdefault("_tls", threading.local())
        buf = getattr(tl, "buf", None)
        if buf is None or len(buf) < cap:
            buf = tl.buf = (ctypes.c_uint8 * cap)()
        return buf

    def _collect(self, fn, ticket, *extra):
        cap = self._cap
        out = self._buffer(cap)
        n = _sz()
        st = fn(self._h, ticket, *extra, ctypes.cast(out, _u8p), cap, ctypes.byref(n))
        if st == IPR_PENDING:
            return None
        if st == -6 and n.value > cap:  # a larger payload: the result is kept for the retry
            cap = n.value
            out = self._buffer(cap)
            st = _svc_poll(self._h, ticket, ctypes.cast(out, _u8p), cap, ctypes.byref(n))
        _check(st, "service_result")
        return ctypes.string_at(out, n.value)

    def poll(self, ticket: int) -> Optional[bytes]:
        """the response, or None while the request runs"""
        return self._collect(_svc_poll, ticket)

    def wait(self, ticket: int, timeout_ms: int = -1) -> Optional[bytes]:
        """the response (None if timeout_ms ran out first)"""
        return self._collect(_svc_wait, ticket, timeout_ms)

    def stats(self) -> ServiceStats:
        st = _ServiceStats()
        _check(_svc_stats(self._h, ctypes.byref(st)), "service_stats")
        return ServiceStats(*[getattr(st, f) for f, _ in _ServiceStats._fields_])

    def reset_stats(self):
        _check(_svc_reset(self._h), "service_reset_stats")

    def diagnose(self) -> str:
        """ipr_service_diagnose: per database lane, the queue, busy slots and the completion
        state of their uploads, compute and streams"""
        buf = ctypes.create_string_buffer(1 << 14)
        _check(_svc_diagnose(self._h, buf, len(buf)), "service_diagnose")
        return buf.value.decode()

    def batch_log(self, cap: int = 4096):
        """the most recent batches, oldest first: dicts of db, payloads, launch/start/ready ms, queue_ms_max"""
        arr = (_ServiceBatch * cap)()
        n = _i32()
        _check(_svc_log(self._h, arr, cap, ctypes.byref(n)), "service_batch_log")
        return [{f: getattr(arr[i], f) for f, _ in _ServiceBatch._fields_} for i in range(n.value)]

    def close(self):
        if self._h and self._h.value:
            _svc_destroy(self._h)
            self._h = _vp()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# the keyword-PIR client on the GPU (ipr_client_*, KeywordClient of src/pir/client/keyword.rs)
# ---------------------------------------------------------------------------
_cl_create = _sig("ipr_client_create", _i32, _i32, ctypes.POINTER(_Plan), ctypes.c_char_p, ctypes.POINTER(_vp))
_cl_query = _sig("ipr_client_query", _i32, _vp, _u64, ctypes.c_uint, ctypes.POINTER(_u64), _u8p, _sz,
                 ctypes.POINTER(_sz))
_cl_decrypt = _sig("ipr_client_decrypt", _i32, _vp, _u8p, _sz, ctypes.POINTER(ctypes.c_uint16), _sz,
                   ctypes.POINTER(_sz))
_cl_key = _sig("ipr_client_secret_key", _i32, _vp, ctypes.POINTER(ctypes.c_int8))
_cl_destroy = _sig("ipr_client_destroy", None, _vp)
_cuckoo = _sig("ipr_cuckoo_positions", _i32, ctypes.c_char_p, _u64, ctypes.c_uint, ctypes.c_char_p, _sz,
               ctypes.POINTER(_u64))


def cuckoo_positions(seed: bytes, num_buckets: int, num_hashes: int, key: bytes) -> List[int]:
    """CuckooHash::all_positions (cuckoo.rs:105-131): the bucket positions of a keyword"""
    out = (_u64 * max(num_hashes, 1))()
    _check(_cuckoo(bytes(seed)[:16].ljust(16, b"\0"), num_buckets, num_hashes, bytes(key), len(key), out),
           "ipr_cuckoo_positions")
    return list(out)[:num_hashes]


class KeywordClient:
    """KeywordClient on the GPU for a server plan: query payloads for buckets (cuckoo
    positions) and decryption of the server's response.  Key and noise are deterministic in
    the 32-byte `seed`; every query takes a fresh nonce (counted up from 0 unless given)."""

    def __init__(self, plan: Plan, seed: bytes, device: int = 0):
        if len(seed) != 32:
            raise ValueError("seed must be 32 bytes")
        self.plan, self.device, self._nonce = plan, device, 0
        self.keyword = None  # the keyword layout, known when built from the public parameters
        self.per = plan.num_items // plan.db_rows
        self.item_elems = plan.item_size_bits // 16
        h = _vp()
        pc = plan._c()
        _check(_cl_create(device, ctypes.byref(pc), bytes(seed), ctypes.byref(h)), "ipr_client_create")
        self._h = h.value

    def query(self, buckets: Sequence[int], nonce: Optional[int] = None) -> bytes:
        """build_query_payload + serialize_query (keyword.rs:193-214) for these buckets"""
        if nonce is None:
            nonce, self._nonce = self._nonce, self._nonce + 1
        b = (_u64 * max(len(buckets), 1))(*buckets)
        need = query_bytes(self.plan.db_rows, len(buckets))
        out = (ctypes.c_uint8 * need)()
        n = _sz()
        _check(_cl_query(self._h, nonce, len(buckets), b, out, need, ctypes.byref(n)), "ipr_client_query")
        return bytes(out)

    def decrypt(self, response: bytes):
        """plaintexts [responses][c][2048] (u16 mod 65535) of a serialized response"""
        import numpy as np
        buf = (ctypes.c_uint8 * max(len(response), 1)).from_buffer_copy(response or b"\0")
        n = _sz()
        st = _cl_decrypt(self._h, buf, len(response), None, 0, ctypes.byref(n))
        if st not in (0, -6):
            _check(st, "ipr_client_decrypt")
        vals = np.zeros(n.value, dtype=np.uint16)
        _check(_cl_decrypt(self._h, buf, len(response), vals.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)),
                           vals.size, ctypes.byref(n)), "ipr_client_decrypt")
        return vals.reshape(-1, self.plan.c, POLY_LEN)

    @classmethod
    def from_public_params(cls, params: dict, seed: bytes, device: int = 0) -> "KeywordClient":
        """KeywordClient::setup_from_public_params (keyword.rs:60-115): the plan from the
        server's public parameters; keeps the keyword layout for query_key / extract_key"""
        kw = params.get("keyword_pir")
        if not kw:
            raise ValueError("server is not in keyword PIR mode")
        if kw["key_size"] == 0 or kw["value_size"] == 0:
            raise ValueError("server keyword and value sizes must be non-zero")
        if kw["entry_size"] < kw["key_size"] + kw["value_size"]:
            raise ValueError("server entry size is smaller than key_size + value_size")
        plan = plan_from_shape(max(1, min(kw.get("num_records", 0) or 1, params["num_items"])), kw["key_size"],
                               kw["value_size"], params["num_items"], params["dim0"])
        if plan.item_size_bits != params["item_size_bits"]:
            raise ValueError("public parameters do not match the scheme's shape")
        c = cls(plan, seed, device)
        c.keyword = kw
        return c

    def positions(self, key: bytes) -> List[int]:
        """positions (keyword.rs:129-137)"""
        kw = self.keyword
        if kw is None:
            raise ValueError("no keyword layout: build the client with from_public_params")
        if len(key) != kw["key_size"]:
            raise ValueError(f"expected {kw['key_size']} keyword bytes, got {len(key)}")
        return cuckoo_positions(bytes(kw["cuckoo_seed"]), self.plan.num_items, kw["num_hashes"], key)

    def query_key(self, key: bytes):
        """query (keyword.rs:193-200) + serialize_query: (positions, payload bytes)"""
        pos = self.positions(key)
        return pos, self.query(pos)

    def extract_key(self, key: bytes, positions: Sequence[int], response: bytes) -> Optional[bytes]:
        """extract_from_serialized_response (keyword.rs:232-300): the value stored under key, from
        the decrypted entry of one of its positions or from the stash, else None"""
        kw = self.keyword
        if kw is None:
            raise ValueError("no keyword layout: build the client with from_public_params")
        if len(key) != kw["key_size"]:
            return None
        ks, vs, es = kw["key_size"], kw["value_size"], kw["entry_size"]
        pts = self.decrypt(response)
        for pos, pt in zip(positions, pts):
            entry = self.extract(pos, pt)
            if entry is not None and len(entry) >= es and entry[:ks] == bytes(key):
                return entry[ks:ks + vs]
        for entry in deserialize_keyword_response(response).stash_entries:
            if len(entry) >= es and entry[:ks] == bytes(key):
                return entry[ks:ks + vs]
        return None

    def extract(self, bucket: int, plaintext) -> Optional[bytes]:
        """the entry bytes of `bucket` from its sub-query's plaintexts (keyword.rs:246-257);
        None when the entry crosses a polynomial boundary and is not all in the returned one"""
        import numpy as np
        col = (bucket % self.per) * self.item_elems
        poly, coeff = col // POLY_LEN, col % POLY_LEN
        if coeff + self.item_elems > POLY_LEN:
            return None
        flat = np.asarray(plaintext, dtype=np.uint16).reshape(-1)
        off = (poly // self.plan.interp) * POLY_LEN + coeff
        return flat[off:off + self.item_elems].astype(">u2").tobytes()

    def secret_key(self):
        import numpy as np
        out = np.zeros(POLY_LEN, dtype=np.int8)
        _check(_cl_key(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int8))), "ipr_client_secret_key")
        return out

    def close(self):
        if getattr(self, "_h", None):
            _cl_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


# ---------------------------------------------------------------------------
# fold-group sharding across GPUs (one process per GPU)
# ---------------------------------------------------------------------------
def shard_plan(plan: Plan, num_shards: int, shard: int):
    """(sub-plan, first instance) of shard `shard` (ipr_plan_shard): a contiguous run of fold groups."""
    out = _Plan()
    first = _u64()
    _check(_plan_shard(ctypes.byref(plan._c()), num_shards, shard, ctypes.byref(out), ctypes.byref(first)),
           "plan_shard")
    return Plan(**{f: getattr(out, f) for f, _ in _Plan._fields_}), first.value


def shard_slices(plan: Plan, num_shards: int, shard: int):
    """element ranges of the shard's slice in each host array of ipr_server_data"""
    sub, first = shard_plan(plan, num_shards, shard)
    n, rows = sub.instances, plan.db_rows
    return sub, {
        "db": (first * POLY_LEN * rows, (first + n) * POLY_LEN * rows),
        "a_hat": (first * POLY_LEN, (first + n) * POLY_LEN),
        "bold_t": (first * 3069 * POLY_LEN, (first + n) * 3069 * POLY_LEN),
        "bold_t_bar": (first * 3069 * POLY_LEN, (first + n) * 3069 * POLY_LEN),
        "bold_t_hat": (first * 3 * POLY_LEN, (first + n) * 3 * POLY_LEN),
    }


def merge_responses(parts: Sequence[bytes]) -> bytes:
    """ipr_response_merge: the unsharded response from the shards' responses (in shard order)."""
    k = len(parts)
    bufs = [(ctypes.c_uint8 * max(len(p), 1)).from_buffer_copy(p if p else b"\0") for p in parts]
    arr = (_u8p * k)(*[ctypes.cast(b, _u8p) for b in bufs])
    lens = (_sz * k)(*[len(p) for p in parts])
    need = _sz()
    st = _merge(arr, lens, k, None, 0, ctypes.byref(need))
    if st not in (0, -6):
        _check(st, "response_merge")
    out = (ctypes.c_uint8 * need.value)()
    _check(_merge(arr, lens, k, ctypes.cast(out, _u8p), need.value, ctypes.byref(need)), "response_merge")
    return bytes(out)


class ShardedKeywordServer:
    """One fold-group shard per process (torch.distributed rank); the ranks
    together answer like one KeywordServer.  ``respond_to_serialized_query``
    is collective: rank 0's query bytes are broadcast, every rank answers its
    groups, and the parts are gathered to rank 0, which returns the merged
    response (other ranks return None).  ``answer`` is the per-rank step:
    any callable bytes -> bytes (a KeywordServer built from the shard's
    slices, or a test stand-in)."""

    def __init__(self, answer, group=None, device=None):
        import torch.distributed as dist
        self._dist = dist
        self._answer = answer
        self._group = group
        self._device = device  # tensors for the collectives live here (a CUDA device under NCCL)
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    def _bcast_bytes(self, data: Optional[bytes]) -> bytes:
        import torch
        dist = self._dist
        n = torch.tensor([len(data) if self.rank == 0 else 0], dtype=torch.int64, device=self._device)
        dist.broadcast(n, 0, group=self._group)
        buf = (torch.frombuffer(bytearray(data), dtype=torch.uint8).to(self._device) if self.rank == 0
               else torch.empty(int(n.item()), dtype=torch.uint8, device=self._device))
        dist.broadcast(buf, 0, group=self._group)
        return bytes(buf.cpu().numpy().tobytes())

    def _gather_bytes(self, data: bytes) -> Optional[List[bytes]]:
        import torch
        dist = self._dist
        n = torch.tensor([len(data)], dtype=torch.int64, device=self._device)
        ns = [torch.zeros(1, dtype=torch.int64, device=self._device) for _ in range(self.world)]
        dist.all_gather(ns, n, group=self._group)
        mx = max(int(x.item()) for x in ns)
        mine = torch.zeros(mx, dtype=torch.uint8, device=self._device)
        if data:
            mine[:len(data)] = torch.frombuffer(bytearray(data), dtype=torch.uint8).to(self._device)
        parts = [torch.empty(mx, dtype=torch.uint8, device=self._device) for _ in range(self.world)]
        dist.all_gather(parts, mine, group=self._group)
        if self.rank != 0:
            return None
        return [bytes(p.cpu().numpy()[:int(k.item())].tobytes()) for p, k in zip(parts, ns)]

    def respond_to_serialized_query(self, query: Optional[bytes]) -> Optional[bytes]:
        q = self._bcast_bytes(query)
        part = self._answer(q)
        parts = self._gather_bytes(part)
        return merge_responses(parts) if parts is not None else None

    def respond_batch(self, queries: Optional[Sequence[bytes]], answer_batch=None) -> Optional[List[bytes]]:
        """collective batch form: rank 0's payloads travel in one broadcast, every rank answers
        them with `answer_batch` (list -> list, e.g. its KeywordServer.respond_batch; default:
        `answer` per payload), the parts come back in one gather and rank 0 merges each
        payload's parts (other ranks return None)"""
        import struct
        if self.rank == 0:
            blob = struct.pack("<I", len(queries)) + b"".join(struct.pack("<Q", len(q)) + bytes(q) for q in queries)
        else:
            blob = None
        blob = self._bcast_bytes(blob)
        n, off, qs = struct.unpack_from("<I", blob)[0], 4, []
        for _ in range(n):
            k = struct.unpack_from("<Q", blob, off)[0]
            qs.append(blob[off + 8:off + 8 + k])
            off += 8 + k
        mine = answer_batch(qs) if answer_batch is not None else [self._answer(q) for q in qs]
        parts = self._gather_bytes(b"".join(struct.pack("<Q", len(r)) + r for r in mine))
        if parts is None:
            return None
        per_rank = []
        for blob_r in parts:
            rs, o = [], 0
            while o < len(blob_r):
                k = struct.unpack_from("<Q", blob_r, o)[0]
                rs.append(blob_r[o + 8:o + 8 + k])
                o += 8 + k
            per_rank.append(rs)
        return [merge_responses([rs[i] for rs in per_rank]) for i in range(n)]


# ---------------------------------------------------------------------------
# kernel-level building blocks on device buffers (pointers to device memory)
# ---------------------------------------------------------------------------
def ntt_batch(d_polys: int, count: int, limb: int, inverse: bool = False, device: int = 0, stream: int = 0):
    """in place: `count` polynomials of 2048 u64 coefficients of CRT limb `limb`"""
    _check(_ntt_batch(device, _vp(d_polys), count, limb, 1 if inverse else 0, _vp(stream)), "ntt_batch")


def automorph_batch(d_in: int, count: int, d_ks: int, nk: int, d_out: int, device: int = 0, stream: int = 0):
    """out[j][p] = NTT-domain automorphism x -> x^ks[j] of in[p] (ks: device u32 array)"""
    _check(_automorph_batch(device, _vp(d_in), count, _vp(d_ks), nk, _vp(d_out), _vp(stream)), "automorph_batch")


def encode_db(d_raw: int, d_encoded: int, db_rows: int, db_cols: int, interp: int, device: int = 0, stream: int = 0):
    """ipr_encode_db on device buffers: raw -> encoded u16 DB ([db_cols][db_rows])"""
    _check(_encode(device, _vp(d_raw), _vp(d_encoded), db_rows, db_cols, interp, _vp(stream)), "encode_db")


def cuckoo_to_raw_db(d_entries: int, d_occupied: int, num_buckets: int, entry_size: int, db_rows: int, db_cols: int,
                     per: int, d_raw: int, device: int = 0, stream: int = 0):
    """ipr_cuckoo_to_raw_db on device buffers"""
    _check(_raw_db(device, _vp(d_entries), _vp(d_occupied), num_buckets, entry_size, db_rows, db_cols, per,
                   _vp(d_raw), _vp(stream)), "cuckoo_to_raw_db")


# --- dataset generation and keyword-server setup from a dataset ------------------------------
# DatasetGenerator / Dataset (src/dataset/generator.rs:16-193, dataset.rs:20-46) and
# setup_keyword_server (src/dataset/keyword.rs:29-44) over the device generator
# ipr_dataset_generate and the device setup path.

KEM_PUBLIC_KEY_LEN = {"ml-kem-512": 800, "ml-kem-768": 1184, "ml-kem-1024": 1568}  # kem.rs:47-54
PUBLIC_KEY_ID_LEN = 32
PUBLIC_KEY_ID_DOMAIN = b"pq-key:v1:"
DEFAULT_DATASET_BATCH_SIZE = 100_000
# CuckooParams of build_cuckoo_table (server/keyword.rs:33-47; cuckoo.rs:29-31, 48-65)
DETERMINISTIC_SEED = bytes([0xDE, 0xAD, 0xBE, 0xEF, 0xCA, 0xFE, 0xBA, 0xBE,
                            0x01, 0x23, 0x45, 0x67, 0x89, 0xAB, 0xCD, 0xEF])
CUCKOO_NUM_HASHES = 2
CUCKOO_MAX_EVICTIONS = 500

_dataset_gen = _sig("ipr_dataset_generate", _i32, _i32, _i32, _u64, _u64, _u64, _vp, _vp)
_dataset_gen_host = _sig("ipr_dataset_generate_host", _i32, _i32, _i32, _u64, _u64, _u64, _vp)


def derive_public_key_id(public_key: bytes, kem_name: str) -> bytes:
    """SHA3-256(domain || kem_name || public_key) (dataset.rs:36-46)"""
    import hashlib
    return hashlib.sha3_256(PUBLIC_KEY_ID_DOMAIN + kem_name.encode() + bytes(public_key)).digest()


def public_key_matches_id(public_key_id: bytes, public_key: bytes, kem_name: str) -> bool:
    """dataset/keyword.rs:22-24"""
    return derive_public_key_id(public_key, kem_name) == bytes(public_key_id)


@dataclass
class DatasetRecord:
    public_key_id: bytes
    public_key: bytes


@dataclass
class Dataset:
    kem_name: str
    public_key_len: int
    records: List[DatasetRecord]


class DatasetGenerator:
    """DatasetGenerator (generator.rs:16-193): seeded ML-KEM public keys with their IDs,
    generated on the GPU (ipr_dataset_generate)."""

    def __init__(self, kem: str, count: int):
        if kem not in KEM_PUBLIC_KEY_LEN:
            raise ValueError(f"unknown KEM {kem!r}")
        self.kem, self.count, self.seed, self.batch_size = kem, count, 1, DEFAULT_DATASET_BATCH_SIZE

    def with_seed(self, seed: int) -> "DatasetGenerator":
        self.seed = seed
        return self

    def with_batch_size(self, batch_size: int) -> "DatasetGenerator":
        self.batch_size = batch_size
        return self

    @property
    def public_key_len(self) -> int:
        return KEM_PUBLIC_KEY_LEN[self.kem]

    @property
    def record_size(self) -> int:
        return PUBLIC_KEY_ID_LEN + self.public_key_len

    def _validate(self):  # generator.rs:150-164
        if self.count == 0:
            raise ValueError("count must be greater than zero")
        if self.batch_size == 0:
            raise ValueError("batch_size must be greater than zero")

    def generate_device(self, d_records: int, first: int = 0, count: Optional[int] = None, device: int = 0,
                        stream: int = 0):
        """records first .. first + count - 1 as id || pk rows into device memory"""
        n = self.count - first if count is None else count
        _check(_dataset_gen(device, int(self.kem.split("-")[-1]), self.seed, first, n, _vp(d_records), _vp(stream)),
               "ipr_dataset_generate")

    def generate_records(self, device: int = 0):
        """all records as one host array [count][32 + pk_len] (uint8), generated on the device
        (ipr_dataset_generate_host)"""
        import numpy as np
        self._validate()
        out = np.empty((self.count, self.record_size), dtype=np.uint8)
        _check(_dataset_gen_host(device, int(self.kem.split("-")[-1]), self.seed, 0, self.count, _vp(out.ctypes.data)),
               "ipr_dataset_generate_host")
        return out

    def generate_in_memory(self, device: int = 0) -> Dataset:
        """generate_in_memory (generator.rs:59-87): the whole dataset on the host; a duplicate
        id is an error, as in the reference"""
        rows = self.generate_records(device)
        ids = set()
        records = []
        for row in rows:
            rid, pk = row[:PUBLIC_KEY_ID_LEN].tobytes(), row[PUBLIC_KEY_ID_LEN:].tobytes()
            if rid in ids:
                raise ValueError("duplicate public key id generated")
            ids.add(rid)
            records.append(DatasetRecord(rid, pk))
        return Dataset(self.kem, self.public_key_len, records)


def build_cuckoo_table(keys: Sequence[bytes], values: Sequence[bytes], num_buckets: int, key_size: int,
                       value_size: int, seed: bytes = DETERMINISTIC_SEED, eviction_seed: int = 0):
    """build_cuckoo_table (server/keyword.rs:33-47) with CuckooTable::insert (cuckoo.rs:199-246):
    each record goes to its first free position of the two SipHash-2-4 positions, else
    evicts at a random hash position up to 500 times, else joins the stash.  The reference
    draws the eviction choice from the unseeded rand::rng(); here it is a seeded generator,
    so the table is reproducible.  Returns (entries [num_buckets][entry] uint8, occupied
    uint8 [num_buckets], stash list of entry bytes)."""
    import random
    import numpy as np
    es = key_size + value_size
    entries = np.zeros((num_buckets, es), dtype=np.uint8)
    occ = np.zeros(num_buckets, dtype=np.uint8)
    stash = []
    rng = random.Random(eviction_seed)

    def positions(k):
        return cuckoo_positions(seed, num_buckets, CUCKOO_NUM_HASHES, k)

    for key, value in zip(keys, values):
        entry = np.zeros(es, dtype=np.uint8)
        entry[:key_size] = np.frombuffer(bytes(key), dtype=np.uint8)
        entry[key_size:key_size + len(value)] = np.frombuffer(bytes(value), dtype=np.uint8)
        placed = False
        for p in positions(bytes(key)):
            if not occ[p]:
                entries[p], occ[p], placed = entry, 1, True
                break
        for _ in range(0 if placed else CUCKOO_MAX_EVICTIONS):
            p = positions(entry[:key_size].tobytes())[rng.randrange(CUCKOO_NUM_HASHES)]
            evicted = entries[p].copy()
            entries[p], occ[p] = entry, 1
            entry = evicted
            for q in positions(entry[:key_size].tobytes()):
                if not occ[q]:
                    entries[q], occ[q], placed = entry, 1, True
                    break
            if placed:
                break
        if not placed:
            stash.append(entry.tobytes())
    return entries, occ, stash


def setup_keyword_server(dataset: Dataset, buckets: Optional[int] = None, dim0: Optional[int] = None,
                         device: int = 0) -> "KeywordServer":
    """setup_keyword_server (dataset/keyword.rs:29-44): records (id -> public key) in a cuckoo
    table under DETERMINISTIC_SEED, its raw DB (to_raw_db, on the device), then
    KeywordServer::setup on the GPU (encode + offline precomputation)."""
    import torch
    plan = plan_from_shape(len(dataset.records), PUBLIC_KEY_ID_LEN, dataset.public_key_len, buckets, dim0)
    entries, occ, stash = build_cuckoo_table([r.public_key_id for r in dataset.records],
                                             [r.public_key for r in dataset.records], plan.num_items,
                                             PUBLIC_KEY_ID_LEN, dataset.public_key_len)
    dev = f"cuda:{device}"
    d_entries = torch.from_numpy(entries.reshape(-1)).to(dev)
    d_occ = torch.from_numpy(occ).to(dev)
    d_raw = torch.empty(plan.db_rows * plan.db_cols, dtype=torch.int16, device=dev)
    cuckoo_to_raw_db(d_entries.data_ptr(), d_occ.data_ptr(), plan.num_items, plan.entry_size, plan.db_rows,
                     plan.db_cols, plan.num_items // plan.db_rows, d_raw.data_ptr(), device=device)
    torch.cuda.synchronize(device)
    raw = d_raw.cpu().numpy().view("uint16")
    return KeywordServer.setup(plan, raw, raw=True, stash=stash, key_size=PUBLIC_KEY_ID_LEN,
                               value_size=dataset.public_key_len, num_records=len(dataset.records),
                               cuckoo_seed=DETERMINISTIC_SEED, device=device)
