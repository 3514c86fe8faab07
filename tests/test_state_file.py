"""Server state file (ipr_server_save / ipr_server_load / ipr_state_file_plan).

The format is restated here in NumPy (header struct, section order and
alignment, the splitmix64-keyed checksum) independently of the C writer:
CPU tests hand-build files with it and check that the library reads the header
and refuses every malformed file before touching a GPU; GPU tests check that a
saved file holds exactly the arrays the server was built from, under checksums
this restatement computes, and that a loaded server answers byte for byte like
the saved one.
"""
import os
import struct

import numpy as np
import pytest

N = 2048
NINNER = 3069
HDR = 4096
MAGIC = b"IPRSTATE"
# magic, version, header_bytes, plan[10], key/value size, records, stash count/entry,
# cuckoo seed, 6 x {offset, bytes, checksum, reserved}, header checksum
FMT = "<8sII10Q5Q16s24QQ"
CK_OFF = struct.calcsize(FMT) - 8
POS_KEY = np.uint64(0x9E3779B97F4A7C15)
SECTIONS = ("db", "a_hat", "bold_t", "bold_t_bar", "bold_t_hat", "stash")


def mix64(x):
    x = x ^ (x >> np.uint64(30))
    x = x * np.uint64(0xBF58476D1CE4E5B9)
    x = x ^ (x >> np.uint64(27))
    x = x * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def checksum(b: bytes) -> int:
    b = bytes(b) + bytes(-len(b) % 8)
    w = np.frombuffer(b, dtype="<u8")
    i = np.arange(w.size, dtype=np.uint64)
    with np.errstate(over="ignore"):
        return int(np.sum(mix64(w + i * POS_KEY), dtype=np.uint64))


def align(x):
    return (x + HDR - 1) // HDR * HDR


def section_bytes(plan, stash_bytes):
    no = plan[6]
    return [plan[4] * plan[5] * 2, no * N * 8, no * NINNER * N * 8, no * NINNER * N * 8, no * 3 * N * 8,
            stash_bytes]


def build_header(plan, sections, key_size=32, value_size=1184, records=10, stash_count=0, stash_entry=0,
                 seed=bytes(range(16)), version=1, checksums=None):
    off, table = HDR, []
    for k, n in enumerate(sections):
        ck = 0 if checksums is None else checksums[k]
        table += [off, n, ck, 0]
        off = align(off + n)
    fields = [MAGIC, version, HDR, *plan, key_size, value_size, records, stash_count, stash_entry, seed, *table, 0]
    raw = struct.pack(FMT, *fields)
    raw = raw[:CK_OFF] + struct.pack("<Q", checksum(raw[:CK_OFF]))
    return raw + bytes(HDR - len(raw)), off


def parse_header(block):
    v = struct.unpack(FMT, block[:struct.calcsize(FMT)])
    plan = list(v[3:13])
    sec = [v[19 + 4 * k: 23 + 4 * k] for k in range(6)]
    return {"magic": v[0], "version": v[1], "plan": plan, "key_size": v[13], "value_size": v[14],
            "num_records": v[15], "stash_count": v[16], "stash_entry": v[17], "seed": v[18], "sec": sec,
            "header_checksum": v[-1]}


# a small plan: 2 packing outputs, interpolation 2, one fold group
PLAN = [32768, 1216, 9728, 2048, 2048, 2 * N, 2, 2, 1, 0]


def _status(pkg, fn, *a):
    try:
        fn(*a)
    except pkg.IprError as e:
        return e.status
    return 0


def test_header_round_trip_without_gpu(pkg, tmp_path):
    hdr, _ = build_header(PLAN, section_bytes(PLAN, 0))
    p = tmp_path / "h.state"
    p.write_bytes(hdr)
    plan = pkg.state_file_plan(str(p))
    assert [getattr(plan, f) for f in ("num_items", "entry_size", "item_size_bits", "dim0", "db_rows", "db_cols",
                                       "instances", "interp", "c", "peak_bytes")] == PLAN


def test_malformed_headers_are_refused(pkg, tmp_path):
    good, _ = build_header(PLAN, section_bytes(PLAN, 0))
    cases = {
        "magic": b"IPRSTATX" + good[8:],
        "version": good[:8] + struct.pack("<I", 2) + good[12:],
        "checksum": good[:100] + bytes([good[100] ^ 1]) + good[101:],
        "short": good[:200],
    }
    for name, blob in cases.items():
        p = tmp_path / f"{name}.state"
        p.write_bytes(blob)
        assert _status(pkg, pkg.state_file_plan, str(p)) == -5, name  # IPR_E_FORMAT
    assert _status(pkg, pkg.state_file_plan, str(tmp_path / "missing.state")) == -9  # IPR_E_IO


def test_load_refuses_bad_tables_before_the_gpu(pkg, tmp_path):
    """every refusal here happens before the loader allocates on a device"""
    secs = section_bytes(PLAN, 0)
    # a section table that disagrees with the plan
    bad = list(secs)
    bad[2] -= 8
    hdr, end = build_header(PLAN, bad)
    p = tmp_path / "table.state"
    p.write_bytes(hdr)
    assert _status(pkg, pkg.KeywordServer.load, str(p)) == -5
    # a right table in a file of the wrong size (truncated)
    hdr, end = build_header(PLAN, secs)
    p = tmp_path / "trunc.state"
    with open(p, "wb") as f:
        f.write(hdr)
        f.truncate(end - HDR)
    assert _status(pkg, pkg.KeywordServer.load, str(p)) == -5
    # an implausible plan (db_cols not instances * 2048)
    plan = list(PLAN)
    plan[5] += 1
    hdr, _ = build_header(plan, secs)
    p = tmp_path / "plan.state"
    p.write_bytes(hdr)
    assert _status(pkg, pkg.KeywordServer.load, str(p)) == -5
    # a stash whose checksum does not match
    st = bytes(range(40))
    hdr, end = build_header(PLAN, section_bytes(PLAN, len(st)), stash_count=2, stash_entry=20,
                            checksums=[0] * 5 + [checksum(st) ^ 1])
    p = tmp_path / "stash.state"
    with open(p, "wb") as f:
        f.write(hdr)
        f.truncate(end)
        f.seek(end - align(len(st)))
        f.write(st)
    assert _status(pkg, pkg.KeywordServer.load, str(p)) == -5


def test_checksum_sees_position_and_padding():
    a = np.arange(64, dtype=np.uint64).tobytes()
    b = np.roll(np.arange(64, dtype=np.uint64), 1).tobytes()
    assert checksum(a) != checksum(b)             # same words, other positions
    assert checksum(b"\x01") == checksum(b"\x01" + bytes(7))
    assert checksum(b"") == 0


def _server(pkg, orc, seed):
    plan = pkg.Plan(*PLAN)
    stash = [bytes([i]) * 1216 for i in (3, 9)]
    sdb = orc.SynthDB(plan.db_rows, plan.instances, plan.interp, plan.c, seed=seed, stash=stash)
    srv = pkg.KeywordServer.from_encoded(plan, sdb.db, sdb.a_hat, sdb.bold_t, sdb.bold_t_bar, sdb.bold_t_hat,
                                         stash=stash, num_records=10, cuckoo_seed=bytes(range(16)))
    return plan, sdb, stash, srv


@pytest.mark.gpu
def test_saved_file_holds_the_setup_arrays(pkg, orc, tmp_path):
    plan, sdb, stash, srv = _server(pkg, orc, 91)
    p = str(tmp_path / "s.state")
    with srv:
        srv.save(p)
    data = open(p, "rb").read()
    h = parse_header(data[:HDR])
    assert h["magic"] == MAGIC and h["version"] == 1
    assert h["plan"] == PLAN
    assert (h["key_size"], h["value_size"], h["num_records"]) == (32, 1184, 10)
    assert (h["stash_count"], h["stash_entry"], h["seed"]) == (2, 1216, bytes(range(16)))
    assert h["header_checksum"] == checksum(data[:CK_OFF])
    want = [np.ascontiguousarray(sdb.db, dtype=np.uint16).tobytes(),
            np.ascontiguousarray(sdb.a_hat, dtype=np.uint64).tobytes(),
            np.ascontiguousarray(sdb.bold_t, dtype=np.uint64).tobytes(),
            np.ascontiguousarray(sdb.bold_t_bar, dtype=np.uint64).tobytes(),
            np.ascontiguousarray(sdb.bold_t_hat, dtype=np.uint64).tobytes(),
            b"".join(stash)]
    off = HDR
    for k, (o, n, ck, _) in enumerate(h["sec"]):
        assert (o, n) == (off, len(want[k])), SECTIONS[k]
        assert data[o:o + n] == want[k], SECTIONS[k]
        assert ck == checksum(want[k]), SECTIONS[k]
        off = align(off + n)
    assert len(data) == off


@pytest.mark.gpu
def test_loaded_server_answers_like_the_saved_one(pkg, orc, tmp_path):
    plan, sdb, stash, srv = _server(pkg, orc, 92)
    p = str(tmp_path / "s.state")
    q = orc.synth_query(17, plan.db_rows, 2)
    with srv:
        want = srv.respond_to_serialized_query(q)
        params = srv.public_params()
        srv.save(p)
    assert want == orc.respond(sdb, q)
    with pkg.KeywordServer.load(p) as loaded:
        assert loaded.plan == plan
        assert loaded.public_params() == params
        assert loaded.respond_to_serialized_query(q) == want
        assert loaded.respond_batch([q, q]) == [want, want]
        # a loaded server saves the same file again
        p2 = str(tmp_path / "s2.state")
        loaded.save(p2)
    assert open(p, "rb").read() == open(p2, "rb").read()


@pytest.mark.gpu
def test_corrupt_section_is_refused(pkg, orc, tmp_path):
    plan, sdb, stash, srv = _server(pkg, orc, 93)
    p = str(tmp_path / "s.state")
    with srv:
        srv.save(p)
    h = parse_header(open(p, "rb").read(HDR))
    for k in (0, 2, 4):  # db, bold_t, bold_t_hat: checked on the device after upload
        o, n = h["sec"][k][0], h["sec"][k][1]
        with open(p, "r+b") as f:
            f.seek(o + n // 2)
            b = f.read(1)
            f.seek(o + n // 2)
            f.write(bytes([b[0] ^ 0x10]))
        with pytest.raises(pkg.IprError) as ei:
            pkg.KeywordServer.load(p)
        assert ei.value.status == -5 and SECTIONS[k] in str(ei.value)
        with open(p, "r+b") as f:  # restore for the next case
            f.seek(o + n // 2)
            f.write(b)
    with pkg.KeywordServer.load(p):
        pass
