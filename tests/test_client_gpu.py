"""The keyword-PIR client on the GPU (ipr_client_*, KeywordClient).

The device client draws its key and noise deterministically from its seed, so
its query bytes must equal, bit for bit, those of the oracle's model of the
same client (`pir_client.SeededClient`: the reference client's query
construction, client/keyword.rs:137-214, with the same key shuffle and noise
streams).  Its decryption must equal the model's decryption of the same
response bytes and the database rows the queries select.  The answering server
is the device library's, built from a raw DB on the device.
"""
import numpy as np
import pytest

import pir_client as pc

N = 2048
SEED = bytes(range(1, 33))


def test_model_key_and_noise(orc):
    """the model's key has 256 entries +1 and 256 entries -1; its noise has sigma ~ 6.4"""
    cl = pc.SeededClient(2048, 8, 1, 16, 608, seed=SEED)
    assert (cl.s == 1).sum() == 256 and (cl.s == -1).sum() == 256
    cl.query([3], nonce=1)
    assert abs(cl._noise.std() - 6.4) < 0.1 and np.abs(cl._noise).max() <= 82
    other = pc.SeededClient(2048, 8, 1, 16, 608, seed=SEED)
    other.query([3], nonce=2)
    assert not np.array_equal(other._noise, cl._noise)  # a fresh nonce draws fresh noise


def _small_plan(pkg, db_rows=2048, instances=2, interp=2, per=6):
    return pkg.Plan(num_items=db_rows * per, entry_size=1216, item_size_bits=9728, dim0=db_rows, db_rows=db_rows,
                    db_cols=instances * N, instances=instances, interp=interp, c=instances // interp, peak_bytes=0)


@pytest.mark.gpu
@pytest.mark.parametrize("shape", ["10k", "rows4096"])
def test_device_query_bytes_equal_model(pkg, shape):
    if shape == "10k":
        plan = pkg.plan_from_shape(10_000, 32, 1184)
    else:  # two first-dimension polynomials per sub-query
        plan = _small_plan(pkg, db_rows=4096, instances=4, interp=2, per=4)
    per = plan.num_items // plan.db_rows
    model = pc.SeededClient(plan.db_rows, plan.interp, plan.c, per, 608, seed=SEED)
    with pkg.KeywordClient(plan, SEED) as dev:
        assert np.array_equal(dev.secret_key(), model.s)
        for nonce, buckets in ((0, [5, plan.num_items - 1]), (9, [plan.num_items // 2]),
                               (3, [1, 2 * per + 4, 7 * per + 3])):
            got = dev.query(buckets, nonce=nonce)
            want, _ = model.query(buckets, nonce=nonce)
            assert len(got) == pkg.query_bytes(plan.db_rows, len(buckets))
            assert got == want, (nonce, buckets)


@pytest.mark.gpu
def test_device_client_round_trip(pkg, orc):
    """device client -> device server (set up from a raw DB on the device) -> device
    decryption: equal to the model's decryption and to the DB rows, and extract returns
    the entries"""
    plan = pkg.plan_from_shape(10_000, 32, 1184)
    per = plan.num_items // plan.db_rows
    rng = np.random.default_rng(12)
    entries = rng.integers(0, 256, (plan.num_items, plan.entry_size), dtype=np.uint8)
    pairs = entries[:, :plan.entry_size // 2 * 2].reshape(plan.num_items, -1, 2)
    pairs[(pairs[..., 0] == 255) & (pairs[..., 1] == 255), 1] = 254  # no DB value 0xFFFF (= 0 mod 65535)
    occ = np.ones(plan.num_items, dtype=np.uint8)
    raw = orc.raw_db(entries, occ, plan.entry_size, plan.db_rows, plan.db_cols, per)
    R = raw.reshape(plan.db_cols, plan.db_rows)
    buckets = [0 * per + 1, 1234 * per + 2, 2047 * per + 4]  # items inside one DB polynomial
    model = pc.SeededClient(plan.db_rows, plan.interp, plan.c, per, 608, seed=SEED)
    with pkg.KeywordServer.setup(plan, raw, raw=True) as srv, pkg.KeywordClient(plan, SEED) as dev:
        q = dev.query(buckets, nonce=4)
        resp = srv.respond_to_serialized_query(q)
        got = dev.decrypt(resp)
    want = model.decrypt(resp)[0]
    assert got.shape == (3, plan.c, N)
    for k, b in enumerate(buckets):
        np.testing.assert_array_equal(got[k], want[k])
        row, col, sub = model.target(b)
        np.testing.assert_array_equal(got[k][0], R[sub * N:(sub + 1) * N, row])
        assert dev.extract(b, got[k]) == entries[b].tobytes()


@pytest.mark.gpu
def test_device_clients_batch_of_64_at_1m(pkg):
    """64 device clients, one batched pass of the 1M server set up from a raw DB, 64
    device decryptions: every result of every client equals the DB row it selects"""
    plan = pkg.plan_from_shape(1_000_000, 32, 1184, 2_097_152, 2048)
    per = plan.num_items // plan.db_rows
    raw = np.random.default_rng(3).integers(0, 65535, plan.db_rows * plan.db_cols, dtype=np.uint16)
    R = raw.reshape(plan.db_cols, plan.db_rows)
    rng = np.random.default_rng(99)
    asks = [[int(x) for x in rng.integers(0, plan.num_items, 2)] for _ in range(64)]
    clients = [pkg.KeywordClient(plan, bytes([i]) * 32) for i in range(64)]
    try:
        qs = [cl.query(b) for cl, b in zip(clients, asks)]
        with pkg.KeywordServer.setup(plan, raw, raw=True) as srv:
            batch = srv.respond_batch(qs)
        for cl, b, resp in zip(clients, asks, batch):
            pt = cl.decrypt(resp)
            for k, bucket in enumerate(b):
                row = bucket // per
                sub = ((bucket % per) * 608 % (plan.interp * N)) // N
                for w in range(plan.c):
                    c0 = (w * plan.interp + sub) * N
                    np.testing.assert_array_equal(pt[k][w], R[c0:c0 + N, row])
    finally:
        for cl in clients:
            cl.close()


@pytest.mark.gpu
def test_device_client_refuses_bad_input(pkg):
    plan = pkg.plan_from_shape(10_000, 32, 1184)
    with pkg.KeywordClient(plan, SEED) as dev:
        with pytest.raises(pkg.IprError) as e:
            dev.query([plan.num_items])  # bucket out of range
        assert e.value.status == -1
        with pytest.raises(pkg.IprError) as e:
            dev.decrypt(b"\x01\x00\x00\x00\x05\x00\x00\x00abcde")  # a result of the wrong length
        assert e.value.status == -5
        assert dev.decrypt(b"\x00\x00\x00\x00\x00\x00\x00\x00").shape == (0, plan.c, N)


@pytest.mark.gpu
def test_device_client_zero_queries_and_stash(pkg, orc):
    """a payload of keys only (0 sub-queries) equals the model's and gets an empty answer;
    a response with a stash block decrypts its results and leaves the stash to the caller"""
    plan = _small_plan(pkg)
    per = plan.num_items // plan.db_rows
    raw = np.random.default_rng(4).integers(0, 65535, plan.db_rows * plan.db_cols, dtype=np.uint16)
    stash = [bytes([i]) * plan.entry_size for i in (1, 2, 3)]
    model = pc.SeededClient(plan.db_rows, plan.interp, plan.c, per, 608, seed=SEED)
    with pkg.KeywordServer.setup(plan, raw, raw=True, stash=stash) as srv, pkg.KeywordClient(plan, SEED) as dev:
        q0 = dev.query([], nonce=11)
        assert q0 == model.query([], nonce=11)[0] and len(q0) == pkg.query_bytes(plan.db_rows, 0)
        r0 = srv.respond_to_serialized_query(q0)
        assert pkg.deserialize_keyword_response(r0).responses == []
        assert dev.decrypt(r0).shape == (0, plan.c, N)
        b = 321 * per + 4
        resp = srv.respond_to_serialized_query(dev.query([b], nonce=12))
    assert pkg.deserialize_keyword_response(resp).stash_entries == stash
    with pkg.KeywordClient(plan, SEED) as dev2:  # the same seed decrypts the same key's answers
        pt = dev2.decrypt(resp)
    row, _, sub = model.target(b)
    np.testing.assert_array_equal(pt[0][0], raw.reshape(plan.db_cols, plan.db_rows)[sub * N:(sub + 1) * N, row])


# --- keyword lookup: cuckoo positions, query by ID, extract the value --------------------------
def test_siphash_paper_vectors():
    """SipHash-2-4 of the paper (Aumasson, Bernstein 2012), key 00..0f: the empty message and the
    15-byte message 00..0e"""
    k0, k1 = int.from_bytes(bytes(range(8)), "little"), int.from_bytes(bytes(range(8, 16)), "little")
    assert pc.siphash24(k0, k1, b"") == 0x726FDB47DD0E0E31
    assert pc.siphash24(k0, k1, bytes(range(15))) == 0xA129CA6149BE45E5


def test_library_positions_equal_oracle(pkg):
    rng = np.random.default_rng(8)
    for seed in (bytes(16), bytes(range(16)), bytes(rng.integers(0, 256, 16, dtype=np.uint8))):
        for klen in (0, 5, 8, 16, 32, 33):
            for _ in range(4):
                key = bytes(rng.integers(0, 256, klen, dtype=np.uint8))
                for nb in (2, 32768, 2_097_152):
                    assert pkg.cuckoo_positions(seed, nb, 2, key) == pc.cuckoo_positions(seed, nb, 2, key)
    assert pkg.cuckoo_positions(bytes(range(16)), 1000, 3, b"abc") == pc.cuckoo_positions(bytes(range(16)), 1000, 3,
                                                                                         b"abc")


def _no_ffff(b):
    a = np.frombuffer(bytearray(b), dtype=np.uint8).copy()
    pairs = a[:len(a) // 2 * 2].reshape(-1, 2)
    pairs[(pairs[:, 0] == 255) & (pairs[:, 1] == 255), 1] = 254  # 0xFFFF reads back as 0 mod 65535
    return a.tobytes()


@pytest.mark.gpu
def test_keyword_lookup_end_to_end(pkg, orc):
    """the reference's end-to-end property (tests/e2e_mlkem.rs: the client retrieves the right
    key): records placed in a cuckoo layout under a non-trivial seed (or in the stash), the
    server set up on the device, and a device client that queries by 32-byte ID and extracts
    the 1184-byte value, or None for an absent ID"""
    plan = pkg.plan_from_shape(10_000, 32, 1184)
    per, es = plan.num_items // plan.db_rows, plan.entry_size
    cseed = bytes(range(100, 116))
    rng = np.random.default_rng(2026)
    entries = np.zeros((plan.num_items, es), dtype=np.uint8)
    occ = np.zeros(plan.num_items, dtype=np.uint8)
    placed, stash = {}, []

    def inside(b):  # the entry lies in one DB polynomial, so one result holds all of it
        return (b % per) * 608 % N + 608 <= N
    while len(placed) < 300:
        key, value = _no_ffff(rng.bytes(32)), _no_ffff(rng.bytes(1184))
        pos = pc.cuckoo_positions(cseed, plan.num_items, 2, key)
        free = [p for p in pos if not occ[p] and inside(p)]
        if free:
            entries[free[0], :32], entries[free[0], 32:1216] = np.frombuffer(key, np.uint8), np.frombuffer(value,
                                                                                                           np.uint8)
            occ[free[0]] = 1
            placed[key] = value
        elif len(stash) < 3:
            stash.append(key + value + bytes(es - 1216))
            placed[key] = value
    raw = orc.raw_db(entries, occ, es, plan.db_rows, plan.db_cols, per)
    with pkg.KeywordServer.setup(plan, raw, raw=True, stash=stash, key_size=32, value_size=1184,
                                 num_records=len(placed), cuckoo_seed=cseed) as srv:
        pp = srv.public_params()
        assert bytes(pp["keyword_pir"]["cuckoo_seed"]) == cseed
        with pkg.KeywordClient.from_public_params(pp, bytes([9]) * 32) as cl:
            keys = list(placed)[:6] + [s[:32] for s in stash]
            for key in keys:
                pos, q = cl.query_key(key)
                assert pos == pc.cuckoo_positions(cseed, plan.num_items, 2, key)
                assert cl.extract_key(key, pos, srv.respond_to_serialized_query(q)) == placed[key]
            absent = _no_ffff(rng.bytes(32))
            pos, q = cl.query_key(absent)
            assert cl.extract_key(absent, pos, srv.respond_to_serialized_query(q)) is None


def test_public_params_are_validated_before_any_device_work(pkg):
    """setup_from_public_params (keyword.rs:64-79): keyword mode, non-zero sizes, entry size"""
    base = {"num_items": 32768, "item_size_bits": 9728, "dim0": 2048,
            "keyword_pir": {"cuckoo_seed": list(range(16)), "num_hashes": 2, "key_size": 32, "value_size": 1184,
                            "entry_size": 1216, "num_records": 10000}}
    for bad in ({"keyword_pir": None}, {"keyword_pir": dict(base["keyword_pir"], key_size=0)},
                {"keyword_pir": dict(base["keyword_pir"], value_size=0)},
                {"keyword_pir": dict(base["keyword_pir"], entry_size=1000)}, {"item_size_bits": 4096}):
        with pytest.raises(ValueError):
            pkg.KeywordClient.from_public_params(dict(base, **bad), bytes(32))
