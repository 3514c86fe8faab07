"""End to end through a real client: a query encrypted under a secret key
decrypts, after respond(), to the database values it asked for.

The reference pins respond() only this way (tests/e2e_mlkem.rs:8-39: the
client decrypts the right key); it has no golden response.  The client here
(oracle/pir_client.py) restates the reference client: ternary secret key,
scaled-Regev first-dimension query under the public seed, RGSW bodies under
RGSW_SEEDS, InspiRING packing keys, the wire format and the decryption after
the modulus switch.  A server whose packing keys, precomputation, fold or
switch were wrong in any step would not decrypt to the DB.

CPU tests run the oracle's respond() on a small server built from a raw DB
(encode and the offline precomputation included); GPU tests build the device
server from records (encode and offline precomputation on the device) at the
10k ML-KEM-768 shape and at the 1M benchmark shape, and decrypt single and
batch-64 answers.
"""
import numpy as np
import pytest

import pir_client as pc

N = 2048


def _entries(rng, buckets, entry_size, fill=0.9):
    """random entries with no aligned 0xFFFF pair (the plaintext modulus is 65535, so the
    DB value 0xFFFF reads back as 0), and the occupancy bitmap"""
    e = rng.integers(0, 256, (buckets, entry_size), dtype=np.uint8)
    pairs = e[:, :entry_size // 2 * 2].reshape(buckets, -1, 2)
    pairs[(pairs[..., 0] == 255) & (pairs[..., 1] == 255), 1] = 254
    occ = (rng.random(buckets) < fill).astype(np.uint8)
    return e, occ


def _check_plaintexts(cl, raw_cm, db_rows, db_cols, buckets, results):
    """every result of every sub-query equals the raw DB row it selects"""
    R = raw_cm.reshape(db_cols, db_rows)
    for b, r in zip(buckets, results):
        row, _, sub = cl.target(b)
        assert r.shape == (cl.c, N)
        for wp in range(cl.c):
            col0 = (wp * cl.interp + sub) * N
            np.testing.assert_array_equal(r[wp], R[col0:col0 + N, row].astype(np.uint64) % 65535,
                                          err_msg=f"bucket {b} group {wp}")


# --- CPU: the oracle server ----------------------------------------------------
SMALL = dict(db_rows=2048, instances=2, interp=2, c=1, per=6, item_elems=608, entry_size=1216)


@pytest.fixture(scope="module")
def small_server(orc):
    s = SMALL
    db_cols = s["instances"] * N
    rng = np.random.default_rng(2026)
    entries, occ = _entries(rng, s["db_rows"] * s["per"], s["entry_size"])
    raw = orc.raw_db(entries, occ, s["entry_size"], s["db_rows"], db_cols, s["per"])
    enc = orc.encode_db(raw, s["db_rows"], db_cols, s["interp"])
    a_hat, bt, btb, bth = orc.offline_precompute(enc, s["db_rows"], s["instances"])
    sdb = orc.SynthDB.__new__(orc.SynthDB)
    sdb.db_rows, sdb.instances, sdb.interp, sdb.c, sdb.seed = s["db_rows"], s["instances"], s["interp"], s["c"], 0
    sdb.db_cols, sdb.db = db_cols, enc
    sdb.a_hat, sdb.bold_t, sdb.bold_t_bar, sdb.bold_t_hat = (np.ascontiguousarray(x).reshape(-1)
                                                               for x in (a_hat, bt, btb, bth))
    sdb.stash, sdb._stash_buf = [], np.zeros(1, dtype=np.uint8)
    return sdb, raw, entries, occ


def _client(seed, s=SMALL):
    return pc.TestClient(s["db_rows"], s["interp"], s["c"], s["per"], s["item_elems"], seed=seed)


def test_oracle_response_decrypts_to_the_db(orc, small_server):
    sdb, raw, entries, occ = small_server
    cl = _client(11)
    per = SMALL["per"]
    # item 0 / 2 lie in DB polynomial 0 (sub-column 0), items 4 / 5 in polynomial 1
    buckets = [7 * per + 0, 1500 * per + 4, 2047 * per + 5, 3 * per + 2]
    q, _ = cl.query(buckets)
    assert len(q) == orc.query_bytes(SMALL["db_rows"], len(buckets))
    results, stash = cl.decrypt(orc.respond(sdb, q))
    assert stash == []
    _check_plaintexts(cl, raw, SMALL["db_rows"], sdb.db_cols, buckets, results)
    for b, r in zip(buckets, results):
        got = cl.extract(b, r)
        assert got == (entries[b].tobytes() if occ[b] else bytes(SMALL["entry_size"]))


def test_another_key_does_not_decrypt(orc, small_server):
    """control: the same response under a different secret key is noise"""
    sdb, raw, _, _ = small_server
    cl, other = _client(12), _client(13)
    b = 100 * SMALL["per"] + 1
    q, _ = cl.query([b])
    resp = orc.respond(sdb, q)
    row, _, sub = cl.target(b)
    want = raw.reshape(sdb.db_cols, SMALL["db_rows"])[sub * N:(sub + 1) * N, row].astype(np.uint64) % 65535
    assert np.array_equal(cl.decrypt(resp)[0][0][0], want)
    assert np.count_nonzero(other.decrypt(resp)[0][0][0] == want) < 16


def test_client_bytes_match_the_package_serializer(pkg):
    cl = _client(14)
    q, f = cl.query([5, 6000])
    p = pkg.KeywordQueryPayload(f["y_body"], f["z_body"], [(r, g) for r, g in f["queries"]])
    assert pkg.serialize_keyword_query(p) == q


# --- GPU: the device server built from records ----------------------------------
@pytest.fixture(scope="module")
def config0(pkg, orc):
    plan = pkg.plan_from_shape(10_000, 32, 1184)
    assert (plan.db_rows, plan.db_cols, plan.instances, plan.interp, plan.c) == (2048, 16384, 8, 8, 1)
    per = plan.num_items // plan.db_rows
    rng = np.random.default_rng(7)
    entries, occ = _entries(rng, plan.num_items, plan.entry_size, fill=10_000 / plan.num_items)
    raw = orc.raw_db(entries, occ, plan.entry_size, plan.db_rows, plan.db_cols, per)
    srv = pkg.KeywordServer.setup(plan, raw, raw=True, key_size=32, value_size=1184, num_records=int(occ.sum()))
    yield plan, per, raw, entries, occ, srv
    srv.close()


@pytest.mark.gpu
def test_device_response_decrypts_to_the_entry(config0):
    plan, per, raw, entries, occ, srv = config0
    cl = pc.TestClient(plan.db_rows, plan.interp, plan.c, per, plan.item_size_bits // 16, seed=21)
    occupied = np.flatnonzero(occ)
    # two positions as the keyword client sends them; entries inside one DB polynomial
    buckets = [int(b) for b in occupied if (b % per) * 608 % N + 608 <= N][:2]
    q, _ = cl.query(buckets)
    results, stash = cl.decrypt(srv.respond_to_serialized_query(q))
    _check_plaintexts(cl, raw, plan.db_rows, plan.db_cols, buckets, results)
    for b, r in zip(buckets, results):
        entry = cl.extract(b, r)
        assert entry == entries[b].tobytes()
        assert entry[32:32 + 1184] == entries[b, 32:1216].tobytes()  # the value after the 32-byte key


@pytest.mark.gpu
def test_device_batch_of_distinct_clients_decrypts(config0):
    plan, per, raw, entries, occ, srv = config0
    rng = np.random.default_rng(5)
    clients = [pc.TestClient(plan.db_rows, plan.interp, plan.c, per, 608, seed=100 + i) for i in range(16)]
    asks = [[int(x) for x in rng.integers(0, plan.num_items, 2)] for _ in clients]
    qs = [cl.query(b)[0] for cl, b in zip(clients, asks)]
    for cl, b, resp in zip(clients, asks, srv.respond_batch(qs)):
        _check_plaintexts(cl, raw, plan.db_rows, plan.db_cols, b, cl.decrypt(resp)[0])


@pytest.mark.gpu
def test_batch_of_64_decrypts_at_1m(pkg):
    """the benchmark configuration: 1M ML-KEM-768 records (buckets 2^21, dim0 2048), the
    server set up on the device from a raw DB, 64 distinct clients in one batched pass"""
    plan = pkg.plan_from_shape(1_000_000, 32, 1184, 2_097_152, 2048)
    assert (plan.db_rows, plan.db_cols, plan.instances, plan.interp, plan.c) == (2048, 720896, 352, 32, 11)
    per = plan.num_items // plan.db_rows
    raw = np.random.default_rng(1).integers(0, 65535, plan.db_rows * plan.db_cols, dtype=np.uint16)
    with pkg.KeywordServer.setup(plan, raw, raw=True, num_records=1_000_000) as srv:
        rng = np.random.default_rng(64)
        clients = [pc.TestClient(plan.db_rows, plan.interp, plan.c, per, 608, seed=500 + i) for i in range(64)]
        asks = [[int(x) for x in rng.integers(0, plan.num_items, 2)] for _ in clients]
        qs = [cl.query(b)[0] for cl, b in zip(clients, asks)]
        batch = srv.respond_batch(qs)
    for cl, b, resp in zip(clients, asks, batch):
        _check_plaintexts(cl, raw, plan.db_rows, plan.db_cols, b, cl.decrypt(resp)[0])


@pytest.mark.gpu
def test_service_state_file_and_shards_decrypt(pkg, orc, tmp_path):
    """the other public entry points answer decryptably too: the serving API, a server
    reloaded from its state file, and two fold-group shards whose parts are merged"""
    plan = pkg.Plan(num_items=8 * 2048, entry_size=1216, item_size_bits=9728, dim0=2048, db_rows=2048,
                    db_cols=4 * N, instances=4, interp=2, c=2, peak_bytes=0)
    per = 8
    rng = np.random.default_rng(77)
    entries, occ = _entries(rng, plan.num_items, plan.entry_size)
    raw = orc.raw_db(entries, occ, plan.entry_size, plan.db_rows, plan.db_cols, per)
    clients = [pc.TestClient(plan.db_rows, plan.interp, plan.c, per, 608, seed=900 + i) for i in range(3)]
    asks = [[1 * per + 0, 2047 * per + 7], [600 * per + 4], [9 * per + 3, 10 * per + 5, 11 * per + 1]]
    qs = [cl.query(b)[0] for cl, b in zip(clients, asks)]

    def check(answers):
        for cl, b, resp in zip(clients, asks, answers):
            _check_plaintexts(cl, raw, plan.db_rows, plan.db_cols, b, cl.decrypt(resp)[0])

    path = str(tmp_path / "real.state")
    with pkg.KeywordServer.setup(plan, raw, raw=True) as srv:
        check([srv.respond_to_serialized_query(q) for q in qs])
        with pkg.KeywordService([srv], max_batch=4) as svc:
            check([svc.wait(t) for t in svc.submit_many(0, qs)])
        srv.save(path)
    with pkg.KeywordServer.load(path) as loaded:
        check(loaded.respond_batch(qs))
    parts = []
    for k in range(2):
        sub, sl = pkg.shard_slices(plan, 2, k)
        lo, hi = sl["db"]
        with pkg.KeywordServer.setup(sub, raw[lo:hi], raw=True) as shard:
            parts.append([shard.respond_to_serialized_query(q) for q in qs])
    check([pkg.merge_responses([parts[0][i], parts[1][i]]) for i in range(len(qs))])


# --- InspiRING packing: packed LWEs decrypt to their messages ------------------------
def _lwes_of_rlwe(cl, msgs):
    """2048 LWE ciphertexts from one RLWE encryption of sum_j scale_k m_j X^j, the public
    polynomial from ChaCha20Rng([2; 32]) as in test_packing_inspir (packing.rs:3428-3526):
    rlwe_to_lwe (client/online.rs:18-24) -> [N + 1][N], column j = the LWE of coefficient j
    (rows: the negacyclic matrix of row 0 = -a, then the b row)"""
    Q = pc.Q
    a = pc._o.random_raw(bytes([2] * 32), N)
    msg = (np.asarray(msgs, dtype=np.uint64) * np.uint64(pc.SCALE_K)) % np.uint64(Q)
    b = pc.from_ntt(pc.ntt_add(pc.to_ntt(cl.noise_raw()), pc.ntt_mul(cl.s_ntt, pc.to_ntt(a)), pc.to_ntt(msg)))
    row0 = (np.uint64(Q) - a) % np.uint64(Q)
    r, j = np.arange(N)[:, None], np.arange(N)[None, :]
    m = row0[(j - r) % N]
    wrap = j < r
    m[wrap] = (np.uint64(Q) - m[wrap]) % np.uint64(Q)
    return np.ascontiguousarray(np.vstack([m, b[None, :]]))


def _decrypt_rlwe(cl, packed):
    """decrypt_matrix_reg + rescale to 65535 of an RLWE [2][N] raw (row 1 may be < 2q)"""
    p0, p1 = (np.asarray(packed[k], dtype=np.uint64) % np.uint64(pc.Q) for k in (0, 1))
    dec = pc.from_ntt(pc.ntt_add(pc.ntt_mul(cl.s_ntt, pc.to_ntt(p0)), pc.to_ntt(p1)))
    return pc._o.rescale_many(dec, pc.Q, pc.P)


def _packing_keys_condensed(cl):
    y, z = cl.packing_keys()
    return (np.stack([pc.condense(y[k]) for k in range(3)]), np.stack([pc.condense(z[k]) for k in range(3)]))


def test_oracle_inspiring_pack_decrypts(orc):
    """test_packing_inspir (packing.rs:3428-3526) with all 2048 LWEs packed (packing_fully_online,
    full keys): the packed RLWE decrypts to every message"""
    cl = _client(31)
    msgs = (np.arange(N, dtype=np.uint64) * 7919) % 65535
    y, z = _packing_keys_condensed(cl)
    packed = orc.inspiring_pack(_lwes_of_rlwe(cl, msgs), y, z)
    np.testing.assert_array_equal(_decrypt_rlwe(cl, packed), msgs)


@pytest.mark.gpu
def test_device_inspiring_pack_decrypts(pkg):
    """ipr_inspiring_pack of two sets of 2048 LWEs under one client's keys (a call takes one
    key pair): each packed RLWE decrypts to its set's messages"""
    import torch
    sets = 2
    cl = _client(40)
    rng = np.random.default_rng(8)
    msgs = [rng.integers(0, 65535, N, dtype=np.uint64) for _ in range(sets)]
    y, z = _packing_keys_condensed(cl)
    lwe = np.stack([_lwes_of_rlwe(cl, m) for m in msgs])
    d_lwe = torch.from_numpy(lwe.view(np.int64)).cuda()
    d_y = torch.from_numpy(y.view(np.int64)).cuda()
    d_z = torch.from_numpy(z.view(np.int64)).cuda()
    d_out = torch.zeros((sets, 2, N), dtype=torch.int64, device="cuda")
    with pkg.InspiringPacker(max_sets=sets) as pk:
        pk.pack(sets, d_lwe.data_ptr(), d_y.data_ptr(), d_z.data_ptr(), d_out.data_ptr())
        torch.cuda.synchronize()
    got = d_out.cpu().numpy().view(np.uint64)
    for c in range(sets):
        np.testing.assert_array_equal(_decrypt_rlwe(cl, got[c]), msgs[c])
