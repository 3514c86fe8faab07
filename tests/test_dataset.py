"""Dataset generation (DatasetGenerator, src/dataset/generator.rs:24-193) and a keyword
server set up from a generated dataset.

CPU: the oracle's FIPS 202 hashes equal hashlib's, its FIPS 203 encapsulation keys equal
those of an independent ML-KEM implementation (pyca/cryptography, from the same 64-byte
seed d || z), its records carry the SHA3-256 IDs of dataset.rs:36-46, and the host logic of
the cuckoo build places every record where a lookup finds it.
GPU: the device generator's records equal the oracle's for ML-KEM-512/-768/-1024, and the
reference's own end-to-end test (tests/e2e_mlkem.rs:8-39) passes through this library: a
10,000-key ML-KEM-768 dataset with seed 7, setup_keyword_server, a client that queries one
record's ID and extracts exactly its public key, whose ID matches.
"""
import hashlib

import numpy as np
import pytest

import pir_client as pc

KEMS = ("ml-kem-512", "ml-kem-768", "ml-kem-1024")


def test_oracle_hashes_match_hashlib(orc):
    rng = np.random.default_rng(3)
    for n in list(range(0, 210)) + [271, 272, 273, 1000, 1203, 1204, 1205, 1577]:
        m = rng.bytes(n)
        assert orc.sha3_256(m) == hashlib.sha3_256(m).digest()
        assert orc.sha3_512(m) == hashlib.sha3_512(m).digest()
        assert orc.shake128(m, 505) == hashlib.shake_128(m).digest(505)
        assert orc.shake256(m, 300) == hashlib.shake_256(m).digest(300)


def test_oracle_mlkem_keys_match_an_independent_implementation(orc):
    mlkem = pytest.importorskip("cryptography.hazmat.primitives.asymmetric.mlkem")
    rng = np.random.default_rng(11)
    for cls, kem in ((mlkem.MLKEM768PrivateKey, "ml-kem-768"), (mlkem.MLKEM1024PrivateKey, "ml-kem-1024")):
        for _ in range(12):
            seed = rng.bytes(64)  # d || z, the seed form of FIPS 203 and of generate_deterministic
            want = cls.from_seed_bytes(seed).public_key().public_bytes_raw()
            assert orc.mlkem_ek(kem, seed[:32]) == want


def test_oracle_mlkem_512_shape_and_range(orc):
    """ML-KEM-512 (k = 2, eta1 = 3) shares the code of the pinned variants; its key holds two
    ByteEncode12 polynomials of coefficients below 3329, then rho = SHA3-512(d || 2)[:32]"""
    d = bytes(range(32))
    ek = orc.mlkem_ek("ml-kem-512", d)
    assert len(ek) == 800
    b = np.frombuffer(ek[:768], dtype=np.uint8).astype(np.int64).reshape(-1, 3)
    c0, c1 = b[:, 0] | ((b[:, 1] & 15) << 8), (b[:, 1] >> 4) | (b[:, 2] << 4)
    assert c0.max() < 3329 and c1.max() < 3329
    assert ek[768:] == hashlib.sha3_512(d + bytes([2])).digest()[:32]


@pytest.mark.parametrize("kem", KEMS)
def test_oracle_record_layout(orc, kem):
    rid, pk = orc.dataset_record(kem, 7, 5)
    assert len(pk) == {"ml-kem-512": 800, "ml-kem-768": 1184, "ml-kem-1024": 1568}[kem]
    assert rid == hashlib.sha3_256(b"pq-key:v1:" + kem.encode() + pk).digest()
    # the record seed is ChaCha20 block 5 of the seed_from_u64(7) key: d = its first 32 bytes
    blk = orc.chacha_blocks(orc.seed_from_u64(7), 0, 5, 1)[0].astype("<u4").tobytes()
    assert orc.mlkem_ek(kem, blk[:32]) == pk
    assert orc.dataset_record(kem, 7, 6)[1] != pk and orc.dataset_record(kem, 8, 5)[1] != pk


def test_host_helpers(pkg):
    pk = bytes(range(200)) * 6
    rid = pkg.derive_public_key_id(pk[:1184], "ml-kem-768")
    assert rid == hashlib.sha3_256(b"pq-key:v1:ml-kem-768" + pk[:1184]).digest()
    assert pkg.public_key_matches_id(rid, pk[:1184], "ml-kem-768")
    assert not pkg.public_key_matches_id(rid, pk[:1184], "ml-kem-512")
    with pytest.raises(ValueError):
        pkg.DatasetGenerator("ml-kem-768", 0)._validate()
    with pytest.raises(ValueError):
        pkg.DatasetGenerator("x25519", 10)


def test_cuckoo_build_places_every_record_where_a_lookup_finds_it(pkg):
    """CuckooTable::insert semantics: each key sits at one of its two SipHash positions or in
    the stash; a crowded table (more keys than half the buckets) forces evictions"""
    rng = np.random.default_rng(8)
    n, buckets = 700, 1024
    keys = [rng.bytes(32) for _ in range(n)]
    vals = [rng.bytes(16) for _ in range(n)]
    entries, occ, stash = pkg.build_cuckoo_table(keys, vals, buckets, 32, 16)
    assert int(occ.sum()) + len(stash) == n
    for k, v in zip(keys, vals):
        pos = pkg.cuckoo_positions(pkg.DETERMINISTIC_SEED, buckets, 2, k)
        hits = [p for p in set(pos) if occ[p] and entries[p, :32].tobytes() == k]  # both hashes may agree
        in_stash = [s for s in stash if s[:32] == k]
        assert len(hits) + len(in_stash) == 1
        row = entries[hits[0]].tobytes() if hits else in_stash[0]
        assert row[32:48] == v
    again = pkg.build_cuckoo_table(keys, vals, buckets, 32, 16)
    assert np.array_equal(again[0], entries) and again[2] == stash  # seeded evictions: reproducible


@pytest.mark.gpu
@pytest.mark.parametrize("kem", KEMS)
def test_device_records_equal_oracle(pkg, orc, kem):
    import torch
    gen = pkg.DatasetGenerator(kem, 300).with_seed(7)
    rows = gen.generate_records()
    for i in list(range(0, 300, 7)) + [299]:
        rid, pk = orc.dataset_record(kem, 7, i)
        assert rows[i, :32].tobytes() == rid and rows[i, 32:].tobytes() == pk, i
    # a window far into a 1M-record dataset: the block counter, not the call, fixes a record
    rs = gen.record_size
    d = torch.empty(4 * rs, dtype=torch.uint8, device="cuda")
    gen.generate_device(d.data_ptr(), first=999_996, count=4)
    torch.cuda.synchronize()
    far = d.cpu().numpy().reshape(4, rs)
    for k in range(4):
        rid, pk = orc.dataset_record(kem, 7, 999_996 + k)
        assert far[k].tobytes() == rid + pk


@pytest.mark.gpu
def test_keyword_pir_roundtrip_mlkem(pkg):
    """tests/e2e_mlkem.rs:8-39 through this library: 10,000 ML-KEM-768 keys from seed 7, a
    target chosen by ChaCha20Rng::seed_from_u64(2026), setup_keyword_server, a keyword client
    from the public parameters: the extracted key is the record's and matches its ID.
    The last record is checked too.  Both lie inside one DB polynomial: the reference's layout
    (to_raw_db puts a row's items back to back) lets a quarter of the records straddle two
    polynomials, and its client gets back only the one holding an item's first value, so such
    records are not retrievable in the reference either (extract returns None here)."""
    ds = pkg.DatasetGenerator("ml-kem-768", 10_000).with_seed(7).generate_in_memory()
    assert ds.kem_name == "ml-kem-768" and len(ds.records) == 10_000
    target = pc.random_range_u32(pc.chacha_u32_stream(2026), 10_000)
    expected = ds.records[target]
    with pkg.setup_keyword_server(ds, None, None) as server:
        pp = server.public_params()
        assert pp["keyword_pir"]["num_records"] == 10_000
        with pkg.KeywordClient.from_public_params(pp, bytes([7]) * 32) as client:
            for rec in (expected, ds.records[-1]):
                pos, query = client.query_key(rec.public_key_id)
                public_key = client.extract_key(rec.public_key_id, pos, server.respond_to_serialized_query(query))
                assert public_key is not None, "query should return the inserted public key"
                assert pkg.public_key_matches_id(rec.public_key_id, public_key, ds.kem_name)
                assert public_key == rec.public_key
