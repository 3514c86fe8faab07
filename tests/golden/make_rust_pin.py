"""Generate the wire-compatibility pin for a maintainer with a Rust toolchain.

The Rust test in INTEGRATION.md ("Wire-compatibility pin") runs inside the reference
crate and compares the crate's own outputs with the values written here by the oracle:

* chacha7_u64: the first 16 StandardUniform u64 draws of ChaCha20Rng::from_seed([7; 32])
  (the stream of the RGSW row-0 mask, src/pir/server/keyword.rs:546-555);
* ntt_neg_a: the first 8 coefficients of each CRT limb of NTT(-a), a = PolyMatrixRaw::
  random_rng(params, 1, 1, ChaCha20Rng::from_seed([7; 32])) (the same lines);
* records: id and SHA3-256 of the public key of records 0..3 of DatasetGenerator::new(
  MlKem768, 300).with_seed(7) (src/dataset/generator.rs:171-193);
* response: respond_to_serialized_query's bytes (their SHA3-256 and the file
  rust_pin_response.bin) for setup_keyword_server(that dataset, Some(32768), None) and
  the query below.

The query is defined by a formula both sides compute: byte 0 = 2 (queries), then the
40,960 56-bit fields of serialize_keyword_query, 7 little-endian bytes each from byte 1,
field f = (splitmix64(2f) mod q0) | (splitmix64(2f + 1) mod q1) << 28.  With 300 records
in 32,768 buckets no cuckoo insertion needs an eviction (checked below), so the table
layout does not depend on the reference's unseeded eviction generator.

Run from the repository root:  python tests/golden/make_rust_pin.py
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))

import oracle as orc  # noqa: E402
import pir_client as pc  # noqa: E402

N = 2048
Q0, Q1 = 268369921, 249561089
M64 = (1 << 64) - 1
DETERMINISTIC_SEED = bytes([0xDE, 0xAD, 0xBE, 0xEF, 0xCA, 0xFE, 0xBA, 0xBE, 0x01, 0x23, 0x45, 0x67, 0x89, 0xAB,
                            0xCD, 0xEF])
RECORDS, BUCKETS = 300, 32768


def splitmix64(i: int) -> int:
    z = (i + 0x9E3779B97F4A7C15) & M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def pin_query(db_rows: int) -> bytes:
    nfields = 3 * N * 2 + 2 * (db_rows + 6 * N)
    f = np.arange(nfields, dtype=np.uint64)

    def mix(x):
        z = x + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))

    lo = mix(np.uint64(2) * f) % np.uint64(Q0)
    hi = mix(np.uint64(2) * f + np.uint64(1)) % np.uint64(Q1)
    v = (lo | (hi << np.uint64(28))).astype("<u8")
    assert int(lo[3]) == splitmix64(6) % Q0  # the vector form equals the scalar definition
    return bytes([2]) + v.view(np.uint8).reshape(-1, 8)[:, :7].tobytes()


def oracle_server(records, plan):
    """the oracle's KeywordServer::setup for the records: cuckoo table (no evictions), raw DB,
    encode, offline precomputation"""
    es = plan["entry_size"]
    entries = np.zeros((plan["num_items"], es), dtype=np.uint8)
    occ = np.zeros(plan["num_items"], dtype=np.uint8)
    for rid, pk in records:
        pos = pc.cuckoo_positions(DETERMINISTIC_SEED, plan["num_items"], 2, rid)
        free = [p for p in pos if not occ[p]]
        assert free, "an eviction would be needed: the layout would depend on the eviction generator"
        entries[free[0], :32] = np.frombuffer(rid, np.uint8)
        entries[free[0], 32:32 + len(pk)] = np.frombuffer(pk, np.uint8)
        occ[free[0]] = 1
    rows, cols = plan["db_rows"], plan["db_cols"]
    raw = orc.raw_db(entries, occ, es, rows, cols, plan["num_items"] // rows)
    enc = orc.encode_db(raw, rows, cols, plan["interp"])
    a_hat, bt, btb, bth = orc.offline_precompute(enc, rows, plan["instances"])
    sdb = orc.SynthDB.__new__(orc.SynthDB)
    sdb.db_rows, sdb.instances, sdb.interp, sdb.c, sdb.seed = rows, plan["instances"], plan["interp"], plan["c"], 0
    sdb.db_cols, sdb.db = cols, enc
    sdb.a_hat, sdb.bold_t, sdb.bold_t_bar, sdb.bold_t_hat = (np.ascontiguousarray(x).reshape(-1)
                                                               for x in (a_hat, bt, btb, bth))
    sdb.stash, sdb._stash_buf = [], np.zeros(1, dtype=np.uint8)
    return sdb


def build():
    seed7 = bytes([7]) * 32
    words = orc.chacha_blocks(seed7, 0, 0, 2).reshape(-1).astype(np.uint64)
    u64 = [int(words[2 * i]) | (int(words[2 * i + 1]) << 32) for i in range(16)]
    q = Q0 * Q1
    a = orc.random_raw(seed7, N)  # u64 draws mod q (poly.rs:211-231)
    neg = [(q - int(x)) % q for x in a]
    raw2 = np.array([[v % Q0 for v in neg], [v % Q1 for v in neg]], dtype=np.uint64)
    ntt = pc.to_ntt(raw2)
    records = [orc.dataset_record("ml-kem-768", 7, i) for i in range(RECORDS)]
    plan = orc.plan_from_shape(RECORDS, 32, 1184, BUCKETS, 0)
    sdb = oracle_server(records, plan)
    query = pin_query(plan["db_rows"])
    resp = orc.respond(sdb, query)
    meta = {
        "chacha7_u64": [str(x) for x in u64],
        "ntt_neg_a_limb0": [int(x) for x in ntt[0][:8]],
        "ntt_neg_a_limb1": [int(x) for x in ntt[1][:8]],
        "records": [{"index": i, "id_hex": records[i][0].hex(),
                     "public_key_sha3_256": hashlib.sha3_256(records[i][1]).hexdigest()} for i in range(4)],
        "dataset": {"kem": "ml-kem-768", "count": RECORDS, "seed": 7, "buckets": BUCKETS},
        "plan": {k: int(plan[k]) for k in ("num_items", "db_rows", "db_cols", "instances", "interp", "c")},
        "query_len": len(query), "query_sha3_256": hashlib.sha3_256(query).hexdigest(),
        "response_len": len(resp), "response_sha3_256": hashlib.sha3_256(resp).hexdigest(),
    }
    return meta, query, resp


def main():
    meta, _, resp = build()
    with open(os.path.join(HERE, "rust_pin.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
        f.write("\n")
    with open(os.path.join(HERE, "rust_pin_response.bin"), "wb") as f:
        f.write(resp)
    print("wrote rust_pin.json and rust_pin_response.bin")


if __name__ == "__main__":
    main()
