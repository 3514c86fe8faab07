"""The wire-compatibility pin (tests/golden/rust_pin.json, rust_pin_response.bin).

The Rust test in INTEGRATION.md runs inside the reference crate and compares the crate's
own ChaCha20Rng([7; 32]) u64 stream, NTT(-a) of the RGSW row-0 mask, DatasetGenerator
records and respond_to_serialized_query bytes with these committed values.  Here:
CPU: the oracle regenerates every committed value (make_rust_pin.py), including the
response of a server set up from the generated dataset (cuckoo table, raw DB, encode,
offline precomputation) to the formula-defined query;
GPU: the device, from DatasetGenerator through setup_keyword_server, returns the committed
response bytes exactly.
"""
import hashlib
import json
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
sys.path.insert(0, GOLDEN)

import make_rust_pin as mrp  # noqa: E402


def _committed():
    with open(os.path.join(GOLDEN, "rust_pin.json")) as f:
        meta = json.load(f)
    with open(os.path.join(GOLDEN, "rust_pin_response.bin"), "rb") as f:
        resp = f.read()
    return meta, resp


def test_oracle_regenerates_the_pin():
    meta, resp = _committed()
    got, query, got_resp = mrp.build()
    assert got == meta
    assert got_resp == resp
    assert hashlib.sha3_256(query).hexdigest() == meta["query_sha3_256"]


@pytest.mark.gpu
def test_device_setup_from_dataset_answers_the_pin(pkg):
    meta, resp = _committed()
    d = meta["dataset"]
    ds = pkg.DatasetGenerator(d["kem"], d["count"]).with_seed(d["seed"]).generate_in_memory()
    for r in meta["records"]:
        rec = ds.records[r["index"]]
        assert rec.public_key_id.hex() == r["id_hex"]
        assert hashlib.sha3_256(rec.public_key).hexdigest() == r["public_key_sha3_256"]
    with pkg.setup_keyword_server(ds, d["buckets"], None) as srv:
        q = mrp.pin_query(srv.plan.db_rows)
        assert srv.respond_to_serialized_query(q) == resp
        assert srv.respond_batch([q, q]) == [resp, resp]
