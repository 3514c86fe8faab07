"""Golden respond() fixtures (tests/golden/, made by tests/golden/make_golden.py).

CPU: the oracle regenerates every fixture's inputs (SHA-256 of the synthetic
state and query) and its response bytes exactly.  GPU: the device path, through
the C ABI, returns the fixture's response bytes — from the single-payload
entry, from the batch entry, and from a server built from host arrays.
"""
import glob
import hashlib
import json
import os

import pytest

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = sorted(os.path.basename(p)[len("respond_"):-len(".json")] for p in glob.glob(os.path.join(HERE, "respond_*.json")))
N = 2048


def _load(name):
    with open(os.path.join(HERE, f"respond_{name}.json")) as f:
        meta = json.load(f)
    with open(os.path.join(HERE, f"respond_{name}.bin"), "rb") as f:
        resp = f.read()
    return meta, resp


def _sha(b):
    return hashlib.sha256(bytes(b)).hexdigest()


def _inputs(orc, meta):
    stash = [bytes.fromhex(s) for s in meta["stash_hex"]]
    sdb = orc.SynthDB(meta["db_rows"], meta["instances"], meta["interp"], meta["c"], seed=meta["db_seed"],
                      stash=stash)
    query = orc.synth_query(meta["query_seed"], meta["db_rows"], meta["num_queries"])
    return sdb, query, stash


def test_fixture_set_present():
    assert len(CASES) >= 5
    for name in CASES:
        meta, resp = _load(name)
        assert len(resp) == meta["response_len"] and _sha(resp) == meta["response_sha256"]


@pytest.mark.parametrize("name", CASES)
def test_oracle_reproduces_golden(orc, name):
    meta, resp = _load(name)
    sdb, query, _ = _inputs(orc, meta)
    assert _sha(sdb.db.tobytes()) == meta["db_sha256"]
    assert _sha(sdb.bold_t.tobytes()) == meta["bold_t_sha256"]
    assert _sha(sdb.bold_t_bar.tobytes()) == meta["bold_t_bar_sha256"]
    assert _sha(sdb.bold_t_hat.tobytes()) == meta["bold_t_hat_sha256"]
    assert _sha(sdb.a_hat.tobytes()) == meta["a_hat_sha256"]
    assert _sha(query) == meta["query_sha256"] and len(query) == meta["query_len"]
    assert orc.respond(sdb, query) == resp


def test_golden_framing(pkg, orc):
    """the fixtures decode with the wire-format parser: counts, lengths, stash echo"""
    for name in CASES:
        meta, resp = _load(name)
        r = pkg.deserialize_keyword_response(resp)
        assert len(r.responses) == meta["num_queries"]
        assert all(len(x) == meta["c"] * 12288 for x in r.responses)
        assert [s.hex() for s in r.stash_entries] == meta["stash_hex"]


def _plan(pkg, meta):
    return pkg.Plan(num_items=max(meta["db_rows"], 32768), entry_size=1216, item_size_bits=9728,
                    dim0=meta["db_rows"], db_rows=meta["db_rows"], db_cols=meta["instances"] * N,
                    instances=meta["instances"], interp=meta["interp"], c=meta["c"], peak_bytes=0)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_device_matches_golden(pkg, orc, name):
    meta, resp = _load(name)
    plan = _plan(pkg, meta)
    query = orc.synth_query(meta["query_seed"], meta["db_rows"], meta["num_queries"])
    if meta["stash_hex"]:
        sdb, _, stash = _inputs(orc, meta)
        srv = pkg.KeywordServer.from_encoded(plan, sdb.db, sdb.a_hat, sdb.bold_t, sdb.bold_t_bar, sdb.bold_t_hat,
                                             stash=stash)
    else:
        srv = pkg.KeywordServer.synthetic(plan, seed=meta["db_seed"])
    with srv:
        assert srv.respond_to_serialized_query(query) == resp
        # batch entry: the same payload three times in one call
        assert srv.respond_batch([query] * 3) == [resp] * 3
