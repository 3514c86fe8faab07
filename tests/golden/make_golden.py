"""Generate the golden respond() fixtures in this folder from the oracle.

The reference has no golden response (its end-to-end test only checks that the
client decrypts the right key, tests/e2e_mlkem.rs:8-39), so the fixtures are
captured from the oracle, whose building blocks are pinned by the reference's
known-answer tests and by its own CUDA kernels.  Each case is a seeded
synthetic server state (the generator shared by the oracle and the device) and
a seeded synthetic query; the fixture records the shape, the seeds, SHA-256
digests of the inputs (so a change of generator is caught) and the full
response bytes.

Run from the repository root:  python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))

import oracle as orc  # noqa: E402

N = 2048

# name -> (db_rows, instances, interp, c, db_seed, query_seed, num_queries, stash entries)
CASES = {
    "config0_q2026": (2048, 8, 8, 1, 7, 2026, 2, ()),
    "i2_p2_q1": (2048, 2, 2, 1, 5, 1, 2, ()),
    "i4_p2_c2_stash": (2048, 4, 2, 2, 44, 9, 1, (b"\x01" * 24, bytes(range(24)))),
    "i3_p1_c3_rows4096": (4096, 3, 1, 3, 61, 3, 2, ()),
    "i6_p3_c2_nq0": (2048, 6, 3, 2, 13, 4, 0, (b"stash-entry-0123",)),
}


def sha(b) -> str:
    return hashlib.sha256(bytes(b)).hexdigest()


def build_case(name):
    db_rows, inst, interp, c, dseed, qseed, nq, stash = CASES[name]
    sdb = orc.SynthDB(db_rows, inst, interp, c, seed=dseed, stash=stash)
    query = orc.synth_query(qseed, db_rows, nq)
    resp = orc.respond(sdb, query)
    meta = {
        "db_rows": db_rows, "instances": inst, "interp": interp, "c": c,
        "db_seed": dseed, "query_seed": qseed, "num_queries": nq,
        "stash_hex": [s.hex() for s in stash],
        "db_sha256": sha(sdb.db.tobytes()),
        "bold_t_sha256": sha(sdb.bold_t.tobytes()),
        "bold_t_bar_sha256": sha(sdb.bold_t_bar.tobytes()),
        "bold_t_hat_sha256": sha(sdb.bold_t_hat.tobytes()),
        "a_hat_sha256": sha(sdb.a_hat.tobytes()),
        "query_sha256": sha(query), "query_len": len(query),
        "response_sha256": sha(resp), "response_len": len(resp),
    }
    return meta, sdb, query, resp


def main():
    for name in CASES:
        meta, _, _, resp = build_case(name)
        with open(os.path.join(HERE, f"respond_{name}.json"), "w") as f:
            json.dump(meta, f, indent=1, sort_keys=True)
            f.write("\n")
        with open(os.path.join(HERE, f"respond_{name}.bin"), "wb") as f:
            f.write(resp)
        print(name, meta["response_len"], meta["response_sha256"][:16])


if __name__ == "__main__":
    main()
