"""Parity at the benchmark's full size: 1M ML-KEM-768 records, buckets 2^21,
dim0 2048 (db 2048 x 720,896, 352 packing outputs, 11 fold groups).

The oracle cannot answer the whole 1M server in test time, but the fold groups
are independent (keyword.rs:558-574) and the synthetic state is generated by
global element index, so the oracle builds one group's slice alone and answers
it; the device's bytes for that group (in every query's result) must equal the
oracle's.  Size-independent properties complete the check: the batch path
(64 distinct clients per pass) returns exactly the single-payload bytes, and
framing, lengths and stash echo follow the wire format.
"""
import pytest

pytestmark = pytest.mark.gpu

RESULT = 12288


@pytest.fixture(scope="module")
def full(pkg):
    plan = pkg.plan_from_shape(1_000_000, 32, 1184, 2_097_152, 2048)
    assert (plan.db_rows, plan.db_cols, plan.instances, plan.interp, plan.c) == (2048, 720896, 352, 32, 11)
    srv = pkg.KeywordServer.synthetic(plan, seed=7)
    yield plan, srv
    srv.close()


def _group_bytes(resp: bytes, plan, group: int, nq: int):
    """bytes of fold group `group` in each query's result (after the framing headers)"""
    assert int.from_bytes(resp[:4], "little") == nq
    out, off = [], 4
    for _ in range(nq):
        n = int.from_bytes(resp[off:off + 4], "little")
        out.append(resp[off + 4 + group * RESULT: off + 4 + (group + 1) * RESULT])
        off += 4 + n
    return out


@pytest.mark.parametrize("group", [0, 10])
def test_fold_group_matches_oracle_at_1m(full, orc, group):
    plan, srv = full
    q = orc.synth_query(4242 + group, plan.db_rows, 2)
    got = srv.respond_to_serialized_query(q)
    assert len(got) == srv.response_bytes(2) == 4 + 2 * (4 + plan.c * RESULT) + 4
    shard = orc.SynthDB.shard_of(plan.db_rows, group * plan.interp, plan.interp, plan.interp, 1, seed=7)
    want = orc.respond(shard, q)  # one fold group: 2 x 12288 result bytes
    assert _group_bytes(got, plan, group, 2) == _group_bytes(want, plan, 0, 2)


def test_batch_of_64_equals_single_at_1m(full, orc):
    plan, srv = full
    qs = [orc.synth_query(9000 + i, plan.db_rows, 2) for i in range(64)]
    batch = srv.respond_batch(qs)
    for i in (0, 31, 63):
        assert batch[i] == srv.respond_to_serialized_query(qs[i])
    # one batched payload's fold group against the oracle as well
    shard = orc.SynthDB.shard_of(plan.db_rows, 5 * plan.interp, plan.interp, plan.interp, 1, seed=7)
    assert _group_bytes(batch[17], plan, 5, 2) == _group_bytes(orc.respond(shard, qs[17]), plan, 0, 2)
    # distinct clients give distinct responses; the stash block is empty
    assert len({b[8:8 + 4096] for b in batch}) == 64
    assert all(b[-4:] == bytes(4) for b in batch)
