"""Parity at the serving workload's shapes: three databases resident on one GPU at
dim0 8192 -- ML-KEM-512 x 4M (buckets 2^23), ML-KEM-768 x 1M (2^21), ML-KEM-1024 x
2M (2^22), seeds 7/8/9 -- answered on the batched INT8 path and through the serving
loop.

The plans come from the reference's derivation (KeywordServerSetupPlan::from_shape,
src/pir/server/keyword.rs:145-233): db 8192 x 524,288 / 196,608 / 524,288 u16, 256 /
96 / 256 packing outputs, interpolation degree 32.  The oracle cannot answer a whole
database in test time, so, as for the 1M benchmark shape, it answers single fold groups
(keyword.rs:558-574), generated alone from the same global element indices, and the
device's bytes for those groups must equal them; the rest is checked by size-independent
properties: every batched response equals the same payload answered alone, and the
serving loop, given the three databases' payloads interleaved, returns exactly the
batch responses.
"""
import pytest

pytestmark = pytest.mark.gpu

RESULT = 12288
SHAPES = (  # (name, records, value bytes, buckets, seed) at dim0 8192
    ("ml-kem-512 x 4M", 4_000_000, 800, 1 << 23, 7),
    ("ml-kem-768 x 1M", 1_000_000, 1184, 1 << 21, 8),
    ("ml-kem-1024 x 2M", 2_000_000, 1568, 1 << 22, 9),
)
BATCH = 16


@pytest.fixture(scope="module")
def three(pkg):
    servers = []
    try:
        for name, records, value, buckets, seed in SHAPES:
            plan = pkg.plan_from_shape(records, 32, value, buckets, 8192)
            srv = pkg.KeywordServer.synthetic(plan, seed=seed)
            srv.prepare_batch(BATCH)
            servers.append((name, plan, seed, srv))
        yield servers
    finally:
        for _, _, _, srv in servers:
            srv.close()


def _group_bytes(resp: bytes, group: int, nq: int = 2):
    assert int.from_bytes(resp[:4], "little") == nq
    out, off = [], 4
    for _ in range(nq):
        n = int.from_bytes(resp[off:off + 4], "little")
        out.append(resp[off + 4 + group * RESULT: off + 4 + (group + 1) * RESULT])
        off += 4 + n
    return out


def test_plans_are_the_reference_derivation(three):
    got = [(p.db_rows, p.db_cols, p.instances, p.interp, p.c) for _, p, _, _ in three]
    assert got == [(8192, 524288, 256, 32, 8), (8192, 196608, 96, 32, 3), (8192, 524288, 256, 32, 8)]


def test_batches_match_oracle_and_single_answers(three, orc):
    for k, (name, plan, seed, srv) in enumerate(three):
        qs = [orc.synth_query(40_000 + 100 * k + i, plan.db_rows, 2) for i in range(BATCH)]
        batch = srv.respond_batch(qs)
        assert len(batch) == BATCH and len({b[8:8 + 4096] for b in batch}) == BATCH
        for i in (0, BATCH - 1):
            assert batch[i] == srv.respond_to_serialized_query(qs[i]), (name, i)
        for group, i in ((0, 3), (plan.c - 1, 11)):
            shard = orc.SynthDB.shard_of(plan.db_rows, group * plan.interp, plan.interp, plan.interp, 1, seed=seed)
            assert _group_bytes(batch[i], group) == _group_bytes(orc.respond(shard, qs[i]), 0), (name, group)
            del shard


def test_serving_loop_over_three_resident_databases(three, pkg, orc):
    """payloads of the three databases submitted interleaved (the serving loop batches them
    per database as they arrive) come back exactly as the batched path answers them"""
    svc = pkg.KeywordService([srv for _, _, _, srv in three], max_batch=BATCH)
    try:
        per_db = [[orc.synth_query(50_000 + 100 * k + i, plan.db_rows, 2) for i in range(BATCH)]
                  for k, (_, plan, _, _) in enumerate(three)]
        tickets = []
        for i in range(BATCH):
            for k in range(3):
                tickets.append((k, i, svc.submit(k, per_db[k][i])))
        got = {(k, i): svc.wait(t) for k, i, t in tickets}
    finally:
        svc.close()
    for k, (name, _, _, srv) in enumerate(three):
        want = srv.respond_batch(per_db[k])
        assert [got[(k, i)] for i in range(BATCH)] == want, name
