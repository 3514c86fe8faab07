"""Fold-group sharding across ranks (the multi-GPU path), on CPU.

The shard plan (ipr_plan_shard), the slicing of the server state, the
collective flow of ShardedKeywordServer (broadcast the query, gather the
parts) and the merge (ipr_response_merge) are product code; here they run as
world_size-2 gloo ranks, each rank answering its shard with the oracle in
place of a GPU, and the merged response must equal the oracle's unsharded
response byte for byte.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
N = 2048


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _plan(pkg, instances, interp, db_rows=2048):
    return pkg.Plan(num_items=max(db_rows, 32768), entry_size=1216, item_size_bits=9728, dim0=db_rows,
                    db_rows=db_rows, db_cols=instances * N, instances=instances, interp=interp,
                    c=instances // interp, peak_bytes=0)


def test_shard_plan_covers_groups(pkg):
    plan = pkg.plan_from_shape(1_000_000, 32, 1184, 2_097_152, 2048)
    for shards in (1, 2, 3, 4, 8, 11):
        firsts, total = [], 0
        for k in range(shards):
            sub, first = pkg.shard_plan(plan, shards, k)
            assert sub.interp == plan.interp and sub.db_rows == plan.db_rows
            assert sub.instances == sub.c * plan.interp and sub.db_cols == sub.instances * N
            assert first == total
            total += sub.instances
            firsts.append(first)
        assert total == plan.instances
        cs = [pkg.shard_plan(plan, shards, k)[0].c for k in range(shards)]
        assert max(cs) - min(cs) <= 1
    with pytest.raises(pkg.IprError):
        pkg.shard_plan(plan, 12, 0)  # 11 fold groups cannot feed 12 shards
    with pytest.raises(pkg.IprError):
        pkg.shard_plan(plan, 2, 2)


@pytest.mark.parametrize("nq", [0, 1, 2, 3])
def test_merge_of_oracle_shards_equals_unsharded(pkg, orc, nq):
    plan = _plan(pkg, 6, 2)  # c = 3 fold groups
    stash = [bytes([7]) * 40, bytes(range(40))]
    full = orc.SynthDB(plan.db_rows, 6, 2, 3, seed=31, stash=stash)
    q = orc.synth_query(40 + nq, plan.db_rows, nq)
    want = orc.respond(full, q)
    for shards in (1, 2, 3):
        parts = []
        for k in range(shards):
            sub, first = pkg.shard_plan(plan, shards, k)
            parts.append(orc.respond(full.shard(first, sub.instances, sub.interp, sub.c), q))
        assert pkg.merge_responses(parts) == want


def test_merge_rejects_inconsistent_parts(pkg):
    a = (1).to_bytes(4, "little") + (3).to_bytes(4, "little") + b"abc" + (0).to_bytes(4, "little")
    b = (2).to_bytes(4, "little") + (1).to_bytes(4, "little") + b"x" + (1).to_bytes(4, "little") + b"y" + bytes(4)
    with pytest.raises(pkg.IprError):
        pkg.merge_responses([a, b])  # different response counts
    with pytest.raises(pkg.IprError):
        pkg.merge_responses([a[:6]])  # truncated
    assert pkg.merge_responses([a, a]) == (1).to_bytes(4, "little") + (6).to_bytes(4, "little") + b"abcabc" + bytes(4)


def _rank_main(rank, world, port, out_q):
    import sys
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import datetime

    import torch.distributed as dist
    from conftest import load_package, load_oracle
    pkg, orc = load_package(), load_oracle()
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        plan = _plan(pkg, 6, 2)
        full = orc.SynthDB(plan.db_rows, 6, 2, 3, seed=31, stash=[b"s" * 16])
        sub, first = pkg.shard_plan(plan, world, rank)
        mine = full.shard(first, sub.instances, sub.interp, sub.c)
        srv = pkg.ShardedKeywordServer(lambda q: orc.respond(mine, q))
        results = []
        for seed, nq in ((1, 2), (2, 1), (3, 0)):
            q = orc.synth_query(seed, plan.db_rows, nq) if rank == 0 else None
            r = srv.respond_to_serialized_query(q)
            if rank == 0:
                results.append(r == orc.respond(full, orc.synth_query(seed, plan.db_rows, nq)))
            else:
                results.append(r is None)
        # the batch collective: one broadcast of three payloads, one gather of the parts
        qs = [orc.synth_query(10 + i, plan.db_rows, 2) for i in range(3)]
        rb = srv.respond_batch(qs if rank == 0 else None, lambda batch: [orc.respond(mine, q) for q in batch])
        results.append(rb == [orc.respond(full, q) for q in qs] if rank == 0 else rb is None)
        out_q.put((rank, results))
    finally:
        dist.destroy_process_group()


def test_sharded_server_gloo_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=240) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got[0] == [True, True, True, True]
    assert got[1] == [True, True, True, True]


@pytest.mark.gpu
def test_shards_on_one_gpu_merge_to_full(pkg, orc):
    """two shard servers built from slices of one state, answered one after the other on
    the same GPU and merged, equal the unsharded server (both single and batch paths)"""
    plan = _plan(pkg, 6, 2)
    stash = [bytes([9]) * 1216]
    full = orc.SynthDB(plan.db_rows, 6, 2, 3, seed=33, stash=stash)
    whole = pkg.KeywordServer.from_encoded(plan, full.db, full.a_hat, full.bold_t, full.bold_t_bar,
                                           full.bold_t_hat, stash=stash)
    shards = []
    for k in range(2):
        sub, first = pkg.shard_plan(plan, 2, k)
        s = full.shard(first, sub.instances, sub.interp, sub.c)
        shards.append(pkg.KeywordServer.from_encoded(sub, s.db, s.a_hat, s.bold_t, s.bold_t_bar, s.bold_t_hat,
                                                     stash=stash))
    try:
        for seed, nq in ((5, 2), (6, 1), (7, 3)):
            q = orc.synth_query(seed, plan.db_rows, nq)
            want = whole.respond_to_serialized_query(q)
            assert want == orc.respond(full, q)
            assert pkg.merge_responses([s.respond_to_serialized_query(q) for s in shards]) == want
        qs = [orc.synth_query(50 + i, plan.db_rows, 2) for i in range(5)]
        per_shard = [s.respond_batch(qs) for s in shards]
        assert [pkg.merge_responses([a, b]) for a, b in zip(*per_shard)] == whole.respond_batch(qs)
    finally:
        for s in shards + [whole]:
            s.close()


def test_synth_shard_of_equals_slice(orc):
    """a fold-group slice generated alone equals the same slice of the whole synthetic state"""
    import numpy as np
    full = orc.SynthDB(2048, 6, 2, 3, seed=31)
    alone = orc.SynthDB.shard_of(2048, 2, 2, 2, 1, seed=31)
    view = full.shard(2, 2, 2, 1)
    for a in ("db", "a_hat", "bold_t", "bold_t_bar", "bold_t_hat"):
        assert np.array_equal(getattr(alone, a), getattr(view, a)), a
    q = orc.synth_query(3, 2048, 2)
    assert orc.respond(alone, q) == orc.respond(view, q)


@pytest.mark.gpu
def test_synthetic_shards_merge_to_full_synthetic(pkg):
    """ipr_server_create_synthetic_shard: each shard generates its own slice of the synthetic
    state on the device; merged, the shards answer like the full synthetic server (single and
    batch paths).  This is how a sharded run builds its per-GPU servers."""
    import numpy as np  # noqa: F401
    sys_orc = __import__("oracle")
    plan = _plan(pkg, 6, 2)
    with pkg.KeywordServer.synthetic(plan, seed=12) as whole:
        for shards in (2, 3):
            parts = [pkg.KeywordServer.synthetic_shard(plan, shards, k, seed=12) for k in range(shards)]
            try:
                qs = [sys_orc.synth_query(80 + i, plan.db_rows, 2) for i in range(4)]
                want = whole.respond_batch(qs)
                for i, q in enumerate(qs[:2]):
                    assert pkg.merge_responses([s.respond_to_serialized_query(q) for s in parts]) == want[i]
                per = [s.respond_batch(qs) for s in parts]
                assert [pkg.merge_responses(list(x)) for x in zip(*per)] == want
            finally:
                for s in parts:
                    s.close()
