"""Serving loop (ipr_service_*): continuous batching over one or more servers.

Every response must equal the payload answered alone (ipr_server_respond) and
the oracle, whether it ran alone, in a batch with other clients, next to
payloads with other query counts, or next to another database's traffic.
"""
import threading
import time

import pytest

N = 2048


def _plan(pkg, instances, interp, db_rows=2048):
    return pkg.Plan(num_items=max(db_rows, 32768), entry_size=1216, item_size_bits=9728, dim0=db_rows,
                    db_rows=db_rows, db_cols=instances * N, instances=instances, interp=interp,
                    c=instances // interp, peak_bytes=0)


@pytest.fixture(scope="module")
def dbs(pkg, orc):
    """two databases of different shapes"""
    out = []
    for inst, interp, seed in ((8, 8, 7), (4, 2, 19)):
        plan = _plan(pkg, inst, interp)
        srv = pkg.KeywordServer.synthetic(plan, seed=seed)
        sdb = orc.SynthDB(plan.db_rows, inst, interp, plan.c, seed=seed)
        out.append((plan, srv, sdb))
    yield out
    for _, srv, _ in out:
        srv.close()


@pytest.mark.gpu
def test_alone_equals_in_mix(pkg, orc, dbs):
    plan, srv, sdb = dbs[0]
    queries = [orc.synth_query(500 + i, plan.db_rows, 2) for i in range(12)]
    queries += [orc.synth_query(600, plan.db_rows, 1), orc.synth_query(601, plan.db_rows, 3),
                orc.synth_query(602, plan.db_rows, 0)]
    alone = [srv.respond_to_serialized_query(q) for q in queries]
    for q, a in zip(queries[:3] + queries[-3:], alone[:3] + alone[-3:]):
        assert a == orc.respond(sdb, q)
    with pkg.KeywordService([srv]) as svc:
        # one at a time
        for q, a in zip(queries, alone):
            assert svc.wait(svc.submit(0, q)) == a
        # all at once: batches form from whatever is pending
        tickets = [svc.submit(0, q) for q in queries]
        got = [svc.wait(t) for t in tickets]
        assert got == alone
        st = svc.stats()
        assert st.completed == 2 * len(queries) and st.failed == 0 and st.in_flight == 0
        assert st.batches >= 1 and st.batched_payloads >= 1 and st.max_batch == 64
        log = svc.batch_log()
        assert len(log) == st.batches and sum(b["payloads"] for b in log) == st.batched_payloads
        assert all(b["launch_ms"] <= b["ready_ms"] and b["start_ms"] <= b["ready_ms"] for b in log)
        assert all(log[i]["ready_ms"] <= log[i + 1]["ready_ms"] for i in range(len(log) - 1))


@pytest.mark.gpu
def test_two_databases_concurrent_clients(pkg, orc, dbs):
    (p0, s0, d0), (p1, s1, d1) = dbs
    q0 = [orc.synth_query(700 + i, p0.db_rows, 2) for i in range(20)]
    q1 = [orc.synth_query(800 + i, p1.db_rows, 2) for i in range(20)]
    want0 = [s0.respond_to_serialized_query(q) for q in q0]
    want1 = [s1.respond_to_serialized_query(q) for q in q1]
    assert want1[0] == orc.respond(d1, q1[0])
    results = {}
    with pkg.KeywordService([s0, s1], max_batch=8) as svc:
        def client(db, qs, key):
            ts = []
            for q in qs:
                ts.append(svc.submit(db, q))
                time.sleep(0.0005)
            results[key] = [svc.wait(t, 60000) for t in ts]
        th = [threading.Thread(target=client, args=(0, q0[:10], "a")),
              threading.Thread(target=client, args=(0, q0[10:], "b")),
              threading.Thread(target=client, args=(1, q1, "c"))]
        for t in th:
            t.start()
        for t in th:
            t.join()
        assert results["a"] + results["b"] == want0
        assert results["c"] == want1
        st = svc.stats()
        assert st.max_batch == 8 and st.failed == 0 and st.completed == 40
        assert st.p50_us > 0 and st.p99_us >= st.p50_us


@pytest.mark.gpu
def test_admission_by_hbm_budget_and_queue(pkg, orc, dbs):
    plan, srv, _ = dbs[0]
    srv.prepare_batch(1)  # the slot-indexed precomputation exists: footprints below are scratch only
    with pytest.raises(pkg.IprError) as ei:
        pkg.KeywordService([srv], hbm_budget_bytes=1 << 20)
    assert ei.value.status == -2  # IPR_E_OOM: not even one payload fits
    # a budget between the 3- and 4-payload footprints admits batches of 3
    probe = [pkg.KeywordService([srv], max_batch=b, hbm_budget_bytes=1 << 40) for b in (3, 4)]
    need3, need4 = probe[0].stats().hbm_bytes, probe[1].stats().hbm_bytes
    for p in probe:
        p.close()
    assert need4 > need3
    with pkg.KeywordService([srv], hbm_budget_bytes=(need3 + need4) // 2) as svc:
        assert svc.stats().max_batch == 3
        q = orc.synth_query(900, plan.db_rows, 2)
        want = srv.respond_to_serialized_query(q)
        ts = [svc.submit(0, q) for _ in range(7)]
        assert all(svc.wait(t) == want for t in ts)
        assert svc.stats().batched_payloads == 7
    with pkg.KeywordService([srv], max_pending=2) as svc:
        q = orc.synth_query(901, plan.db_rows, 2)
        ts, busy = [], 0
        for _ in range(40):
            try:
                ts.append(svc.submit(0, q))
            except pkg.IprError as e:
                assert e.status == -8  # IPR_E_BUSY
                busy += 1
        assert busy > 0 and svc.stats().rejected == busy
        want = srv.respond_to_serialized_query(q)
        assert all(svc.wait(t) == want for t in ts)


@pytest.mark.gpu
def test_database_added_to_a_running_service(pkg, orc, dbs):
    """ipr_service_add_database: a second database joins while the first one's traffic runs;
    both answer exactly, and a database that does not fit what is left of the budget is
    refused with IPR_E_OOM"""
    (p0, s0, d0), (p1, s1, d1) = dbs
    q0 = [orc.synth_query(1100 + i, p0.db_rows, 2) for i in range(10)]
    q1 = [orc.synth_query(1200 + i, p1.db_rows, 2) for i in range(6)] + [orc.synth_query(1300, p1.db_rows, 1)]
    want0 = [s0.respond_to_serialized_query(q) for q in q0]
    want1 = [s1.respond_to_serialized_query(q) for q in q1]
    assert want1[-1] == orc.respond(d1, q1[-1])
    with pkg.KeywordService([s0], max_batch=8, hbm_budget_bytes=1 << 40) as svc:
        first = [svc.submit(0, q) for q in q0[:5]]
        db = svc.add_database(s1)
        assert db == 1
        second = [svc.submit(1, q) for q in q1] + [svc.submit(0, q) for q in q0[5:]]
        assert [svc.wait(t) for t in first] == want0[:5]
        got = [svc.wait(t) for t in second]
        assert got[:len(q1)] == want1 and got[len(q1):] == want0[5:]
        with pytest.raises(pkg.IprError):
            svc.add_database(s1)  # already served
    s0.prepare_batch(2)
    s1.prepare_batch(2)
    with pkg.KeywordService([s0], max_batch=2, hbm_budget_bytes=1 << 40) as probe:
        need = probe.stats().hbm_bytes
    with pkg.KeywordService([s0], max_batch=2, hbm_budget_bytes=need) as svc:
        with pytest.raises(pkg.IprError) as ei:
            svc.add_database(s1)
        assert ei.value.status == -2  # IPR_E_OOM: nothing of the budget is left
        assert svc.wait(svc.submit(0, q0[0])) == want0[0]


@pytest.mark.gpu
def test_service_errors_and_poll(pkg, orc, dbs):
    plan, srv, _ = dbs[0]
    with pkg.KeywordService([srv]) as svc:
        with pytest.raises(pkg.IprError):
            svc.submit(5, b"\x02")  # no such database
        with pytest.raises(pkg.IprError):
            svc.submit(0, b"\x02" + bytes(100))  # shorter than two queries need
        t = svc.submit(0, orc.synth_query(902, plan.db_rows, 2))
        r = None
        for _ in range(20000):
            r = svc.poll(t)
            if r is not None:
                break
            time.sleep(0.001)
        assert r == srv.respond_to_serialized_query(orc.synth_query(902, plan.db_rows, 2))
        with pytest.raises(pkg.IprError):
            svc.poll(t)  # collected tickets are released


@pytest.mark.gpu
def test_bounded_wait_reports_timeout_and_device_stays_usable(pkg, orc):
    """failure detection without a GPU fault: a kernel's bounded mbarrier wait on a barrier
    nothing arrives on gives up and is reported as IPR_E_TIMEOUT; afterwards the same
    process answers a query bit-exactly"""
    import time
    t0 = time.perf_counter()
    assert pkg.selftest_bounded_wait(5_000) == -4  # 5 ms limit
    assert time.perf_counter() - t0 < 5.0
    assert "bounded wait ran out" in (pkg.lib.ipr_last_error() or b"").decode()
    assert pkg.selftest_bounded_wait(2_000_000) == -1  # limits above one second are refused
    plan = pkg.plan_from_shape(10_000, 32, 1184)
    with pkg.KeywordServer.synthetic(plan, seed=3) as srv:
        sdb = orc.SynthDB(plan.db_rows, plan.instances, plan.interp, plan.c, seed=3)
        q = orc.synth_query(9, plan.db_rows, 2)
        assert srv.respond_to_serialized_query(q) == orc.respond(sdb, q)


@pytest.mark.gpu
def test_submit_many_answers_each_payload_like_alone(pkg, orc):
    """ipr_service_submit_batch: a burst queued atomically, every response bit-exact"""
    plan = pkg.plan_from_shape(10_000, 32, 1184)
    sdb = orc.SynthDB(plan.db_rows, plan.instances, plan.interp, plan.c, seed=5)
    qs = [orc.synth_query(40 + i, plan.db_rows, 2) for i in range(70)] + [orc.synth_query(9, plan.db_rows, 1)]
    with pkg.KeywordServer.synthetic(plan, seed=5) as srv:
        svc = pkg.KeywordService([srv], max_batch=64)
        try:
            tickets = svc.submit_many(0, qs)
            got = [svc.wait(t) for t in tickets]
            with pytest.raises(pkg.IprError):
                svc.submit_many(0, [qs[0], b""])  # one malformed payload: none queued
        finally:
            svc.close()
    for q, g in zip(qs, got):
        assert g == orc.respond(sdb, q)


@pytest.mark.gpu
def test_full_batches_staged_at_once_and_diagnose(pkg, orc, dbs):
    """a queue holding several full batches fills both I/O slots at once (no staging lead);
    every response equals the payload answered alone, and ipr_service_diagnose reports the
    lane idle afterwards"""
    plan, srv, sdb = dbs[0]
    qs = [orc.synth_query(900 + i, plan.db_rows, 2) for i in range(40)]
    alone = [srv.respond_to_serialized_query(q) for q in qs]
    svc = pkg.KeywordService([srv], max_batch=8)
    try:
        tickets = svc.submit_many(0, qs)
        got = [svc.wait(t, 60_000) for t in tickets]
        for _ in range(100):  # the scheduler frees the last slot just after completing its requests
            text = svc.diagnose()
            if "0 slots busy" in text:
                break
            time.sleep(0.01)
        st = svc.stats()
    finally:
        svc.close()
    assert got == alone
    assert got[0] == orc.respond(sdb, qs[0]) and got[-1] == orc.respond(sdb, qs[-1])
    assert st.batches >= 5 and st.pending == 0 and st.in_flight == 0
    assert "db 0: max_batch 8, 0 pending, 0 slots busy" in text
    assert "slot 0:" in text and "slot 1:" in text and "server stream done" in text


@pytest.mark.gpu
def test_injected_allocation_failures_are_clean(pkg, orc):
    """every device allocation of server creation, a first respond and batch preparation fails
    once in turn (ipr_debug_fail_allocation): the call that needed it returns IPR_E_OOM, the
    server stays usable and bit-exact, and closing everything returns the device memory"""
    import torch
    plan = pkg.plan_from_shape(10_000, 32, 1184)
    sdb = orc.SynthDB(plan.db_rows, plan.instances, plan.interp, plan.c, seed=3)
    q = orc.synth_query(77, plan.db_rows, 2)
    want = orc.respond(sdb, q)
    with pkg.KeywordServer.synthetic(plan, seed=3) as warm:  # first-use tables and context
        assert warm.respond_to_serialized_query(q) == want
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    fired = 0
    for n in range(200):
        pkg.fail_allocation_after(n)
        srv = None
        try:
            srv = pkg.KeywordServer.synthetic(plan, seed=3)
            for step in (lambda: srv.respond_to_serialized_query(q), lambda: srv.prepare_batch(4),
                         lambda: srv.respond_batch([q, q])):
                try:
                    step()
                except pkg.IprError as e:
                    assert e.status == -2, e  # IPR_E_OOM
                    fired += 1
        except pkg.IprError as e:
            assert e.status == -2, e
            fired += 1
            continue
        finally:
            pkg.fail_allocation_after(-1)
        try:
            # after the failure, the same server answers bit-exactly
            assert srv.respond_to_serialized_query(q) == want
            assert srv.respond_batch([q, q]) == [want, want]
        finally:
            srv.close()
        if fired < n + 1 and n > 0:  # the countdown outlived every allocation: all points covered
            break
    assert fired >= 10
    torch.cuda.synchronize()
    assert abs(torch.cuda.mem_get_info()[0] - free0) < (64 << 20)


@pytest.mark.gpu
def test_service_with_autotuned_servers_answers_exactly(pkg, orc):
    plan = pkg.plan_from_shape(10_000, 32, 1184)
    sdb = orc.SynthDB(plan.db_rows, plan.instances, plan.interp, plan.c, seed=21)
    qs = [orc.synth_query(300 + i, plan.db_rows, 2) for i in range(12)]
    with pkg.KeywordServer.synthetic(plan, seed=21) as srv:
        svc = pkg.KeywordService([srv], max_batch=8, autotune=True)
        try:
            got = [svc.wait(t) for t in svc.submit_many(0, qs)]
        finally:
            svc.close()
    assert got == [orc.respond(sdb, q) for q in qs]
