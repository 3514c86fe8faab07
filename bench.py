#!/usr/bin/env python3
"""Benchmark of the B200 respond() path (InsPIRe keyword PIR, rkdud007/inspire-rs).

Workload: 1,000,000 ML-KEM-768 records (32-byte IDs + 1184-byte keys), cuckoo
buckets 2^21 (the reference default for 1M records; 262,144 is rejected by the
reference because buckets < records), dim0 = 2048 -> DB 2048 x 720,896 u16,
352 packing outputs, interpolation degree 32, 11 fold groups.  One step = one
batch of B (default 64) KeywordQueryPayloads (2 cuckoo sub-queries each) from
B distinct clients, answered together on the INT8-limb tensor-core path;
`--batch 1` times the batch-1 path.  The same run also times the plain batch-1
u64 path (CUDA-core GEMV and packing) on the same GPU.  Server state is seeded synthetic data of the reference's
shapes (the reference's own timing mode, engine.rs:693-729); queries are
seeded synthetic payloads.

  value : payloads/s with queries resident in HBM (ipr_server_respond_batch_device)
  e2e   : payloads/s through the serving API (KeywordService: submit host
          bytes, wait for host bytes; H2D queries and D2H responses of every
          batch inside the timed region)
  serving: p50/p99 latency and throughput under Poisson arrivals at stated
          loads (default 1000 and 2500 payloads/s, 3 s each)

--impl reference times the CPU restatement of the reference's respond() on the
host cores (the reference's Rust CPU path cannot be built here).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))

RECORDS, KEY, VALUE, BUCKETS, DIM0 = 1_000_000, 32, 1184, 2_097_152, 2048
N = 2048
METRIC = "queries/s at 1M ML-KEM-768 keys, batch-64 INT8-limb vs batch-1 u64, bit-exact"
UNIT = "payloads/s"


def load_package():
    import importlib.util
    if "inspire_rs_b200" in sys.modules:
        return sys.modules["inspire_rs_b200"]
    d = os.path.join(ROOT, "inspire-rs_b200")
    spec = importlib.util.spec_from_file_location("inspire_rs_b200", os.path.join(d, "__init__.py"),
                                                  submodule_search_locations=[d])
    m = importlib.util.module_from_spec(spec)
    sys.modules["inspire_rs_b200"] = m
    spec.loader.exec_module(m)
    return m


def load_oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    return oracle


class ClockSampler:
    """nvidia-smi samples of SM clock, power and throttle reasons.  Each sample carries the
    driver's own timestamp, so that the summary covers only [begin(), end()] when those are
    marked: the 20 ms samples taken before and after the timed region run at idle clocks."""
    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index, interval_ms=20):
        self.gpu = gpu_index
        self.interval = interval_ms
        self.proc = None
        self.lines = []
        self.t0 = self.t1 = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", str(self.interval)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def begin(self):
        self.t0 = time.time()

    def end(self):
        self.t1 = time.time()

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    @staticmethod
    def _when(ts):
        import datetime
        try:
            return datetime.datetime.strptime(ts, "%Y/%m/%d %H:%M:%S.%f").timestamp()
        except ValueError:
            return None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 10:
                continue
            try:
                rows.append((self._when(f[0]), float(f[2]), float(f[3]), float(f[4]), f[6:10]))
            except ValueError:
                continue
        window = "whole run"
        if self.t0 is not None and self.t1 is not None:
            inside = [r for r in rows if r[0] is not None and self.t0 <= r[0] <= self.t1]
            if inside:
                rows, window = inside, "timed region"
        sm = [r[1] for r in rows]
        mx = rows[-1][2] if rows else None
        power = [r[3] for r in rows]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for nm, v in zip(names, r[4]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "sm_mhz_min": min(sm) if sm else None, "power_w": statistics.median(power) if power else None,
                "reasons": sorted(reasons), "samples": len(sm), "window": window}


def read_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def read_bf16_peak(sustained=False):
    """dense bf16 TFLOP/s of a cuBLAS GEMM timed alone (burst) or in a seconds-long loop under
    the power cap (sustained), measured or the fallback"""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops_sustained" if sustained else "bf16_tflops"]), "measured"
    except Exception:
        return (1400.0 if sustained else 1590.0), "fallback"


def read_traffic(kernel="k_pack"):
    """dram bytes per launch of `kernel` from its committed ncu summary (scaled to the full launch), or None"""
    path = os.path.join(ROOT, "profiles", f"{kernel}_1M_dram.md")
    try:
        for ln in open(path):
            if ln.startswith("traffic_bytes_per_full_launch:"):
                return float(ln.split(":")[1])
    except OSError:
        pass
    return None


class CpuFullRespond:
    """The oracle's respond() (the CPU restatement of KeywordServer::respond,
    src/pir/server/keyword.rs:534-628) on the whole 1M workload, measured, not scaled.
    The 11 fold groups are independent (keyword.rs:558-574): each group's slice of the
    synthetic server state (its 65,536 DB columns and 32 packing outputs, 3.2 GB) is
    generated on its own, untimed, and answered for every payload, so a payload's time is
    the sum of its 11 measured group answers (the query is parsed once per group).  Only
    one group's state is held at a time."""

    def __init__(self, orc):
        self.orc = orc
        self.plan = orc.plan_from_shape(RECORDS, KEY, VALUE, BUCKETS, DIM0)
        self.groups = self.plan["c"]
        self.q = orc.synth_query(2026, self.plan["db_rows"], 2)

    def run(self, warmup, steps):
        """seconds per payload for `steps` payloads, after `warmup` untimed ones per group"""
        p, orc = self.plan, self.orc
        per = [0.0] * steps
        for g in range(self.groups):
            sdb = orc.SynthDB.shard_of(p["db_rows"], g * p["interp"], p["interp"], p["interp"], 1, seed=7)
            for _ in range(warmup):
                orc.respond(sdb, self.q)
            for k in range(steps):
                t0 = time.perf_counter()
                orc.respond(sdb, self.q)
                per[k] += time.perf_counter() - t0
            del sdb
        return per

    def describe(self, per_payload, steps):
        return {"value": 1.0 / per_payload, "unit": UNIT, "cores": int(self.orc.threads()), "kind": "port",
                "sample": f"oracle respond() of {steps} full payloads (2 queries): all {self.groups} fold groups "
                          f"answered, each on its own slice of the 1M state generated in turn (untimed); "
                          f"{per_payload:.2f} s/payload"}


def cpu_sample(orc, payloads=3):
    s = CpuFullRespond(orc)
    per = s.run(1, payloads)
    return s.describe(statistics.median(per), payloads)


SERVICE_WAIT_S = 120.0  # no request of these loads waits that long unless the service is stuck


def svc_wait(svc, ticket, timeout_s=SERVICE_WAIT_S):
    """a service response within timeout_s; otherwise the service's counters and its last
    batches go to stderr and the process ends (a stuck wait would hold the GPU indefinitely)"""
    r = svc.wait(ticket, int(timeout_s * 1000))
    if r is None:
        try:
            st = svc.stats()
            print(f"service wait timed out after {timeout_s:.0f} s on ticket {ticket}: {st}", file=sys.stderr)
            print(svc.diagnose(), file=sys.stderr)
            for b in svc.batch_log(16):
                print(f"  batch {b}", file=sys.stderr)
            sys.stderr.flush()
            smi = subprocess.run(["nvidia-smi", "--query-gpu=utilization.gpu,clocks.sm,power.draw,memory.used",
                                  "--format=csv"], capture_output=True, text=True, timeout=30)
            print(smi.stdout, file=sys.stderr)
        finally:
            sys.stderr.flush()
            sys.stdout.flush()
            os._exit(3)
    return r


def poisson_load(svc, payloads, rate, seconds, per_db=None):
    """Poisson arrivals at `rate` payloads/s for `seconds`; latency = submit -> response ready
    inside the service (p50/p99 over all requests), throughput = completions / elapsed.
    With `per_db` (one payload list per database) each arrival picks a database uniformly."""
    import queue
    import random
    svc.reset_stats()
    rng = random.Random(int(rate))
    pick = random.Random(int(rate) + 1)
    n = max(1, int(rate * seconds))
    q = queue.Queue()
    done = []

    def collector():
        while True:
            t = q.get()
            if t is None:
                return
            svc_wait(svc, t)
            done.append(time.perf_counter())

    th = threading.Thread(target=collector, daemon=True)
    th.start()
    t_start = time.perf_counter()
    t_next = t_start
    try:
        for i in range(n):
            t_next += rng.expovariate(rate)
            d = t_next - time.perf_counter()
            if d > 0:
                time.sleep(d)
            if per_db:
                db = pick.randrange(len(per_db))
                q.put(svc.submit(db, per_db[db][i % len(per_db[db])]))
            else:
                q.put(svc.submit(0, payloads[i % len(payloads)]))
        offered_s = time.perf_counter() - t_start
    finally:
        q.put(None)  # the collector ends even when a submission raised
    th.join()
    st = svc.stats()
    return {"offered_payloads_per_s": rate, "arrived_payloads_per_s": n / offered_s, "payloads": n,
            "completed_payloads_per_s": n / (done[-1] - t_start), "p50_ms": st.p50_us / 1e3,
            "p99_ms": st.p99_us / 1e3, "mean_ms": st.mean_us / 1e3, "max_ms": st.max_us / 1e3,
            "mean_batch": st.batched_payloads / max(st.batches, 1), "failed": st.failed,
            "batch_ms_mean": st.batch_ms_mean, "batch_ms_max": st.batch_ms_max,
            "queue_ms_mean": st.queue_ms_mean, "queue_ms_max": st.queue_ms_max}


CONFIG4 = (  # (name, records, key bytes, value bytes, buckets, seed): three databases at dim0 = 8192
    ("ML-KEM-512 x 4M", 4_000_000, 32, 800, 1 << 23, 7),
    ("ML-KEM-768 x 1M", 1_000_000, 32, 1184, 1 << 21, 8),
    ("ML-KEM-1024 x 2M", 2_000_000, 32, 1568, 1 << 22, 9),
)


def serve_config4(pkg, rates, seconds):
    """Serving three databases from one GPU (ML-KEM-512 x 4M, -768 x 1M, -1024 x 2M records,
    dim0 8192, seeds 7/8/9): saturation throughput of the serving loop and p50/p99 latency
    under Poisson arrivals spread uniformly over the databases.  One JSON line."""
    import numpy as np
    import torch
    torch.cuda.set_device(0)
    servers, plans, per_db = [], [], []
    t0 = time.perf_counter()

    def progress(what):  # phase marks on stderr: the JSON line on stdout comes only at the end
        print(f"[serve-config4 {time.perf_counter() - t0:7.1f} s] {what}", file=sys.stderr, flush=True)

    for name, rec, key, val, buckets, seed in CONFIG4:
        plan = pkg.plan_from_shape(rec, key, val, buckets, 8192)
        srv = pkg.KeywordServer.synthetic(plan, seed=seed)
        servers.append(srv)
        plans.append(plan)
        rng = np.random.default_rng(seed)
        pays = []
        for _ in range(32):
            nvals = 3 * N * 2 + 2 * (plan.db_rows + 6 * N)
            lo = rng.integers(0, 268369921, nvals, dtype=np.uint64)
            hi = rng.integers(0, 249561089, nvals, dtype=np.uint64)
            v = (lo | (hi << np.uint64(28))).astype("<u8")
            pays.append(bytes([2]) + v.view(np.uint8).reshape(-1, 8)[:, :7].tobytes())
        per_db.append(pays)
    svc = pkg.KeywordService(servers, max_batch=64)
    setup_s = time.perf_counter() - t0
    progress("three databases and the service are up")
    for db in range(3):
        for t in [svc.submit(db, per_db[db][i % 32]) for i in range(64)]:
            svc_wait(svc, t)
    # saturation: every database kept full, 16 batches of 64 per database; the median of
    # three repetitions (a single short burst varies with host scheduling)
    n_each = 16 * 64
    sat_runs = []
    for _ in range(3):
        t1 = time.perf_counter()
        tickets = [svc.submit(i % 3, per_db[i % 3][(i // 3) % 32]) for i in range(3 * n_each)]
        for t in tickets:
            svc_wait(svc, t)
        sat_runs.append(3 * n_each / (time.perf_counter() - t1))
    sat = statistics.median(sat_runs)
    progress(f"saturation runs {[round(x) for x in sat_runs]} payloads/s")
    poisson_load(svc, None, rates[0], 0.5, per_db=per_db)  # warm-up at the first load, not reported
    clocks = ClockSampler(0, interval_ms=100)
    clocks.start()
    time.sleep(0.5)
    clocks.begin()
    # at least 1,000 arrivals per load, so that a p99 rests on ten or more samples
    serving = []
    for r in rates:
        serving.append(poisson_load(svc, None, r, max(seconds, 1000.0 / r), per_db=per_db))
        progress(f"Poisson load {r:g}/s: p99 {serving[-1]['p99_ms']:.1f} ms")
    clocks.end()
    clk = clocks.stop()
    st = svc.stats()
    free_b, total_b = torch.cuda.mem_get_info()
    hbm = total_b - free_b  # the whole device in use while serving
    svc.close()
    for s in servers:
        s.close()
    line = {"metric": "serving three keyword databases on one GPU (Poisson arrivals, uniform over databases)",
            "value": sat, "unit": "payloads/s at saturation", "n_gpus": 1, "higher_is_better": True,
            "data": "synthetic",
            "config": {"workload": "config 4: " + ", ".join(c[0] for c in CONFIG4) + ", dim0 8192",
                       "databases": [{"name": c[0], "db_rows": p.db_rows, "db_cols": p.db_cols,
                                      "instances": p.instances, "c": p.c} for c, p in zip(CONFIG4, plans)],
                       "max_batch": st.max_batch, "device_bytes_in_use": hbm, "setup_s": setup_s,
                       "saturation_runs": sat_runs, "saturation_payloads_per_run": 3 * n_each},
            "serving": serving, "clocks": clk}
    print(json.dumps(line))
    return 0


def micro_bench(pkg, steps, warmup):
    """Kernel microbenchmarks on seeded data: batched limb NTT / INTT of 4096 polynomials
    (64 MB of u64 coefficients in and out per prime) and NTT-domain automorphisms of the
    same batch under all 2048 odd t < 4096 (137 GB of writes per prime, produced 64 t at a
    time into a 4 GB rotating output).  One JSON line per measurement."""
    import numpy as np
    import torch
    torch.cuda.set_device(0)
    peak, peak_kind = read_peaks()
    count = 4096
    lines = []

    def roofline(nbytes, ms):
        gbs = nbytes / (ms / 1000.0) / 1e9
        return {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
                "peak_source": peak_kind}

    for limb, q in ((0, 268369921), (1, 249561089)):
        rng = np.random.default_rng(limb)
        polys = torch.from_numpy(rng.integers(0, q, (count, N), dtype=np.uint64).view(np.int64)).cuda()
        for inverse in (False, True):
            for _ in range(warmup):
                pkg.ntt_batch(polys.data_ptr(), count, limb, inverse=inverse)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            for _ in range(steps):
                pkg.ntt_batch(polys.data_ptr(), count, limb, inverse=inverse)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / steps
            lines.append({"metric": f"{'intt' if inverse else 'ntt'} limb {limb}: 4096 x 2048 u64 coefficients",
                          "value": count / (ms / 1000.0), "unit": "polys/s", "ms_per_launch": ms,
                          "roofline": roofline(2 * count * N * 8, ms)})
        nk = 64
        ks_all = np.arange(1, 4096, 2, dtype=np.uint32)
        d_ks = torch.from_numpy(ks_all.view(np.int32)).cuda()
        out = torch.empty((nk, count, N), dtype=torch.int64, device="cuda")
        launches = len(ks_all) // nk
        for w in range(min(warmup, launches)):
            pkg.automorph_batch(polys.data_ptr(), count, d_ks.data_ptr() + 4 * nk * w, nk, out.data_ptr())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for i in range(launches):
            pkg.automorph_batch(polys.data_ptr(), count, d_ks.data_ptr() + 4 * nk * i, nk, out.data_ptr())
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        written = len(ks_all) * count * N * 8
        lines.append({"metric": f"galois limb {limb}: 4096 polys x all 2048 odd t",
                      "value": written / (ms / 1000.0) / 1e9, "unit": "GB/s written", "ms_total": ms,
                      "roofline": roofline(written, ms)})
        del out
    # setup-time DB encode at the 1M shape: 2048 x 720,896 u16, interpolation degree 32
    rows, cols, interp = 2048, 720896, 32
    raw = torch.randint(0, 65535, (rows * cols,), dtype=torch.int32, device="cuda").to(torch.int16)
    enc = torch.empty_like(raw)
    for _ in range(warmup):
        pkg.encode_db(raw.data_ptr(), enc.data_ptr(), rows, cols, interp)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        pkg.encode_db(raw.data_ptr(), enc.data_ptr(), rows, cols, interp)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    lines.append({"metric": "DB encode (1M ML-KEM-768 shape: 2048 x 720896 u16, interp 32)", "value": ms,
                  "unit": "ms", "higher_is_better": False, "roofline": roofline(2 * rows * cols * 2, ms)})
    del raw
    # offline precomputation at the 1M shape: 352 packing instances from the encoded DB above
    inst = cols // N
    a_hat = torch.empty(inst * N, dtype=torch.int64, device="cuda")
    bt = torch.empty(inst * 3069 * N, dtype=torch.int64, device="cuda")
    btb = torch.empty_like(bt)
    bth = torch.empty(inst * 3 * N, dtype=torch.int64, device="cuda")
    args = (enc.data_ptr(), rows, inst, a_hat.data_ptr(), bt.data_ptr(), btb.data_ptr(), bth.data_ptr())
    pkg.offline_precompute(*args)  # warm-up
    reps = 3
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        pkg.offline_precompute(*args)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    # bytes that must cross HBM once: the DB read, bold_t + bold_t_bar + bold_t_hat + a_hat written
    algo = rows * cols * 2 + (2 * 3069 + 3 + 1) * N * 8 * inst
    line = {"metric": "offline precomputation (1M ML-KEM-768 shape: 352 instances, db_rows 2048)", "value": ms,
            "unit": "ms", "higher_is_better": False, "roofline": roofline(algo, ms)}
    try:  # the oracle on one instance of the same DB, scaled to 352 (reference CPU loops)
        sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle"))
        import oracle as orc
        db0 = enc[: N * rows].cpu().numpy().view(np.uint16).copy()
        t0 = time.perf_counter()
        orc.offline_precompute(db0, rows, 1)
        cpu_s = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": cpu_s * inst * 1000.0, "unit": "ms", "cores": orc.threads(),
                                "kind": "port", "sample": f"1 of {inst} instances ({cpu_s:.1f} s), scaled"}
    except Exception as exc:  # the timing line stands without it
        line["cpu_baseline"] = {"unavailable": str(exc)[:120]}
    lines.append(line)
    del a_hat, bt, btb, bth, enc
    # InspiRING: pack 2048 LWEs (uniform mod q, seeded) into one RLWE, packing_fully_online;
    # one set alone (latency) and 16 sets per call (throughput)
    rng = np.random.default_rng(2048)
    qq = 268369921 * 249561089
    max_sets = 16
    lwe = torch.from_numpy(rng.integers(0, qq, (max_sets, N + 1, N), dtype=np.uint64).view(np.int64)).cuda()
    keys = (rng.integers(0, 268369921, (2, 3, N), dtype=np.uint64)
            | (rng.integers(0, 249561089, (2, 3, N), dtype=np.uint64) << np.uint64(32)))
    d_y = torch.from_numpy(keys[0].view(np.int64)).cuda()
    d_z = torch.from_numpy(keys[1].view(np.int64)).cuda()
    out = torch.empty((max_sets, 2, N), dtype=torch.int64, device="cuda")
    with pkg.InspiringPacker(max_sets=max_sets) as pk:
        for sets in (1, max_sets):
            for _ in range(max(warmup, 1)):
                pk.pack(sets, lwe.data_ptr(), d_y.data_ptr(), d_z.data_ptr(), out.data_ptr())
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            for _ in range(steps):
                pk.pack(sets, lwe.data_ptr(), d_y.data_ptr(), d_z.data_ptr(), out.data_ptr())
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / steps
            line = {"metric": f"InspiRING pack: {sets} x 2048 LWEs -> {sets} RLWE (packing_fully_online)",
                    "value": sets * 2048 / (ms / 1000.0), "unit": "LWEs packed/s", "ms_per_call": ms}
            if sets == 1:
                try:
                    import oracle as orc
                    l0 = lwe[0].cpu().numpy().view(np.uint64).copy()
                    t0 = time.perf_counter()
                    orc.inspiring_pack(l0, keys[0], keys[1])
                    cpu_s = time.perf_counter() - t0
                    line["cpu_baseline"] = {"value": 2048 / cpu_s, "unit": "LWEs packed/s", "cores": orc.threads(),
                                            "kind": "port", "sample": f"1 set ({cpu_s:.1f} s)"}
                except Exception as exc:
                    line["cpu_baseline"] = {"unavailable": str(exc)[:120]}
            lines.append(line)
    # dataset generation (DatasetGenerator): 1M ML-KEM-768 records (id || key) into device memory
    gen = pkg.DatasetGenerator("ml-kem-768", RECORDS).with_seed(7)
    recs = torch.empty(RECORDS * gen.record_size, dtype=torch.uint8, device="cuda")
    gen.generate_device(recs.data_ptr(), 0, 65536)  # warm-up
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    gen.generate_device(recs.data_ptr())
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    line = {"metric": "dataset generation: 1M ML-KEM-768 records (ChaCha20 seed, FIPS 203 key, SHA3-256 id)",
            "value": RECORDS / (ms / 1000.0), "unit": "records/s", "ms_total": ms}
    try:  # the oracle's restatement of the same records on the host cores (one thread per call)
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as orc
        n_cpu = 2000
        t0 = time.perf_counter()
        for i in range(n_cpu):
            orc.dataset_record("ml-kem-768", 7, i)
        cpu_s = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": n_cpu / cpu_s, "unit": "records/s", "cores": 1, "kind": "port",
                                "sample": f"{n_cpu} records on one host thread ({cpu_s:.1f} s)"}
    except Exception as exc:
        line["cpu_baseline"] = {"unavailable": str(exc)[:120]}
    lines.append(line)
    del recs
    # the client on the GPU (ipr_client_*) at the 1M plan: one payload of 2 sub-queries built
    # and serialized (host bytes out), and one 2 x 11-result response decrypted (host bytes in)
    plan = pkg.plan_from_shape(RECORDS, KEY, VALUE, BUCKETS, DIM0)
    resp_len = 4 + 2 * (4 + plan.c * 12288) + 4
    rb = bytearray(np.random.default_rng(5).integers(0, 256, resp_len, dtype=np.uint8).tobytes())
    rb[0:4] = (2).to_bytes(4, "little")
    for k in range(2):
        o = 4 + k * (4 + plan.c * 12288)
        rb[o:o + 4] = (plan.c * 12288).to_bytes(4, "little")
    rb[-4:] = bytes(4)
    resp = bytes(rb)
    buckets = [12345, 1_500_000]
    with pkg.KeywordClient(plan, bytes(range(32))) as cl:
        for name, fn in (("query generation", lambda i: cl.query(buckets, nonce=i)),
                         ("response decryption", lambda i: cl.decrypt(resp))):
            for i in range(max(warmup, 1)):
                fn(i)
            t0 = time.perf_counter()
            for i in range(steps):
                fn(1000 + i)
            ms = (time.perf_counter() - t0) * 1000.0 / steps
            line = {"metric": f"client {name} on the GPU (1M plan, 2 sub-queries, host bytes)",
                    "value": 1000.0 / ms, "unit": "payloads/s", "ms_per_call": ms}
            try:
                sys.path.insert(0, os.path.join(ROOT, "oracle"))
                import pir_client as pcl
                model = pcl.SeededClient(plan.db_rows, plan.interp, plan.c, plan.num_items // plan.db_rows, 608,
                                         seed=bytes(range(32)))
                t0 = time.perf_counter()
                if name == "query generation":
                    model.query(buckets, nonce=1)
                else:
                    model.decrypt(resp)
                cpu_s = time.perf_counter() - t0
                line["cpu_baseline"] = {"value": 1.0 / cpu_s, "unit": "payloads/s", "cores": 1, "kind": "port",
                                        "sample": f"1 payload, oracle model of the client ({cpu_s * 1000:.1f} ms)"}
            except Exception as exc:
                line["cpu_baseline"] = {"unavailable": str(exc)[:120]}
            lines.append(line)
    for ln in lines:
        print(json.dumps(ln))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--records", type=int, default=RECORDS, help="workload override (profiling small cases)")
    ap.add_argument("--buckets", type=int, default=None)
    ap.add_argument("--plan", type=int, nargs=2, metavar=("INSTANCES", "INTERP"), default=None,
                    help="profiling case: a synthetic plan of INSTANCES packing outputs and interpolation degree "
                         "INTERP (db_rows 2048, INSTANCES / INTERP fold groups) instead of a record count")
    ap.add_argument("--dim0", type=int, default=None)
    ap.add_argument("--batch", type=int, default=64, help="payloads per step (1 = batch-1 u64 packing path)")
    ap.add_argument("--no-batch1", action="store_true", help="skip the batch-1 comparison measurement")
    ap.add_argument("--shard", action="store_true",
                    help="under torchrun: one database split by fold groups over the ranks (each rank answers its "
                         "groups of every payload; NCCL broadcast of the queries and gather of the parts) "
                         "instead of one replica per rank")
    ap.add_argument("--fold-form", type=int, default=3, choices=[1, 2, 3, 4, 5],
                    help="3: fold with the packing post-process fused in, one chain per CTA, two or three CTAs "
                         "per SM by chain count (default); 4 / 5: always three / two per SM; 2: the same on two "
                         "chains per CTA; 1: separate INTT + CRT pass")
    ap.add_argument("--cuda-core-gemv", type=int, default=None, metavar="FORM",
                    help="with --batch 1: the first dimension on the CUDA-core GEMV of this IPR_OPT_GEMV_FORM "
                         "instead of the tensor-core GEMV (a profiling case for that kernel)")
    ap.add_argument("--no-serving", action="store_true", help="skip the Poisson serving measurement")
    ap.add_argument("--serve-rates", type=float, nargs="*", default=[1000.0, 2500.0],
                    help="offered Poisson loads (payloads/s) for the serving measurement")
    ap.add_argument("--serve-seconds", type=float, default=3.0)
    ap.add_argument("--serve-config4", action="store_true",
                    help="serve three databases (ML-KEM-512 x4M, -768 x1M, -1024 x2M at dim0 8192) under Poisson load")
    ap.add_argument("--micro", action="store_true",
                    help="kernel microbenchmarks (batched NTT / INTT, Galois automorphisms) instead of the step")
    args = ap.parse_args()
    small = args.records != RECORDS or args.plan is not None
    if args.micro:
        return micro_bench(load_package(), max(args.steps, 3), max(args.warmup, 1))
    if args.serve_config4:
        rates = args.serve_rates if args.serve_rates != [1000.0, 2500.0] else [100.0, 300.0, 1200.0, 2500.0]
        return serve_config4(load_package(), rates, args.serve_seconds)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        s = CpuFullRespond(load_oracle())
        times = s.run(args.warmup, args.steps)
        v = args.steps / sum(times)
        cb = s.describe(sum(times) / args.steps, args.steps)
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / v, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": "1M ML-KEM-768 respond(), buckets 2^21, dim0 2048, 2 queries/payload",
                       "records": RECORDS, "buckets": BUCKETS, "dim0": DIM0, "batch": 1},
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }))
        return 0

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()

    pkg = load_package()
    if args.plan is not None:
        inst, interp = args.plan
        plan = pkg.Plan(num_items=32768, entry_size=KEY + VALUE, item_size_bits=8 * (KEY + VALUE), dim0=2048,
                        db_rows=2048, db_cols=inst * N, instances=inst, interp=interp, c=inst // interp, peak_bytes=0)
    elif small:
        plan = pkg.plan_from_shape(args.records, KEY, VALUE, args.buckets, args.dim0)
    else:
        plan = pkg.plan_from_shape(RECORDS, KEY, VALUE, BUCKETS, DIM0)
    shard = args.shard and world > 1
    if shard:  # this rank's fold groups of one synthetic database
        srv = pkg.KeywordServer.synthetic_shard(plan, world, rank, seed=7, device=dev)
    else:
        srv = pkg.KeywordServer.synthetic(plan, seed=7 + rank, device=dev)
    local = srv.plan  # the rank's share: the whole plan for a replica, a fold-group slice for a shard
    if args.fold_form != 3:
        srv.set_option(pkg.KeywordServer.OPT_FOLD_REGISTER_NTT, args.fold_form)
    if args.cuda_core_gemv is not None:
        srv.set_option(pkg.KeywordServer.OPT_TENSOR_GEMV, 0)
        srv.set_option(pkg.KeywordServer.OPT_GEMV_FORM, args.cuda_core_gemv)
    qbytes = srv.query_bytes(2)
    rbytes = srv.response_bytes(2)

    import numpy as np

    def synth_payload(seed):
        # a structurally valid payload: uniform 28-bit residues below each prime
        rng = np.random.default_rng(seed)
        nvals = 3 * N * 2 + 2 * (plan.db_rows + 6 * N)
        lo = rng.integers(0, 268369921, nvals, dtype=np.uint64)
        hi = rng.integers(0, 249561089, nvals, dtype=np.uint64)
        v = (lo | (hi << np.uint64(28))).astype("<u8")
        return bytes([2]) + v.view(np.uint8).reshape(-1, 8)[:, :7].tobytes()

    B = max(1, args.batch)
    # one batched pass answers up to 64 payloads (the packing GEMM's N = 64 clients x 4 byte
    # limbs = 256 columns); larger batches run as consecutive passes of 64
    PASS = 64
    passes = (B + PASS - 1) // PASS if B > 1 else 1
    npay = max(2 * B, 4)
    payloads = [synth_payload((0 if shard else 1000 * rank) + i) for i in range(npay)]
    assert len(payloads[0]) == qbytes
    stream = torch.cuda.ExternalStream(srv.stream_handle(), device=dev)
    # HBM-resident inputs: two distinct batches of B payloads, alternated
    d_batches = [torch.frombuffer(bytearray(b"".join(payloads[k * B:(k + 1) * B])), dtype=torch.uint8).to(dev)
                 for k in range(2)]
    d_out = torch.empty(B * rbytes, dtype=torch.uint8, device=dev)
    tune = None
    if B > 1:
        srv.prepare_batch(min(B, PASS))
        # the autotuner times the exact candidate configurations of the batch path and keeps the fastest
        tune = srv.autotune(min(B, PASS), 5)

    def run_device(i):
        d = d_batches[i % 2]
        if B > 1:
            for c0 in range(0, B, PASS):
                srv.respond_batch_device(min(PASS, B - c0), d.data_ptr() + c0 * qbytes, d_out.data_ptr() + c0 * rbytes)
        else:
            srv.respond_device(d.data_ptr(), qbytes, d_out.data_ptr(), rbytes)

    def run_host(i):
        batch = payloads[(i % 2) * B:(i % 2 + 1) * B]
        if B > 1:
            srv.respond_batch(batch)
        else:
            srv.respond_to_serialized_query(batch[0])

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # the clock sampler runs from the warm-up on (nvidia-smi takes a moment to start); its
    # summary keeps only the samples inside the timed region
    clocks = ClockSampler(dev if world == 1 else local)
    clocks.start()
    for i in range(args.warmup):
        run_device(i)
        run_host(i)
    srv.sync()

    # ---- device-resident timed region -------------------------------------------------
    srv.set_profiling(True)
    barrier()
    clocks.begin()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(args.steps):
        run_device(i)
    e1.record(stream)
    srv.sync()
    clocks.end()
    barrier()
    dev_ms = e0.elapsed_time(e1)
    stage_ms, calls = srv.stage_times()
    plan_response_bytes = 4 + 2 * (4 + plan.c * 12288) + 4  # the merged (whole-database) response
    srv.set_profiling(False)
    clk = clocks.stop()

    # ---- end-to-end through the serving API: host buffers, H2D + D2H of every batch ---------
    # (KeywordService: continuous batching, pinned staging, copies overlapped with compute)
    svc = pkg.KeywordService([srv], max_batch=min(B, PASS)) if B > 1 and not shard else None
    barrier()
    # the blocking call (ipr_server_respond_batch / ipr_server_respond), for comparison
    t0 = time.perf_counter()
    for i in range(args.steps):
        run_host(i)
    blocking_ms = (time.perf_counter() - t0) * 1000
    e2e_ms = blocking_ms
    e2e_steps = args.steps  # batches of B payloads in the end-to-end timed region
    if shard:
        # the public sharded API: rank 0's host payloads broadcast over NCCL, every rank answers
        # its groups (ipr_server_respond_batch, host bytes), the parts gathered and merged on rank 0
        sks = pkg.ShardedKeywordServer(srv.respond_to_serialized_query, device=torch.device("cuda", dev))
        sks.respond_batch(payloads[:B] if rank == 0 else None, srv.respond_batch)
        barrier()
        t0 = time.perf_counter()
        for i in range(args.steps):
            batch = payloads[(i % 2) * B:(i % 2 + 1) * B]
            sks.respond_batch(batch if rank == 0 else None, srv.respond_batch)
        barrier()
        e2e_ms = (time.perf_counter() - t0) * 1000
    if svc is not None:
        for t in [svc.submit(0, payloads[i % npay]) for i in range(2 * B)]:
            svc_wait(svc, t)
        barrier()
        # at least 64 batches (about a second): the pipeline's fill and drain, one batch each,
        # and host scheduling noise then weigh little in the rate
        e2e_steps = max(args.steps, 64)
        t0 = time.perf_counter()
        # handed over a batch's worth at a time (ipr_service_submit_batch): the first dispatch
        # already fills a whole batch, and later bursts are staged while earlier ones compute
        tickets = []
        for s0 in range(0, e2e_steps * B, B):
            tickets += svc.submit_many(0, [payloads[i % npay] for i in range(s0, min(s0 + B, e2e_steps * B))])
        for t in tickets:
            svc_wait(svc, t)
        e2e_ms = (time.perf_counter() - t0) * 1000
    barrier()

    # ---- serving at stated Poisson loads (1-GPU runs) -----------------------------------
    serving = []
    if svc is not None and world == 1 and not args.no_serving:
        poisson_load(svc, payloads, args.serve_rates[0], 0.5)  # warm-up at the first load, not reported
        for rate in args.serve_rates:
            serving.append(poisson_load(svc, payloads, rate, args.serve_seconds))
    if svc is not None:
        svc.close()

    # ---- the plain batch-1 u64 path on the same GPU (CUDA-core GEMV + packing) ----------
    # the CUDA-core GEMV is timed in each of its forms (DB columns per warp); the fastest is
    # the u64 figure, its stage time against HBM (2 bytes per DB element, both queries in one
    # pass) is its roofline
    b1, u64_forms = {}, []
    if B > 1 and not args.no_batch1 and not shard:
        d1 = torch.frombuffer(bytearray(payloads[0]), dtype=torch.uint8).to(dev)
        d1o = torch.empty(rbytes, dtype=torch.uint8, device=dev)
        k1 = max(5, min(args.steps, 20))

        def single_rate():
            for _ in range(2):
                srv.respond_device(d1.data_ptr(), qbytes, d1o.data_ptr(), rbytes)
            srv.sync()
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record(stream)
            for _ in range(k1):
                srv.respond_device(d1.data_ptr(), qbytes, d1o.data_ptr(), rbytes)
            a1.record(stream)
            srv.sync()
            return k1 / (a0.elapsed_time(a1) / 1000.0)

        def single_gemv_ms():
            srv.set_profiling(True)
            for _ in range(k1):
                srv.respond_device(d1.data_ptr(), qbytes, d1o.data_ptr(), rbytes)
            srv.sync()
            st_ms, n_calls = srv.stage_times()
            srv.set_profiling(False)
            return st_ms["gemv"] / max(n_calls, 1)

        srv.set_option(pkg.KeywordServer.OPT_TENSOR_GEMV, 0)
        gemv_bytes = 2 * plan.db_rows * plan.db_cols
        forms = {0: "8 columns per warp, registers", 1: "4 columns per warp, registers",
                 2: "2 columns per warp, registers", 3: "8 columns per warp, cp.async ring in shared memory",
                 4: "8 columns per warp, exact products on the FP64 pipe",
                 5: "8 columns per warp, cp.async ring, FP64 pipe, residues converted once into shared memory",
                 6: "a lane per column, 16 warps, TMA-fed stages, FP64 pipe, residues broadcast"}
        for form, name in forms.items():
            srv.set_option(pkg.KeywordServer.OPT_GEMV_FORM, form)
            rate = single_rate()
            gms = single_gemv_ms()
            u64_forms.append({"form": form, "name": name, "payloads_per_s": rate, "gemv_ms": gms,
                              "gemv_gbs": gemv_bytes / (gms / 1000.0) / 1e9})
        best = min(u64_forms, key=lambda f: f["gemv_ms"])
        srv.set_option(pkg.KeywordServer.OPT_GEMV_FORM, best["form"])
        b1["u64"] = max(f["payloads_per_s"] for f in u64_forms)
        srv.set_option(pkg.KeywordServer.OPT_TENSOR_GEMV, 1)
        b1["tensor_gemv"] = single_rate()
        b1["u64_gemv"] = dict(best, bytes=gemv_bytes)

    t = torch.tensor([dev_ms, e2e_ms], dtype=torch.float64, device=dev)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dev_ms, e2e_ms = float(t[0]), float(t[1])
    total = args.steps * B * (1 if shard else world)  # a shard answers part of every payload
    value = total / (dev_ms / 1000.0)
    e2e = total * e2e_steps / args.steps / (e2e_ms / 1000.0)

    peak, peak_kind = read_peaks()
    pack_ms = stage_ms["pack"] / max(calls, 1)
    if B > 1:  # the packing GEMM streams the slot-indexed precomputation once per batch
        pack_bytes = N * 2 * ((local.instances + 31) // 32) * 128 * 3 * N  # [slot][limb][tile][128 rows][6144]
        kname = "k_pack_mma_pair" if min(B, PASS) >= 48 else "k_pack_mma"  # the server's default choice of form
    else:
        pack_bytes = local.instances * (2 * 3069 + 3) * N * 8  # bold_t + bold_t_bar + bold_t_hat per launch
        kname = "k_pack"
    achieved = pack_bytes / (pack_ms / 1000.0) / 1e9
    tensor = None
    if B > 1:
        # the packing GEMM multiplies every precomputation byte with every client byte column:
        # 2 ops x bytes streamed x N, N = 4 byte limbs x clients of a pass, rounded to 16
        nt = max(16, (4 * min(B, PASS) + 15) // 16 * 16)
        ops = 2.0 * pack_bytes * nt
        bf16, bf16_kind = read_bf16_peak()
        bf16s, _ = read_bf16_peak(sustained=True)
        i8_peak = 2 * bf16  # dense int8 issues at twice the bf16 rate on B200 (4.5 vs 2.25 P nominal)
        i8_sus = 2 * bf16s
        hbm_floor_ms, tensor_floor_ms = pack_bytes / (peak * 1e9) * 1e3, ops / (i8_peak * 1e12) * 1e3
        tensor = {"bound": "tensor", "kernel": kname, "ops_per_launch": ops,
                  "achieved_tops": ops / (pack_ms / 1000.0) / 1e12, "peak_tops": i8_peak,
                  "peak_source": f"2 x {bf16_kind} bf16 TFLOP/s" + ("" if bf16_kind == "measured"
                                                                     else " (MEASURED_PEAKS.json absent)"),
                  "frac": tensor_floor_ms / pack_ms,
                  # the launch runs inside a multi-step timed region, so the sustained rate under the
                  # power cap is its ceiling too
                  "peak_tops_sustained": i8_sus, "frac_sustained": ops / (i8_sus * 1e12) * 1e3 / pack_ms,
                  "hbm_floor_ms": hbm_floor_ms,
                  "tensor_floor_ms": tensor_floor_ms,
                  "binding": "tensor" if tensor_floor_ms > hbm_floor_ms else "hbm"}

    out = None
    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline and world == 1 and not small:
            try:
                cpu = cpu_sample(load_oracle())
            except Exception as ex:  # reported, never fatal to the GPU number
                cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "port", "sample": f"failed: {ex}"}
        stage_avg = {k: round(v / max(calls, 1), 4) for k, v in stage_ms.items()}
        wl = (f"1M ML-KEM-768 respond(), buckets 2^21, dim0 2048, 2 queries/payload, batch {B}"
              + (" (INT8-limb tcgen05 GEMMs)" if B > 1 else " (u64 packing)"))
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
            "scaling": "strong" if shard else "weak", "vs_baseline": None,
            "dtype": "u8 limbs -> s32 / u64" if B > 1 else "u64",
            "data": "synthetic",
            "config": {"workload": wl if not small else (
                           f"profiling case: {plan.instances} packing outputs, interp {plan.interp}"
                           if args.plan is not None else f"{args.records} ML-KEM-768 records (profiling case)"),
                       "records": args.records, "buckets": plan.num_items, "dim0": plan.dim0, "db_rows": plan.db_rows,
                       "db_cols": plan.db_cols, "instances": plan.instances, "interp": plan.interp, "c": plan.c,
                       "batch_payloads": B,
                       "parallelism": f"fold-group shards x{world}" if shard else f"replica x{world}",
                       "rank0_share": {"instances": local.instances, "c": local.c, "db_cols": local.db_cols},
                       "autotune": ({"chosen": tune["chosen"], "candidates": tune["candidates"]} if tune else None),
                       "l2": "inputs larger than L2 (packing stream of %.1f GB + DB of %.2f GB per step)" % (
                           pack_bytes / 1e9, plan.db_rows * plan.db_cols * 2 / 1e9)},
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": B * qbytes,
                    "d2h_bytes_per_step": B * (plan_response_bytes if shard else rbytes),
                    "api": ("ShardedKeywordServer.respond_batch (NCCL broadcast / gather, ipr_response_merge)" if shard
                            else f"KeywordService (ipr_service_submit_batch per {B} payloads / ipr_service_wait)"
                            if B > 1 else "ipr_server_respond"),
                    "steps": e2e_steps,
                    "blocking_batch_call_payloads_per_s": args.steps * B / (blocking_ms / 1000.0)},
            "serving": serving or None,
            "batch1": ({"u64_payloads_per_s": b1["u64"], "tensor_gemv_payloads_per_s": b1["tensor_gemv"],
                        "speedup_vs_batch1_u64": value / world / b1["u64"],
                        "u64_gemv_roofline": {"bound": "hbm", "kernel": "k_gemv (u64, CUDA cores)",
                                              "form": b1["u64_gemv"]["name"],
                                              "avg_launch_ms": b1["u64_gemv"]["gemv_ms"],
                                              "algorithmic_bytes": b1["u64_gemv"]["bytes"],
                                              "achieved": b1["u64_gemv"]["gemv_gbs"], "peak": peak, "unit": "GB/s",
                                              "frac": b1["u64_gemv"]["gemv_gbs"] / peak},
                        "u64_forms": u64_forms} if b1 else None),
            "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": ("measured (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                                         else "fallback 6.65 TB/s (MEASURED_PEAKS.json absent)"),
                         "traffic": read_traffic(kname), "algorithmic_bytes": pack_bytes, "avg_launch_ms": pack_ms},
            "tensor_roofline": tensor,
            "stage_ms": stage_avg,
            "gpu_launches": (7 * passes if B > 1 else 6) * args.steps,
            "clocks": clk,
            "cpu_baseline": cpu,
        }
        print(json.dumps(out))
    srv.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
