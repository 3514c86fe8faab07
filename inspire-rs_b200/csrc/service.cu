// service.cu — continuous-batching serving loop over one or more keyword servers.
//
// The reference serves one payload at a time (KeywordServer::respond behind a
// sequential TCP loop, rkdud007/inspire-rs src/pir/server/keyword.rs:534-640).
// Here requests are queued per database; one scheduler thread forms a batch
// from whatever is pending the moment a device slot frees (up to the admitted
// batch size), so the batch grows with the load and a lone request is not
// held back.  Each database gets two I/O slots: while one batch computes on the
// server stream, the next batch's queries are staged in pinned memory and
// copied up on a separate stream, and the previous batch's responses copied
// down.  Completion is signalled by a host callback on the copy stream.
//
// Admission: the batch size is the largest B <= max_batch whose batch-path
// device memory (slot-indexed precomputation + scratch + I/O slots) fits the
// HBM budget for all databases together; a database added later
// (ipr_service_add_database) gets the largest batch size that still fits what is
// left of the budget.  Submissions beyond max_pending queued requests are refused
// with IPR_E_BUSY.  Responses are byte-identical
// to ipr_server_respond: the batch path is bit-exact per payload.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "ipr_b200.h"
#include "server_internal.hpp"

namespace {

using Clock = std::chrono::steady_clock;
constexpr size_t kBatchLog = 4096;
constexpr int kMaxDatabases = 64;  // lanes are allocated once, so adding one never moves the others

int svc_fail(int code, const std::string& msg) {
    ipr::set_last_error(msg.c_str());
    return code;
}

int cuda_fail(cudaError_t e, const char* what) {
    return svc_fail(e == cudaErrorMemoryAllocation ? IPR_E_OOM : IPR_E_CUDA,
                    std::string(what) + ": " + cudaGetErrorString(e));
}

struct Request {
    uint64_t ticket = 0;
    int db = 0;
    std::vector<uint8_t> query;
    std::vector<uint8_t> resp;
    int status = IPR_PENDING;
    Clock::time_point t_submit, t_done;
};

struct Lane;

struct Slot {
    ipr_service* svc = nullptr;
    Lane* lane = nullptr;
    uint8_t *h_q = nullptr, *h_r = nullptr;
    int* h_err = nullptr;
    uint8_t *d_q = nullptr, *d_r = nullptr;
    cudaEvent_t up = nullptr, computed = nullptr;
    std::vector<Request*> batch;
    bool ready = false;  // set by the host callback once the responses are in h_r
    Clock::time_point t_launch, t_ready;
};

struct Lane {
    ipr_server* s = nullptr;
    int max_batch = 0;  // 0: no batch path, every payload is answered alone
    uint64_t qb = 0, rb = 0;
    std::deque<Request*> pending;
    Slot slot[2];
    int head = 0, nbusy = 0;  // slots complete in the order they were filled
    cudaStream_t up = nullptr, down = nullptr;
    // device time per batch size (moving average of completed batches, 0 = not seen yet) and
    // the estimated moment the device finishes the batches already enqueued
    double est_ms[ipr::kMaxBatchPayloads + 1] = {0};
    Clock::time_point free_at;
    Clock::time_point last_ready;

    double estimate(int B) const {
        if (est_ms[B] > 0) return est_ms[B];
        for (int d = 1; d <= ipr::kMaxBatchPayloads; d++) {  // nearest measured size
            if (B - d >= 1 && est_ms[B - d] > 0) return est_ms[B - d];
            if (B + d <= ipr::kMaxBatchPayloads && est_ms[B + d] > 0) return est_ms[B + d];
        }
        return 0;
    }
};

}  // namespace

struct ipr_service {
    std::vector<Lane> lanes;          // kMaxDatabases entries; [0, nlanes) are in use
    std::atomic<int> nlanes{0};       // published after a lane is fully set up
    uint64_t budget = 0;              // the HBM budget the admissions share
    ipr_service_config cfg{};
    std::mutex mu;
    std::mutex add_mu;  // serialises ipr_service_add_database
    std::condition_variable cv_work, cv_done;
    std::unordered_map<uint64_t, Request*> reqs;
    uint64_t next_ticket = 1;
    std::thread sched;
    bool stop = false;
    uint64_t submitted = 0, completed = 0, rejected = 0, failed = 0, batches = 0, batched_payloads = 0;
    uint64_t npending = 0, in_flight = 0;
    std::vector<double> lat_us;
    double batch_ms_sum = 0, batch_ms_max = 0, queue_ms_sum = 0, queue_ms_max = 0;
    Clock::time_point t0 = Clock::now();
    std::vector<ipr_service_batch> log;  // ring of the most recent batches
    uint64_t log_next = 0;
    uint64_t timed_batches = 0, queued_requests = 0;
    std::atomic<uint64_t> hbm{0};  // device bytes of the batch paths and I/O slots
    int admitted_batch = 0;
};

namespace {

void CUDART_CB on_slot_done(void* arg) {
    Slot* sl = static_cast<Slot*>(arg);
    ipr_service* v = sl->svc;
    {
        std::lock_guard<std::mutex> lk(v->mu);
        sl->ready = true;
        sl->t_ready = Clock::now();
    }
    v->cv_work.notify_one();
}

// record results of finished requests (caller holds no lock)
void complete(ipr_service* v, std::vector<Request*>& done) {
    const auto now = Clock::now();
    {
        std::lock_guard<std::mutex> lk(v->mu);
        for (Request* r : done) {
            r->t_done = now;
            v->completed++;
            if (r->status != IPR_OK) v->failed++;
            if (v->lat_us.size() < (1u << 22))
                v->lat_us.push_back(std::chrono::duration<double, std::micro>(r->t_done - r->t_submit).count());
            v->in_flight--;
        }
    }
    v->cv_done.notify_all();
    done.clear();
}

// answer one payload through the single-payload path (odd query counts, no batch path)
void answer_single(ipr_service* v, Lane& ln, Request* r) {
    const uint64_t cap = ipr_server_response_bytes(ln.s, r->query.empty() ? 0 : r->query[0]);
    r->resp.resize(cap);
    size_t n = 0;
    {
        std::lock_guard<std::mutex> lk(ln.s->mu);
        cudaSetDevice(ln.s->device);
        r->status = ipr::server_respond_locked(ln.s, r->query.data(), r->query.size(), r->resp.data(), cap, &n);
    }
    r->resp.resize(r->status == IPR_OK ? n : 0);
    std::vector<Request*> one{r};
    complete(v, one);
}

// stage and enqueue one batch into the lane's next free slot
void launch_batch(ipr_service* v, Lane& ln, std::vector<Request*>& batch) {
    ipr::NvtxRange nvtx_range("ipr_service batch launch");
    Slot& sl = ln.slot[(ln.head + ln.nbusy) & 1];
    const int B = (int)batch.size();
    for (int b = 0; b < B; b++) std::memcpy(sl.h_q + (size_t)b * ln.qb, batch[b]->query.data(), ln.qb);
    sl.batch.swap(batch);
    sl.ready = false;
    int st = IPR_OK;
    cudaError_t e;
    cudaSetDevice(ln.s->device);
    if ((e = cudaMemcpyAsync(sl.d_q, sl.h_q, (size_t)B * ln.qb, cudaMemcpyHostToDevice, ln.up)) != cudaSuccess ||
        (e = cudaEventRecord(sl.up, ln.up)) != cudaSuccess) {
        st = cuda_fail(e, "service upload");
    } else {
        std::lock_guard<std::mutex> lk(ln.s->mu);
        cudaStream_t cs = ln.s->stream;
        if ((e = cudaStreamWaitEvent(cs, sl.up, 0)) != cudaSuccess ||
            (e = cudaMemsetAsync(ln.s->d_err, 0, sizeof(int), cs)) != cudaSuccess) {
            st = cuda_fail(e, "service enqueue");
        } else if ((st = ipr::server_enqueue_batch(ln.s, B, sl.d_q, sl.d_r)) == IPR_OK) {
            if ((e = cudaMemcpyAsync(sl.h_err, ln.s->d_err, sizeof(int), cudaMemcpyDeviceToHost, cs)) != cudaSuccess ||
                (e = cudaEventRecord(sl.computed, cs)) != cudaSuccess)
                st = cuda_fail(e, "service enqueue");
        }
    }
    if (st == IPR_OK) {
        if ((e = cudaStreamWaitEvent(ln.down, sl.computed, 0)) != cudaSuccess ||
            (e = cudaMemcpyAsync(sl.h_r, sl.d_r, (size_t)B * ln.rb, cudaMemcpyDeviceToHost, ln.down)) != cudaSuccess ||
            (e = cudaLaunchHostFunc(ln.down, on_slot_done, &sl)) != cudaSuccess)
            st = cuda_fail(e, "service download");
    }
    if (st != IPR_OK) {  // nothing of this batch will complete on the device: fail its requests now
        for (Request* r : sl.batch) r->status = st;
        complete(v, sl.batch);
        return;
    }
    ln.nbusy++;
    sl.t_launch = Clock::now();
    const auto start = ln.nbusy == 1 || ln.free_at < sl.t_launch ? sl.t_launch : ln.free_at;
    ln.free_at = start + std::chrono::microseconds((int64_t)(ln.estimate(B) * 1000.0));
    std::lock_guard<std::mutex> lk(v->mu);
    v->batches++;
    v->batched_payloads += B;
}

// copy a finished slot's responses into its requests
void harvest(ipr_service* v, Lane& ln, Slot& sl) {
    const int err = *sl.h_err;
    {  // device time of this batch: from its launch, or from the previous batch's end if that was later
        const auto start = sl.t_launch > ln.last_ready ? sl.t_launch : ln.last_ready;
        const double ms = std::chrono::duration<double, std::milli>(sl.t_ready - start).count();
        double& e = ln.est_ms[sl.batch.size()];
        e = e > 0 ? 0.8 * e + 0.2 * ms : ms;
        ln.last_ready = sl.t_ready;
        std::lock_guard<std::mutex> lk(v->mu);
        v->timed_batches++;
        v->batch_ms_sum += ms;
        v->batch_ms_max = std::max(v->batch_ms_max, ms);
        double qmax = 0;
        for (Request* r : sl.batch) {  // time from submission to the launch of the request's batch
            const double qms = std::chrono::duration<double, std::milli>(sl.t_launch - r->t_submit).count();
            v->queued_requests++;
            v->queue_ms_sum += qms;
            v->queue_ms_max = std::max(v->queue_ms_max, qms);
            qmax = std::max(qmax, qms);
        }
        ipr_service_batch rec;
        rec.db = (int)(&ln - v->lanes.data());
        rec.payloads = (int)sl.batch.size();
        rec.launch_ms = std::chrono::duration<double, std::milli>(sl.t_launch - v->t0).count();
        rec.start_ms = std::chrono::duration<double, std::milli>(start - v->t0).count();
        rec.ready_ms = std::chrono::duration<double, std::milli>(sl.t_ready - v->t0).count();
        rec.queue_ms_max = qmax;
        if (v->log.size() < kBatchLog) v->log.push_back(rec);
        else v->log[v->log_next % kBatchLog] = rec;
        v->log_next++;
    }
    for (size_t b = 0; b < sl.batch.size(); b++) {
        Request* r = sl.batch[b];
        if (err) {
            r->status = IPR_E_TIMEOUT;
        } else {
            r->resp.assign(sl.h_r + b * ln.rb, sl.h_r + (b + 1) * ln.rb);
            r->status = IPR_OK;
        }
    }
    complete(v, sl.batch);
}

void scheduler(ipr_service* v) {
    size_t rr = 0;  // round-robin start over databases
    std::vector<Request*> take;
    for (;;) {
        bool progressed = false;
        // 1. finished batches, oldest first per database
        const int nl = v->nlanes.load(std::memory_order_acquire);
        for (int li = 0; li < nl; li++) {
            Lane& ln = v->lanes[li];
            while (ln.nbusy > 0) {
                Slot& sl = ln.slot[ln.head];
                {
                    std::lock_guard<std::mutex> lk(v->mu);
                    if (!sl.ready) break;
                }
                harvest(v, ln, sl);
                ln.head ^= 1;
                ln.nbusy--;
                progressed = true;
            }
        }
        // 2. dispatch.  An idle database takes what is pending at once; with one batch in
        // flight the second slot is filled only when that batch is about to end (the
        // staging lead), so it carries everything that arrived meanwhile -- unless a full
        // batch is already waiting, which gains nothing by waiting and is staged at once.
        Clock::time_point wake = Clock::time_point::max();
        const auto now = Clock::now();
        for (int i = 0; i < nl; i++) {
            Lane& ln = v->lanes[(rr + i) % nl];
            while (ln.max_batch == 0 || ln.nbusy < 2) {
                bool full = false;
                if (ln.max_batch > 0 && ln.nbusy == 1) {
                    std::lock_guard<std::mutex> lk(v->mu);
                    full = ln.pending.size() >= (size_t)ln.max_batch;
                }
                if (ln.max_batch > 0 && ln.nbusy == 1 && !full) {
                    const auto lead = std::chrono::microseconds(
                        (int64_t)std::max(1500.0, 250.0 * ln.estimate(ln.max_batch)));
                    if (now + lead < ln.free_at) {
                        wake = std::min(wake, ln.free_at - lead);
                        break;
                    }
                }
                take.clear();
                Request* single = nullptr;
                {
                    std::lock_guard<std::mutex> lk(v->mu);
                    while (!ln.pending.empty()) {
                        Request* r = ln.pending.front();
                        const bool batchable = ln.max_batch > 0 && r->query[0] == 2;
                        if (!batchable) {
                            if (take.empty()) {
                                single = r;
                                ln.pending.pop_front();
                                v->npending--;
                            }
                            break;
                        }
                        if ((int)take.size() == ln.max_batch) break;
                        take.push_back(r);
                        ln.pending.pop_front();
                        v->npending--;
                    }
                }
                if (single) {
                    answer_single(v, ln, single);
                    progressed = true;
                    continue;
                }
                if (take.empty()) break;
                launch_batch(v, ln, take);
                progressed = true;
            }
        }
        rr++;
        if (progressed) continue;
        // 3. idle: wait for a submission, a finished slot, the next dispatch moment or shutdown
        std::unique_lock<std::mutex> lk(v->mu);
        auto ready = [&] {
            if (v->stop) return true;
            for (int li = 0; li < v->nlanes.load(std::memory_order_acquire); li++) {
                const Lane& ln = v->lanes[li];
                if (ln.nbusy > 0 && ln.slot[ln.head].ready) return true;
                if (!ln.pending.empty() && (ln.max_batch == 0 || ln.nbusy == 0)) return true;
            }
            return false;
        };
        if (wake == Clock::time_point::max()) v->cv_work.wait(lk, ready);
        else v->cv_work.wait_until(lk, wake, ready);
        if (v->stop) {
            bool busy = false;
            for (int li = 0; li < nl; li++) busy = busy || v->lanes[li].nbusy > 0;
            if (!busy) break;
            // let the batches in flight finish before leaving
            lk.unlock();
            for (int li = 0; li < nl; li++)
                if (v->lanes[li].nbusy) cudaStreamSynchronize(v->lanes[li].down);
        }
    }
}

void free_lane(Lane& ln) {
    if (!ln.s) return;
    cudaSetDevice(ln.s->device);
    for (Slot& sl : ln.slot) {
        if (sl.h_q) cudaFreeHost(sl.h_q);
        if (sl.h_r) cudaFreeHost(sl.h_r);
        if (sl.h_err) cudaFreeHost(sl.h_err);
        if (sl.d_q) cudaFree(sl.d_q);
        if (sl.d_r) cudaFree(sl.d_r);
        if (sl.up) cudaEventDestroy(sl.up);
        if (sl.computed) cudaEventDestroy(sl.computed);
        sl = Slot();
    }
    if (ln.up) cudaStreamDestroy(ln.up);
    if (ln.down) cudaStreamDestroy(ln.down);
    ln.up = ln.down = nullptr;
}

int setup_lane(ipr_service* v, Lane& ln) {
    cudaError_t e;
    if ((e = cudaSetDevice(ln.s->device)) != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    if ((e = cudaStreamCreateWithFlags(&ln.up, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&ln.down, cudaStreamNonBlocking)) != cudaSuccess)
        return cuda_fail(e, "service streams");
    if (ln.max_batch == 0) return IPR_OK;
    {
        std::lock_guard<std::mutex> lk(ln.s->mu);
        const int st = ipr::server_ensure_batch(ln.s, ln.max_batch);
        if (st) return st;
    }
    for (Slot& sl : ln.slot) {
        sl.svc = v;
        sl.lane = &ln;
        const size_t qbytes = (size_t)ln.max_batch * ln.qb, rbytes = (size_t)ln.max_batch * ln.rb;
        if ((e = cudaMallocHost(&sl.h_q, qbytes)) != cudaSuccess || (e = cudaMallocHost(&sl.h_r, rbytes)) != cudaSuccess ||
            (e = cudaMallocHost(&sl.h_err, sizeof(int))) != cudaSuccess || (e = cudaMalloc(&sl.d_q, qbytes)) != cudaSuccess ||
            (e = cudaMalloc(&sl.d_r, rbytes)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&sl.up, cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&sl.computed, cudaEventDisableTiming)) != cudaSuccess)
            return cuda_fail(e, "service I/O slots");
        *sl.h_err = 0;
        v->hbm += qbytes + rbytes;
    }
    return IPR_OK;
}

}  // namespace

extern "C" {

int ipr_service_create(ipr_server* const* servers, int num_servers, const ipr_service_config* cfg, ipr_service** out) {
    if (!servers || num_servers < 1 || !out) return svc_fail(IPR_E_ARGS, "null argument or no servers");
    *out = nullptr;
    ipr_service_config c{};
    if (cfg) c = *cfg;
    if (c.max_batch <= 0 || c.max_batch > ipr::kMaxBatchPayloads) c.max_batch = ipr::kMaxBatchPayloads;
    if (c.max_pending <= 0) c.max_pending = 4096;
    for (int i = 0; i < num_servers; i++)
        for (int j = 0; j < i; j++)
            if (!servers[i] || servers[i] == servers[j]) return svc_fail(IPR_E_ARGS, "null or repeated server");
    // admission: the largest common batch size whose batch-path memory fits the budget
    uint64_t budget = c.hbm_budget_bytes;
    if (budget == 0) {
        size_t free_b = 0, total_b = 0;
        cudaSetDevice(servers[0]->device);
        cudaError_t e = cudaMemGetInfo(&free_b, &total_b);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMemGetInfo");
        budget = free_b > (2ull << 30) ? free_b - (2ull << 30) : 0;
    }
    auto need = [&](int B) {
        uint64_t tot = 0;
        for (int i = 0; i < num_servers; i++) {
            ipr_server* s = servers[i];
            if (!s->gemv_tc) continue;
            tot += ipr::server_batch_bytes(s, B) +
                   2ull * B * (ipr::query_bytes(s->plan.db_rows, 2) + s->response_bytes(2));
        }
        return tot;
    };
    int B = c.max_batch;
    while (B > 0 && need(B) > budget) B--;
    bool any_tc = false;
    for (int i = 0; i < num_servers; i++) any_tc = any_tc || servers[i]->gemv_tc;
    if (any_tc && B == 0) {
        char msg[256];
        snprintf(msg, sizeof msg, "HBM budget of %llu bytes admits no batch (one payload per database needs %llu)",
                 (unsigned long long)budget, (unsigned long long)need(1));
        return svc_fail(IPR_E_OOM, msg);
    }
    auto* v = new ipr_service();
    v->cfg = c;
    v->admitted_batch = B;
    if (num_servers > kMaxDatabases) {
        delete v;
        return svc_fail(IPR_E_ARGS, "more than 64 databases");
    }
    v->budget = budget;
    v->lanes.resize(kMaxDatabases);
    for (int i = 0; i < num_servers; i++) {
        Lane& ln = v->lanes[i];
        ln.s = servers[i];
        ln.max_batch = ln.s->gemv_tc ? B : 0;
        ln.qb = ipr::query_bytes(ln.s->plan.db_rows, 2);
        ln.rb = ln.s->response_bytes(2);
        if (ln.max_batch) v->hbm += ipr::server_batch_bytes(ln.s, ln.max_batch);
        const int st = setup_lane(v, ln);
        if (st) {
            for (Lane& l2 : v->lanes) free_lane(l2);
            delete v;
            return st;
        }
    }
    v->nlanes.store(num_servers, std::memory_order_release);
    v->sched = std::thread(scheduler, v);
    *out = v;
    return IPR_OK;
}

int ipr_service_add_database(ipr_service* v, ipr_server* server, int* db) {
    if (!v || !server || !db) return svc_fail(IPR_E_ARGS, "null argument");
    std::lock_guard<std::mutex> add_lk(v->add_mu);  // one admission at a time
    const int n = v->nlanes.load(std::memory_order_acquire);
    if (n >= kMaxDatabases) return svc_fail(IPR_E_ARGS, "the service holds 64 databases already");
    for (int i = 0; i < n; i++)
        if (v->lanes[i].s == server) return svc_fail(IPR_E_ARGS, "server already served");
    uint64_t used;
    {
        std::lock_guard<std::mutex> lk(v->mu);
        if (v->stop) return svc_fail(IPR_E_STATE, "service is shutting down");
        used = v->hbm.load();
    }
    const uint64_t left = v->budget > used ? v->budget - used : 0;
    int B = 0;
    if (server->gemv_tc) {
        auto need = [&](int b) {
            return ipr::server_batch_bytes(server, b) +
                   2ull * b * (ipr::query_bytes(server->plan.db_rows, 2) + server->response_bytes(2));
        };
        B = v->cfg.max_batch;
        while (B > 0 && need(B) > left) B--;
        if (B == 0) {
            char msg[256];
            snprintf(msg, sizeof msg, "HBM budget has %llu bytes left; one payload of this database needs %llu",
                     (unsigned long long)left, (unsigned long long)need(1));
            return svc_fail(IPR_E_OOM, msg);
        }
    }
    Lane& ln = v->lanes[n];  // not visible to the scheduler until nlanes is raised
    ln.s = server;
    ln.max_batch = B;
    ln.qb = ipr::query_bytes(server->plan.db_rows, 2);
    ln.rb = server->response_bytes(2);
    uint64_t batch_bytes = B ? ipr::server_batch_bytes(server, B) : 0;
    const uint64_t hbm_before = v->hbm.load();
    int st = setup_lane(v, ln);
    if (st) {
        free_lane(ln);
        ln = Lane();
        std::lock_guard<std::mutex> lk(v->mu);
        v->hbm.store(hbm_before);
        return st;
    }
    {
        std::lock_guard<std::mutex> lk(v->mu);
        v->hbm += batch_bytes;
    }
    v->nlanes.store(n + 1, std::memory_order_release);
    *db = n;
    v->cv_work.notify_one();
    return IPR_OK;
}

int ipr_service_submit(ipr_service* v, int db, const uint8_t* query, size_t len, uint64_t* ticket) {
    if (!v || !query || !ticket) return svc_fail(IPR_E_ARGS, "null argument");
    if (db < 0 || db >= v->nlanes.load(std::memory_order_acquire)) return svc_fail(IPR_E_ARGS, "no such database");
    Lane& ln = v->lanes[db];
    if (len < 1) return svc_fail(IPR_E_FORMAT, "empty query");
    const uint64_t want = ipr_server_query_bytes(ln.s, query[0]);
    if (len < want) return svc_fail(IPR_E_FORMAT, "query shorter than its query count needs");
    auto* r = new Request();
    r->db = db;
    r->query.assign(query, query + want);
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(v->mu);
        if (v->stop) {
            delete r;
            return svc_fail(IPR_E_STATE, "service is shutting down");
        }
        if (v->npending >= (uint64_t)v->cfg.max_pending) {
            v->rejected++;
            delete r;
            return svc_fail(IPR_E_BUSY, "request queue is full");
        }
        r->ticket = v->next_ticket++;
        v->reqs[r->ticket] = r;
        ln.pending.push_back(r);
        v->npending++;
        v->in_flight++;
        v->submitted++;
        *ticket = r->ticket;
    }
    v->cv_work.notify_one();
    return IPR_OK;
}

int ipr_service_submit_batch(ipr_service* v, int db, int n, const uint8_t* const* queries, const size_t* lens,
                             uint64_t* tickets) {
    if (!v || n < 0 || (n && (!queries || !lens || !tickets))) return svc_fail(IPR_E_ARGS, "null argument");
    if (db < 0 || db >= v->nlanes.load(std::memory_order_acquire)) return svc_fail(IPR_E_ARGS, "no such database");
    Lane& ln = v->lanes[db];
    std::vector<Request*> rs;
    rs.reserve((size_t)n);
    auto drop = [&]() {
        for (Request* r : rs) delete r;
    };
    for (int i = 0; i < n; i++) {  // every query is checked before any is queued
        if (!queries[i] || lens[i] < 1) {
            drop();
            return svc_fail(IPR_E_FORMAT, "empty query");
        }
        const uint64_t want = ipr_server_query_bytes(ln.s, queries[i][0]);
        if (lens[i] < want) {
            drop();
            return svc_fail(IPR_E_FORMAT, "query shorter than its query count needs");
        }
        auto* r = new Request();
        r->db = db;
        r->query.assign(queries[i], queries[i] + want);
        rs.push_back(r);
    }
    {
        std::lock_guard<std::mutex> lk(v->mu);
        if (v->stop) {
            drop();
            return svc_fail(IPR_E_STATE, "service is shutting down");
        }
        if (v->npending + (uint64_t)n > (uint64_t)v->cfg.max_pending) {
            v->rejected += (uint64_t)n;
            drop();
            return svc_fail(IPR_E_BUSY, "request queue cannot take all of them");
        }
        const auto now = Clock::now();
        for (int i = 0; i < n; i++) {
            Request* r = rs[(size_t)i];
            r->t_submit = now;
            r->ticket = v->next_ticket++;
            v->reqs[r->ticket] = r;
            ln.pending.push_back(r);
            tickets[i] = r->ticket;
        }
        v->npending += (uint64_t)n;
        v->in_flight += (uint64_t)n;
        v->submitted += (uint64_t)n;
    }
    v->cv_work.notify_one();
    return IPR_OK;
}

static int collect_locked(ipr_service* v, Request* r, uint8_t* out, size_t cap, size_t* out_len) {
    if (out_len) *out_len = r->resp.size();
    const int st = r->status;
    if (st == IPR_OK) {
        if (!out || cap < r->resp.size()) return svc_fail(IPR_E_SPACE, "response buffer too small");
        std::memcpy(out, r->resp.data(), r->resp.size());
    }
    v->reqs.erase(r->ticket);
    delete r;
    return st;
}

int ipr_service_poll(ipr_service* v, uint64_t ticket, uint8_t* out, size_t cap, size_t* out_len) {
    if (!v) return svc_fail(IPR_E_ARGS, "null service");
    std::lock_guard<std::mutex> lk(v->mu);
    auto it = v->reqs.find(ticket);
    if (it == v->reqs.end()) return svc_fail(IPR_E_ARGS, "unknown ticket");
    Request* r = it->second;
    if (r->t_done == Clock::time_point()) return IPR_PENDING;
    return collect_locked(v, r, out, cap, out_len);
}

int ipr_service_wait(ipr_service* v, uint64_t ticket, int timeout_ms, uint8_t* out, size_t cap, size_t* out_len) {
    if (!v) return svc_fail(IPR_E_ARGS, "null service");
    std::unique_lock<std::mutex> lk(v->mu);
    auto it = v->reqs.find(ticket);
    if (it == v->reqs.end()) return svc_fail(IPR_E_ARGS, "unknown ticket");
    Request* r = it->second;
    auto done = [&] { return r->t_done != Clock::time_point(); };
    if (timeout_ms < 0) {
        v->cv_done.wait(lk, done);
    } else if (!v->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done)) {
        return IPR_PENDING;
    }
    return collect_locked(v, r, out, cap, out_len);
}

int ipr_service_get_stats(ipr_service* v, ipr_service_stats* out) {
    if (!v || !out) return svc_fail(IPR_E_ARGS, "null argument");
    std::vector<double> lat;
    {
        std::lock_guard<std::mutex> lk(v->mu);
        out->submitted = v->submitted;
        out->completed = v->completed;
        out->rejected = v->rejected;
        out->failed = v->failed;
        out->batches = v->batches;
        out->batched_payloads = v->batched_payloads;
        out->pending = v->npending;
        out->in_flight = v->in_flight;
        out->max_batch = v->admitted_batch;
        out->hbm_bytes = v->hbm.load();
        lat = v->lat_us;
    }
    out->p50_us = out->p99_us = out->mean_us = out->max_us = 0;
    if (!lat.empty()) {
        std::sort(lat.begin(), lat.end());
        auto pct = [&](double p) {
            size_t k = (size_t)(p * (double)(lat.size() - 1) + 0.5);
            return lat[std::min(k, lat.size() - 1)];
        };
        out->p50_us = pct(0.50);
        out->p99_us = pct(0.99);
        double sum = 0;
        for (double x : lat) sum += x;
        out->mean_us = sum / (double)lat.size();
        out->max_us = lat.back();
    }
    out->latency_samples = lat.size();
    {
        std::lock_guard<std::mutex> lk(v->mu);
        out->batch_ms_mean = v->timed_batches ? v->batch_ms_sum / (double)v->timed_batches : 0;
        out->batch_ms_max = v->batch_ms_max;
        out->queue_ms_mean = v->queued_requests ? v->queue_ms_sum / (double)v->queued_requests : 0;
        out->queue_ms_max = v->queue_ms_max;
    }
    return IPR_OK;
}

int ipr_service_batch_log(ipr_service* v, ipr_service_batch* out, int cap, int* n) {
    if (!v || !n || cap < 0 || (cap && !out)) return svc_fail(IPR_E_ARGS, "null argument");
    std::lock_guard<std::mutex> lk(v->mu);
    const size_t have = v->log.size();
    const size_t k = std::min(have, (size_t)cap);
    // oldest first among the last k recorded
    for (size_t i = 0; i < k; i++) {
        const uint64_t idx = v->log_next - k + i;
        out[i] = v->log[have < kBatchLog ? idx : idx % kBatchLog];
    }
    *n = (int)k;
    return IPR_OK;
}

int ipr_service_reset_stats(ipr_service* v) {
    if (!v) return svc_fail(IPR_E_ARGS, "null service");
    std::lock_guard<std::mutex> lk(v->mu);
    v->lat_us.clear();
    v->batch_ms_sum = v->batch_ms_max = v->queue_ms_sum = v->queue_ms_max = 0;
    v->timed_batches = v->queued_requests = 0;
    v->log.clear();
    v->log_next = 0;
    v->batches = v->batched_payloads = 0;
    v->submitted = v->completed = v->rejected = v->failed = 0;
    return IPR_OK;
}

int ipr_service_diagnose(ipr_service* v, char* out, size_t cap) {
    if (!v || !out || cap == 0) return svc_fail(IPR_E_ARGS, "null argument");
    auto q = [](cudaError_t e) { return e == cudaSuccess ? "done" : e == cudaErrorNotReady ? "busy" : "error"; };
    std::string txt;
    char line[320];
    const int nl = v->nlanes.load(std::memory_order_acquire);
    for (int li = 0; li < nl; li++) {
        Lane& ln = v->lanes[li];
        size_t pending;
        bool ready[2];
        size_t nb[2];
        {
            std::lock_guard<std::mutex> lk(v->mu);
            pending = ln.pending.size();
            for (int k = 0; k < 2; k++) {
                ready[k] = ln.slot[k].ready;
                nb[k] = ln.slot[k].batch.size();
            }
        }
        // the scheduler owns nbusy / head; a racing read only misstates this one line
        std::snprintf(line, sizeof line, "db %d: max_batch %d, %zu pending, %d slots busy (head %d); server stream %s, "
                                         "download stream %s\n",
                      li, ln.max_batch, pending, ln.nbusy, ln.head, q(cudaStreamQuery(ln.s->stream)),
                      ln.down ? q(cudaStreamQuery(ln.down)) : "none");
        txt += line;
        for (int k = 0; k < 2 && ln.max_batch > 0; k++) {
            const Slot& sl = ln.slot[k];
            const double age = std::chrono::duration<double, std::milli>(Clock::now() - sl.t_launch).count();
            std::snprintf(line, sizeof line, "  slot %d: %zu payloads, uploaded %s, computed %s, ready %d, launched %.1f ms ago\n",
                          k, nb[k], sl.up ? q(cudaEventQuery(sl.up)) : "none",
                          sl.computed ? q(cudaEventQuery(sl.computed)) : "none", (int)ready[k], age);
            txt += line;
        }
    }
    const size_t n = std::min(cap - 1, txt.size());
    std::memcpy(out, txt.data(), n);
    out[n] = 0;
    return IPR_OK;
}

void ipr_service_destroy(ipr_service* v) {
    if (!v) return;
    {
        std::lock_guard<std::mutex> lk(v->mu);
        v->stop = true;
        for (int li = 0; li < v->nlanes.load(); li++) v->lanes[li].pending.clear();  // never started; freed below
        v->npending = 0;
    }
    v->cv_work.notify_all();
    if (v->sched.joinable()) v->sched.join();
    // requests still queued were never started; uncollected results are dropped
    for (auto& kv : v->reqs) delete kv.second;
    v->reqs.clear();
    for (Lane& ln : v->lanes) free_lane(ln);
    delete v;
}

}  // extern "C"
