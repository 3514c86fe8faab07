// server.cu — keyword server handle and the C ABI of include/ipr_b200.h.
//
// One ipr_server owns the device-resident state of one database (encoded DB,
// packing precomputation, NTT tables, RGSW mask row) plus the per-request
// scratch, a stream, and one CUDA graph per query count.  respond() runs
// (rkdud007/inspire-rs src/pir/server/keyword.rs:534-640):
//   H2D query bytes -> parse -> GEMV (both queries, one DB pass) -> packing
//   (once per payload) -> INTT/CRT -> fold + modulus switch -> framing -> D2H.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <algorithm>
#include <atomic>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "host_math.hpp"
#include "ipr_b200.h"
#include "bounds.cuh"
#include "kernels.cuh"
#include "server_internal.hpp"

namespace {

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

#define CU(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return fail(e_ == cudaErrorMemoryAllocation ? IPR_E_OOM : IPR_E_CUDA, "%s: %s (%s:%d)", \
                        #call, cudaGetErrorString(e_), __FILE__, __LINE__);                   \
    } while (0)

constexpr int kN = 2048;
constexpr int kNInner = 3069;
constexpr int kMaxProfileSlots = 8192;

}  // namespace

namespace ipr {
int encode_db_device(const uint16_t* d_raw, uint16_t* d_out, uint64_t db_rows, uint64_t db_cols, uint64_t interp,
                     cudaStream_t st);
int offline_precompute_device(const uint16_t* d_db, uint64_t db_rows, uint64_t instances, uint64_t* d_a_hat,
                              uint64_t* d_bt, uint64_t* d_btb, uint64_t* d_bth, uint64_t scratch_budget,
                              cudaStream_t st);
// lets other translation units of the library report through ipr_last_error()
void set_last_error(const char* msg) { g_last_error = msg; }
}  // namespace ipr

namespace {

void destroy_graphs(ipr_server* s) {
    for (auto& kv : s->graphs) cudaGraphExecDestroy(kv.second);
    s->graphs.clear();
}

// query-byte rows: 7 per query (the bytes of its CRT-composed value); a tile of nt rows
// (the MMA's N, a multiple of 16) carries nt / 7 whole queries.  The buffer holds 256 rows
// beyond the queries, so that every tile box lies inside it.
constexpr unsigned kQbPadRows = 256;
unsigned qb_rows(unsigned nq) { return 7 * nq + kQbPadRows; }

// the GEMM's tile height: the smallest multiple of 16 that holds all nq queries, at most 224
// (32 queries), lowered under the server option's cap to a multiple of 112 (16 queries, no
// unused rows) when the cap allows one, else to a multiple of 16
int g1_nt(const ipr_server* s, unsigned nq) {
    int nt = (int)(7 * nq + 15) / 16 * 16;
    if (nt > 224) nt = 224;
    if (s->g1_tile && s->g1_tile < nt) nt = s->g1_tile >= 112 ? s->g1_tile / 112 * 112 : s->g1_tile / 16 * 16;
    return nt < 16 ? 16 : nt;
}
int g1_tiles(unsigned nq, int nt) { return (int)((nq + nt / 7 - 1) / (nt / 7)); }

int qb_map(ipr_server* s, int nt, const CUtensorMap** out) {
    auto it = s->tm_qb.find(nt);
    if (it == s->tm_qb.end()) {
        CUtensorMap m;
        CU(ipr::make_u8_tile_map(&m, s->d_qb, s->plan.db_rows, qb_rows(s->cap_q), (uint32_t)nt));
        it = s->tm_qb.emplace(nt, m).first;
    }
    *out = &it->second;
    return IPR_OK;
}

int ensure_scratch(ipr_server* s, unsigned nq) {
    const unsigned want = nq < 2 ? 2 : nq;
    if (want <= s->cap_q) return IPR_OK;
    CU(cudaStreamSynchronize(s->stream));  // work already enqueued may still use the old buffers
    destroy_graphs(s);
    for (void* p : {(void*)s->d_query, (void*)s->d_ail, (void*)s->d_gsw, (void*)s->d_c, (void*)s->d_resp,
                    (void*)s->d_qb})
        if (p) s->free_ptr(p);
    s->tm_qb.clear();
    if (s->h_query) cudaFreeHost(s->h_query);
    if (s->h_resp) cudaFreeHost(s->h_resp);
    s->h_query = s->h_resp = nullptr;
    const uint64_t rows = s->plan.db_rows, cols = s->plan.db_cols;
    const unsigned groups = (want + 1) / 2;
    int st;
    if ((st = s->alloc(&s->d_query, ipr::query_bytes(rows, want) + 16))) return st;
    if ((st = s->alloc(&s->d_ail, (size_t)groups * rows * 4 * 4))) return st;
    if ((st = s->alloc(&s->d_gsw, (size_t)want * 12 * kN * 4))) return st;
    if ((st = s->alloc(&s->d_c, (size_t)want * cols * 8))) return st;
    if ((st = s->alloc(&s->d_resp, s->response_bytes(want)))) return st;
    if ((st = s->alloc(&s->d_qb, (size_t)qb_rows(want) * rows))) return st;
    CU(cudaMallocHost(&s->h_query, ipr::query_bytes(rows, want) + 16));
    CU(cudaMallocHost(&s->h_resp, s->response_bytes(want)));
    s->cap_q = want;
    return IPR_OK;
}

// The one-chain fold's occupancy for `chains` chains: two CTAs per SM staging the RGSW bodies
// in shared memory, or three per SM reading them from L2 (more warps to hide latency, 80
// registers).  Chains run in rounds of (CTAs per SM x SMs); a round of three per SM takes
// about 1.22x as long as one of two per SM (measured at the 1M shape), so the three-per-SM
// form wins where it needs fewer rounds in proportion, e.g. 1,408 chains (64 payloads) on
// 148 SMs: 4 rounds x 1.22 against 5 rounds.  Forms 4 / 5 force one occupancy.
bool fold_staged(const ipr_server* s, int chains) {
    if (s->fold_mode == 4) return false;
    if (s->fold_mode == 5) return true;
    const int sm = s->sm_count > 0 ? s->sm_count : 1;
    const int64_t r2 = (chains + 2 * sm - 1) / (2 * sm), r3 = (chains + 3 * sm - 1) / (3 * sm);
    return r3 * 122 >= r2 * 100;
}

// enqueue the device pipeline for one payload; `prof` = event slot base or -1
int enqueue(ipr_server* s, unsigned nq, const uint8_t* d_query, uint8_t* d_resp, int prof) {
    cudaStream_t st = s->stream;
    const ipr::Plan& p = s->plan;
    auto rec = [&](int stage) {
        if (prof >= 0) cudaEventRecord(s->events[(size_t)prof * (IPR_NSTAGES + 1) + stage], st);
    };
    rec(0);
    if (nq > 0) {
        CU(ipr::launch_parse_query(d_query, (int)nq, (int)p.db_rows, s->d_y, s->d_z, s->d_ail, s->d_gsw,
                                   s->gemv_tc ? s->d_qb : nullptr, 0, st));
        rec(1);
        if (s->gemv_tc) {
            const int nt = g1_nt(s, nq);
            const CUtensorMap* tq;
            int e = qb_map(s, nt, &tq);
            if (e) return e;
            CU(ipr::launch_gemm1(&s->tm_db, tq, (int)p.db_rows, (int64_t)p.db_cols, nt, g1_tiles(nq, nt),
                                 (int)nq, s->d_c, s->d_err, s->sm_count, st));
        } else {
            for (unsigned g = 0; 2 * g < nq; g++) {
                const int ng = nq - 2 * g >= 2 ? 2 : 1;
                // forms 4 and 5 hold exact sums only up to 16,384 rows; beyond, form 0
                const int form =
                    ((s->gemv_form == 4 || s->gemv_form == 5) && p.db_rows > 16384) ? 0 : s->gemv_form;
                CU(ipr::launch_gemv(s->d_db, (int)p.db_rows, (int64_t)p.db_cols, ng,
                                    s->d_ail + (size_t)g * p.db_rows * 4, s->d_c + (size_t)2 * g * p.db_cols,
                                    s->sm_count, st, form, s->d_err));
            }
        }
        rec(2);
        CU(ipr::launch_pack(s->d_bt, s->d_btb, s->d_bth, s->d_y, s->d_z, s->d_S, (int)p.instances, st));
        rec(3);
        if (s->fold_mode >= 2) {
            const bool chain = s->fold_mode >= 3;
            CU(ipr::launch_fold_prep(s->d_S, (int64_t)p.instances, nullptr, nullptr, 1, s->hp.ninv, s->sm_count, st,
                                     chain ? s->d_gsw : nullptr, (int)nq, s->hp.ninvr));
            rec(4);
            if (chain) {
                ipr::FoldExtents ext{(int64_t)p.instances * 2 * kN, (int64_t)nq * 12 * kN,
                                     (int64_t)p.instances * kN, (int64_t)nq * (int64_t)p.db_cols,
                                     (int64_t)s->response_bytes(nq)};
                if (ipr::kBoundsChecked) ext.s_words -= ipr::g_fold_extent_cut.load();
                CU(ipr::launch_fold4(s->d_row0m, s->d_gsw, s->d_ahat, s->d_S, 0, s->d_c, s->d_fwi, s->d_iwi,
                                     (int)p.interp, (int)p.c, (int)nq, (int64_t)p.db_cols, (int)nq, d_resp, 0,
                                     (int64_t)(4 + s->per_query_bytes()), ext, st,
                                     fold_staged(s, (int)(nq * p.c))));
            }
            else
                CU(ipr::launch_fold3(s->d_row0s, s->d_gsw, s->d_ahat, s->d_S, 0, s->d_c, s->d_fwi, s->d_iwi,
                                     s->hp.ninv, (int)p.interp, (int)p.c, (int)nq, (int64_t)p.db_cols, (int)nq, d_resp,
                                     0, (int64_t)(4 + s->per_query_bytes()), st));
        } else if (s->fold_mode == 1) {
            CU(ipr::launch_intt_crt(s->d_S, s->d_iw, s->d_iwp, s->d_R, (int)p.instances, st));
            rec(4);
            CU(ipr::launch_fold2(s->d_row0, s->d_gsw, s->d_ahat, s->d_R, 0, s->d_c, s->d_fw, s->d_fwp, s->d_iw,
                                 s->d_iwp, (int)p.interp, (int)p.c, (int)nq, (int64_t)p.db_cols, (int)nq, d_resp, 0,
                                 (int64_t)(4 + s->per_query_bytes()), st));
        } else {
            CU(ipr::launch_intt_crt(s->d_S, s->d_iw, s->d_iwp, s->d_R, (int)p.instances, st));
            rec(4);
            CU(ipr::launch_fold_switch(s->d_row0, s->d_gsw, s->d_ahat, s->d_R, s->d_c, s->d_fw, s->d_fwp, s->d_iw,
                                       s->d_iwp, (int)p.interp, (int)p.c, (int)nq, (int64_t)p.db_cols, d_resp + 8,
                                       (int64_t)(4 + s->per_query_bytes()), st));
        }
    } else {
        rec(1); rec(2); rec(3); rec(4);
    }
    CU(ipr::launch_response_frame(d_resp, (int)nq, (int64_t)s->per_query_bytes(), s->d_stash,
                                  (int64_t)s->stash_count, (int64_t)s->stash_entry, st));
    rec(5);
    return IPR_OK;
}

int harvest_profile(ipr_server* s) {
    if (!s->slots_used) return IPR_OK;
    CU(cudaStreamSynchronize(s->stream));
    for (int slot = 0; slot < s->slots_used; slot++) {
        for (int k = 0; k < IPR_NSTAGES; k++) {
            float ms = 0;
            cudaEvent_t a = s->events[(size_t)slot * (IPR_NSTAGES + 1) + k];
            cudaEvent_t b = s->events[(size_t)slot * (IPR_NSTAGES + 1) + k + 1];
            CU(cudaEventElapsedTime(&ms, a, b));
            s->stage_ms[k] += ms;
        }
        s->calls++;
    }
    s->slots_used = 0;
    return IPR_OK;
}

int next_profile_slot(ipr_server* s) {
    if (!s->profiling) return -1;
    if (s->slots_used == kMaxProfileSlots && harvest_profile(s)) return -1;
    return s->slots_used++;
}

constexpr int kMaxBatch = ipr::kMaxBatchPayloads;

// build the slot-indexed precomputation once (35.4 GB at 1M records)
int ensure_tpp(ipr_server* s) {
    if (s->d_tpp) return IPR_OK;
    if (!s->gemv_tc) return fail(IPR_E_STATE, "batched respond needs the tensor-core first dimension (db_rows <= 32768)");
    const uint64_t bytes = ipr::tpp_bytes((int)s->plan.instances);
    size_t free_b = 0, total_b = 0;
    CU(cudaMemGetInfo(&free_b, &total_b));
    if (bytes + (1ull << 30) > free_b)
        return fail(IPR_E_OOM, "batched packing needs %llu more bytes of HBM, %zu free", (unsigned long long)bytes, free_b);
    int st = s->alloc(&s->d_tpp, bytes);
    if (st) return st;
    CU(ipr::launch_relayout_tpp(s->d_bt, s->d_btb, s->d_tpp, (int)s->plan.instances, s->stream));
    CU(cudaStreamSynchronize(s->stream));
    const uint64_t rows = bytes / (3 * kN);
    CU(ipr::make_u8_tile_map(&s->tm_tpp, s->d_tpp, 3 * kN, rows, 128));
    return IPR_OK;
}

int ensure_batch(ipr_server* s, int B) {
    if (B <= s->bcap) return IPR_OK;
    int st = ensure_tpp(s);
    if (st) return st;
    CU(cudaStreamSynchronize(s->stream));  // work already enqueued may still use the old buffers
    if ((st = ensure_scratch(s, 2 * (unsigned)B))) return st;
    for (void* p : {(void*)s->d_bq, (void*)s->d_ybs, (void*)s->d_zbs, (void*)s->d_y8, (void*)s->d_bS, (void*)s->d_bR,
                    (void*)s->d_bresp})
        if (p) s->free_ptr(p);
    if (s->h_bq) cudaFreeHost(s->h_bq);
    if (s->h_bresp) cudaFreeHost(s->h_bresp);
    s->h_bq = s->h_bresp = nullptr;
    s->tm_y8.clear();
    const uint64_t qb = ipr::query_bytes(s->plan.db_rows, 2), rb = s->response_bytes(2);
    const uint64_t no = s->plan.instances;
    s->y8_np = ipr::pack_mma_nt(B);
    s->d_bR = nullptr;
    if ((st = s->alloc(&s->d_bq, (size_t)B * qb)) || (st = s->alloc(&s->d_ybs, (size_t)B * 3 * kN * 8)) ||
        (st = s->alloc(&s->d_zbs, (size_t)B * 3 * kN * 8)) || (st = s->alloc(&s->d_y8, (size_t)2 * s->y8_np * 3 * kN)) ||
        (st = s->alloc(&s->d_bS, (size_t)B * no * 2 * kN * 4)) ||
        (s->fold_mode < 2 && (st = s->alloc(&s->d_bR, (size_t)B * no * kN * 8))) ||
        (st = s->alloc(&s->d_bresp, (size_t)B * rb)))
        return st;
    CU(cudaMallocHost(&s->h_bq, (size_t)B * qb));
    CU(cudaMallocHost(&s->h_bresp, (size_t)B * rb));
    s->bcap = B;
    return IPR_OK;
}

int y8_map(ipr_server* s, int nt, const CUtensorMap** out) {
    auto it = s->tm_y8.find(nt);
    if (it == s->tm_y8.end()) {
        CUtensorMap m;
        CU(ipr::make_u8_tile_map(&m, s->d_y8, 3 * kN, 2 * (uint64_t)s->y8_np, (uint32_t)nt));
        it = s->tm_y8.emplace(nt, m).first;
    }
    *out = &it->second;
    return IPR_OK;
}

// B payloads of 2 queries each: queries at d_queries + p*qbytes, responses at d_resps + p*rbytes
int enqueue_batch(ipr_server* s, int B, const uint8_t* d_queries, uint8_t* d_resps, int prof) {
    cudaStream_t st = s->stream;
    const ipr::Plan& p = s->plan;
    auto rec = [&](int stage) {
        if (prof >= 0) cudaEventRecord(s->events[(size_t)prof * (IPR_NSTAGES + 1) + stage], st);
    };
    const int64_t qb = (int64_t)ipr::query_bytes(p.db_rows, 2), rb = (int64_t)s->response_bytes(2);
    const int nqt = 2 * B;
    rec(0);
    CU(ipr::launch_parse_batch(d_queries, B, qb, 2, (int)p.db_rows, s->d_ybs, s->d_zbs, s->d_gsw, s->d_qb, st));
    rec(1);
    {
        const int nt = g1_nt(s, (unsigned)nqt);
        const CUtensorMap* tq;
        int e = qb_map(s, nt, &tq);
        if (e) return e;
        CU(ipr::launch_gemm1(&s->tm_db, tq, (int)p.db_rows, (int64_t)p.db_cols, nt, g1_tiles((unsigned)nqt, nt),
                             nqt, s->d_c, s->d_err, s->sm_count, st));
    }
    rec(2);
    {
        const int nt = ipr::pack_mma_nt(B);
        const bool pair = s->pack_pair == 1 || (s->pack_pair == 2 && B >= 48);
        const CUtensorMap* ty;
        int e = y8_map(s, pair ? nt / 2 : nt, &ty);  // the pair form loads half the client rows per CTA
        if (e) return e;
        CU(ipr::launch_build_y8(s->d_ybs, s->d_y8, B, s->y8_np, st));
        if (pair)
            CU(ipr::launch_pack_mma_pair(&s->tm_tpp, ty, (int)p.instances, B, s->y8_np, s->d_bS, s->d_err, s->sm_count,
                                         st));
        else
            CU(ipr::launch_pack_mma(&s->tm_tpp, ty, (int)p.instances, B, s->y8_np, s->d_bS, s->d_err, s->sm_count,
                                    st));
    }
    rec(3);
    if (s->fold_mode >= 2) {
        const bool chain = s->fold_mode >= 3;
        CU(ipr::launch_fold_prep(s->d_bS, (int64_t)B * p.instances, s->d_zbs, s->d_bth, (int)p.instances, s->hp.ninv,
                                 s->sm_count, st, chain ? s->d_gsw : nullptr, nqt, s->hp.ninvr));
        rec(4);
        if (chain) {
            ipr::FoldExtents ext{(int64_t)B * (int64_t)p.instances * 2 * kN, (int64_t)nqt * 12 * kN,
                                 (int64_t)p.instances * kN, (int64_t)nqt * (int64_t)p.db_cols, (int64_t)B * rb};
            if (ipr::kBoundsChecked) ext.s_words -= ipr::g_fold_extent_cut.load();
            CU(ipr::launch_fold4(s->d_row0m, s->d_gsw, s->d_ahat, s->d_bS, (int64_t)(p.instances * 2 * kN), s->d_c,
                                 s->d_fwi, s->d_iwi, (int)p.interp, (int)p.c, nqt, (int64_t)p.db_cols, 2, d_resps, rb,
                                 (int64_t)(4 + s->per_query_bytes()), ext, st, fold_staged(s, (int)(nqt * p.c))));
        }
        else
            CU(ipr::launch_fold3(s->d_row0s, s->d_gsw, s->d_ahat, s->d_bS, (int64_t)(p.instances * 2 * kN), s->d_c,
                                 s->d_fwi, s->d_iwi, s->hp.ninv, (int)p.interp, (int)p.c, nqt, (int64_t)p.db_cols, 2,
                                 d_resps, rb, (int64_t)(4 + s->per_query_bytes()), st));
    } else {
        if (!s->d_bR) return fail(IPR_E_STATE, "batch scratch lacks the INTT output (fold form changed mid-batch)");
        CU(ipr::launch_intt_crt(s->d_bS, s->d_iw, s->d_iwp, s->d_bR, (int)(B * p.instances), st, s->d_zbs, s->d_bth,
                                (int)p.instances));
        rec(4);
        CU(ipr::launch_fold2(s->d_row0, s->d_gsw, s->d_ahat, s->d_bR, (int64_t)(p.instances * kN), s->d_c, s->d_fw,
                             s->d_fwp, s->d_iw, s->d_iwp, (int)p.interp, (int)p.c, nqt, (int64_t)p.db_cols, 2, d_resps,
                             rb, (int64_t)(4 + s->per_query_bytes()), st));
    }
    CU(ipr::launch_response_frame(d_resps, 2, (int64_t)s->per_query_bytes(), s->d_stash, (int64_t)s->stash_count,
                                  (int64_t)s->stash_entry, st, B, rb));
    rec(5);
    return IPR_OK;
}

int get_graph(ipr_server* s, unsigned nq, cudaGraphExec_t* out) {
    auto it = s->graphs.find(nq);
    if (it != s->graphs.end()) {
        *out = it->second;
        return IPR_OK;
    }
    const size_t qb = ipr::query_bytes(s->plan.db_rows, nq), rb = s->response_bytes(nq);
    cudaGraph_t g;
    CU(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(s->d_err, 0, sizeof(int), s->stream);
    cudaMemcpyAsync(s->d_query, s->h_query, qb, cudaMemcpyHostToDevice, s->stream);
    int st = enqueue(s, nq, s->d_query, s->d_resp, -1);
    cudaMemcpyAsync(s->h_resp, s->d_resp, rb, cudaMemcpyDeviceToHost, s->stream);
    cudaMemcpyAsync(s->h_err, s->d_err, sizeof(int), cudaMemcpyDeviceToHost, s->stream);
    cudaError_t e = cudaStreamEndCapture(s->stream, &g);
    if (st) return st;
    CU(e);
    cudaGraphExec_t ex;
    e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    CU(e);
    s->graphs[nq] = ex;
    *out = ex;
    return IPR_OK;
}

int init_common(ipr_server* s, int device, const ipr_plan* plan) {
    if (!plan || plan->db_rows < (uint64_t)kN || (plan->db_rows & 255) || plan->instances == 0 ||
        plan->interp == 0 || plan->c == 0 || plan->c * plan->interp > plan->instances ||
        plan->db_cols != plan->instances * kN)
        return fail(IPR_E_ARGS, "invalid plan");
    s->device = device;
    CU(cudaSetDevice(device));
    CU(cudaDeviceGetAttribute(&s->sm_count, cudaDevAttrMultiProcessorCount, device));
    s->plan.num_items = plan->num_items;
    s->plan.entry_size = plan->entry_size;
    s->plan.item_size_bits = plan->item_size_bits;
    s->plan.dim0 = plan->dim0;
    s->plan.db_rows = plan->db_rows;
    s->plan.db_cols = plan->db_cols;
    s->plan.instances = plan->instances;
    s->plan.interp = plan->interp;
    s->plan.c = plan->c;
    s->plan.peak_bytes = plan->peak_bytes;
    // HBM preflight (the reference's check, keyword.rs:368-387, on the resident footprint)
    const uint64_t resident = plan->db_rows * plan->db_cols * 2 + plan->instances * kN * 8 +
                              2 * plan->instances * (uint64_t)kNInner * kN * 8 + plan->instances * 3ull * kN * 8;
    size_t free_b = 0, total_b = 0;
    CU(cudaMemGetInfo(&free_b, &total_b));
    if (resident > free_b)
        return fail(IPR_E_OOM,
                    "insufficient GPU memory: requires %llu bytes, only %zu bytes available (db_rows=%llu, "
                    "db_cols=%llu, instances=%llu)",
                    (unsigned long long)resident, free_b, (unsigned long long)plan->db_rows,
                    (unsigned long long)plan->db_cols, (unsigned long long)plan->instances);
    int lo, hi;
    CU(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    CU(cudaStreamCreateWithPriority(&s->stream, cudaStreamNonBlocking, hi));
    CU(ipr::init_device_kernels());
    CU(ipr::init_gemm1_kernel());
    CU(ipr::init_fold2_kernel());
    CU(ipr::init_fold3_kernel());
    CU(ipr::init_pack_mma_kernel());
    CU(ipr::init_pack_pair_kernel());
    ipr::host_params_init(s->hp);
    CU(ipr::set_constants(s->hp.barrett, s->hp.q0_inv_mod_q1));
    int st;
    const size_t tb = 2 * kN * 4;
    if ((st = s->alloc(&s->d_fw, tb)) || (st = s->alloc(&s->d_fwp, tb)) || (st = s->alloc(&s->d_iw, tb)) ||
        (st = s->alloc(&s->d_iwp, tb)) || (st = s->alloc(&s->d_row0, tb)) || (st = s->alloc(&s->d_fwi, 2 * tb)) ||
        (st = s->alloc(&s->d_iwi, 2 * tb)) || (st = s->alloc(&s->d_row0s, tb)) || (st = s->alloc(&s->d_row0m, tb)))
        return st;
    CU(cudaMemcpy(s->d_fwi, s->hp.fwi.data(), 2 * tb, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(s->d_iwi, s->hp.iwi.data(), 2 * tb, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(s->d_row0s, s->hp.row0s.data(), tb, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(s->d_row0m, s->hp.row0m.data(), tb, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(s->d_fw, s->hp.fw.data(), tb, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(s->d_fwp, s->hp.fwp.data(), tb, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(s->d_iw, s->hp.iw.data(), tb, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(s->d_iwp, s->hp.iwp.data(), tb, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(s->d_row0, s->hp.row0.data(), tb, cudaMemcpyHostToDevice));
    const uint64_t no = plan->instances;
    if ((st = s->alloc(&s->d_db, plan->db_rows * plan->db_cols * 2)) || (st = s->alloc(&s->d_ahat, no * kN * 8)) ||
        (st = s->alloc(&s->d_bt, no * (uint64_t)kNInner * kN * 8)) ||
        (st = s->alloc(&s->d_btb, no * (uint64_t)kNInner * kN * 8)) || (st = s->alloc(&s->d_bth, no * 3 * kN * 8)) ||
        (st = s->alloc(&s->d_y, 3 * kN * 8)) || (st = s->alloc(&s->d_z, 3 * kN * 8)) ||
        (st = s->alloc(&s->d_S, no * 2 * kN * 4)) || (st = s->alloc(&s->d_R, no * kN * 8)))
        return st;
    s->gemv_tc = plan->db_rows <= 32768 && plan->db_rows % 128 == 0 && plan->db_cols % 128 == 0;
    if ((st = s->alloc(&s->d_db8, plan->db_rows * plan->db_cols * 2)) || (st = s->alloc(&s->d_err, sizeof(int))))
        return st;
    CU(cudaMemset(s->d_err, 0, sizeof(int)));
    CU(cudaMallocHost(&s->h_err, sizeof(int)));
    *s->h_err = 0;
    CU(ipr::make_u8_tile_map(&s->tm_db, s->d_db8, plan->db_rows, 2 * plan->db_cols, 128));
    s->events.resize((size_t)kMaxProfileSlots * (IPR_NSTAGES + 1), nullptr);
    return ensure_scratch(s, 2);
}

int check_payload(ipr_server* s, const uint8_t* query, size_t len, unsigned* nq) {
    if (!query || len < 1) return fail(IPR_E_FORMAT, "empty query");
    *nq = query[0];
    const uint64_t need = ipr::query_bytes(s->plan.db_rows, *nq);
    if (len < need)
        return fail(IPR_E_FORMAT, "query has %zu bytes, %u queries need %llu", len, *nq, (unsigned long long)need);
    return IPR_OK;
}

int respond_locked(ipr_server* s, const uint8_t* query, size_t len, uint8_t* out, size_t cap, size_t* out_len) {
    unsigned nq;
    int st = check_payload(s, query, len, &nq);
    if (st) return st;
    const uint64_t rb = s->response_bytes(nq);
    if (out_len) *out_len = rb;
    if (!out || cap < rb) return fail(IPR_E_SPACE, "response needs %llu bytes", (unsigned long long)rb);
    CU(cudaSetDevice(s->device));
    if ((st = ensure_scratch(s, nq))) return st;
    const uint64_t qb = ipr::query_bytes(s->plan.db_rows, nq);
    std::memcpy(s->h_query, query, qb);
    if (s->profiling) {
        CU(cudaMemsetAsync(s->d_err, 0, sizeof(int), s->stream));
        CU(cudaMemcpyAsync(s->d_query, s->h_query, qb, cudaMemcpyHostToDevice, s->stream));
        if ((st = enqueue(s, nq, s->d_query, s->d_resp, next_profile_slot(s)))) return st;
        CU(cudaMemcpyAsync(s->h_resp, s->d_resp, rb, cudaMemcpyDeviceToHost, s->stream));
        CU(cudaMemcpyAsync(s->h_err, s->d_err, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    } else {
        cudaGraphExec_t g;
        if ((st = get_graph(s, nq, &g))) return st;
        CU(cudaGraphLaunch(g, s->stream));
    }
    CU(cudaStreamSynchronize(s->stream));
    if (*s->h_err) return fail(IPR_E_TIMEOUT, "a device-side wait ran out (code %d)", *s->h_err);
    std::memcpy(out, s->h_resp, rb);
    return IPR_OK;
}

}  // namespace

namespace ipr {
namespace {
std::atomic<int64_t> g_alloc_fault{-1};  // allocations left before the injected failure; -1 = off
}
bool alloc_fault_due() {
    int64_t v = g_alloc_fault.load(std::memory_order_relaxed);
    while (v >= 0 && !g_alloc_fault.compare_exchange_weak(v, v - 1)) {
    }
    return v == 0;
}
}  // namespace ipr

int ipr_server::alloc_failed(size_t bytes, cudaError_t e) const {
    return fail(IPR_E_OOM, "cudaMalloc(%zu bytes) failed on device %d: %s", bytes, device, cudaGetErrorString(e));
}

namespace ipr {

int server_ensure_batch(ipr_server* s, int payloads) { return ensure_batch(s, payloads); }

int server_enqueue_batch(ipr_server* s, int payloads, const uint8_t* d_queries, uint8_t* d_resps) {
    return enqueue_batch(s, payloads, d_queries, d_resps, next_profile_slot(s));
}

int server_respond_locked(ipr_server* s, const uint8_t* query, size_t len, uint8_t* out, size_t cap,
                          size_t* out_len) {
    return respond_locked(s, query, len, out, cap, out_len);
}

uint64_t server_batch_bytes(const ipr_server* s, int B) {
    const ipr::Plan& p = s->plan;
    const uint64_t rows = p.db_rows, cols = p.db_cols, no = p.instances, nq = 2ull * B;
    const uint64_t qb = ipr::query_bytes(rows, 2), rb = s->response_bytes(2);
    const uint64_t tpp = s->d_tpp ? 0 : ipr::tpp_bytes((int)no);
    // ensure_scratch(2B) + ensure_batch(B) allocations
    const uint64_t scratch = ipr::query_bytes(rows, (unsigned)nq) + 16 + (nq + 1) / 2 * rows * 16 + nq * 12 * kN * 4 +
                             nq * cols * 8 + s->response_bytes((unsigned)nq) + qb_rows((unsigned)nq) * rows;
    const uint64_t batch = B * qb + 2ull * B * 3 * kN * 8 + 2ull * ipr::pack_mma_nt(B) * 3 * kN +
                           B * no * 2 * kN * 4 + (s->fold_mode < 2 ? B * no * kN * 8 : 0) + B * rb;
    return tpp + scratch + batch;
}

int server_init(ipr_server* s, int device, const ipr_plan* plan) { return init_common(s, device, plan); }

int server_finish(ipr_server* s, bool raw_db, const ipr_server_data* data) {
    const ipr::Plan& plan = s->plan;
    int st;
    if (raw_db) {  // encode on the device: the byte-plane buffer has the DB's size and is free until below
        uint16_t* tmp = reinterpret_cast<uint16_t*>(s->d_db8);
        if ((st = ipr::encode_db_device(s->d_db, tmp, plan.db_rows, plan.db_cols, plan.interp, s->stream))) return st;
        CU(cudaMemcpyAsync(s->d_db, tmp, plan.db_rows * plan.db_cols * 2, cudaMemcpyDeviceToDevice, s->stream));
    }
    CU(ipr::launch_db_to_planes(s->d_db, s->d_db8, (int64_t)(plan.db_rows * plan.db_cols), s->stream));
    CU(cudaStreamSynchronize(s->stream));
    s->stash_count = data->stash_count;
    s->stash_entry = data->stash_entry_bytes;
    if (s->stash_count) {
        if ((st = s->alloc(&s->d_stash, s->stash_count * s->stash_entry))) return st;
        CU(cudaMemcpy(s->d_stash, data->stash, s->stash_count * s->stash_entry, cudaMemcpyHostToDevice));
    }
    s->key_size = data->key_size;
    s->value_size = data->value_size;
    s->num_records = data->num_records;
    std::memcpy(s->cuckoo_seed, data->cuckoo_seed, 16);
    // response buffers depend on the stash size: rebuild scratch
    s->cap_q = 0;
    return ensure_scratch(s, 2);
}

}  // namespace ipr

extern "C" {

int ipr_plan_from_shape(uint64_t record_count, uint64_t key_size, uint64_t value_size, uint64_t buckets,
                        uint64_t dim0, ipr_plan* out) {
    if (!out) return fail(IPR_E_ARGS, "null output");
    ipr::Plan p;
    int st = ipr::plan_from_shape(record_count, key_size, value_size, buckets, dim0, p);
    if (st) return fail(st, "invalid keyword server shape (records=%llu, buckets=%llu, dim0=%llu)",
                        (unsigned long long)record_count, (unsigned long long)buckets, (unsigned long long)dim0);
    out->num_items = p.num_items;
    out->entry_size = p.entry_size;
    out->item_size_bits = p.item_size_bits;
    out->dim0 = p.dim0;
    out->db_rows = p.db_rows;
    out->db_cols = p.db_cols;
    out->instances = p.instances;
    out->interp = p.interp;
    out->c = p.c;
    out->peak_bytes = p.peak_bytes;
    return IPR_OK;
}

uint64_t ipr_query_bytes(uint64_t db_rows, unsigned num_queries) { return ipr::query_bytes(db_rows, num_queries); }

int ipr_plan_shard(const ipr_plan* full, int num_shards, int shard, ipr_plan* out, uint64_t* first_instance) {
    if (!full || !out || num_shards < 1 || shard < 0 || shard >= num_shards)
        return fail(IPR_E_ARGS, "bad shard arguments");
    if ((uint64_t)num_shards > full->c)
        return fail(IPR_E_ARGS, "%d shards for %llu fold groups: every shard needs a group", num_shards,
                    (unsigned long long)full->c);
    if (full->c * full->interp != full->instances || full->db_cols != full->instances * kN)
        return fail(IPR_E_ARGS, "plan is not a whole number of fold groups");
    const uint64_t base = full->c / num_shards, rem = full->c % num_shards, k = (uint64_t)shard;
    const uint64_t groups = base + (k < rem ? 1 : 0);
    const uint64_t first_group = k * base + (k < rem ? k : rem);
    *out = *full;
    out->c = groups;
    out->instances = groups * full->interp;
    out->db_cols = out->instances * kN;
    // the reference's setup estimate for the slice (keyword.rs:105-141)
    const uint64_t nph = 1024;
    out->peak_bytes = out->db_rows * out->db_cols * 2 + out->db_cols * 2 * kN * 8 +
                      2 * out->instances * nph * 2 * kN * 8 + 2 * out->instances * (nph - 1) * 3 * kN * 8;
    if (first_instance) *first_instance = first_group * full->interp;
    return IPR_OK;
}

int ipr_response_merge(const uint8_t* const* parts, const size_t* lens, int num_parts, uint8_t* out, size_t cap,
                       size_t* out_len) {
    if (!parts || !lens || num_parts < 1) return fail(IPR_E_ARGS, "no parts");
    auto rd32 = [](const uint8_t* p) {
        return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
    };
    auto wr32 = [](uint8_t* p, uint32_t v) {
        for (int i = 0; i < 4; i++) p[i] = (uint8_t)(v >> (8 * i));
    };
    // parse every part: count, per query (len, bytes), then the stash block
    std::vector<std::vector<std::pair<size_t, uint32_t>>> q(num_parts);  // (offset, length) per query
    std::vector<size_t> stash_at(num_parts);
    uint32_t count = 0;
    for (int k = 0; k < num_parts; k++) {
        const uint8_t* p = parts[k];
        const size_t n = lens[k];
        if (!p || n < 8) return fail(IPR_E_FORMAT, "part %d is too short", k);
        const uint32_t c = rd32(p);
        if (k == 0) count = c;
        else if (c != count) return fail(IPR_E_FORMAT, "part %d has %u responses, part 0 has %u", k, c, count);
        size_t off = 4;
        for (uint32_t i = 0; i < c; i++) {
            if (off + 4 > n) return fail(IPR_E_FORMAT, "part %d is truncated", k);
            const uint32_t l = rd32(p + off);
            if (off + 4 + l > n) return fail(IPR_E_FORMAT, "part %d is truncated", k);
            q[k].push_back({off + 4, l});
            off += 4 + (size_t)l;
        }
        if (off + 4 > n) return fail(IPR_E_FORMAT, "part %d has no stash block", k);
        stash_at[k] = off;
    }
    const size_t stash_bytes = lens[0] - stash_at[0];
    size_t total = 4 + stash_bytes;
    for (uint32_t i = 0; i < count; i++) {
        uint64_t l = 0;
        for (int k = 0; k < num_parts; k++) l += q[k][i].second;
        if (l > 0xffffffffull) return fail(IPR_E_FORMAT, "merged response %u is too long", i);
        total += 4 + l;
    }
    if (out_len) *out_len = total;
    if (!out || cap < total) return fail(IPR_E_SPACE, "merged response needs %zu bytes", total);
    wr32(out, count);
    size_t o = 4;
    for (uint32_t i = 0; i < count; i++) {
        uint32_t l = 0;
        for (int k = 0; k < num_parts; k++) l += q[k][i].second;
        wr32(out + o, l);
        o += 4;
        for (int k = 0; k < num_parts; k++) {
            std::memcpy(out + o, parts[k] + q[k][i].first, q[k][i].second);
            o += q[k][i].second;
        }
    }
    std::memcpy(out + o, parts[0] + stash_at[0], stash_bytes);  // the stash echo of the first part
    return IPR_OK;
}

static int create_server(int device, const ipr_plan* plan, const ipr_server_data* data, bool raw_db,
                         ipr_server** out);

int ipr_server_create(int device, const ipr_plan* plan, const ipr_server_data* data, ipr_server** out) {
    ipr::NvtxRange nvtx_range("ipr_server_create");
    return create_server(device, plan, data, false, out);
}

int ipr_server_create_from_raw(int device, const ipr_plan* plan, const ipr_server_data* data, ipr_server** out) {
    return create_server(device, plan, data, true, out);
}

static int create_server(int device, const ipr_plan* plan, const ipr_server_data* data, bool raw_db,
                         ipr_server** out) {
    if (!out || !data || !data->db || !data->a_hat || !data->bold_t || !data->bold_t_bar || !data->bold_t_hat)
        return fail(IPR_E_ARGS, "null argument");
    if (data->stash_count && (!data->stash || !data->stash_entry_bytes)) return fail(IPR_E_ARGS, "bad stash");
    *out = nullptr;
    auto* s = new ipr_server();
    int st = init_common(s, device, plan);
    if (st) {
        ipr_server_destroy(s);
        return st;
    }
    const uint64_t no = plan->instances;
    auto up = [&](void* dst, const void* src, size_t bytes) -> int {
        CU(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice));
        return IPR_OK;
    };
    if ((st = up(s->d_db, data->db, plan->db_rows * plan->db_cols * 2)) || (st = up(s->d_ahat, data->a_hat, no * kN * 8)) ||
        (st = up(s->d_bt, data->bold_t, no * (uint64_t)kNInner * kN * 8)) ||
        (st = up(s->d_btb, data->bold_t_bar, no * (uint64_t)kNInner * kN * 8)) ||
        (st = up(s->d_bth, data->bold_t_hat, no * 3 * kN * 8)) || (st = ipr::server_finish(s, raw_db, data))) {
        ipr_server_destroy(s);
        return st;
    }
    *out = s;
    return IPR_OK;
}

int ipr_debug_fail_allocation(int64_t after) {
    ipr::g_alloc_fault.store(after < 0 ? -1 : after);
    return IPR_OK;
}

int ipr_server_setup(int device, const ipr_plan* plan, const ipr_server_data* data, int db_is_raw,
                     ipr_server** out) {
    ipr::NvtxRange nvtx_range("ipr_server_setup");
    if (!out || !data || !data->db) return fail(IPR_E_ARGS, "null argument");
    if (data->stash_count && (!data->stash || !data->stash_entry_bytes)) return fail(IPR_E_ARGS, "bad stash");
    *out = nullptr;
    auto* s = new ipr_server();
    int st = init_common(s, device, plan);
    auto bail = [&](int code) {
        ipr_server_destroy(s);
        return code;
    };
    if (st) return bail(st);
    const uint64_t db_bytes = plan->db_rows * plan->db_cols * 2;
    if (cudaMemcpy(s->d_db, data->db, db_bytes, cudaMemcpyHostToDevice) != cudaSuccess)
        return bail(fail(IPR_E_CUDA, "DB upload: %s", cudaGetErrorString(cudaGetLastError())));
    if (db_is_raw) {  // encode first: the precomputation reads the encoded DB
        uint16_t* tmp = reinterpret_cast<uint16_t*>(s->d_db8);
        if ((st = ipr::encode_db_device(s->d_db, tmp, plan->db_rows, plan->db_cols, plan->interp, s->stream)))
            return bail(st);
        if (cudaMemcpyAsync(s->d_db, tmp, db_bytes, cudaMemcpyDeviceToDevice, s->stream) != cudaSuccess)
            return bail(fail(IPR_E_CUDA, "encoded DB copy: %s", cudaGetErrorString(cudaGetLastError())));
    }
    if ((st = ipr::offline_precompute_device(s->d_db, plan->db_rows, plan->instances, s->d_ahat, s->d_bt, s->d_btb,
                                             s->d_bth, 0, s->stream)) ||
        (st = ipr::server_finish(s, false, data)))
        return bail(st);
    *out = s;
    return IPR_OK;
}

namespace {
// a synthetic server holding instances [first, first + plan->instances) of a synthetic state
int create_synthetic(int device, const ipr_plan* plan, uint64_t seed, uint64_t first, ipr_server** out) {
    if (!out) return fail(IPR_E_ARGS, "null output");
    *out = nullptr;
    auto* s = new ipr_server();
    int st = init_common(s, device, plan);
    if (st) {
        ipr_server_destroy(s);
        return st;
    }
    const int64_t no = (int64_t)plan->instances;
    const uint64_t f = first;
    cudaStream_t t = s->stream;
    auto chk = [&](cudaError_t e) -> int {
        if (e != cudaSuccess) return fail(IPR_E_CUDA, "synthetic fill: %s", cudaGetErrorString(e));
        return IPR_OK;
    };
    if ((st = chk(ipr::launch_synth_db(s->d_db, (int64_t)(plan->db_rows * plan->db_cols), seed, t,
                                       f * kN * plan->db_rows))) ||
        (st = chk(ipr::launch_synth_modq(s->d_ahat, no * kN, seed, 2, t, f * kN))) ||
        (st = chk(ipr::launch_synth_condensed(s->d_bt, no * kNInner * kN, seed, 3, t, f * kNInner * kN))) ||
        (st = chk(ipr::launch_synth_condensed(s->d_btb, no * kNInner * kN, seed, 4, t, f * kNInner * kN))) ||
        (st = chk(ipr::launch_synth_condensed(s->d_bth, no * 3 * kN, seed, 5, t, f * 3 * kN))) ||
        (st = chk(ipr::launch_db_to_planes(s->d_db, s->d_db8, (int64_t)(plan->db_rows * plan->db_cols), t))) ||
        (st = chk(cudaStreamSynchronize(t)))) {
        ipr_server_destroy(s);
        return st;
    }
    s->key_size = 32;
    s->value_size = plan->entry_size > 32 ? plan->entry_size - 32 : 0;
    *out = s;
    return IPR_OK;
}
}  // namespace

int ipr_server_create_synthetic(int device, const ipr_plan* plan, uint64_t seed, ipr_server** out) {
    ipr::NvtxRange nvtx_range("ipr_server_create_synthetic");
    return create_synthetic(device, plan, seed, 0, out);
}

int ipr_server_create_synthetic_shard(int device, const ipr_plan* full, int num_shards, int shard, uint64_t seed,
                                      ipr_server** out) {
    ipr::NvtxRange nvtx_range("ipr_server_create_synthetic_shard");
    if (!full || !out) return fail(IPR_E_ARGS, "null argument");
    ipr_plan sub;
    uint64_t first = 0;
    int st = ipr_plan_shard(full, num_shards, shard, &sub, &first);
    if (st) return st;
    return create_synthetic(device, &sub, seed, first, out);
}

void ipr_server_destroy(ipr_server* s) {
    if (!s) return;
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    destroy_graphs(s);
    for (auto e : s->events)
        if (e) cudaEventDestroy(e);
    for (void* p : s->allocs) cudaFree(p);
    if (s->h_query) cudaFreeHost(s->h_query);
    if (s->h_resp) cudaFreeHost(s->h_resp);
    if (s->h_err) cudaFreeHost(s->h_err);
    if (s->h_bq) cudaFreeHost(s->h_bq);
    if (s->h_bresp) cudaFreeHost(s->h_bresp);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

int ipr_server_public_params_json(const ipr_server* s, char* out, size_t cap, size_t* out_len) {
    if (!s) return fail(IPR_E_ARGS, "null server");
    std::string j = "{\"num_items\":" + std::to_string(s->plan.num_items) +
                    ",\"item_size_bits\":" + std::to_string(s->plan.entry_size * 8) +
                    ",\"dim0\":" + std::to_string(s->plan.dim0) + ",\"keyword_pir\":{\"cuckoo_seed\":[";
    for (int i = 0; i < 16; i++) j += (i ? "," : "") + std::to_string((int)s->cuckoo_seed[i]);
    j += "],\"num_hashes\":2,\"key_size\":" + std::to_string(s->key_size) +
         ",\"value_size\":" + std::to_string(s->value_size) + ",\"entry_size\":" + std::to_string(s->plan.entry_size) +
         ",\"num_records\":" + std::to_string(s->num_records) + "}}";
    if (out_len) *out_len = j.size();
    if (!out || cap < j.size() + 1) return fail(IPR_E_SPACE, "public params need %zu bytes", j.size() + 1);
    std::memcpy(out, j.c_str(), j.size() + 1);
    return IPR_OK;
}

uint64_t ipr_server_query_bytes(const ipr_server* s, unsigned nq) {
    return s ? ipr::query_bytes(s->plan.db_rows, nq) : 0;
}
uint64_t ipr_server_response_bytes(const ipr_server* s, unsigned nq) { return s ? s->response_bytes(nq) : 0; }

int ipr_server_hbm_bytes(const ipr_server* s, uint64_t* out) {
    if (!s || !out) return fail(IPR_E_ARGS, "null argument");
    *out = s->hbm;
    return IPR_OK;
}

int ipr_server_plan(const ipr_server* s, ipr_plan* out) {
    if (!s || !out) return fail(IPR_E_ARGS, "null argument");
    out->num_items = s->plan.num_items;
    out->entry_size = s->plan.entry_size;
    out->item_size_bits = s->plan.item_size_bits;
    out->dim0 = s->plan.dim0;
    out->db_rows = s->plan.db_rows;
    out->db_cols = s->plan.db_cols;
    out->instances = s->plan.instances;
    out->interp = s->plan.interp;
    out->c = s->plan.c;
    out->peak_bytes = s->plan.peak_bytes;
    return IPR_OK;
}

int ipr_server_respond(ipr_server* s, const uint8_t* query, size_t len, uint8_t* out, size_t cap, size_t* out_len) {
    ipr::NvtxRange nvtx_range("ipr_server_respond");
    if (!s) return fail(IPR_E_ARGS, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    return respond_locked(s, query, len, out, cap, out_len);
}

int ipr_server_respond_batch(ipr_server* s, int n, const uint8_t* const* queries, const size_t* lens,
                             uint8_t* const* outs, const size_t* caps, size_t* out_lens, int* statuses) {
    ipr::NvtxRange nvtx_range("ipr_server_respond_batch");
    if (!s || n < 0 || (n && (!queries || !lens || !outs || !caps))) return fail(IPR_E_ARGS, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    const uint64_t qb = ipr::query_bytes(s->plan.db_rows, 2), rb = s->response_bytes(2);
    // payloads with the usual two cuckoo queries go through the tensor-core batch
    // path, up to 64 at a time; anything else is answered one by one
    std::vector<int> batchable, single;
    for (int i = 0; i < n; i++) {
        const bool ok2 = queries[i] && lens[i] >= qb && queries[i][0] == 2 && outs[i] && caps[i] >= rb;
        (ok2 && n >= 2 && s->gemv_tc ? batchable : single).push_back(i);
    }
    int worst = IPR_OK;
    auto note = [&](int i, int st, size_t ol) {
        if (out_lens) out_lens[i] = ol;
        if (statuses) statuses[i] = st;
        if (st && !worst) worst = st;
    };
    for (size_t c0 = 0; c0 < batchable.size(); c0 += kMaxBatch) {
        const int B = (int)std::min<size_t>(kMaxBatch, batchable.size() - c0);
        int st = ensure_batch(s, B);
        if (st == IPR_OK) {
            CU(cudaSetDevice(s->device));
            for (int b = 0; b < B; b++) std::memcpy(s->h_bq + (size_t)b * qb, queries[batchable[c0 + b]], qb);
            CU(cudaMemsetAsync(s->d_err, 0, sizeof(int), s->stream));
            CU(cudaMemcpyAsync(s->d_bq, s->h_bq, (size_t)B * qb, cudaMemcpyHostToDevice, s->stream));
            st = enqueue_batch(s, B, s->d_bq, s->d_bresp, next_profile_slot(s));
            if (st == IPR_OK) {
                CU(cudaMemcpyAsync(s->h_bresp, s->d_bresp, (size_t)B * rb, cudaMemcpyDeviceToHost, s->stream));
                CU(cudaMemcpyAsync(s->h_err, s->d_err, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
                CU(cudaStreamSynchronize(s->stream));
                if (*s->h_err) st = fail(IPR_E_TIMEOUT, "a device-side wait ran out (code %d)", *s->h_err);
            }
        }
        for (int b = 0; b < B; b++) {
            const int i = batchable[c0 + b];
            if (st == IPR_OK) std::memcpy(outs[i], s->h_bresp + (size_t)b * rb, rb);
            note(i, st, rb);
        }
    }
    for (int i : single) {
        size_t ol = 0;
        int st = respond_locked(s, queries[i], lens[i], outs[i], caps[i], &ol);
        note(i, st, ol);
    }
    return worst;
}

int ipr_server_prepare_batch(ipr_server* s, int max_payloads) {
    if (!s || max_payloads < 1) return fail(IPR_E_ARGS, "bad argument");
    std::lock_guard<std::mutex> lk(s->mu);
    CU(cudaSetDevice(s->device));
    return ensure_batch(s, max_payloads < kMaxBatch ? max_payloads : kMaxBatch);
}

int ipr_server_respond_batch_device(ipr_server* s, int n, const uint8_t* d_queries, uint8_t* d_out) {
    ipr::NvtxRange nvtx_range("ipr_server_respond_batch_device");
    if (!s || !d_queries || !d_out || n < 1 || n > kMaxBatch) return fail(IPR_E_ARGS, "bad argument (1 <= n <= 64)");
    std::lock_guard<std::mutex> lk(s->mu);
    CU(cudaSetDevice(s->device));
    int st = ensure_batch(s, n);
    if (st) return st;
    CU(cudaMemsetAsync(s->d_err, 0, sizeof(int), s->stream));
    return enqueue_batch(s, n, d_queries, d_out, next_profile_slot(s));
}

int ipr_server_respond_device(ipr_server* s, const uint8_t* d_query, size_t len, uint8_t* d_out, size_t cap,
                              size_t* out_len) {
    ipr::NvtxRange nvtx_range("ipr_server_respond_device");
    if (!s || !d_query || !d_out) return fail(IPR_E_ARGS, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    CU(cudaSetDevice(s->device));
    // the query count follows from the exact length (the count byte stays on the device)
    const uint64_t base = ipr::query_bytes(s->plan.db_rows, 0), per = ipr::query_bytes(s->plan.db_rows, 1) - base;
    if (len < base || (len - base) % per || (len - base) / per > 255)
        return fail(IPR_E_FORMAT, "device query length %zu is not an exact payload size", len);
    const unsigned nq = (unsigned)((len - base) / per);
    const uint64_t rb = s->response_bytes(nq);
    if (out_len) *out_len = rb;
    if (cap < rb) return fail(IPR_E_SPACE, "response needs %llu bytes", (unsigned long long)rb);
    int st = ensure_scratch(s, nq);
    if (st) return st;
    CU(cudaMemsetAsync(s->d_err, 0, sizeof(int), s->stream));
    return enqueue(s, nq, d_query, d_out, next_profile_slot(s));
}

int ipr_server_stream(ipr_server* s, void** stream) {
    if (!s || !stream) return fail(IPR_E_ARGS, "null argument");
    *stream = (void*)s->stream;
    return IPR_OK;
}

int ipr_server_sync(ipr_server* s) {
    if (!s) return fail(IPR_E_ARGS, "null server");
    CU(cudaStreamSynchronize(s->stream));
    int flag = 0;
    CU(cudaMemcpy(&flag, s->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) return fail(IPR_E_TIMEOUT, "a device-side wait ran out (code %d)", flag);
    return IPR_OK;
}

int ipr_server_autotune(ipr_server* s, int payloads, int reps, ipr_autotune_result* out) {
    ipr::NvtxRange nvtx_range("ipr_server_autotune");
    if (!s || !out || payloads < 1 || payloads > kMaxBatch || reps < 1 || reps > 100)
        return fail(IPR_E_ARGS, "bad argument (1 <= payloads <= 64, 1 <= reps <= 100)");
    std::lock_guard<std::mutex> lk(s->mu);
    CU(cudaSetDevice(s->device));
    if (!s->gemv_tc) return fail(IPR_E_STATE, "the batch path needs the tensor-core first dimension");
    int st = ensure_batch(s, payloads);
    if (st) return st;
    // synthetic payloads: a count byte of 2, then 56-bit fields of residues below each prime
    const uint64_t qb = ipr::query_bytes(s->plan.db_rows, 2);
    uint64_t x = 0x9E3779B97F4A7C15ull;
    auto next = [&x]() {
        uint64_t z = (x += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    for (int b = 0; b < payloads; b++) {
        uint8_t* q = s->h_bq + (size_t)b * qb;
        q[0] = 2;
        for (uint64_t f = 0; f < (qb - 1) / 7; f++) {
            const uint64_t v = (next() % 268369921ull) | ((next() % 249561089ull) << 28);
            for (int k = 0; k < 7; k++) q[1 + 7 * f + k] = (uint8_t)(v >> (8 * k));
        }
    }
    CU(cudaMemcpyAsync(s->d_bq, s->h_bq, (size_t)payloads * qb, cudaMemcpyHostToDevice, s->stream));
    const int old_pair = s->pack_pair, old_tile = s->g1_tile;
    // CTA pairs pay off only for large batches, so the automatic threshold (2) competes with
    // pairs never (0) and always (1), and every candidate is timed at the requested batch
    // size and at a quarter of it: the score is the device time per payload summed over both
    static const int pairs[] = {2, 0, 1}, tiles[] = {0, 128};
    *out = ipr_autotune_result{};
    for (int pr : pairs)
        for (int tl : tiles) {
            out->pack_cta_pair[out->candidates] = pr;
            out->gemv_tile[out->candidates++] = tl ? tl : 256;
        }
    const int nc = out->candidates;
    const int sizes[2] = {payloads, payloads >= 4 ? payloads / 4 : 0};
    const int nsz = sizes[1] ? 2 : 1;
    out->small_payloads = sizes[1];
    // candidates interleaved round-robin, one event pair per timed batch, so that clock drift
    // under the power cap falls on every candidate alike
    std::vector<cudaEvent_t> ev((size_t)2 * nc * reps * nsz, nullptr);
    auto cleanup = [&]() {
        for (cudaEvent_t e : ev)
            if (e) cudaEventDestroy(e);
    };
    for (auto& e : ev)
        if (cudaEventCreate(&e) != cudaSuccess) {
            e = nullptr;
            cleanup();
            return fail(IPR_E_CUDA, "event");
        }
    auto use = [&](int i) {
        s->pack_pair = out->pack_cta_pair[i];
        s->g1_tile = out->gemv_tile[i] == 256 ? 0 : out->gemv_tile[i];
    };
    auto evi = [&](int z, int r, int i) { return (size_t)2 * ((z * reps + r) * nc + i); };
    cudaMemsetAsync(s->d_err, 0, sizeof(int), s->stream);
    for (int z = 0; z < nsz; z++)
        for (int i = 0; i < nc && !st; i++) {  // one warm-up batch per candidate and size
            use(i);
            st = enqueue_batch(s, sizes[z], s->d_bq, s->d_bresp, -1);
        }
    for (int r = 0; r < reps && !st; r++)
        for (int z = 0; z < nsz && !st; z++)
            for (int i = 0; i < nc && !st; i++) {
                use(i);
                cudaEventRecord(ev[evi(z, r, i)], s->stream);
                st = enqueue_batch(s, sizes[z], s->d_bq, s->d_bresp, -1);
                cudaEventRecord(ev[evi(z, r, i) + 1], s->stream);
            }
    int flag = 0;
    if (!st && (cudaStreamSynchronize(s->stream) != cudaSuccess ||
                cudaMemcpy(&flag, s->d_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess))
        st = fail(IPR_E_CUDA, "autotune: %s", cudaGetErrorString(cudaGetLastError()));
    if (!st && flag) st = fail(IPR_E_TIMEOUT, "a device-side wait ran out during autotuning (code %d)", flag);
    int best = -1;
    double best_score = 0;
    for (int i = 0; i < nc && !st; i++) {
        double score = 0;
        for (int z = 0; z < nsz && !st; z++) {
            double sum = 0;
            for (int r = 0; r < reps && !st; r++) {
                float ms = 0;
                if (cudaEventElapsedTime(&ms, ev[evi(z, r, i)], ev[evi(z, r, i) + 1]) != cudaSuccess)
                    st = fail(IPR_E_CUDA, "event timing: %s", cudaGetErrorString(cudaGetLastError()));
                sum += ms;
            }
            (z ? out->ms_small : out->ms)[i] = sum / reps;
            score += sum / reps / sizes[z];
        }
        if (best < 0 || score < best_score) {
            best = i;
            best_score = score;
        }
    }
    cleanup();
    if (st) {
        cudaStreamSynchronize(s->stream);
        s->pack_pair = old_pair;
        s->g1_tile = old_tile;
        return st;
    }
    s->pack_pair = out->pack_cta_pair[best];
    s->g1_tile = out->gemv_tile[best] == 256 ? 0 : out->gemv_tile[best];
    out->chosen = best;
    if (s->g1_tile != old_tile) destroy_graphs(s);  // the single-payload graphs bake in the tile
    return IPR_OK;
}

int ipr_server_set_option(ipr_server* s, int option, int64_t value) {
    if (!s) return fail(IPR_E_ARGS, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    switch (option) {
        case IPR_OPT_TENSOR_GEMV:
            if (value && !(s->plan.db_rows <= 32768 && s->plan.db_rows % 128 == 0))
                return fail(IPR_E_ARGS, "tensor-core first dimension needs db_rows <= 32768, a multiple of 128");
            s->gemv_tc = value != 0;
            destroy_graphs(s);
            return IPR_OK;
        case IPR_OPT_FOLD_REGISTER_NTT: {
            if (value < 0 || value > 5) return fail(IPR_E_ARGS, "IPR_OPT_FOLD_REGISTER_NTT takes 0 to 5");
            const bool had_r = s->fold_mode < 2;
            s->fold_mode = (int)value;
            destroy_graphs(s);
            if ((s->fold_mode < 2) != had_r && s->bcap) {  // the batch scratch changes shape
                CU(cudaStreamSynchronize(s->stream));
                s->bcap = 0;
            }
            return IPR_OK;
        }
        case IPR_OPT_GEMV_FORM:
            if (value < 0 || value > 6) return fail(IPR_E_ARGS, "IPR_OPT_GEMV_FORM takes 0 to 6");
            s->gemv_form = (int)value;
            destroy_graphs(s);
            return IPR_OK;
        case IPR_OPT_PACK_CTA_PAIR:
            if (value < 0 || value > 2) return fail(IPR_E_ARGS, "IPR_OPT_PACK_CTA_PAIR takes 0, 1 or 2");
            s->pack_pair = (int)value;
            return IPR_OK;
        case IPR_OPT_GEMV_TILE:
            if (value && (value < 16 || value > 256 || (256 % value)))
                return fail(IPR_E_ARGS, "IPR_OPT_GEMV_TILE takes 0 or a divisor of 256 from 16 up");
            s->g1_tile = (int)value;
            destroy_graphs(s);
            return IPR_OK;
        default:
            return fail(IPR_E_ARGS, "unknown option %d", option);
    }
}

int ipr_server_set_profiling(ipr_server* s, int on) {
    if (!s) return fail(IPR_E_ARGS, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    CU(cudaSetDevice(s->device));
    if (on && !s->events[0])
        for (auto& e : s->events) CU(cudaEventCreate(&e));
    int st = harvest_profile(s);
    if (st) return st;
    s->profiling = on != 0;
    for (double& v : s->stage_ms) v = 0;
    s->calls = 0;
    return IPR_OK;
}

int ipr_server_stage_times(ipr_server* s, double* ms_sum, uint64_t* calls) {
    if (!s || !ms_sum) return fail(IPR_E_ARGS, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    int st = harvest_profile(s);
    if (st) return st;
    for (int k = 0; k < IPR_NSTAGES; k++) ms_sum[k] = s->stage_ms[k];
    if (calls) *calls = s->calls;
    return IPR_OK;
}

const char* ipr_last_error(void) { return g_last_error.c_str(); }
const char* ipr_version(void) { return "inspire-rs_b200 0.1 (sm_100a)"; }

}  // extern "C"
