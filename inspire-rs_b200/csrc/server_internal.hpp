// server_internal.hpp — the ipr_server handle shared by server.cu and service.cu
// (library-internal; the public interface is include/ipr_b200.h).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <mutex>
#include <vector>

#include "host_math.hpp"
#include "ipr_b200.h"

#include <nvtx3/nvToolsExt.h>

namespace ipr {
// a named NVTX range over a host API call (visible in Nsight Systems; inert without a tool)
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// allocation-failure injection (ipr_debug_fail_allocation): true for the one device allocation
// of a server that the armed countdown reaches, which then fails as an out-of-memory would
bool alloc_fault_due();
}

namespace ipr {
void set_last_error(const char* msg);
}

struct ipr_server {
    int device = 0;
    int sm_count = 148;
    ipr::Plan plan{};
    ipr::HostParams hp;
    cudaStream_t stream = nullptr;
    // resident state
    uint16_t* d_db = nullptr;
    uint8_t* d_db8 = nullptr;  // [2][db_cols][db_rows] byte planes for the tensor-core GEMM
    CUtensorMap tm_db;
    bool gemv_tc = false;      // first dimension on tcgen05 (db_rows <= 32768)
    int fold_mode = 3;         // 3 fused fold, one chain per CTA (k_fold_prep + k_fold4), two or three
                               // CTAs per SM by chain count (4: three, 5: two), 2 fused fold
                               // on two chains per CTA (k_fold_prep + k_fold3), 1 k_intt_crt + k_fold2,
                               // 0 smem fold
    int pack_pair = 2;         // batch packing GEMM on CTA pairs: 0 never, 1 always, 2 from 48 payloads up
    int g1_tile = 0;           // first-dimension GEMM query-byte tile height cap (0 = 256)
    int gemv_form = 6;         // form of the CUDA-core GEMV (IPR_OPT_GEMV_FORM)
    std::map<int, CUtensorMap> tm_qb;  // per query-byte tile height
    uint64_t *d_ahat = nullptr, *d_bt = nullptr, *d_btb = nullptr, *d_bth = nullptr;
    uint8_t* d_stash = nullptr;
    uint64_t stash_count = 0, stash_entry = 0;
    uint32_t *d_fw = nullptr, *d_fwp = nullptr, *d_iw = nullptr, *d_iwp = nullptr, *d_row0 = nullptr;
    uint32_t *d_fwi = nullptr, *d_iwi = nullptr, *d_row0s = nullptr;  // the fused fold's tables
    uint32_t* d_row0m = nullptr;  // row 0 x N^-1 x 2^32 for the one-chain fold's Montgomery reductions
    // per-request scratch
    unsigned cap_q = 0;
    uint8_t* d_query = nullptr;
    uint64_t *d_y = nullptr, *d_z = nullptr;
    uint32_t *d_ail = nullptr, *d_gsw = nullptr, *d_S = nullptr;
    uint64_t *d_R = nullptr, *d_c = nullptr;
    uint8_t* d_resp = nullptr;
    uint8_t* d_qb = nullptr;  // query bytes [q*7 + byte][db_rows], bytes of the CRT-composed values
    int* d_err = nullptr;     // device-side wait failures (bounded waits)
    uint8_t *h_query = nullptr, *h_resp = nullptr;
    int* h_err = nullptr;
    std::map<unsigned, cudaGraphExec_t> graphs;
    std::mutex mu;
    // batched path: precomputation re-indexed by slot (Tpp), batch scratch
    uint8_t* d_tpp = nullptr;
    CUtensorMap tm_tpp;
    int bcap = 0, y8_np = 0;
    uint8_t* d_bq = nullptr;
    uint64_t *d_ybs = nullptr, *d_zbs = nullptr;
    uint8_t* d_y8 = nullptr;
    std::map<int, CUtensorMap> tm_y8;
    uint32_t* d_bS = nullptr;
    uint64_t* d_bR = nullptr;
    uint8_t* d_bresp = nullptr;
    uint8_t *h_bq = nullptr, *h_bresp = nullptr;
    // profiling
    bool profiling = false;
    std::vector<cudaEvent_t> events;  // kMaxProfileSlots * (IPR_NSTAGES + 1)
    int slots_used = 0;
    double stage_ms[IPR_NSTAGES] = {0};
    uint64_t calls = 0;
    // public parameters
    uint64_t key_size = 0, value_size = 0, num_records = 0;
    uint8_t cuckoo_seed[16] = {0};
    uint64_t hbm = 0;
    std::vector<void*> allocs;

    int alloc_failed(size_t bytes, cudaError_t e) const;  // records the message, returns IPR_E_OOM
    template <typename T>
    int alloc(T** p, size_t bytes) {
        if (ipr::alloc_fault_due()) return alloc_failed(bytes, cudaErrorMemoryAllocation);  // injected
        void* v = nullptr;
        cudaError_t e = cudaMalloc(&v, bytes ? bytes : 16);
        if (e != cudaSuccess)
            return alloc_failed(bytes, e);
        allocs.push_back(v);
        hbm += bytes;
        *p = static_cast<T*>(v);
        return IPR_OK;
    }
    void free_ptr(void* p) {
        for (size_t i = 0; i < allocs.size(); i++)
            if (allocs[i] == p) {
                cudaFree(p);
                allocs.erase(allocs.begin() + i);
                return;
            }
    }
    uint64_t per_query_bytes() const { return plan.c * IPR_RESULT_BYTES; }
    uint64_t response_bytes(unsigned nq) const {
        return 4 + (uint64_t)nq * (4 + per_query_bytes()) + 4 + stash_count * (4 + stash_entry);
    }
};

namespace ipr {
// payloads per tensor-core batch pass (N = 4 bytes x clients <= 256 in the packing GEMM)
constexpr int kMaxBatchPayloads = 64;
// entry points of server.cu for the serving loop; the caller holds s->mu and has set the device
int server_ensure_batch(ipr_server* s, int payloads);
int server_enqueue_batch(ipr_server* s, int payloads, const uint8_t* d_queries, uint8_t* d_resps);
int server_respond_locked(ipr_server* s, const uint8_t* query, size_t len, uint8_t* out, size_t cap, size_t* out_len);
// setup steps shared with the state-file loader: validate the plan, allocate the resident
// state and tables (server_init); after the resident arrays hold the setup outputs, encode
// a raw DB if asked, build the byte planes, upload the stash, set the public parameters
// and the request scratch (server_finish)
int server_init(ipr_server* s, int device, const ipr_plan* plan);
int server_finish(ipr_server* s, bool raw_db, const ipr_server_data* data);
// device bytes the batch path holds for `payloads` (slot-indexed precomputation + scratch)
uint64_t server_batch_bytes(const ipr_server* s, int payloads);
}  // namespace ipr
