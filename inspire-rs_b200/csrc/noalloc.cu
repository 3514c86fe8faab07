// noalloc.cu — a first-dimension GEMV query that allocates no device memory.
//
// Who needs it: callers that cannot call cudaMalloc.  A serving process whose
// framework reserves all free HBM for its own memory pool at start-up cannot
// get more from cudaMalloc (the call fails, or competes with that pool), and a
// latency-critical request path cannot afford the device-wide synchronisation
// that cudaMalloc/cudaFree imply.  gpu_gemv_query (the reference-named entry
// point in compat.cu) allocates a device copy of the query row and of the
// result on every call; ipr_gemv_query_noalloc computes the same GEMV but
// stages both in one fixed device array compiled into this library.
//
// The array holds at most 65,536 query-row entries and 1,048,576 result
// entries (8 bytes each, 8.5 MiB in total).  Every GPU that loads the library
// holds it until the process exits.  All calls share it and it keeps the last
// call's contents: each call first overwrites the query region, and the
// kernel writes every result entry that is copied back, so nothing needs
// clearing.  Calls whose work overlaps on the GPU (several host threads, or
// streams running at once) race on the array; issue them one after another.
//
// The first call on each device looks up the array's device address
// (cudaGetSymbolAddress, with that device current) and loads the modular
// reduction constants; make that first call before any stream capture on the
// device.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "host_math.hpp"
#include "ipr_b200.h"
#include "ipr_device.cuh"
#include "kernels.cuh"

namespace ipr {
void set_last_error(const char* msg);  // server.cu: the text ipr_last_error() returns
}

namespace {

constexpr uint64_t kMaxRows = 65536;       // query-row entries (db_rows)
constexpr uint64_t kMaxCols = 1ull << 20;  // result entries (b_cols)
constexpr int kMaxDevices = 64;

// query row at [0, kMaxRows), result at [kMaxRows, kMaxRows + kMaxCols)
static __device__ __align__(256) uint64_t g_gemv_scratch[kMaxRows + kMaxCols];

std::mutex g_setup_mu;
uint64_t* g_scratch_ptr[kMaxDevices] = {nullptr};
int g_sm_count[kMaxDevices] = {0};

int noalloc_fail(int code, const char* msg, cudaError_t e = cudaSuccess) {
    char buf[320];
    if (e != cudaSuccess) snprintf(buf, sizeof(buf), "ipr_gemv_query_noalloc: %s: %s", msg, cudaGetErrorString(e));
    else snprintf(buf, sizeof(buf), "ipr_gemv_query_noalloc: %s", msg);
    ipr::set_last_error(buf);
    return code;
}

// once per device, with that device current: resolve the array's device
// address (the host-side name is only a stand-in) and load the constants
int setup_device(int dev, uint64_t** out) {
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (g_scratch_ptr[dev]) {
        *out = g_scratch_ptr[dev];
        return IPR_OK;
    }
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_gemv_scratch);
    if (e != cudaSuccess) return noalloc_fail(IPR_E_CUDA, "cudaGetSymbolAddress failed", e);
    uint64_t br[2];
    uint32_t q0inv;
    ipr::host_moduli_constants(br, &q0inv);
    e = ipr::set_constants(br, q0inv);
    if (e != cudaSuccess) return noalloc_fail(IPR_E_CUDA, "loading constants failed", e);
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return noalloc_fail(IPR_E_CUDA, "device query failed", e);
    g_sm_count[dev] = sms;
    g_scratch_ptr[dev] = static_cast<uint64_t*>(p);
    *out = g_scratch_ptr[dev];
    return IPR_OK;
}

}  // namespace

extern "C" int ipr_gemv_query_noalloc(uint64_t* h_c, const uint64_t* h_a, const uint16_t* d_db, int db_rows,
                                      int b_cols) {
    if (!h_c || !h_a || !d_db) return noalloc_fail(IPR_E_ARGS, "null pointer argument");
    if (db_rows < 256 || (db_rows & 255) || (uint64_t)db_rows > kMaxRows)
        return noalloc_fail(IPR_E_ARGS, "db_rows must be a multiple of 256 in [256, 65536]");
    if (b_cols < 16 || (b_cols & 15) || (uint64_t)b_cols > kMaxCols)
        return noalloc_fail(IPR_E_ARGS, "b_cols must be a multiple of 16 in [16, 1048576]");
    // the kernel's 64-bit partial sums stay exact only for reduced residues (at 65,536 rows a
    // full 32-bit limb could wrap them), so an unreduced query row is refused
    for (int k = 0; k < db_rows; k++)
        if ((uint32_t)h_a[k] >= ipr::Q0 || (uint32_t)(h_a[k] >> 32) >= ipr::Q1)
            return noalloc_fail(IPR_E_ARGS, "query row entry not reduced (need lo32 < q0 and hi32 < q1)");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return noalloc_fail(IPR_E_CUDA, "no current device", e);
    if (dev >= kMaxDevices) return noalloc_fail(IPR_E_ARGS, "device ordinal above 63");
    uint64_t* scratch = nullptr;
    int st = setup_device(dev, &scratch);
    if (st) return st;
    uint64_t* d_a = scratch;
    uint64_t* d_c = scratch + kMaxRows;
    cudaStream_t s = cudaStreamPerThread;
    if ((e = cudaMemcpyAsync(d_a, h_a, (size_t)db_rows * 8, cudaMemcpyHostToDevice, s)) != cudaSuccess)
        return noalloc_fail(IPR_E_CUDA, "query copy failed", e);
    // the condensed query row (lo32 = mod q0, hi32 = mod q1) is the one-query operand layout
    if ((e = ipr::launch_gemv(d_db, db_rows, b_cols, 1, reinterpret_cast<const uint32_t*>(d_a), d_c,
                              g_sm_count[dev], s)) != cudaSuccess)
        return noalloc_fail(IPR_E_CUDA, "kernel launch failed", e);
    if ((e = cudaMemcpyAsync(h_c, d_c, (size_t)b_cols * 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
        return noalloc_fail(IPR_E_CUDA, "result copy failed", e);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return noalloc_fail(IPR_E_CUDA, "synchronize failed", e);
    return IPR_OK;
}
