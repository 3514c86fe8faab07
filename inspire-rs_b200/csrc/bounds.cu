// bounds.cu — host side of the bounds-checked debug build (bounds.cuh): the allocation-range
// check of launch arguments, the registry of the translation units' device flags and the
// C-ABI report.  In the release build the C-ABI functions remain and report nothing.
#include <cuda.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "bounds.cuh"
#include "ipr_b200.h"

namespace ipr {

std::atomic<int64_t> g_fold_extent_cut{0};

#ifdef IPR_BOUNDS_CHECK
namespace {
std::mutex g_bounds_mu;
std::string g_host_failures;  // one line per failed range check since the last report
int g_host_count = 0;

std::vector<BoundsTake>& registry() {
    static std::vector<BoundsTake> r;
    return r;
}

using GetRangeFn = CUresult (*)(CUdeviceptr*, size_t*, CUdeviceptr);
GetRangeFn g_get_range = nullptr;
}  // namespace

void bounds_register(BoundsTake fn) {
    std::lock_guard<std::mutex> lk(g_bounds_mu);
    registry().push_back(fn);
}

cudaError_t check_extent(const void* p, uint64_t bytes, const char* what) {
    if (bytes == 0) return cudaSuccess;
    if (!g_get_range) {
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuMemGetAddressRange", (void**)&g_get_range, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !g_get_range) {
            g_get_range = nullptr;
            return cudaErrorNotSupported;
        }
    }
    CUdeviceptr base = 0;
    size_t size = 0;
    const CUdeviceptr a = (CUdeviceptr)(uintptr_t)p;
    const bool ok = p && g_get_range(&base, &size, a) == CUDA_SUCCESS && a + bytes <= base + size;
    if (ok) return cudaSuccess;
    char line[256];
    std::snprintf(line, sizeof line, "%s: needs %llu bytes at %p, the allocation holds %llu from %p\n", what,
                  (unsigned long long)bytes, p, (unsigned long long)size, (void*)(uintptr_t)base);
    std::lock_guard<std::mutex> lk(g_bounds_mu);
    if (g_host_count++ < 16) g_host_failures += line;
    return cudaErrorInvalidValue;
}
#endif

}  // namespace ipr

extern "C" {

int ipr_bounds_checked_build(void) { return ipr::kBoundsChecked ? 1 : 0; }

int ipr_debug_check_extent(const void* d_ptr, uint64_t bytes) {
#ifdef IPR_BOUNDS_CHECK
    const cudaError_t e = ipr::check_extent(d_ptr, bytes, "ipr_debug_check_extent");
    return e == cudaSuccess ? IPR_OK : e == cudaErrorInvalidValue ? IPR_E_ARGS : IPR_E_CUDA;
#else
    (void)d_ptr;
    (void)bytes;
    return IPR_E_STATE;
#endif
}

int ipr_debug_cut_fold_extent(int64_t words) {
    if (words < 0) return IPR_E_ARGS;
#ifdef IPR_BOUNDS_CHECK
    ipr::g_fold_extent_cut.store(words);
    return IPR_OK;
#else
    return IPR_E_STATE;
#endif
}

int ipr_bounds_report(char* out, size_t cap) {
    if (out && cap) out[0] = 0;
#ifdef IPR_BOUNDS_CHECK
    std::string txt;
    int failures = 0;
    if (cudaDeviceSynchronize() == cudaSuccess) {  // kernels still running may yet record
        std::vector<ipr::BoundsTake> regs;
        {
            std::lock_guard<std::mutex> lk(ipr::g_bounds_mu);
            regs = ipr::registry();
        }
        for (ipr::BoundsTake take : regs) {
            const int site = take();
            if (site != 0) {
                failures++;
                txt += "device check failed at site " + std::to_string(site) + "\n";
            }
        }
    } else {
        failures++;
        txt += "device synchronisation failed before reading the device flags\n";
    }
    {
        std::lock_guard<std::mutex> lk(ipr::g_bounds_mu);
        failures += ipr::g_host_count;
        txt += ipr::g_host_failures;
        ipr::g_host_failures.clear();
        ipr::g_host_count = 0;
    }
    if (out && cap) {
        const size_t n = txt.size() < cap - 1 ? txt.size() : cap - 1;
        std::memcpy(out, txt.data(), n);
        out[n] = 0;
    }
    return failures;
#else
    return 0;
#endif
}

}  // extern "C"
