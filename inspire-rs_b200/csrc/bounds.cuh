// bounds.cuh — the bounds-checked debug build of the respond() path.
//
// `make -C inspire-rs_b200 debug` builds libipr_b200_dbg.so from the same sources with
// -DIPR_BOUNDS_CHECK.  That build checks two things that the release build compiles away:
//  1. before every launch of the path, the byte range that each buffer argument will be read
//     or written over, computed from the launch's own parameters, against the device
//     allocation that holds the pointer (cuMemGetAddressRange).  A range outside it fails the
//     launch with cudaErrorInvalidValue and records which buffer it was;
//  2. inside the fold and its scaling pass, every global index against the extent the launch
//     passes.  A failed check skips its access and records its site id in a device flag of
//     the translation unit (the first failure wins); nothing traps or waits, so a failing
//     case leaves the context usable.
// ipr_bounds_report() returns and clears both records.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>

namespace ipr {

#ifdef IPR_BOUNDS_CHECK
constexpr bool kBoundsChecked = true;

// this translation unit's device flag: the site id of the first failed check, 0 if none
static __device__ int g_bounds_site;

__device__ __forceinline__ bool in_bounds(bool ok, int site) {
    if (!ok) atomicCAS(&g_bounds_site, 0, site);
    return ok;
}

// the allocation holding p covers [p, p + bytes); otherwise records `what` and fails
cudaError_t check_extent(const void* p, uint64_t bytes, const char* what);

using BoundsTake = int (*)();  // reads and clears one translation unit's device flag
void bounds_register(BoundsTake fn);

namespace {
int bounds_take_tu() {
    int v = 0, z = 0;
    if (cudaMemcpyFromSymbol(&v, g_bounds_site, sizeof v) != cudaSuccess) return -1;
    cudaMemcpyToSymbol(g_bounds_site, &z, sizeof z);
    return v;
}
const int g_bounds_registered = (bounds_register(&bounds_take_tu), 0);
}  // namespace

#else
constexpr bool kBoundsChecked = false;

__device__ __forceinline__ constexpr bool in_bounds(bool, int) { return true; }
inline cudaError_t check_extent(const void*, uint64_t, const char*) { return cudaSuccess; }
#endif

// words taken off the packing-output extent the fold is told (ipr_debug_cut_fold_extent, debug
// build): the fold's own index checks then trip on real, allocated words, which it skips
extern std::atomic<int64_t> g_fold_extent_cut;

// device check sites (ids reported by ipr_bounds_report)
enum BoundsSite : int {
    kSitePrepZb = 32,
    kSitePrepBth = 33,
    kSiteFoldS = 41,
    kSiteFoldAhat = 42,
    kSiteFoldC = 43,
    kSiteFoldResp = 44,
    kSiteFoldGsw = 45,
};

}  // namespace ipr
