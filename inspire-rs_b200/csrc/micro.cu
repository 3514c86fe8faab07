// micro.cu — kernel-level entry points over device buffers: batched negacyclic
// NTT / INTT of one CRT limb and batched NTT-domain Galois automorphisms.
//
// These are the building blocks respond() uses internally (ntt_forward /
// ntt_inverse, src/core/ntt.rs:111-160, 731-780 of rkdud007/inspire-rs; the
// rotation gather of native/cuda/rotation_kernel.cu:21-59 in the closed form
// of generate_automorph_tables_brute_force, src/pir/packing.rs:1423-1468),
// exposed on their own so they can be checked and timed in isolation.
// Polynomials are 2048 u64 coefficients (one limb, canonical residues), the
// reference's per-limb storage.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>
#include <vector>

#include "host_math.hpp"
#include "ipr_b200.h"
#include "ipr_device.cuh"
#include "ntt_regs.cuh"
#include "umma.cuh"

namespace ipr {
void set_last_error(const char* msg);

namespace {

constexpr int M_POLYS = 4;  // polynomials per 256-thread CTA (one twiddle load feeds 4 butterflies)

// One CTA of 256 threads per M_POLYS polynomials.  Global memory is read and written in
// natural order (coalesced 8-byte accesses); the register layouts the transforms start
// from and end in are reached through shared memory.
template <bool INVERSE>
__global__ void __launch_bounds__(256) k_ntt_limb(uint64_t* __restrict__ polys, int64_t count, uint32_t q,
                                                  const uint32_t* __restrict__ w, const uint32_t* __restrict__ wp) {
    __shared__ uint32_t xbuf[M_POLYS * N];
    const int t = threadIdx.x;
    const int64_t p0 = (int64_t)blockIdx.x * M_POLYS;
    uint32_t v[M_POLYS][nttr::EPT];
#pragma unroll
    for (int p = 0; p < M_POLYS; p++) {
        const bool live = p0 + p < count;
        const uint64_t* src = polys + (p0 + p) * N;
#pragma unroll
        for (int m = 0; m < nttr::EPT; m++) {
            const uint32_t x = live ? (uint32_t)src[nttr::eA(t, m)] : 0u;
            if (INVERSE) xbuf[p * N + nttr::eA(t, m)] = x;  // to layout D below
            else v[p][m] = x;
        }
    }
    if (INVERSE) {
        __syncthreads();
#pragma unroll
        for (int p = 0; p < M_POLYS; p++)
#pragma unroll
            for (int m = 0; m < nttr::EPT; m++) v[p][m] = xbuf[p * N + nttr::eD(t, m)];
        __syncthreads();
        nttr::inverse<M_POLYS>(v, t, xbuf, 1, w, wp, q);  // ends in layout A
    } else {
        nttr::forward<M_POLYS>(v, t, xbuf, 1, w, wp, q);  // ends in layout D
        __syncthreads();
#pragma unroll
        for (int p = 0; p < M_POLYS; p++)
#pragma unroll
            for (int m = 0; m < nttr::EPT; m++) xbuf[p * N + nttr::eD(t, m)] = v[p][m];
        __syncthreads();
#pragma unroll
        for (int p = 0; p < M_POLYS; p++)
#pragma unroll
            for (int m = 0; m < nttr::EPT; m++) v[p][m] = xbuf[p * N + nttr::eA(t, m)];
    }
#pragma unroll
    for (int p = 0; p < M_POLYS; p++) {
        if (p0 + p >= count) break;
        uint64_t* dst = polys + (p0 + p) * N;
#pragma unroll
        for (int m = 0; m < nttr::EPT; m++) dst[nttr::eA(t, m)] = v[p][m];
    }
}

// out[j][p][s] = in[p][auto_src(ks[j], s)]: one CTA stages one input polynomial in shared
// memory and writes its image under every requested automorphism
__global__ void __launch_bounds__(256) k_automorph(const uint64_t* __restrict__ in, int64_t count,
                                                   const uint32_t* __restrict__ ks, int nk,
                                                   uint64_t* __restrict__ out) {
    __shared__ uint64_t poly[N];
    for (int64_t p = blockIdx.x; p < count; p += gridDim.x) {
        __syncthreads();
        for (int s = threadIdx.x; s < N; s += blockDim.x) poly[s] = in[p * N + s];
        __syncthreads();
        for (int j = 0; j < nk; j++) {
            const uint32_t k = __ldg(ks + j);
            uint64_t* o = out + ((int64_t)j * count + p) * N;
            for (int s = threadIdx.x; s < N; s += blockDim.x) o[s] = poly[auto_src(k, (uint32_t)s)];
        }
    }
}

// The bounded wait the tensor-core kernels use on their mbarriers (umma::mbar_wait), on a
// barrier nothing arrives on: the wait gives up after `limit_ns` of global time and the kernel
// reports it instead of hanging, as the GEMM kernels do through their error flags.
__global__ void k_wait_selftest(uint64_t limit_ns, int* out) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        umma::mbar_init(&bar, 1);
        umma::fence_mbar_init();
    }
    __syncthreads();
    const bool done = umma::mbar_wait(&bar, 0, limit_ns);  // phase 0 never completes
    if (threadIdx.x == 0) *out = done ? 1 : 0;
}

// per-device NTT tables (fw, fwp, iw, iwp: [4][2 limbs][N] u32), built on first use
std::mutex g_mu;
std::vector<uint32_t*> g_tables;

int tables_for(int device, const uint32_t** out) {
    std::lock_guard<std::mutex> lk(g_mu);
    if ((int)g_tables.size() <= device) g_tables.resize(device + 1, nullptr);
    uint32_t*& d = g_tables[device];
    if (!d) {
        HostParams hp;
        host_params_init(hp);
        std::vector<uint32_t> h(8 * N);
        std::copy(hp.fw.begin(), hp.fw.end(), h.begin());
        std::copy(hp.fwp.begin(), hp.fwp.end(), h.begin() + 2 * N);
        std::copy(hp.iw.begin(), hp.iw.end(), h.begin() + 4 * N);
        std::copy(hp.iwp.begin(), hp.iwp.end(), h.begin() + 6 * N);
        cudaError_t e = cudaMalloc(&d, h.size() * sizeof(uint32_t));
        if (e == cudaSuccess) e = cudaMemcpy(d, h.data(), h.size() * sizeof(uint32_t), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            if (d) cudaFree(d);
            d = nullptr;
            set_last_error(cudaGetErrorString(e));
            return e == cudaErrorMemoryAllocation ? IPR_E_OOM : IPR_E_CUDA;
        }
    }
    *out = d;
    return IPR_OK;
}

int cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return IPR_OK;
    set_last_error(cudaGetErrorString(e));
    return IPR_E_CUDA;
}

}  // namespace
}  // namespace ipr

extern "C" {

int ipr_ntt_batch(int device, uint64_t* d_polys, uint64_t count, int limb, int inverse, void* stream) {
    if (!d_polys || (limb != 0 && limb != 1) || count > (1ull << 36)) {
        ipr::set_last_error("ipr_ntt_batch: bad argument (null buffer, limb not 0/1, or too many polynomials)");
        return IPR_E_ARGS;
    }
    if (count == 0) return IPR_OK;
    int st = ipr::cuda_status(cudaSetDevice(device));
    if (st) return st;
    const uint32_t* tb;
    if ((st = ipr::tables_for(device, &tb))) return st;
    const int n = ipr::N;
    const uint32_t q = limb ? ipr::Q1 : ipr::Q0;
    const uint32_t* w = tb + (inverse ? 4 * n : 0) + limb * n;
    const uint32_t* wp = tb + (inverse ? 6 * n : 2 * n) + limb * n;
    const unsigned blocks = (unsigned)((count + ipr::M_POLYS - 1) / ipr::M_POLYS);
    auto cs = static_cast<cudaStream_t>(stream);
    if (inverse) ipr::k_ntt_limb<true><<<blocks, 256, 0, cs>>>(d_polys, (int64_t)count, q, w, wp);
    else ipr::k_ntt_limb<false><<<blocks, 256, 0, cs>>>(d_polys, (int64_t)count, q, w, wp);
    return ipr::cuda_status(cudaGetLastError());
}

int ipr_automorph_batch(int device, const uint64_t* d_in, uint64_t count, const uint32_t* d_ks, int nk,
                        uint64_t* d_out, void* stream) {
    if (!d_in || !d_out || !d_ks || nk < 0 || count > (1ull << 36)) {
        ipr::set_last_error("ipr_automorph_batch: bad argument");
        return IPR_E_ARGS;
    }
    if (count == 0 || nk == 0) return IPR_OK;
    int st = ipr::cuda_status(cudaSetDevice(device));
    if (st) return st;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int64_t grid = std::min<int64_t>((int64_t)count, (int64_t)sms * 8);
    ipr::k_automorph<<<(unsigned)grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(d_in, (int64_t)count, d_ks, nk,
                                                                                   d_out);
    return ipr::cuda_status(cudaGetLastError());
}

int ipr_device_binary_version(int device, int* binary_version) {
    if (!binary_version) return IPR_E_ARGS;
    int st = ipr::cuda_status(cudaSetDevice(device));
    if (st) return st;
    cudaFuncAttributes a{};
    st = ipr::cuda_status(cudaFuncGetAttributes(&a, ipr::k_wait_selftest));
    if (st) return st;
    *binary_version = a.binaryVersion;
    return IPR_OK;
}

int ipr_selftest_bounded_wait(int device, uint32_t limit_us) {
    if (limit_us == 0 || limit_us > 1000000u) {
        ipr::set_last_error("ipr_selftest_bounded_wait: limit_us must be in [1, 1000000]");
        return IPR_E_ARGS;
    }
    int st = ipr::cuda_status(cudaSetDevice(device));
    if (st) return st;
    int* d = nullptr;
    int h = -1;
    cudaError_t e = cudaMalloc(&d, sizeof(int));
    if (e == cudaSuccess) {
        ipr::k_wait_selftest<<<1, 32>>>((uint64_t)limit_us * 1000u, d);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpy(&h, d, sizeof(int), cudaMemcpyDeviceToHost);
        cudaFree(d);
    }
    if (e != cudaSuccess) return ipr::cuda_status(e);
    if (h == 0) {
        ipr::set_last_error("bounded wait ran out (self-test: nothing arrives on the barrier)");
        return IPR_E_TIMEOUT;
    }
    ipr::set_last_error("bounded wait self-test: the barrier completed unexpectedly");
    return IPR_E_STATE;
}

}  // extern "C"
