// fold.cu — RGSW interpolation fold + modulus switch with register-resident NTTs.
//
// Restates the fold closure of KeywordServer::respond (rkdud007/inspire-rs,
// src/pir/server/keyword.rs:543-581): per (query, fold group wp)
//   s = 0; for i = interp-1 .. 0:  s = from_ntt(CT * to_ntt(G^-1(s))) + packed[wp*interp + i]  (mod q)
// then switch_and_keep (src/pir/modulus_switch.rs:45-73).
//
// One CTA of 512 threads per chain, two groups of 256 threads, group l owning
// CRT limb l.  A limb-NTT of 2048 points runs in registers, 8 elements per
// thread, with the Harvey butterflies of ntt_forward / ntt_inverse
// (src/core/ntt.rs:111-160, 731-780):
//   layout A: thread t holds e = t + 256 m          (stages with distance 1024, 512, 256)
//   layout B: thread t holds e = (t/32)*256 + t%32 + 32 m  (distances 128, 64, 32)
//   distances 16 .. 1 pair lanes of one warp in layout B: warp shuffles.
// A forward NTT goes A -> B with one shared-memory exchange; an inverse NTT
// goes B -> A.  Per fold step each group runs the 6 forward NTTs of the gadget
// digits of its limb, accumulates both rows of the 2x6 product in registers,
// and the 2 inverse NTTs; the two limbs meet only at the CRT compose.
#include <cuda_runtime.h>

#include <cstdint>

#include "ipr_device.cuh"
#include "kernels.cuh"

namespace ipr {

namespace {

constexpr int F_THREADS = 512;
constexpr int GT = 256;  // threads per limb group
constexpr int EPT = 8;   // elements per thread

__device__ __forceinline__ int eA(int t, int m) { return t + 256 * m; }
__device__ __forceinline__ int eB(int t, int m) { return (t >> 5) * 256 + (t & 31) + 32 * m; }

__device__ __forceinline__ void group_bar(int g) { asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(GT) : "memory"); }

// forward Harvey butterfly on a register pair: x in [0,4q), y in [0,4q) -> outputs in [0,4q)
__device__ __forceinline__ void fwd_bfly(uint32_t& x, uint32_t& y, uint32_t w, uint32_t wp, uint32_t q) {
    const uint32_t two_q = 2 * q;
    uint32_t xx = x >= two_q ? x - two_q : x;
    uint32_t qn = shoup_lazy(y, w, wp, q);
    x = xx + qn;
    y = xx + two_q - qn;
}

// inverse Gentleman-Sande butterfly with halving: x, y in [0,2q) -> outputs in [0,2q)
__device__ __forceinline__ void inv_bfly(uint32_t& x, uint32_t& y, uint32_t w, uint32_t wp, uint32_t q) {
    const uint32_t two_q = 2 * q;
    uint32_t tt = two_q - y + x;
    uint32_t cx = x + y - ((2 * x >= tt) ? two_q : 0);
    x = (cx + ((tt & 1) ? q : 0)) >> 1;
    y = w * tt - __umulhi(tt, wp) * q;
}

__device__ __forceinline__ uint32_t canon(uint32_t v, uint32_t q) {
    v = v >= 2 * q ? v - 2 * q : v;
    return v >= q ? v - q : v;
}

// forward NTT of one limb: v[] in layout A on entry, layout B (canonical) on exit
__device__ __forceinline__ void ntt_fwd_group(uint32_t (&v)[EPT], int t, int g, uint32_t* xbuf,
                                              const uint32_t* __restrict__ fw, const uint32_t* __restrict__ fwp,
                                              uint32_t q) {
    // distances 1024, 512, 256 (layout A): pair (m, m + d), block index m >> (3 - mm)
#pragma unroll
    for (int mm = 0; mm < 3; mm++) {
        const int d = 4 >> mm;
#pragma unroll
        for (int m = 0; m < EPT; m++) {
            if (m & d) continue;
            const int idx = (1 << mm) + (m >> (3 - mm));
            fwd_bfly(v[m], v[m + d], __ldg(fw + idx), __ldg(fwp + idx), q);
        }
    }
#pragma unroll
    for (int m = 0; m < EPT; m++) xbuf[eA(t, m)] = v[m];
    group_bar(g);
#pragma unroll
    for (int m = 0; m < EPT; m++) v[m] = xbuf[eB(t, m)];
    group_bar(g);
    // distances 128, 64, 32 (layout B): block index (blk << (mm-3)) + (m >> (6-mm))
    const int blk = t >> 5, r = t & 31;
#pragma unroll
    for (int mm = 3; mm < 6; mm++) {
        const int d = 4 >> (mm - 3);
#pragma unroll
        for (int m = 0; m < EPT; m++) {
            if (m & d) continue;
            const int idx = (1 << mm) + (blk << (mm - 3)) + (m >> (6 - mm));
            fwd_bfly(v[m], v[m + d], __ldg(fw + idx), __ldg(fwp + idx), q);
        }
    }
    // distances 16 .. 1 across lanes of the warp
#pragma unroll
    for (int mm = 6; mm < 11; mm++) {
        const int d = 1024 >> mm;
        const bool upper = r & d;
#pragma unroll
        for (int m = 0; m < EPT; m++) {
            const int e = blk * 256 + r + 32 * m;
            const int idx = (1 << mm) + (e >> (11 - mm));
            const uint32_t w = __ldg(fw + idx), wp = __ldg(fwp + idx);
            const uint32_t mine = v[m];
            const uint32_t wy = upper ? shoup_lazy(mine, w, wp, q) : 0u;
            const uint32_t recv = __shfl_xor_sync(0xffffffffu, upper ? wy : mine, d);
            if (!upper) {
                const uint32_t xx = mine >= 2 * q ? mine - 2 * q : mine;
                v[m] = xx + recv;
            } else {
                const uint32_t xx = recv >= 2 * q ? recv - 2 * q : recv;
                v[m] = xx + 2 * q - wy;
            }
        }
    }
#pragma unroll
    for (int m = 0; m < EPT; m++) v[m] = canon(v[m], q);
}

// inverse NTT of one limb: v[] in layout B on entry, layout A (canonical) on exit
__device__ __forceinline__ void ntt_inv_group(uint32_t (&v)[EPT], int t, int g, uint32_t* xbuf,
                                              const uint32_t* __restrict__ iw, const uint32_t* __restrict__ iwp,
                                              uint32_t q) {
    const int blk = t >> 5, r = t & 31;
    // distances 1 .. 16 across lanes
#pragma unroll
    for (int mm = 10; mm >= 6; mm--) {
        const int d = 1024 >> mm;
        const bool upper = r & d;
#pragma unroll
        for (int m = 0; m < EPT; m++) {
            const int e = blk * 256 + r + 32 * m;
            const int idx = (1 << mm) + (e >> (11 - mm));
            const uint32_t w = __ldg(iw + idx), wp = __ldg(iwp + idx);
            const uint32_t mine = v[m];
            const uint32_t other = __shfl_xor_sync(0xffffffffu, mine, d);
            uint32_t x = upper ? other : mine, y = upper ? mine : other;
            inv_bfly(x, y, w, wp, q);
            v[m] = upper ? y : x;
        }
    }
    // distances 32, 64, 128 (layout B)
#pragma unroll
    for (int mm = 5; mm >= 3; mm--) {
        const int d = 4 >> (mm - 3);
#pragma unroll
        for (int m = 0; m < EPT; m++) {
            if (m & d) continue;
            const int idx = (1 << mm) + (blk << (mm - 3)) + (m >> (6 - mm));
            inv_bfly(v[m], v[m + d], __ldg(iw + idx), __ldg(iwp + idx), q);
        }
    }
#pragma unroll
    for (int m = 0; m < EPT; m++) xbuf[eB(t, m)] = v[m];
    group_bar(g);
#pragma unroll
    for (int m = 0; m < EPT; m++) v[m] = xbuf[eA(t, m)];
    group_bar(g);
    // distances 256, 512, 1024 (layout A)
#pragma unroll
    for (int mm = 2; mm >= 0; mm--) {
        const int d = 4 >> mm;
#pragma unroll
        for (int m = 0; m < EPT; m++) {
            if (m & d) continue;
            const int idx = (1 << mm) + (m >> (3 - mm));
            inv_bfly(v[m], v[m + d], __ldg(iw + idx), __ldg(iwp + idx), q);
        }
    }
#pragma unroll
    for (int m = 0; m < EPT; m++) v[m] = canon(v[m], q);
}

__device__ __forceinline__ uint64_t rescale_to(uint64_t v, uint64_t out_mod) {
    // rescale (src/core/arith.rs:436-452) of a canonical v in [0, q)
    const uint64_t half = QQ / 2;
    const bool neg = v >= half;
    const uint64_t u = neg ? QQ - v : v;
    const unsigned __int128 num = (unsigned __int128)u * out_mod + half;
    const uint64_t rr = (uint64_t)(num / QQ);
    const uint64_t rm = rr % out_mod;
    return neg ? (rm ? out_mod - rm : 0) : rm;
}

}  // namespace

// chains: blockIdx.x = fold group wp, blockIdx.y = query qg (global over the batch).
// Query qg belongs to payload qg / qpp; R and the response layout are per payload.
__global__ void __launch_bounds__(F_THREADS, 1)
    k_fold2(const uint32_t* __restrict__ row0, const uint32_t* __restrict__ gsw, const uint64_t* __restrict__ a_hat,
            const uint64_t* __restrict__ R, int64_t r_payload_stride, const uint64_t* __restrict__ cvec,
            const uint32_t* __restrict__ fw, const uint32_t* __restrict__ fwp, const uint32_t* __restrict__ iw,
            const uint32_t* __restrict__ iwp, int interp, int64_t db_cols, int qpp, uint8_t* __restrict__ resp,
            int64_t resp_payload_stride, int64_t resp_query_stride) {
    extern __shared__ uint64_t fold_smem[];
    uint64_t(*sum)[N] = reinterpret_cast<uint64_t(*)[N]>(fold_smem);                   // [2 rows][N]
    uint32_t(*xbuf)[N] = reinterpret_cast<uint32_t(*)[N]>(fold_smem + 2 * N);          // [2 limbs][N]
    uint32_t(*lbuf)[2][N] = reinterpret_cast<uint32_t(*)[2][N]>(fold_smem + 3 * N);    // [limb][row][slot]
    const int wp = blockIdx.x, qg = blockIdx.y;
    const int payload = qg / qpp, qin = qg % qpp;
    const uint64_t* Rp = R + (int64_t)payload * r_payload_stride;
    const uint32_t* body = gsw + (int64_t)qg * 12 * N;  // [6][2][N]
    const uint64_t* cq = cvec + (int64_t)qg * db_cols;
    const int g = threadIdx.x >> 8, t = threadIdx.x & 255;
    const uint32_t q = g ? Q1 : Q0;
    const uint64_t br = g ? BR1 : BR0;
    const uint32_t* fwl = fw + g * N;
    const uint32_t* fwpl = fwp + g * N;
    const uint32_t* iwl = iw + g * N;
    const uint32_t* iwpl = iwp + g * N;
    const uint64_t mask = (1ull << GADGET_BITS) - 1;

    // first step: s = 0, the product vanishes -> s = packed[interp-1] mod q
    {
        const int j = wp * interp + interp - 1;
        for (int i = threadIdx.x; i < 2 * N; i += F_THREADS) {
            const int rr = i >> 11, e = i & (N - 1);
            const uint64_t pk = rr == 0 ? a_hat[(int64_t)j * N + e] : cq[(int64_t)j * N + e] + Rp[(int64_t)j * N + e];
            sum[rr][e] = pk % QQ;
        }
        __syncthreads();
    }
    for (int step = interp - 2; step >= 0; step--) {
        const int j = wp * interp + step;
        uint32_t acc0[EPT];
        uint64_t acc1[EPT];
#pragma unroll
        for (int m = 0; m < EPT; m++) {
            acc0[m] = 0;
            acc1[m] = 0;
        }
#pragma unroll 1
        for (int p = 0; p < 6; p++) {  // gadget row p = r + 2k holds digit k of row r
            const int rr = p & 1, k = p >> 1;
            uint32_t v[EPT];
#pragma unroll
            for (int m = 0; m < EPT; m++) v[m] = (uint32_t)((sum[rr][eA(t, m)] >> (k * GADGET_BITS)) & mask);
            ntt_fwd_group(v, t, g, xbuf[g], fwl, fwpl, q);
            const uint32_t* bp = body + (p * 2 + g) * N;
#pragma unroll
            for (int m = 0; m < EPT; m++) {
                acc0[m] += v[m];  // < 6q
                acc1[m] += (uint64_t)__ldg(bp + eB(t, m)) * v[m];  // 6 terms < 2^59
            }
        }
        uint32_t p0[EPT], p1[EPT];
#pragma unroll
        for (int m = 0; m < EPT; m++) {
            const uint32_t a0 = mod64(acc0[m], q, br);
            p0[m] = mod64((uint64_t)__ldg(row0 + g * N + eB(t, m)) * a0, q, br);
            p1[m] = mod64(acc1[m], q, br);
        }
        ntt_inv_group(p0, t, g, xbuf[g], iwl, iwpl, q);
        ntt_inv_group(p1, t, g, xbuf[g], iwl, iwpl, q);
#pragma unroll
        for (int m = 0; m < EPT; m++) {
            lbuf[g][0][eA(t, m)] = p0[m];
            lbuf[g][1][eA(t, m)] = p1[m];
        }
        __syncthreads();
        for (int i = threadIdx.x; i < 2 * N; i += F_THREADS) {
            const int rr = i >> 11, e = i & (N - 1);
            uint64_t v = crt2(lbuf[0][rr][e], lbuf[1][rr][e], Q0INV, BR1);
            v += rr == 0 ? a_hat[(int64_t)j * N + e] : cq[(int64_t)j * N + e] + Rp[(int64_t)j * N + e];  // < 3q
            v = v >= QQ ? v - QQ : v;
            v = v >= QQ ? v - QQ : v;
            sum[rr][e] = v;
        }
        __syncthreads();
    }
    // switch_and_keep: row 0 -> 28-bit fields (2 per 7 bytes), row 1 -> 20-bit fields (2 per 5 bytes)
    uint8_t* out = resp + (int64_t)payload * resp_payload_stride + 8 + (int64_t)qin * resp_query_stride +
                   (int64_t)wp * RESULT_BYTES;
    for (int tt = threadIdx.x; tt < N / 2; tt += F_THREADS) {
        const uint64_t v = rescale_to(sum[0][2 * tt], QP2) | (rescale_to(sum[0][2 * tt + 1], QP2) << 28);
#pragma unroll
        for (int b = 0; b < 7; b++) out[7 * tt + b] = (uint8_t)(v >> (8 * b));
        const uint64_t w = rescale_to(sum[1][2 * tt], QP1) | (rescale_to(sum[1][2 * tt + 1], QP1) << 20);
#pragma unroll
        for (int b = 0; b < 5; b++) out[7 * N / 2 + 5 * tt + b] = (uint8_t)(w >> (8 * b));
    }
}

constexpr int FOLD2_SMEM = 2 * N * 8 + 2 * N * 4 + 4 * N * 4;  // 80 KB

cudaError_t init_fold2_kernel() {
    return cudaFuncSetAttribute(k_fold2, cudaFuncAttributeMaxDynamicSharedMemorySize, FOLD2_SMEM);
}

cudaError_t launch_fold2(const uint32_t* row0, const uint32_t* gsw, const uint64_t* a_hat, const uint64_t* R,
                         int64_t r_payload_stride, const uint64_t* cvec, const uint32_t* fw, const uint32_t* fwp,
                         const uint32_t* iw, const uint32_t* iwp, int interp, int c_groups, int num_queries,
                         int64_t db_cols, int qpp, uint8_t* resp, int64_t resp_payload_stride,
                         int64_t resp_query_stride, cudaStream_t st) {
    if (interp < 1 || c_groups < 1 || num_queries < 1 || num_queries > 65535 || qpp < 1) return cudaErrorInvalidValue;
    dim3 grid(c_groups, num_queries);
    k_fold2<<<grid, F_THREADS, FOLD2_SMEM, st>>>(row0, gsw, a_hat, R, r_payload_stride, cvec, fw, fwp, iw, iwp, interp,
                                        db_cols, qpp, resp, resp_payload_stride, resp_query_stride);
    return cudaGetLastError();
}

}  // namespace ipr
