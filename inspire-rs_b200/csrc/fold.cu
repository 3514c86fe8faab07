// fold.cu — RGSW interpolation fold + modulus switch with register-resident NTTs.
//
// Restates the fold closure of KeywordServer::respond (rkdud007/inspire-rs,
// src/pir/server/keyword.rs:543-581): per (query, fold group wp)
//   s = 0; for i = interp-1 .. 0:  s = from_ntt(CT * to_ntt(G^-1(s))) + packed[wp*interp + i]  (mod q)
// then switch_and_keep (src/pir/modulus_switch.rs:45-73).
//
// One CTA of 512 threads per chain, two groups of 256 threads, group l owning
// CRT limb l.  Limb NTTs run in registers (ntt_regs.cuh).  Per fold step each
// group transforms the 6 gadget-digit polynomials of its limb together (one
// twiddle load per 6 butterflies, one exchange barrier pair for all six),
// accumulates both rows of the 2x6 product in registers, and runs the 2
// inverse NTTs together; the two limbs meet only at the CRT compose.
#include <cuda_runtime.h>

#include <cstdint>

#include "ipr_device.cuh"
#include "kernels.cuh"
#include "ntt_regs.cuh"

namespace ipr {

namespace {

constexpr int F_THREADS = 512;
constexpr int EPT = nttr::EPT;
#ifndef IPR_FOLD_FWD_BATCH
#define IPR_FOLD_FWD_BATCH 6
#endif
constexpr int FP = IPR_FOLD_FWD_BATCH;  // gadget-digit polynomials transformed together
static_assert(6 % FP == 0, "forward batch must divide the 6 gadget rows");

using nttr::eA;
using nttr::eD;

// the 8 consecutive words of layout D held by thread t (two 16-byte loads)
__device__ __forceinline__ void load_d(uint32_t (&r)[EPT], const uint32_t* __restrict__ poly, int t) {
    const uint4* src = reinterpret_cast<const uint4*>(poly + eD(t, 0));
    const uint4 a = __ldg(src), b = __ldg(src + 1);
    r[0] = a.x; r[1] = a.y; r[2] = a.z; r[3] = a.w;
    r[4] = b.x; r[5] = b.y; r[6] = b.z; r[7] = b.w;
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
    uint64_t(*sum)[N] = reinterpret_cast<uint64_t(*)[N]>(fold_smem);                  // [2 rows][N]
    uint32_t* xbase = reinterpret_cast<uint32_t*>(fold_smem + 2 * N);                 // [2 limbs][FP][N]
    const int wp = blockIdx.x, qg = blockIdx.y;
    const int payload = qg / qpp, qin = qg % qpp;
    const uint64_t* Rp = R + (int64_t)payload * r_payload_stride;
    const uint32_t* body = gsw + (int64_t)qg * 12 * N;  // [6][2][N]
    const uint64_t* cq = cvec + (int64_t)qg * db_cols;
    const int g = threadIdx.x >> 8, t = threadIdx.x & 255;
    const int bar = 1 + g;
    const uint32_t q = g ? Q1 : Q0;
    const uint64_t br = g ? BR1 : BR0;
    uint32_t* xbuf = xbase + g * FP * N;
    // after the inverse transforms a group's exchange buffer holds its limb of both rows
    const uint32_t* lb0 = xbase;
    const uint32_t* lb1 = xbase + FP * N;
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
        for (int pb = 0; pb < 6; pb += FP) {  // gadget row p = r + 2k holds digit k of row r
            uint32_t v[FP][EPT];
#pragma unroll
            for (int pp = 0; pp < FP; pp++) {
                const int p = pb + pp, rr = p & 1, k = p >> 1;
#pragma unroll
                for (int m = 0; m < EPT; m++) v[pp][m] = (uint32_t)((sum[rr][eA(t, m)] >> (k * GADGET_BITS)) & mask);
            }
            nttr::forward<FP>(v, t, xbuf, bar, fwl, fwpl, q);
#pragma unroll
            for (int pp = 0; pp < FP; pp++) {
                uint32_t bv[EPT];
                load_d(bv, body + ((pb + pp) * 2 + g) * N, t);
#pragma unroll
                for (int m = 0; m < EPT; m++) {
                    acc0[m] += v[pp][m];                         // < 6q
                    acc1[m] += (uint64_t)bv[m] * v[pp][m];       // 6 terms < 2^59
                }
            }
        }
        uint32_t pr[2][EPT], r0[EPT];
        load_d(r0, row0 + g * N, t);
#pragma unroll
        for (int m = 0; m < EPT; m++) {
            const uint32_t a0 = mod64(acc0[m], q, br);
            pr[0][m] = mod64((uint64_t)r0[m] * a0, q, br);
            pr[1][m] = mod64(acc1[m], q, br);
        }
        nttr::inverse<2>(pr, t, xbuf, bar, iwl, iwpl, q);
#pragma unroll
        for (int m = 0; m < EPT; m++) {
            xbuf[eA(t, m)] = pr[0][m];
            xbuf[N + eA(t, m)] = pr[1][m];
        }
        __syncthreads();
        for (int i = threadIdx.x; i < 2 * N; i += F_THREADS) {
            const int rr = i >> 11, e = i & (N - 1);
            uint64_t v = crt2(lb0[rr * N + e], lb1[rr * N + e], Q0INV, BR1);
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

constexpr int FOLD2_SMEM = 2 * N * 8 + 2 * FP * N * 4;  // 128 KB at FP = 6

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
