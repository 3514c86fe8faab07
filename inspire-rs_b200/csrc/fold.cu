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
// inverse NTTs together; the two limbs meet only at the CRT compose.  The
// query's RGSW bodies sit in shared memory for the whole chain, and each
// step's packed operands are copied in asynchronously while its transforms run.
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
constexpr int XB = 3;  // polynomials per exchange buffer (the 6 forward transforms pass in two halves)

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(smem)),
                 "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

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
    uint64_t(*sum)[N] = reinterpret_cast<uint64_t(*)[N]>(fold_smem);             // [2 rows][N]
    uint64_t(*pk)[N] = reinterpret_cast<uint64_t(*)[N]>(fold_smem + 2 * N);      // a_hat, c, R rows of step j
    uint32_t* sbody = reinterpret_cast<uint32_t*>(fold_smem + 5 * N);            // [6][2][N] RGSW bodies
    uint32_t* xbase = reinterpret_cast<uint32_t*>(fold_smem + 11 * N);           // [2 limbs][XB][N]
    const int wp = blockIdx.x, qg = blockIdx.y;
    const int payload = qg / qpp, qin = qg % qpp;
    const uint64_t* Rp = R + (int64_t)payload * r_payload_stride;
    const uint64_t* cq = cvec + (int64_t)qg * db_cols;
    const int g = threadIdx.x >> 8, t = threadIdx.x & 255;
    const int bar = 1 + g;
    const uint32_t q = g ? Q1 : Q0;
    const uint64_t br = g ? BR1 : BR0;
    uint32_t* xbuf = xbase + g * XB * N;
    // after the inverse transforms a group's exchange buffer holds its limb of both rows
    const uint32_t* lb0 = xbase;
    const uint32_t* lb1 = xbase + XB * N;
    const uint32_t* fwl = fw + g * N;
    const uint32_t* fwpl = fwp + g * N;
    const uint32_t* iwl = iw + g * N;
    const uint32_t* iwpl = iwp + g * N;
    const uint64_t mask = (1ull << GADGET_BITS) - 1;

    // the rows of packed[j] (a_hat[j]; c[j], R[j] of this query / payload) land in pk while the
    // step's transforms run: 3 x 16 KB in 16-byte asynchronous copies
    auto fetch_packed = [&](int j) {
        for (int i = threadIdx.x; i < 3 * N / 2; i += F_THREADS) {
            const int r = i / (N / 2), o = (i % (N / 2)) * 2;
            const uint64_t* src = r == 0 ? a_hat : (r == 1 ? cq : Rp);
            cp_async16(&pk[r][o], src + (int64_t)j * N + o);
        }
        cp_async_commit();
    };

    // the query's six RGSW bodies stay in shared memory for the whole chain
    {
        const uint32_t* gb = gsw + (int64_t)qg * 12 * N;
        for (int i = threadIdx.x; i < 12 * N / 4; i += F_THREADS) cp_async16(sbody + 4 * i, gb + 4 * i);
    }
    // first step: s = 0, the product vanishes -> s = packed[interp-1] mod q
    fetch_packed(wp * interp + interp - 1);
    cp_async_wait_all();
    __syncthreads();
    for (int i = threadIdx.x; i < 2 * N; i += F_THREADS) {
        const int rr = i >> 11, e = i & (N - 1);
        sum[rr][e] = (rr == 0 ? pk[0][e] : pk[1][e] + pk[2][e]) % QQ;
    }
    __syncthreads();
    for (int step = interp - 2; step >= 0; step--) {
        fetch_packed(wp * interp + step);
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
            nttr::forward<FP, XB, true>(v, t, xbuf, bar, fwl, fwpl, q);  // outputs in [0, 2q)
#pragma unroll
            for (int pp = 0; pp < FP; pp++) {
                const uint4* bp = reinterpret_cast<const uint4*>(sbody + ((pb + pp) * 2 + g) * N + eD(t, 0));
                const uint4 b0 = bp[0], b1 = bp[1];
                const uint32_t bv[EPT] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
                for (int m = 0; m < EPT; m++) {
                    acc0[m] += v[pp][m];                         // 6 terms < 12q < 2^32
                    acc1[m] += (uint64_t)bv[m] * v[pp][m];       // 6 terms < 2q * q < 2^61
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
        nttr::inverse<2, XB>(pr, t, xbuf, bar, iwl, iwpl, q);
#pragma unroll
        for (int m = 0; m < EPT; m++) {
            xbuf[eA(t, m)] = pr[0][m];
            xbuf[N + eA(t, m)] = pr[1][m];
        }
        cp_async_wait_all();
        __syncthreads();
        for (int i = threadIdx.x; i < 2 * N; i += F_THREADS) {
            const int rr = i >> 11, e = i & (N - 1);
            uint64_t v = crt2(lb0[rr * N + e], lb1[rr * N + e], Q0INV, BR1);
            v += rr == 0 ? pk[0][e] : pk[1][e] + pk[2][e];  // < 3q
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

// sum 32 KB + packed rows 48 KB + RGSW bodies 96 KB + exchange buffers 2 x 3 x 8 KB = 224 KB
constexpr int FOLD2_SMEM = (2 + 3 + 6 + 3) * N * 8;

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
