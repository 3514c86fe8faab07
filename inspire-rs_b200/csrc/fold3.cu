// fold3.cu — RGSW interpolation fold with the packing post-process fused in, plus the
// modulus switch, on register-resident NTTs.
//
// Restates, per (query, fold group wp), the fold closure of KeywordServer::respond
// (rkdud007/inspire-rs src/pir/server/keyword.rs:543-581)
//   s = 0; for i = interp-1 .. 0:  s = from_ntt(CT * to_ntt(G^-1(s))) + packed[wp*interp + i]  (mod q)
// followed by switch_and_keep (src/pir/modulus_switch.rs:45-73), where the packed
// ciphertexts are the online-packing post-process (src/pir/gpu/packing_online.rs:359-397):
//   packed[j] = (a_hat[j], from_ntt(S[j]) + c[j*N .. (j+1)*N]).
// from_ntt is linear, so INTT(CT * NTT(G^-1(s)))[row 1] + INTT(S[j]) is one inverse
// transform of the sum: the packing output S[j] joins the fold's own row-1 accumulator
// in the NTT domain and no separate INTT + CRT pass (nor its u64 output array) exists.
//
// Layout of the work: a CTA of 512 threads takes two fold groups (chains) of one query;
// each team of 256 threads runs one chain alone (its own named barrier), both teams
// sharing the query's six RGSW bodies in shared memory.  A thread owns 8 coefficients
// (layout A of ntt_regs.cuh, e = t + 256 m) of both rows of s as u64 values mod q, kept
// in a shared-memory slot only that thread touches, and runs the transforms of both CRT
// limbs itself, so the CRT compose, the packed-row add and the gadget decomposition need
// no exchange between threads.
//
// Arithmetic: the inverse transforms are Gentleman-Sande butterflies with the plain
// inverse twiddles (the reference pre-halves them, ntt.rs:93-96, to fold in N^-1);
// here N^-1 is folded into the operands instead: into row 0 of the RGSW matrix and the
// query's bodies (once per chain) and into S (by k_fold_prep).  Inverse transforms are
// unique, so the canonical outputs equal the reference's.  The forward transforms of the
// gadget digits (< 2^19) skip the conditional subtraction in their first seven stages,
// where the values provably stay below 2^19 + 14q < 16q < 2^32.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "bounds.cuh"
#include "ipr_device.cuh"
#include "kernels.cuh"
#include "ntt_regs.cuh"

namespace ipr {

namespace {

constexpr int F3_TEAM = 256;
constexpr int F3_THREADS = 2 * F3_TEAM;
constexpr int EPT = nttr::EPT;
constexpr int XP = 4;  // polynomials per team exchange buffer

using nttr::csub;
using nttr::eA;
using nttr::eB;
using nttr::eC;
using nttr::eD;

// x < 16q (< 2^32) to [0, 2q) by three conditional subtractions on the ALU pipe: the fold is
// bound by its integer multiplies, so these cost less than a Barrett reduction's two
__device__ __forceinline__ uint32_t red16(uint32_t x, uint32_t q) {
    return csub(csub(csub(x, 8 * q), 4 * q), 2 * q);
}

// forward butterfly by stage: MODE 0 leaves x unreduced (the bound grows by 2q), MODE 1
// first brings x (< 16q) to [0, 2q).  Outputs: x + w*y, x - w*y + 2q, w*y in [0, 2q).
template <int MODE>
__device__ __forceinline__ void fwd_b(uint32_t& x, uint32_t& y, uint32_t w, uint32_t wp, uint32_t q) {
    const uint32_t xx = MODE == 1 ? red16(x, q) : x;
    const uint32_t qn = shoup_lazy(y, w, wp, q);
    x = xx + qn;
    y = xx + 2 * q - qn;
}

// twiddle tables interleaved with their Shoup companions ([limb][N] of (w, wp)): one 8-byte
// load per twiddle, half the L1 requests of two separate tables.  The twiddle of element k of
// a thread is (1 << mm) + (e >> (11 - mm)) with e = hi + k * RS + lo in every layout: hi, the
// thread's part, is a multiple of 2^(11 - mm) at the stages run in that layout, and lo (the
// thread bits below the register stride RS) never carries into the shifted value.  So the
// index is the thread's base plus a compile-time constant, and the elements of one stage that
// share a twiddle share its load.  Layout A: hi = 0, RS = 256; B: hi = 256 w, RS = 32;
// C: hi = 256 w + 32 (l / 4), RS = 4; D: hi = 256 w + 8 l, RS = 1 (w = t / 32, l = t % 32).
template <int RS>
__device__ __forceinline__ int tw_idx(int mm, int hi, int k) {
    return (1 << mm) + (hi >> (11 - mm)) + ((k * RS) >> (11 - mm));
}

template <int P, int MODE, int RS>
__device__ __forceinline__ void fstage(uint32_t (&v)[P][EPT], int mm, int dd, int hi, const uint2* __restrict__ tw,
                                       uint32_t q) {
#pragma unroll
    for (int k = 0; k < EPT; k++) {
        if (k & dd) continue;
        const uint2 w = __ldg(tw + tw_idx<RS>(mm, hi, k));
#pragma unroll
        for (int p = 0; p < P; p++) fwd_b<MODE>(v[p][k], v[p][k + dd], w.x, w.y, q);
    }
}

// Team exchanges through xbuf.  The intra-warp transposes (B <-> C <-> D) use only the warp's
// own 256-word region of each polynomial and synchronise only the warp, so the cross-warp
// exchanges are fenced by where they write: A -> B stores into every warp's region, so a
// team barrier first lets every warp finish with its region; its loads read the warp's own
// region, which nothing else writes before the next such barrier.  B -> A stores into the
// warp's own region (no other warp reads it until the barrier) and loads from all regions,
// which nothing writes before the next A -> B barrier.
template <int P>
__device__ __forceinline__ void xchg_a2b(uint32_t (&v)[P][EPT], int t, uint32_t* xbuf, int bar) {
    nttr::group_bar(bar);
#pragma unroll
    for (int p = 0; p < P; p++)
#pragma unroll
        for (int m = 0; m < EPT; m++) xbuf[p * N + eA(t, m)] = v[p][m];
    nttr::group_bar(bar);
#pragma unroll
    for (int p = 0; p < P; p++)
#pragma unroll
        for (int m = 0; m < EPT; m++) v[p][m] = xbuf[p * N + eB(t, m)];
}

// XB < P: the buffer holds XB polynomials, moved XB at a time; a later chunk's stores wait at
// a team barrier for every warp to finish loading the previous chunk from this warp's region
template <int P, int XB = P>
__device__ __forceinline__ void xchg_b2a(uint32_t (&v)[P][EPT], int t, uint32_t* xbuf, int bar) {
#pragma unroll
    for (int c0 = 0; c0 < P; c0 += XB) {
        if (c0) nttr::group_bar(bar);
#pragma unroll
        for (int p = c0; p < c0 + XB && p < P; p++)
#pragma unroll
            for (int m = 0; m < EPT; m++) xbuf[(p - c0) * N + eB(t, m)] = v[p][m];
        nttr::group_bar(bar);
#pragma unroll
        for (int p = c0; p < c0 + XB && p < P; p++)
#pragma unroll
            for (int m = 0; m < EPT; m++) v[p][m] = xbuf[(p - c0) * N + eA(t, m)];
    }
}

// forward NTT of P gadget-digit polynomials (< 2^19) of one limb: layout A in, layout D out
// in [0, 2q); xbuf holds XP >= P polynomials of this team.  Bounds: after stage s <= 6 every
// value is below 2^19 + 2q (s + 1) <= 2^19 + 14q; stage 7 reduces x first (outputs < 4q);
// stages 8..10 add 2q each (< 10q < 2^32); one reduction at the end.
template <int P>
__device__ __forceinline__ void forward_digits(uint32_t (&v)[P][EPT], int t, uint32_t* xbuf, int bar,
                                               const uint2* __restrict__ tw, uint32_t q) {
    const int l = t & 31, w = t >> 5;
    uint32_t* wb = xbuf + w * 256;
    const int hb = 256 * w, hc = 256 * w + 32 * (l >> 2), hd = 256 * w + 8 * l;
    fstage<P, 0, 256>(v, 0, 4, 0, tw, q);
    fstage<P, 0, 256>(v, 1, 2, 0, tw, q);
    fstage<P, 0, 256>(v, 2, 1, 0, tw, q);
    xchg_a2b<P>(v, t, xbuf, bar);
    fstage<P, 0, 32>(v, 3, 4, hb, tw, q);
    fstage<P, 0, 32>(v, 4, 2, hb, tw, q);
    fstage<P, 0, 32>(v, 5, 1, hb, tw, q);
    nttr::b_to_c<P>(v, l, wb);
    fstage<P, 0, 4>(v, 6, 4, hc, tw, q);
    fstage<P, 1, 4>(v, 7, 2, hc, tw, q);
    fstage<P, 0, 4>(v, 8, 1, hc, tw, q);
    nttr::c_to_d<P>(v, l, wb);
    fstage<P, 0, 1>(v, 9, 2, hd, tw, q);
    fstage<P, 0, 1>(v, 10, 1, hd, tw, q);
#pragma unroll
    for (int p = 0; p < P; p++)
#pragma unroll
        for (int k = 0; k < EPT; k++) v[p][k] = red16(v[p][k], q);
}

// Gentleman-Sande butterfly with a plain inverse twiddle: x + y, (x - y) * w.  Inputs below
// OFF * q; the difference is taken as x + OFF q - y (< 2 OFF q <= 16q < 2^32); the product
// lands in [0, 2q); the sum (< 2 OFF q <= 16q) is reduced to [0, 2q) when RED.
template <int OFF, bool RED>
__device__ __forceinline__ void inv_b(uint32_t& x, uint32_t& y, uint32_t w, uint32_t wp, uint32_t q) {
    const uint32_t s = x + y;
    const uint32_t d = x + OFF * q - y;
    x = RED ? red16(s, q) : s;
    y = shoup_lazy(d, w, wp, q);
}

// one inverse stage over 2 * PL polynomials: [0, PL) of limb 0, [PL, 2 PL) of limb 1
template <int PL, int OFF, bool RED, int RS>
__device__ __forceinline__ void istage(uint32_t (&v)[2 * PL][EPT], int mm, int dd, int hi, const uint2* __restrict__ iw) {
#pragma unroll
    for (int k = 0; k < EPT; k++) {
        if (k & dd) continue;
        const int idx = tw_idx<RS>(mm, hi, k);
        const uint2 w0 = __ldg(iw + idx), w1 = __ldg(iw + N + idx);
#pragma unroll
        for (int p = 0; p < PL; p++) inv_b<OFF, RED>(v[p][k], v[p][k + dd], w0.x, w0.y, Q0);
#pragma unroll
        for (int p = PL; p < 2 * PL; p++) inv_b<OFF, RED>(v[p][k], v[p][k + dd], w1.x, w1.y, Q1);
    }
}

// N * INTT of 2 * PL canonical polynomials (PL per limb): layout D in, layout A canonical out;
// xbuf holds XB polynomials.  Value bounds entering each stage: q, 2q, 4q, 8q (then the sums
// are reduced), 2q, 4q, 8q (reduced), 2q, 4q, 8q (reduced), 2q; below 4q at the end.
template <int PL, int XB = 2 * PL>
__device__ __forceinline__ void inverse_limbs(uint32_t (&v)[2 * PL][EPT], int t, uint32_t* xbuf, int bar,
                                              const uint2* __restrict__ iw) {
    const int l = t & 31, w = t >> 5;
    uint32_t* wb = xbuf + w * 256;
    const int hb = 256 * w, hc = 256 * w + 32 * (l >> 2), hd = 256 * w + 8 * l;
    istage<PL, 1, false, 1>(v, 10, 1, hd, iw);
    istage<PL, 2, false, 1>(v, 9, 2, hd, iw);
    nttr::d_to_c<2 * PL, XB>(v, l, wb);
    istage<PL, 4, false, 4>(v, 8, 1, hc, iw);
    istage<PL, 8, true, 4>(v, 7, 2, hc, iw);
    istage<PL, 2, false, 4>(v, 6, 4, hc, iw);
    nttr::c_to_b<2 * PL, XB>(v, l, wb);
    istage<PL, 4, false, 32>(v, 5, 1, hb, iw);
    istage<PL, 8, true, 32>(v, 4, 2, hb, iw);
    istage<PL, 2, false, 32>(v, 3, 4, hb, iw);
    xchg_b2a<2 * PL, XB>(v, t, xbuf, bar);
    istage<PL, 4, false, 256>(v, 2, 1, 0, iw);
    istage<PL, 8, true, 256>(v, 1, 2, 0, iw);
    istage<PL, 2, false, 256>(v, 0, 4, 0, iw);
#pragma unroll
    for (int p = 0; p < 2 * PL; p++)
#pragma unroll
        for (int k = 0; k < EPT; k++) {
            const uint32_t q = p < PL ? Q0 : Q1;
            v[p][k] = csub(csub(v[p][k], 2 * q), q);
        }
}

// the 8 consecutive words of layout D held by thread t (two 16-byte loads)
__device__ __forceinline__ void load_d8(uint32_t (&r)[EPT], const uint32_t* __restrict__ p) {
    const uint4 a = __ldg(reinterpret_cast<const uint4*>(p)), b = __ldg(reinterpret_cast<const uint4*>(p) + 1);
    r[0] = a.x; r[1] = a.y; r[2] = a.z; r[3] = a.w;
    r[4] = b.x; r[5] = b.y; r[6] = b.z; r[7] = b.w;
}

__device__ __forceinline__ uint32_t mul_canon(uint32_t x, uint32_t w, uint32_t wp, uint32_t q) {
    return csub(shoup_lazy(x, w, wp, q), q);
}

__device__ __forceinline__ uint64_t add_q(uint64_t a, uint64_t b) {  // a, b < q
    const uint64_t v = a + b;
    return v >= QQ ? v - QQ : v;
}

__device__ __forceinline__ uint64_t rescale_q(uint64_t v, uint64_t out_mod) {
    // rescale (src/core/arith.rs:436-452) of a canonical v in [0, q)
    const uint64_t half = QQ / 2;
    const bool neg = v >= half;
    const uint64_t u = neg ? QQ - v : v;
    const unsigned __int128 num = (unsigned __int128)u * out_mod + half;
    const uint64_t rr = (uint64_t)(num / QQ);
    const uint64_t rm = rr % out_mod;
    return neg ? (rm ? out_mod - rm : 0) : rm;
}

// switch_and_keep (src/pir/modulus_switch.rs:45-73) of thread t's coefficients e = t + 256 m of s:
// row 0 -> 28-bit fields (2 per 7 bytes), row 1 -> 20-bit fields (2 per 5 bytes), LSB first;
// coefficient e + 1 sits in the next lane of the same warp
template <typename SA>
__device__ __forceinline__ void switch_keep(SA S_AT, int t, uint8_t* __restrict__ out) {
#pragma unroll
    for (int m = 0; m < EPT; m++) {
        const uint64_t a = rescale_q(S_AT(0, m), QP2), b = rescale_q(S_AT(1, m), QP1);
        const uint64_t an = __shfl_down_sync(0xffffffffu, a, 1), bn = __shfl_down_sync(0xffffffffu, b, 1);
        if (!(t & 1)) {
            const int tt = eA(t, m) >> 1;
            const uint64_t v = a | (an << 28), w = b | (bn << 20);
#pragma unroll
            for (int x = 0; x < 7; x++) out[7 * tt + x] = (uint8_t)(v >> (8 * x));
#pragma unroll
            for (int x = 0; x < 5; x++) out[7 * N / 2 + 5 * tt + x] = (uint8_t)(w >> (8 * x));
        }
    }
}

// 16- and 8-byte asynchronous copies global -> shared (sm_80+ cp.async); a thread waits for
// its own copies with cp_wait
__device__ __forceinline__ void cp16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int PENDING>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(PENDING) : "memory");
}

}  // namespace

// N^-1 mod q_l and its Shoup companion, per limb
struct NInv {
    uint32_t w[2], wp[2];
};

// S[f][l][z] <- (S[f][l][z] + sum_k zb[f / instances][k][z] * That[f % instances][k][z]) * N^-1 mod q_l
// (the z_body x That term of packing_online_kernel.cu:76-83, then the N^-1 the fold's inverse
// transforms leave out); zb null: the scaling alone.  One thread per 4 slots of one output.
__global__ void __launch_bounds__(256) k_fold_prep(uint32_t* __restrict__ S, int64_t count,
                                                   const uint64_t* __restrict__ zb, const uint64_t* __restrict__ bth,
                                                   int instances, NInv ni, uint32_t* __restrict__ gsw,
                                                   int64_t gsw_words, int64_t zb_words, int64_t bth_words, NInv nb) {
    // the queries' RGSW bodies [query][6 gadget rows][2 limbs][N], scaled by N^-1 in place for
    // the fold form that reads them straight from global memory
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < gsw_words / 4;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int lb = (int)((4 * i / N) & 1);
        const uint32_t q = lb ? Q1 : Q0, w = nb.w[lb], wq = nb.wp[lb];
        uint4* g = reinterpret_cast<uint4*>(gsw) + i;
        const uint4 b = *g;
        *g = make_uint4(mul_canon(b.x, w, wq, q), mul_canon(b.y, w, wq, q), mul_canon(b.z, w, wq, q),
                        mul_canon(b.w, w, wq, q));
    }
    const int64_t n4 = count * (N / 4);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n4; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t f = i / (N / 4);
        const int z0 = (int)(i % (N / 4)) * 4;
        uint4* s0 = reinterpret_cast<uint4*>(S + (f * 2) * N + z0);
        uint4* s1 = reinterpret_cast<uint4*>(S + (f * 2 + 1) * N + z0);
        const uint4 a = *s0, b = *s1;
        uint64_t acc0[4] = {a.x, a.y, a.z, a.w}, acc1[4] = {b.x, b.y, b.z, b.w};
        if (zb && in_bounds((f / instances + 1) * T_EXP * N <= zb_words, kSitePrepZb) &&
            in_bounds((f % instances + 1) * T_EXP * N <= bth_words, kSitePrepBth)) {
            const uint64_t* zc = zb + (f / instances) * T_EXP * N + z0;
            const uint64_t* th = bth + (f % instances) * T_EXP * N + z0;
#pragma unroll
            for (int k = 0; k < T_EXP; k++) {
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const ulonglong2 zv = __ldg(reinterpret_cast<const ulonglong2*>(zc + k * N) + h);
                    const ulonglong2 tv = __ldg(reinterpret_cast<const ulonglong2*>(th + k * N) + h);
                    acc0[2 * h] += (uint64_t)(uint32_t)zv.x * (uint32_t)tv.x;
                    acc0[2 * h + 1] += (uint64_t)(uint32_t)zv.y * (uint32_t)tv.y;
                    acc1[2 * h] += (zv.x >> 32) * (tv.x >> 32);
                    acc1[2 * h + 1] += (zv.y >> 32) * (tv.y >> 32);
                }
            }
        }
        uint32_t o0[4], o1[4];
#pragma unroll
        for (int m = 0; m < 4; m++) {
            o0[m] = mul_canon(mod64(acc0[m], Q0, BR0), ni.w[0], ni.wp[0], Q0);
            o1[m] = mul_canon(mod64(acc1[m], Q1, BR1), ni.w[1], ni.wp[1], Q1);
        }
        *s0 = make_uint4(o0[0], o0[1], o0[2], o0[3]);
        *s1 = make_uint4(o1[0], o1[1], o1[2], o1[3]);
    }
}

// chains: blockIdx.x = fold-group pair (groups 2x, 2x + 1), blockIdx.y = query qg (global over
// the batch); query qg belongs to payload qg / qpp.  S: the prepared packing outputs
// (k_fold_prep) of payload p at S + p * s_payload_stride, [instances][2][N].
__global__ void __launch_bounds__(F3_THREADS, 1)
    k_fold3(const uint32_t* __restrict__ row0s, const uint32_t* __restrict__ gsw, const uint64_t* __restrict__ a_hat,
            const uint32_t* __restrict__ S, int64_t s_payload_stride, const uint64_t* __restrict__ cvec,
            const uint2* __restrict__ fwi, const uint2* __restrict__ iwi, NInv ni, int interp, int c_groups,
            int64_t db_cols, int qpp,
            uint8_t* __restrict__ resp, int64_t resp_payload_stride, int64_t resp_query_stride) {
    extern __shared__ uint32_t f3_smem[];
    uint32_t* sbody = f3_smem;  // [6 gadget rows][2 limbs][N]: N^-1 x the query's RGSW bodies
    const int team = threadIdx.x >> 8, t = threadIdx.x & (F3_TEAM - 1);
    uint32_t* xbuf = f3_smem + 12 * N + team * XP * N;
    // s of this team: [row][m][t] u64, word (row, m) of thread t read back only by thread t
    uint64_t* sst = reinterpret_cast<uint64_t*>(f3_smem + (12 + 2 * XP) * N) + team * 2 * N;
    auto S_AT = [&](int row, int m) -> uint64_t& { return sst[(row * EPT + m) * F3_TEAM + t]; };
    const int qg = blockIdx.y;
    const int wp = 2 * blockIdx.x + team;
    {
        const uint4* gb = reinterpret_cast<const uint4*>(gsw + (int64_t)qg * 12 * N);
        uint4* sb = reinterpret_cast<uint4*>(sbody);
        for (int i = threadIdx.x; i < 12 * N / 4; i += F3_THREADS) {
            const int lb = ((4 * i) / N) & 1;  // word (p * 2 + l) * N + z
            const uint32_t q = lb ? Q1 : Q0, w = ni.w[lb], wq = ni.wp[lb];
            const uint4 b = __ldg(gb + i);
            sb[i] = make_uint4(mul_canon(b.x, w, wq, q), mul_canon(b.y, w, wq, q), mul_canon(b.z, w, wq, q),
                               mul_canon(b.w, w, wq, q));
        }
    }
    __syncthreads();
    if (wp >= c_groups) return;  // the second team of an odd group count has no chain
    const int bar = 1 + team;
    const int payload = qg / qpp, qin = qg % qpp;
    const uint32_t* Sq = S + (int64_t)payload * s_payload_stride;
    const uint64_t* cq = cvec + (int64_t)qg * db_cols;
    const uint64_t mask = (1ull << GADGET_BITS) - 1;
    const int zd = eD(t, 0);

    {  // first step: G^-1(0) = 0, so s = (a_hat[j], INTT(S[j]) + c[j]) mod q
        const int j = wp * interp + interp - 1;
        uint32_t pr[2][EPT];
        load_d8(pr[0], Sq + ((int64_t)j * 2) * N + zd);
        load_d8(pr[1], Sq + ((int64_t)j * 2 + 1) * N + zd);
        uint64_t pc[EPT];
#pragma unroll
        for (int m = 0; m < EPT; m++) {
            S_AT(0, m) = __ldg(a_hat + (int64_t)j * N + eA(t, m));
            pc[m] = __ldg(cq + (int64_t)j * N + eA(t, m));
        }
        inverse_limbs<1>(pr, t, xbuf, bar, iwi);
#pragma unroll
        for (int m = 0; m < EPT; m++) S_AT(1, m) = add_q(crt2(pr[0][m], pr[1][m], Q0INV, BR1), pc[m]);
    }

    for (int step = interp - 2; step >= 0; step--) {
        const int j = wp * interp + step;
        uint32_t pr[4][EPT];  // [row 0 limb 0, row 1 limb 0, row 0 limb 1, row 1 limb 1]
#pragma unroll
        for (int l = 0; l < 2; l++) {
            const uint32_t q = l ? Q1 : Q0;
            const uint64_t br = l ? BR1 : BR0;
            uint32_t sv[EPT];
            load_d8(sv, Sq + ((int64_t)j * 2 + l) * N + zd);
            uint32_t acc0[EPT], acc1[EPT];  // acc1 reduced after every batch of three digits
#pragma unroll
            for (int m = 0; m < EPT; m++) {
                acc0[m] = 0;
                acc1[m] = sv[m];
            }
#pragma unroll 1
            for (int r = 0; r < 2; r++) {  // gadget rows p = r + 2k hold digit k of row r (gadget.rs:44-58)
                uint32_t v[3][EPT];
#pragma unroll
                for (int m = 0; m < EPT; m++) {
                    const uint64_t x = S_AT(r, m);
#pragma unroll
                    for (int k = 0; k < 3; k++) v[k][m] = (uint32_t)((x >> (k * GADGET_BITS)) & mask);
                }
                forward_digits<3>(v, t, xbuf, bar, fwi + l * N, q);
                uint64_t part[EPT];
#pragma unroll
                for (int m = 0; m < EPT; m++) part[m] = acc1[m];
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    const uint4* bp = reinterpret_cast<const uint4*>(sbody + ((r + 2 * k) * 2 + l) * N + zd);
                    const uint4 b0 = bp[0], b1 = bp[1];
                    const uint32_t bv[EPT] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
                    for (int m = 0; m < EPT; m++) {
                        acc0[m] += v[k][m];                    // 6 terms < 12q < 2^32
                        part[m] += (uint64_t)bv[m] * v[k][m];  // q + 3 terms < q + 6 q^2 < 2^60
                    }
                }
#pragma unroll
                for (int m = 0; m < EPT; m++) acc1[m] = mod64(part[m], q, br);
            }
            uint32_t r0[EPT];
            load_d8(r0, row0s + l * N + zd);
            if (l == 0) {
#pragma unroll
                for (int m = 0; m < EPT; m++) {
                    pr[0][m] = mod64((uint64_t)r0[m] * acc0[m], q, br);
                    pr[1][m] = acc1[m];
                }
            } else {
#pragma unroll
                for (int m = 0; m < EPT; m++) {
                    pr[2][m] = mod64((uint64_t)r0[m] * acc0[m], q, br);
                    pr[3][m] = acc1[m];
                }
            }
        }
        uint64_t pa[EPT], pc[EPT];  // packed row j, fetched while the inverse transforms run
#pragma unroll
        for (int m = 0; m < EPT; m++) {
            pa[m] = __ldg(a_hat + (int64_t)j * N + eA(t, m));
            pc[m] = __ldg(cq + (int64_t)j * N + eA(t, m));
        }
        inverse_limbs<2>(pr, t, xbuf, bar, iwi);
#pragma unroll
        for (int m = 0; m < EPT; m++) {
            S_AT(0, m) = add_q(crt2(pr[0][m], pr[2][m], Q0INV, BR1), pa[m]);
            S_AT(1, m) = add_q(crt2(pr[1][m], pr[3][m], Q0INV, BR1), pc[m]);
        }
    }

    switch_keep(S_AT, t, resp + (int64_t)payload * resp_payload_stride + 8 + (int64_t)qin * resp_query_stride +
                             (int64_t)wp * RESULT_BYTES);
}

// One chain (query qg = blockIdx.y, fold group wp = blockIdx.x) per CTA of 256 threads, two
// CTAs per SM, so that the grid's c x queries chains fill the SMs' 296 chain slots in waves
// without the idle half-CTAs of an odd group count.  The RGSW bodies (already scaled by N^-1,
// k_fold_prep) stay in global memory (L2-resident: 48 KB per query per limb); each batch of
// three gadget digits stages the matching three bodies, with the packing output and row 0 of
// its limb, through cp.async into shared memory while its forward transforms run, and the
// packed row j (a_hat, c) lands in s's own slots while the inverse transforms run.
// Shared memory: exchange buffer of 3 polynomials (24 KB), s (32 KB), staging (40 KB).
constexpr int F4_THREADS = nttr::EPT * 32;  // 256: one chain, 8 coefficients per thread
constexpr int F4_XB = 3;
constexpr int F4_SMEM = F4_XB * N * 4 + 2 * N * 8 + 5 * N * 4;
// without the staging area (STAGE false: bodies, packing output and row 0 read straight from
// global memory where they are used) a CTA needs 56 KB and three fit on an SM
constexpr int F4_SMEM_UNSTAGED = F4_XB * N * 4 + 2 * N * 8;

template <bool STAGE>
__global__ void __launch_bounds__(F4_THREADS, STAGE ? 2 : 3)
    k_fold4(const uint32_t* __restrict__ row0s, const uint32_t* __restrict__ gsw, const uint64_t* __restrict__ a_hat,
            const uint32_t* __restrict__ S, int64_t s_payload_stride, const uint64_t* __restrict__ cvec,
            const uint2* __restrict__ fwi, const uint2* __restrict__ iwi, int interp, int c_groups, int64_t db_cols,
            int qpp, uint8_t* __restrict__ resp, int64_t resp_payload_stride, int64_t resp_query_stride,
            FoldExtents ext) {
    extern __shared__ uint4 f4_smem[];
    uint32_t* xbuf = reinterpret_cast<uint32_t*>(f4_smem);  // [F4_XB][N]
    uint64_t* sst = reinterpret_cast<uint64_t*>(xbuf + F4_XB * N);  // [row][m][t]: read back only by thread t
    uint32_t* stg = xbuf + F4_XB * N + 4 * N;  // [5][N]: bodies of digits 0..2, row 0, packing output
    const int t = threadIdx.x;
    auto S_AT = [&](int row, int m) -> uint64_t& { return sst[(row * EPT + m) * F4_THREADS + t]; };
    const int wp = blockIdx.x, qg = blockIdx.y;
    if (wp >= c_groups) return;
    constexpr int bar = 1;
    const int payload = qg / qpp, qin = qg % qpp;
    const uint32_t* Sq = S + (int64_t)payload * s_payload_stride;
    const uint64_t* cq = cvec + (int64_t)qg * db_cols;
    const uint32_t* gq = gsw + (int64_t)qg * 12 * N;
    const int z8 = 8 * t;  // layout D: thread t's 8 consecutive words (eD(t, k) = 8 t + k)
    const uint64_t mask = (1ull << GADGET_BITS) - 1;
    // the debug build's index checks (bounds.cuh); the release build keeps none of them
    const int64_t s_off = (int64_t)payload * s_payload_stride, c_off = (int64_t)qg * db_cols;
    auto s_ok = [&](int64_t row) { return in_bounds(s_off + (row + 1) * N <= ext.s_words, kSiteFoldS); };
    auto ac_ok = [&](int j) {  // rows j of a_hat and of this query's c, every word this thread reads
        const bool a = in_bounds(((int64_t)j + 1) * N <= ext.ahat_words, kSiteFoldAhat);
        return in_bounds(c_off + ((int64_t)j + 1) * N <= ext.c_words, kSiteFoldC) && a;
    };

    {  // first step: G^-1(0) = 0, so s = (a_hat[j], INTT(S[j]) + c[j]) mod q
        const int j = wp * interp + interp - 1;
        uint32_t pr[2][EPT] = {};
        if (s_ok((int64_t)j * 2 + 1)) {
            load_d8(pr[0], Sq + ((int64_t)j * 2) * N + z8);
            load_d8(pr[1], Sq + ((int64_t)j * 2 + 1) * N + z8);
        }
        uint64_t pc[EPT];
        const bool acj = ac_ok(j);
#pragma unroll
        for (int m = 0; m < EPT; m++) {
            S_AT(0, m) = acj ? __ldg(a_hat + (int64_t)j * N + eA(t, m)) : 0;
            pc[m] = acj ? __ldg(cq + (int64_t)j * N + eA(t, m)) : 0;
        }
        inverse_limbs<1, 2>(pr, t, xbuf, bar, iwi);
#pragma unroll
        for (int m = 0; m < EPT; m++) S_AT(1, m) = add_q(crt2m(pr[0][m], pr[1][m]), pc[m]);
    }

    for (int step = interp - 2; step >= 0; step--) {
        const int j = wp * interp + step;
        uint32_t pr[4][EPT];  // [row 0 limb 0, row 1 limb 0, row 0 limb 1, row 1 limb 1]
#pragma unroll
        for (int l = 0; l < 2; l++) {
            const uint32_t q = l ? Q1 : Q0;
            // acc0: the six digit transforms' sum (< 12q); acc1: the packing output plus each
            // batch's Montgomery-reduced MAC (< q + 2 x 2q = 5q), canonicalised after both batches
            uint32_t acc0[EPT], acc1[EPT];
#pragma unroll
            for (int m = 0; m < EPT; m++) acc0[m] = 0;
#pragma unroll 1
            for (int r = 0; r < 2; r++) {  // gadget rows p = r + 2k hold digit k of row r (gadget.rs:44-58)
                if constexpr (STAGE) {
                    // every thread's reads of the staging area (the previous batch) are done
                    nttr::group_bar(bar);
#pragma unroll
                    for (int k = 0; k < 3; k++) {
                        const int64_t row = (int64_t)qg * 12 + (r + 2 * k) * 2 + l;
                        if (!in_bounds((row + 1) * N <= ext.gsw_words, kSiteFoldGsw)) continue;
                        const uint32_t* src = gq + (int64_t)((r + 2 * k) * 2 + l) * N + z8;
                        cp16(stg + k * N + z8, src);
                        cp16(stg + k * N + z8 + 4, src + 4);
                    }
                    if (r == 0) {
                        cp16(stg + 3 * N + z8, row0s + l * N + z8);
                        cp16(stg + 3 * N + z8 + 4, row0s + l * N + z8 + 4);
                        if (s_ok((int64_t)j * 2 + l)) {
                            const uint32_t* sp = Sq + ((int64_t)j * 2 + l) * N + z8;
                            cp16(stg + 4 * N + z8, sp);
                            cp16(stg + 4 * N + z8 + 4, sp + 4);
                        }
                    }
                    cp_commit();
                }
                uint32_t v[3][EPT];
#pragma unroll
                for (int m = 0; m < EPT; m++) {
                    const uint64_t x = S_AT(r, m);
#pragma unroll
                    for (int k = 0; k < 3; k++) v[k][m] = (uint32_t)((x >> (k * GADGET_BITS)) & mask);
                }
                forward_digits<3>(v, t, xbuf, bar, fwi + l * N, q);
                if (l == 1 && r == 1) {
                    // s is consumed (the team barriers of the transforms ordered every read of
                    // it): the packed row j lands in its slots while the inverse transforms run
                    if (ac_ok(j)) {
#pragma unroll
                        for (int m = 0; m < EPT; m++) {
                            cp8(&S_AT(0, m), a_hat + (int64_t)j * N + eA(t, m));
                            cp8(&S_AT(1, m), cq + (int64_t)j * N + eA(t, m));
                        }
                    }
                    cp_commit();
                    if constexpr (STAGE) cp_wait<1>();
                } else if constexpr (STAGE) {
                    cp_wait<0>();
                }
                if (r == 0) {
                    if constexpr (STAGE) {
                        const uint4 a = *reinterpret_cast<const uint4*>(stg + 4 * N + z8);
                        const uint4 b = *reinterpret_cast<const uint4*>(stg + 4 * N + z8 + 4);
                        acc1[0] = a.x; acc1[1] = a.y; acc1[2] = a.z; acc1[3] = a.w;
                        acc1[4] = b.x; acc1[5] = b.y; acc1[6] = b.z; acc1[7] = b.w;
                    } else {
#pragma unroll
                        for (int m = 0; m < EPT; m++) acc1[m] = 0;
                        if (s_ok((int64_t)j * 2 + l)) load_d8(acc1, Sq + ((int64_t)j * 2 + l) * N + z8);
                    }
                }
                uint64_t part[EPT];
#pragma unroll
                for (int m = 0; m < EPT; m++) part[m] = 0;
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    uint4 b0, b1;
                    if constexpr (STAGE) {
                        b0 = *reinterpret_cast<const uint4*>(stg + k * N + z8);
                        b1 = *reinterpret_cast<const uint4*>(stg + k * N + z8 + 4);
                    } else {
                        const int64_t row = (int64_t)qg * 12 + (r + 2 * k) * 2 + l;
                        b0 = b1 = make_uint4(0, 0, 0, 0);
                        if (in_bounds((row + 1) * N <= ext.gsw_words, kSiteFoldGsw)) {
                            const uint4* src = reinterpret_cast<const uint4*>(gq + (int64_t)((r + 2 * k) * 2 + l) * N + z8);
                            b0 = __ldg(src);
                            b1 = __ldg(src + 1);
                        }
                    }
                    const uint32_t bv[EPT] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
                    for (int m = 0; m < EPT; m++) {
                        acc0[m] += v[k][m];                    // 6 terms < 12q < 2^32
                        part[m] += (uint64_t)bv[m] * v[k][m];  // 3 terms < 6 q^2 < q 2^32
                    }
                }
#pragma unroll
                for (int m = 0; m < EPT; m++) acc1[m] += redc(part[m], q);
            }
            uint32_t r0[EPT];
            if constexpr (STAGE) {
                const uint4 ra = *reinterpret_cast<const uint4*>(stg + 3 * N + z8);
                const uint4 rb = *reinterpret_cast<const uint4*>(stg + 3 * N + z8 + 4);
                r0[0] = ra.x; r0[1] = ra.y; r0[2] = ra.z; r0[3] = ra.w;
                r0[4] = rb.x; r0[5] = rb.y; r0[6] = rb.z; r0[7] = rb.w;
            } else {
                load_d8(r0, row0s + l * N + z8);
            }
#pragma unroll
            for (int m = 0; m < EPT; m++) {
                pr[2 * l][m] = csub(redc((uint64_t)r0[m] * acc0[m], q), q);  // < 12 q^2 < q 2^32
                pr[2 * l + 1][m] = csub(csub(csub(acc1[m], 4 * q), 2 * q), q);  // < 5q -> [0, q)
            }
        }
        inverse_limbs<2, 2>(pr, t, xbuf, bar, iwi);
        cp_wait<0>();  // the packed row j in s's slots
#pragma unroll
        for (int m = 0; m < EPT; m++) {
            S_AT(0, m) = add_q(crt2m(pr[0][m], pr[2][m]), S_AT(0, m));
            S_AT(1, m) = add_q(crt2m(pr[1][m], pr[3][m]), S_AT(1, m));
        }
    }

    const int64_t o = (int64_t)payload * resp_payload_stride + 8 + (int64_t)qin * resp_query_stride +
                      (int64_t)wp * RESULT_BYTES;
    if (in_bounds(o + RESULT_BYTES <= ext.resp_bytes, kSiteFoldResp)) switch_keep(S_AT, t, resp + o);
}

// RGSW bodies 96 KB + two team exchange buffers of 4 polynomials (2 x 32 KB) + the two
// teams' s (2 x 32 KB) = 224 KB
constexpr int FOLD3_SMEM = (12 + 2 * XP) * N * 4 + 2 * 2 * N * 8;

cudaError_t init_fold3_kernel() {
    cudaError_t e = cudaFuncSetAttribute(k_fold3, cudaFuncAttributeMaxDynamicSharedMemorySize, FOLD3_SMEM);
    if (e != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_fold4<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, F4_SMEM)) != cudaSuccess)
        return e;
    return cudaFuncSetAttribute(k_fold4<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, F4_SMEM_UNSTAGED);
}

cudaError_t launch_fold_prep(uint32_t* S, int64_t count, const uint64_t* zb, const uint64_t* bth, int instances,
                             const uint32_t ninv[4], int sm_count, cudaStream_t st, uint32_t* gsw, int gsw_queries,
                             const uint32_t* ninv_bodies) {
    if (count < 1 || (zb && instances < 1) || (gsw && gsw_queries < 1)) return cudaErrorInvalidValue;
    NInv ni{{ninv[0], ninv[2]}, {ninv[1], ninv[3]}};
    const uint32_t* nbv = ninv_bodies ? ninv_bodies : ninv;
    NInv nb{{nbv[0], nbv[2]}, {nbv[1], nbv[3]}};
    const int64_t n4 = count * (N / 4);
    const int64_t blocks = std::min<int64_t>((n4 + 255) / 256, (int64_t)sm_count * 8);
    const int64_t gsw_words = gsw ? (int64_t)gsw_queries * 12 * N : 0;
    const int64_t zb_words = zb ? (count + instances - 1) / instances * T_EXP * N : 0;
    const int64_t bth_words = zb ? (int64_t)instances * T_EXP * N : 0;
    cudaError_t e;
    if ((e = check_extent(S, (uint64_t)count * 2 * N * 4, "fold scaling: packing outputs")) != cudaSuccess ||
        (e = check_extent(zb, (uint64_t)zb_words * 8, "fold scaling: z bodies")) != cudaSuccess ||
        (e = check_extent(bth, (uint64_t)bth_words * 8, "fold scaling: condensed T-hat")) != cudaSuccess ||
        (e = check_extent(gsw, (uint64_t)gsw_words * 4, "fold scaling: RGSW bodies")) != cudaSuccess)
        return e;
    k_fold_prep<<<(unsigned)blocks, 256, 0, st>>>(S, count, zb, bth, instances, ni, gsw, gsw_words, zb_words,
                                                  bth_words, nb);
    return cudaGetLastError();
}

cudaError_t launch_fold3(const uint32_t* row0s, const uint32_t* gsw, const uint64_t* a_hat, const uint32_t* S,
                         int64_t s_payload_stride, const uint64_t* cvec, const uint32_t* fwi, const uint32_t* iwi,
                         const uint32_t ninv[4], int interp, int c_groups,
                         int num_queries, int64_t db_cols, int qpp, uint8_t* resp, int64_t resp_payload_stride,
                         int64_t resp_query_stride, cudaStream_t st) {
    if (interp < 1 || c_groups < 1 || num_queries < 1 || num_queries > 65535 || qpp < 1) return cudaErrorInvalidValue;
    NInv ni{{ninv[0], ninv[2]}, {ninv[1], ninv[3]}};
    dim3 grid((c_groups + 1) / 2, num_queries);
    k_fold3<<<grid, F3_THREADS, FOLD3_SMEM, st>>>(row0s, gsw, a_hat, S, s_payload_stride, cvec,
                                                   reinterpret_cast<const uint2*>(fwi),
                                                   reinterpret_cast<const uint2*>(iwi), ni, interp, c_groups, db_cols,
                                                   qpp, resp, resp_payload_stride, resp_query_stride);
    return cudaGetLastError();
}

cudaError_t launch_fold4(const uint32_t* row0s, const uint32_t* gsw_scaled, const uint64_t* a_hat, const uint32_t* S,
                         int64_t s_payload_stride, const uint64_t* cvec, const uint32_t* fwi, const uint32_t* iwi,
                         int interp, int c_groups, int num_queries, int64_t db_cols, int qpp, uint8_t* resp,
                         int64_t resp_payload_stride, int64_t resp_query_stride, const FoldExtents& ext,
                         cudaStream_t st, bool staged) {
    if (interp < 1 || c_groups < 1 || num_queries < 1 || num_queries > 65535 || qpp < 1) return cudaErrorInvalidValue;
    cudaError_t e;
    if ((e = check_extent(row0s, 2ull * N * 4, "fold: row 0")) != cudaSuccess ||
        (e = check_extent(gsw_scaled, (uint64_t)ext.gsw_words * 4, "fold: RGSW bodies")) != cudaSuccess ||
        (e = check_extent(a_hat, (uint64_t)ext.ahat_words * 8, "fold: a_hat")) != cudaSuccess ||
        (e = check_extent(S, (uint64_t)ext.s_words * 4, "fold: packing outputs")) != cudaSuccess ||
        (e = check_extent(cvec, (uint64_t)ext.c_words * 8, "fold: first-dimension outputs")) != cudaSuccess ||
        (e = check_extent(fwi, 2ull * N * 8, "fold: forward twiddles")) != cudaSuccess ||
        (e = check_extent(iwi, 2ull * N * 8, "fold: inverse twiddles")) != cudaSuccess ||
        (e = check_extent(resp, (uint64_t)ext.resp_bytes, "fold: responses")) != cudaSuccess)
        return e;
    dim3 grid(c_groups, num_queries);
    if (staged)
        k_fold4<true><<<grid, F4_THREADS, F4_SMEM, st>>>(
            row0s, gsw_scaled, a_hat, S, s_payload_stride, cvec, reinterpret_cast<const uint2*>(fwi),
            reinterpret_cast<const uint2*>(iwi), interp, c_groups, db_cols, qpp, resp, resp_payload_stride,
            resp_query_stride, ext);
    else
        k_fold4<false><<<grid, F4_THREADS, F4_SMEM_UNSTAGED, st>>>(
            row0s, gsw_scaled, a_hat, S, s_payload_stride, cvec, reinterpret_cast<const uint2*>(fwi),
            reinterpret_cast<const uint2*>(iwi), interp, c_groups, db_cols, qpp, resp, resp_payload_stride,
            resp_query_stride, ext);
    return cudaGetLastError();
}

}  // namespace ipr
