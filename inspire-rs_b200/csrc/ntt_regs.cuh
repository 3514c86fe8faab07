// ntt_regs.cuh — register-resident negacyclic NTTs of 2048 points, one CRT
// limb per group of 256 threads, 8 elements per thread, P polynomials of the
// same limb transformed together (each twiddle load feeds P butterflies).
//
// Butterflies are the Harvey forms of ntt_forward / ntt_inverse
// (rkdud007/inspire-rs src/core/ntt.rs:111-160, 731-780) with the tables of
// build_ntt_tables (ntt.rs:74-108); outputs are canonical, so results equal
// the reference's transforms exactly.
//   layout A: thread t holds e = t + 256 m                  (distances 1024, 512, 256)
//   layout B: thread t holds e = (t/32)*256 + t%32 + 32 m    (distances 128, 64, 32)
//   distances 16 .. 1 pair lanes of one warp in layout B (warp shuffles).
// Forward: A -> B (one shared-memory exchange).  Inverse: B -> A.
#pragma once
#include <cstdint>

#include "ipr_device.cuh"

namespace ipr {
namespace nttr {

constexpr int GT = 256;  // threads per limb group
constexpr int EPT = 8;   // elements per thread

__device__ __forceinline__ int eA(int t, int m) { return t + 256 * m; }
__device__ __forceinline__ int eB(int t, int m) { return (t >> 5) * 256 + (t & 31) + 32 * m; }

// named barrier 1 or 2 over one group (literal ids keep the CTA's barrier count at 3)
__device__ __forceinline__ void group_bar(int id) {
    if (id == 1) asm volatile("bar.sync 1, 256;" ::: "memory");
    else asm volatile("bar.sync 2, 256;" ::: "memory");
}

__device__ __forceinline__ void fwd_bfly(uint32_t& x, uint32_t& y, uint32_t w, uint32_t wp, uint32_t q) {
    const uint32_t two_q = 2 * q;
    const uint32_t xx = x >= two_q ? x - two_q : x;
    const uint32_t qn = shoup_lazy(y, w, wp, q);
    x = xx + qn;
    y = xx + two_q - qn;
}

__device__ __forceinline__ void inv_bfly(uint32_t& x, uint32_t& y, uint32_t w, uint32_t wp, uint32_t q) {
    const uint32_t two_q = 2 * q;
    const uint32_t tt = two_q - y + x;
    const uint32_t cx = x + y - ((2 * x >= tt) ? two_q : 0);
    x = (cx + ((tt & 1) ? q : 0)) >> 1;
    y = w * tt - __umulhi(tt, wp) * q;
}

__device__ __forceinline__ uint32_t canon(uint32_t v, uint32_t q) {
    v = v >= 2 * q ? v - 2 * q : v;
    return v >= q ? v - q : v;
}

// A <-> B exchange of P polynomials through xbuf (P * 2048 words), group barrier id bar
template <int P, bool A_TO_B>
__device__ __forceinline__ void exchange(uint32_t (&v)[P][EPT], int t, uint32_t* xbuf, int bar) {
#pragma unroll
    for (int p = 0; p < P; p++)
#pragma unroll
        for (int m = 0; m < EPT; m++) xbuf[p * N + (A_TO_B ? eA(t, m) : eB(t, m))] = v[p][m];
    group_bar(bar);
#pragma unroll
    for (int p = 0; p < P; p++)
#pragma unroll
        for (int m = 0; m < EPT; m++) v[p][m] = xbuf[p * N + (A_TO_B ? eB(t, m) : eA(t, m))];
    group_bar(bar);
}

// forward NTT of P polynomials of one limb: layout A in, layout B canonical out
template <int P>
__device__ __forceinline__ void forward(uint32_t (&v)[P][EPT], int t, uint32_t* xbuf, int bar,
                                        const uint32_t* __restrict__ fw, const uint32_t* __restrict__ fwp,
                                        uint32_t q) {
#pragma unroll
    for (int mm = 0; mm < 3; mm++) {  // distances 1024, 512, 256
        const int d = 4 >> mm;
#pragma unroll
        for (int m = 0; m < EPT; m++) {
            if (m & d) continue;
            const int idx = (1 << mm) + (m >> (3 - mm));
            const uint32_t w = __ldg(fw + idx), wp = __ldg(fwp + idx);
#pragma unroll
            for (int p = 0; p < P; p++) fwd_bfly(v[p][m], v[p][m + d], w, wp, q);
        }
    }
    exchange<P, true>(v, t, xbuf, bar);
    const int blk = t >> 5, r = t & 31;
#pragma unroll
    for (int mm = 3; mm < 6; mm++) {  // distances 128, 64, 32
        const int d = 4 >> (mm - 3);
#pragma unroll
        for (int m = 0; m < EPT; m++) {
            if (m & d) continue;
            const int idx = (1 << mm) + (blk << (mm - 3)) + (m >> (6 - mm));
            const uint32_t w = __ldg(fw + idx), wp = __ldg(fwp + idx);
#pragma unroll
            for (int p = 0; p < P; p++) fwd_bfly(v[p][m], v[p][m + d], w, wp, q);
        }
    }
#pragma unroll
    for (int mm = 6; mm < 11; mm++) {  // distances 16 .. 1 across lanes
        const int d = 1024 >> mm;
        const bool upper = r & d;
#pragma unroll
        for (int m = 0; m < EPT; m++) {
            const int idx = (1 << mm) + ((blk * 256 + r + 32 * m) >> (11 - mm));
            const uint32_t w = __ldg(fw + idx), wp = __ldg(fwp + idx);
#pragma unroll
            for (int p = 0; p < P; p++) {
                const uint32_t mine = v[p][m];
                const uint32_t wy = shoup_lazy(mine, w, wp, q);  // used by the upper lane only
                const uint32_t recv = __shfl_xor_sync(0xffffffffu, upper ? wy : mine, d);
                const uint32_t x = upper ? recv : mine;
                const uint32_t xx = x >= 2 * q ? x - 2 * q : x;
                v[p][m] = upper ? xx + 2 * q - wy : xx + recv;
            }
        }
    }
#pragma unroll
    for (int p = 0; p < P; p++)
#pragma unroll
        for (int m = 0; m < EPT; m++) v[p][m] = canon(v[p][m], q);
}

// inverse NTT of P polynomials of one limb: layout B in, layout A canonical out
template <int P>
__device__ __forceinline__ void inverse(uint32_t (&v)[P][EPT], int t, uint32_t* xbuf, int bar,
                                        const uint32_t* __restrict__ iw, const uint32_t* __restrict__ iwp,
                                        uint32_t q) {
    const int blk = t >> 5, r = t & 31;
#pragma unroll
    for (int mm = 10; mm >= 6; mm--) {  // distances 1 .. 16 across lanes
        const int d = 1024 >> mm;
        const bool upper = r & d;
#pragma unroll
        for (int m = 0; m < EPT; m++) {
            const int idx = (1 << mm) + ((blk * 256 + r + 32 * m) >> (11 - mm));
            const uint32_t w = __ldg(iw + idx), wp = __ldg(iwp + idx);
#pragma unroll
            for (int p = 0; p < P; p++) {
                const uint32_t mine = v[p][m];
                const uint32_t other = __shfl_xor_sync(0xffffffffu, mine, d);
                uint32_t x = upper ? other : mine, y = upper ? mine : other;
                inv_bfly(x, y, w, wp, q);
                v[p][m] = upper ? y : x;
            }
        }
    }
#pragma unroll
    for (int mm = 5; mm >= 3; mm--) {  // distances 32, 64, 128
        const int d = 4 >> (mm - 3);
#pragma unroll
        for (int m = 0; m < EPT; m++) {
            if (m & d) continue;
            const int idx = (1 << mm) + (blk << (mm - 3)) + (m >> (6 - mm));
            const uint32_t w = __ldg(iw + idx), wp = __ldg(iwp + idx);
#pragma unroll
            for (int p = 0; p < P; p++) inv_bfly(v[p][m], v[p][m + d], w, wp, q);
        }
    }
    exchange<P, false>(v, t, xbuf, bar);
#pragma unroll
    for (int mm = 2; mm >= 0; mm--) {  // distances 256, 512, 1024
        const int d = 4 >> mm;
#pragma unroll
        for (int m = 0; m < EPT; m++) {
            if (m & d) continue;
            const int idx = (1 << mm) + (m >> (3 - mm));
            const uint32_t w = __ldg(iw + idx), wp = __ldg(iwp + idx);
#pragma unroll
            for (int p = 0; p < P; p++) inv_bfly(v[p][m], v[p][m + d], w, wp, q);
        }
    }
#pragma unroll
    for (int p = 0; p < P; p++)
#pragma unroll
        for (int m = 0; m < EPT; m++) v[p][m] = canon(v[p][m], q);
}

}  // namespace nttr
}  // namespace ipr
