// ntt_regs.cuh — register-resident negacyclic NTTs of 2048 points, one CRT
// limb per group of 256 threads, 8 elements per thread, P polynomials of the
// same limb transformed together (each twiddle load feeds P butterflies).
//
// Butterflies are the Harvey forms of ntt_forward / ntt_inverse
// (rkdud007/inspire-rs src/core/ntt.rs:111-160, 731-780) with the tables of
// build_ntt_tables (ntt.rs:74-108); outputs are canonical, so results equal
// the reference's transforms exactly.
// Thread t of the group (warp w = t / 32, lane l = t % 32) holds 8 elements
// whose index bits are split between the thread and the register number, so
// every butterfly pairs two registers of one thread:
//   layout A: e = t + 256 m                          (distances 1024, 512, 256)
//   layout B: e = 256 w + l + 32 m                   (distances 128, 64, 32)
//   layout C: e = 256 w + 32 (l/4) + 4 k + l%4       (distances 16, 8, 4)
//   layout D: e = 256 w + 8 l + k                    (distances 2, 1)
// A <-> B moves data between the group's warps (shared memory + group
// barrier); B <-> C <-> D stay inside one warp's 256 elements (shared memory,
// XOR-swizzled so that every access is free of bank conflicts, + __syncwarp).
// Forward: A -> D.  Inverse: D -> A.
#pragma once
#include <cstdint>

#include "ipr_device.cuh"

namespace ipr {
namespace nttr {

constexpr int GT = 256;  // threads per limb group
constexpr int EPT = 8;   // elements per thread

__device__ __forceinline__ int eA(int t, int m) { return t + 256 * m; }
__device__ __forceinline__ int eB(int t, int m) { return (t >> 5) * 256 + (t & 31) + 32 * m; }
__device__ __forceinline__ int eC(int t, int k) { return (t >> 5) * 256 + ((t & 31) >> 2) * 32 + 4 * k + (t & 3); }
__device__ __forceinline__ int eD(int t, int k) { return (t >> 5) * 256 + (t & 31) * 8 + k; }

// swizzled word of local index i (< 256) inside a warp's 256-word block: the
// row i / 32 flips bits 2..4 of the column, keeping aligned groups of 4 words
__device__ __forceinline__ int swz(int i) { return i ^ (((i >> 5) & 7) << 2); }

// named barrier 1 or 2 over one group (literal ids keep the CTA's barrier count at 3)
__device__ __forceinline__ void group_bar(int id) {
    if (id == 1) asm volatile("bar.sync 1, 256;" ::: "memory");
    else asm volatile("bar.sync 2, 256;" ::: "memory");
}

// conditional subtractions as unsigned minima: for v < 4q, min(v, v - 2q) is v - 2q when
// v >= 2q and v otherwise (the difference wraps above v)
__device__ __forceinline__ uint32_t csub(uint32_t v, uint32_t m) { return min(v, v - m); }

__device__ __forceinline__ void fwd_bfly(uint32_t& x, uint32_t& y, uint32_t w, uint32_t wp, uint32_t q) {
    const uint32_t two_q = 2 * q;
    const uint32_t xx = csub(x, two_q);
    const uint32_t qn = shoup_lazy(y, w, wp, q);
    x = xx + qn;
    y = xx + two_q - qn;
}

__device__ __forceinline__ void inv_bfly(uint32_t& x, uint32_t& y, uint32_t w, uint32_t wp, uint32_t q) {
    const uint32_t two_q = 2 * q;
    const uint32_t tt = two_q - y + x;
    const uint32_t cx = csub(x + y, two_q);  // x + y >= 2q exactly when 2x >= tt
    x = (cx + (q & (0u - (tt & 1)))) >> 1;
    y = w * tt - __umulhi(tt, wp) * q;
}

__device__ __forceinline__ uint32_t canon(uint32_t v, uint32_t q) { return csub(csub(v, 2 * q), q); }

// A <-> B exchange of P polynomials through xbuf (XP * 2048 words, XP <= P polynomials at a
// time), group barrier id bar.  The intra-warp transposes use only the warp's own 256-word
// region of each polynomial and synchronise only the warp.  A -> B stores into every warp's
// region, so its barrier comes before the stores (every warp of the group is done with its
// region, e.g. the transposes of a previous transform) and its loads read the warp's own
// region; B -> A stores into the warp's own region and loads from all regions, so its second
// barrier lets every warp finish loading before anything writes there again.
template <int P, bool A_TO_B, int XP = P>
__device__ __forceinline__ void exchange(uint32_t (&v)[P][EPT], int t, uint32_t* xbuf, int bar) {
#pragma unroll
    for (int c0 = 0; c0 < P; c0 += XP) {
        if (A_TO_B) group_bar(bar);
#pragma unroll
        for (int p = c0; p < c0 + XP && p < P; p++)
#pragma unroll
            for (int m = 0; m < EPT; m++) xbuf[(p - c0) * N + (A_TO_B ? eA(t, m) : eB(t, m))] = v[p][m];
        group_bar(bar);
#pragma unroll
        for (int p = c0; p < c0 + XP && p < P; p++)
#pragma unroll
            for (int m = 0; m < EPT; m++) v[p][m] = xbuf[(p - c0) * N + (A_TO_B ? eB(t, m) : eA(t, m))];
        if (!A_TO_B) group_bar(bar);
    }
}

// intra-warp transposes; wb = the warp's 256-word block of the buffer's polynomial 0, the
// buffer holding XP polynomials (P are moved, XP at a time)
__device__ __forceinline__ int c_word(int l, int k) { return swz((l >> 2) * 32 + 4 * k + (l & 3)); }
__device__ __forceinline__ int b_word(int l, int m) { return swz(l + 32 * m); }
// layout D's 8 words of lane l sit in two aligned 4-word groups: swz(8 l + k)
__device__ __forceinline__ int d_off(int l, int h) { return (l >> 2) * 32 + 4 * ((2 * (l & 3) + h) ^ (l >> 2)); }

template <int P, int XP = P>
__device__ __forceinline__ void b_to_c(uint32_t (&v)[P][EPT], int l, uint32_t* wb) {
#pragma unroll
    for (int c0 = 0; c0 < P; c0 += XP) {
#pragma unroll
        for (int p = c0; p < c0 + XP && p < P; p++)
#pragma unroll
            for (int m = 0; m < EPT; m++) wb[(p - c0) * N + b_word(l, m)] = v[p][m];
        __syncwarp();
#pragma unroll
        for (int p = c0; p < c0 + XP && p < P; p++)
#pragma unroll
            for (int k = 0; k < EPT; k++) v[p][k] = wb[(p - c0) * N + c_word(l, k)];
        __syncwarp();
    }
}

template <int P, int XP = P>
__device__ __forceinline__ void c_to_b(uint32_t (&v)[P][EPT], int l, uint32_t* wb) {
#pragma unroll
    for (int c0 = 0; c0 < P; c0 += XP) {
#pragma unroll
        for (int p = c0; p < c0 + XP && p < P; p++)
#pragma unroll
            for (int k = 0; k < EPT; k++) wb[(p - c0) * N + c_word(l, k)] = v[p][k];
        __syncwarp();
#pragma unroll
        for (int p = c0; p < c0 + XP && p < P; p++)
#pragma unroll
            for (int m = 0; m < EPT; m++) v[p][m] = wb[(p - c0) * N + b_word(l, m)];
        __syncwarp();
    }
}

template <int P, int XP = P>
__device__ __forceinline__ void c_to_d(uint32_t (&v)[P][EPT], int l, uint32_t* wb) {
#pragma unroll
    for (int c0 = 0; c0 < P; c0 += XP) {
#pragma unroll
        for (int p = c0; p < c0 + XP && p < P; p++)
#pragma unroll
            for (int k = 0; k < EPT; k++) wb[(p - c0) * N + c_word(l, k)] = v[p][k];
        __syncwarp();
#pragma unroll
        for (int p = c0; p < c0 + XP && p < P; p++) {
            const uint4 a = *reinterpret_cast<const uint4*>(wb + (p - c0) * N + d_off(l, 0));
            const uint4 b = *reinterpret_cast<const uint4*>(wb + (p - c0) * N + d_off(l, 1));
            v[p][0] = a.x; v[p][1] = a.y; v[p][2] = a.z; v[p][3] = a.w;
            v[p][4] = b.x; v[p][5] = b.y; v[p][6] = b.z; v[p][7] = b.w;
        }
        __syncwarp();
    }
}

template <int P, int XP = P>
__device__ __forceinline__ void d_to_c(uint32_t (&v)[P][EPT], int l, uint32_t* wb) {
#pragma unroll
    for (int c0 = 0; c0 < P; c0 += XP) {
#pragma unroll
        for (int p = c0; p < c0 + XP && p < P; p++) {
            *reinterpret_cast<uint4*>(wb + (p - c0) * N + d_off(l, 0)) = make_uint4(v[p][0], v[p][1], v[p][2], v[p][3]);
            *reinterpret_cast<uint4*>(wb + (p - c0) * N + d_off(l, 1)) = make_uint4(v[p][4], v[p][5], v[p][6], v[p][7]);
        }
        __syncwarp();
#pragma unroll
        for (int p = c0; p < c0 + XP && p < P; p++)
#pragma unroll
            for (int k = 0; k < EPT; k++) v[p][k] = wb[(p - c0) * N + c_word(l, k)];
        __syncwarp();
    }
}

// in-register stage with register distance dd and twiddle index (1 << mm) + (e(k) >> (11 - mm))
template <int P, bool FWD, typename E>
__device__ __forceinline__ void reg_stage(uint32_t (&v)[P][EPT], int mm, int dd, E e, const uint32_t* __restrict__ w_t,
                                          const uint32_t* __restrict__ wp_t, uint32_t q) {
#pragma unroll
    for (int k = 0; k < EPT; k++) {
        if (k & dd) continue;
        const int idx = (1 << mm) + (e(k) >> (11 - mm));
        const uint32_t w = __ldg(w_t + idx), wp = __ldg(wp_t + idx);
#pragma unroll
        for (int p = 0; p < P; p++) {
            if (FWD) fwd_bfly(v[p][k], v[p][k + dd], w, wp, q);
            else inv_bfly(v[p][k], v[p][k + dd], w, wp, q);
        }
    }
}

// forward NTT of P polynomials of one limb: layout A in, layout D canonical out (in [0, 2q)
// instead with HALF_REDUCED, for callers that only accumulate the outputs).
// xbuf holds XP * 2048 words for this group.
template <int P, int XP = P, bool HALF_REDUCED = false>
__device__ __forceinline__ void forward(uint32_t (&v)[P][EPT], int t, uint32_t* xbuf, int bar,
                                        const uint32_t* __restrict__ fw, const uint32_t* __restrict__ fwp,
                                        uint32_t q) {
    const int l = t & 31;
    uint32_t* wb = xbuf + (t >> 5) * 256;
#pragma unroll
    for (int mm = 0; mm < 3; mm++) reg_stage<P, true>(v, mm, 4 >> mm, [&](int k) { return eA(t, k); }, fw, fwp, q);
    exchange<P, true, XP>(v, t, xbuf, bar);
#pragma unroll
    for (int mm = 3; mm < 6; mm++)
        reg_stage<P, true>(v, mm, 4 >> (mm - 3), [&](int k) { return eB(t, k); }, fw, fwp, q);
    b_to_c<P, XP>(v, l, wb);
#pragma unroll
    for (int mm = 6; mm < 9; mm++)
        reg_stage<P, true>(v, mm, 4 >> (mm - 6), [&](int k) { return eC(t, k); }, fw, fwp, q);
    c_to_d<P, XP>(v, l, wb);
#pragma unroll
    for (int mm = 9; mm < 11; mm++)
        reg_stage<P, true>(v, mm, 2 >> (mm - 9), [&](int k) { return eD(t, k); }, fw, fwp, q);
#pragma unroll
    for (int p = 0; p < P; p++)
#pragma unroll
        for (int k = 0; k < EPT; k++) v[p][k] = HALF_REDUCED ? csub(v[p][k], 2 * q) : canon(v[p][k], q);
}

// inverse NTT of P polynomials of one limb: layout D in, layout A canonical out
template <int P, int XP = P>
__device__ __forceinline__ void inverse(uint32_t (&v)[P][EPT], int t, uint32_t* xbuf, int bar,
                                        const uint32_t* __restrict__ iw, const uint32_t* __restrict__ iwp,
                                        uint32_t q) {
    const int l = t & 31;
    uint32_t* wb = xbuf + (t >> 5) * 256;
#pragma unroll
    for (int mm = 10; mm >= 9; mm--)
        reg_stage<P, false>(v, mm, 2 >> (mm - 9), [&](int k) { return eD(t, k); }, iw, iwp, q);
    d_to_c<P, XP>(v, l, wb);
#pragma unroll
    for (int mm = 8; mm >= 6; mm--)
        reg_stage<P, false>(v, mm, 4 >> (mm - 6), [&](int k) { return eC(t, k); }, iw, iwp, q);
    c_to_b<P, XP>(v, l, wb);
#pragma unroll
    for (int mm = 5; mm >= 3; mm--)
        reg_stage<P, false>(v, mm, 4 >> (mm - 3), [&](int k) { return eB(t, k); }, iw, iwp, q);
    exchange<P, false, XP>(v, t, xbuf, bar);
#pragma unroll
    for (int mm = 2; mm >= 0; mm--) reg_stage<P, false>(v, mm, 4 >> mm, [&](int k) { return eA(t, k); }, iw, iwp, q);
#pragma unroll
    for (int p = 0; p < P; p++)
#pragma unroll
        for (int k = 0; k < EPT; k++) v[p][k] = canon(v[p][k], q);
}

}  // namespace nttr
}  // namespace ipr
