// ipr_device.cuh — device-side modular arithmetic and negacyclic NTTs for the
// InsPIRe respond() path on sm_100a.
//
// Arithmetic domain (src/pir/params.rs:8-9 of rkdud007/inspire-rs): two NTT
// primes q0 = 268369921, q1 = 249561089 (both < 2^28), q = q0*q1 < 2^56,
// ring dimension N = 2048.  Every value that leaves a kernel is canonical, so
// any correct reduction strategy reproduces the reference's outputs exactly.
#pragma once
#include <cstdint>

namespace ipr {

constexpr int N = 2048;
constexpr int LOGN = 11;
constexpr int T_EXP = 3;                 // t_exp_left = t_gsw (wire.rs:424)
constexpr int NROT = N / 2 - 1;          // 1023 rotations (packing.rs:1766)
constexpr int NINNER = NROT * T_EXP;     // 3069 key-switch rows per output
constexpr uint32_t Q0 = 268369921u;
constexpr uint32_t Q1 = 249561089u;
constexpr uint64_t QQ = (uint64_t)Q0 * (uint64_t)Q1;
constexpr uint32_t PT = 65535u;          // plaintext modulus (wire.rs:421)
constexpr uint64_t QP1 = 1ull << 20;     // q'_1 (params.rs:346-348)
constexpr uint64_t QP2 = 268369921ull;   // q'_2 = Q2_VALUES[28] (core/params.rs:37)
constexpr int RESULT_BYTES = 12288;      // (28 + 20) * 2048 / 8 (modulus_switch.rs:45-73)
constexpr int GADGET_BITS = 19;          // floor(56/3)+1 (gadget.rs:3-9)
constexpr uint64_t BR0 = 68736257792ull;  // floor(2^64 / q0)
constexpr uint64_t BR1 = 73916747789ull;  // floor(2^64 / q1)
constexpr uint32_t Q0INV = 97389680u;     // q0^-1 mod q1

// Per-limb constants kept in __constant__ memory (filled by the host).
struct LimbConst {
    uint32_t q[2];
    uint64_t barrett[2];     // floor(2^64 / q_l)
    uint32_t q0_inv_mod_q1;  // Garner CRT coefficient
};

// exact x mod q for any 64-bit x (Barrett with floor(2^64/q), one correction)
__device__ __forceinline__ uint32_t mod64(uint64_t x, uint32_t q, uint64_t br) {
    uint64_t t = __umul64hi(x, br);
    uint64_t r = x - t * q;
    return (uint32_t)(r >= q ? r - q : r);
}

// Shoup multiply: y * w mod q in [0, 2q), wp = floor(w * 2^32 / q)
__device__ __forceinline__ uint32_t shoup_lazy(uint32_t y, uint32_t w, uint32_t wp, uint32_t q) {
    uint32_t qt = __umulhi(y, wp);
    return y * w - qt * q;
}

// CRT compose of canonical residues (x mod q0, y mod q1) -> value mod q0*q1 in
// [0, q): Garner form v = x + q0 * ((y - x) * q0^-1 mod q1).  Same canonical
// result as crt_compose_2 (core/params.rs:203-215), which is a unique CRT lift.
__device__ __forceinline__ uint64_t crt2(uint32_t x, uint32_t y, uint32_t q0inv, uint64_t br1) {
    uint32_t xm = x >= Q1 ? x - Q1 : x;            // x < q0 < 2*q1
    uint32_t d = y >= xm ? y - xm : y + Q1 - xm;   // (y - x) mod q1
    uint32_t k = mod64((uint64_t)d * q0inv, Q1, br1);
    return (uint64_t)x + (uint64_t)Q0 * k;
}

// Montgomery reduction with R = 2^32 (Montgomery, "Modular multiplication without trial
// division", 1985): for x < q R, x R^-1 mod q in [0, 2q) from one 32-bit and one 32x32->64
// multiply, against about six for a Barrett reduction of a 64-bit value.  The one-chain fold
// keeps its RGSW bodies and row 0 multiplied by R, so reducing a product with them leaves the
// plain product; the first-dimension GEMM's epilogue reduces its recombined sums the same way.
constexpr uint32_t neg_inv32(uint32_t q) {  // -q^-1 mod 2^32 for odd q (Newton iteration)
    uint32_t x = q;
    for (int i = 0; i < 5; i++) x *= 2u - q * x;
    return 0u - x;
}
constexpr uint32_t QNEG0 = neg_inv32(Q0), QNEG1 = neg_inv32(Q1);
constexpr uint32_t Q0INV_R = (uint32_t)(((uint64_t)Q0INV << 32) % Q1);  // q0^-1 R mod q1
__device__ __forceinline__ uint32_t redc(uint64_t x, uint32_t q) {
    const uint32_t m = (uint32_t)x * (q == Q0 ? QNEG0 : QNEG1);
    return (uint32_t)((x + (uint64_t)m * q) >> 32);
}
// any 64-bit v to [0, q) by one Montgomery reduction: with v = vh 2^32 + vl,
// x = vh (2^64 mod q) + vl (2^32 mod q) < 2 q 2^32 and redc(x) = v mod q in [0, 3q)
constexpr uint32_t R1_0 = (uint32_t)((1ull << 32) % Q0), R1_1 = (uint32_t)((1ull << 32) % Q1);
constexpr uint32_t R2_0 = (uint32_t)((uint64_t)R1_0 * R1_0 % Q0), R2_1 = (uint32_t)((uint64_t)R1_1 * R1_1 % Q1);
__device__ __forceinline__ uint32_t mod64m(uint64_t v, uint32_t q) {
    const uint64_t x = (uint64_t)(uint32_t)(v >> 32) * (q == Q0 ? R2_0 : R2_1) +
                       (uint64_t)(uint32_t)v * (q == Q0 ? R1_0 : R1_1);
    const uint32_t t = redc(x, q), t1 = min(t, t - 2 * q);
    return min(t1, t1 - q);
}

// w0 + 2^32 w1 (w0 < 2^64, w1 < 2^56) to [0, q) by one Montgomery reduction: with
// t = w1 + (w0 >> 32) = th 2^32 + tl, x = (w0 mod 2^32)(2^32 mod q) + tl (2^64 mod q)
// + th (2^96 mod q) < 2^62 and redc(x) = (w0 + 2^32 w1) mod q in [0, 4q)
constexpr uint32_t R3_0 = (uint32_t)((uint64_t)R2_0 * R1_0 % Q0), R3_1 = (uint32_t)((uint64_t)R2_1 * R1_1 % Q1);
__device__ __forceinline__ uint32_t mod96m(uint64_t w0, uint64_t w1, uint32_t q) {
    const uint64_t t = w1 + (w0 >> 32);
    const uint64_t x = (uint64_t)(uint32_t)w0 * (q == Q0 ? R1_0 : R1_1) +
                       (uint64_t)(uint32_t)t * (q == Q0 ? R2_0 : R2_1) + (t >> 32) * (q == Q0 ? R3_0 : R3_1);
    const uint32_t r = redc(x, q), r1 = min(r, r - 2 * q);
    return min(r1, r1 - q);
}

// crt2 with the Garner coefficient in Montgomery form: (y - x) q0^-1 mod q1 by one reduction
__device__ __forceinline__ uint64_t crt2m(uint32_t x, uint32_t y) {
    const uint32_t xm = x >= Q1 ? x - Q1 : x;            // x < q0 < 2 q1
    const uint32_t d = y >= xm ? y - xm : y + Q1 - xm;   // (y - x) mod q1
    const uint32_t kr = redc((uint64_t)d * Q0INV_R, Q1);  // d q0inv R < q1^2 < q1 R
    const uint32_t k = min(kr, kr - Q1);
    return (uint64_t)x + (uint64_t)Q0 * k;
}

// ---------------------------------------------------------------------------
// Shared-memory negacyclic NTTs over u32 residues, executed cooperatively by
// all threads of a CTA on `npoly` independent polynomials laid out at
// smem + p * N.  Twiddles: w/wp for forward (bit-reversed psi powers) and the
// pre-halved inverse tables, exactly the tables of build_ntt_tables
// (src/core/ntt.rs:74-108).  Butterflies are the Harvey forms of
// ntt_forward (ntt.rs:111-160) and ntt_inverse (ntt.rs:731-780); outputs are
// reduced to [0, q).  limb_of(p) selects the prime of polynomial p.
// ---------------------------------------------------------------------------
template <int NPOLY, typename LimbOf>
__device__ __forceinline__ void ntt_forward_smem(uint32_t* smem, const uint32_t* __restrict__ fw,
                                                 const uint32_t* __restrict__ fwp, LimbOf limb_of) {
#pragma unroll 1
    for (int mm = 0; mm < LOGN; mm++) {
        const int m = 1 << mm, t = N >> (mm + 1);
        for (int idx = threadIdx.x; idx < NPOLY * (N / 2); idx += blockDim.x) {
            const int p = idx >> (LOGN - 1);
            const int b = idx & (N / 2 - 1);
            const int i = b >> (LOGN - 1 - mm);        // b / t
            const int j = b & (t - 1);
            const int l = limb_of(p);
            const uint32_t q = l ? Q1 : Q0, two_q = 2 * q;
            const uint32_t w = __ldg(fw + l * N + m + i), wp = __ldg(fwp + l * N + m + i);
            uint32_t* o = smem + p * N + 2 * t * i + j;
            uint32_t x = o[0], y = o[t];
            x -= (x >= two_q) ? two_q : 0;
            uint32_t qn = shoup_lazy(y, w, wp, q);
            o[0] = x + qn;
            o[t] = x + two_q - qn;
        }
        __syncthreads();
    }
    for (int idx = threadIdx.x; idx < NPOLY * N; idx += blockDim.x) {
        const int l = limb_of(idx >> LOGN);
        const uint32_t q = l ? Q1 : Q0;
        uint32_t v = smem[idx];
        v -= (v >= 2 * q) ? 2 * q : 0;
        v -= (v >= q) ? q : 0;
        smem[idx] = v;
    }
    __syncthreads();
}

template <int NPOLY, typename LimbOf>
__device__ __forceinline__ void ntt_inverse_smem(uint32_t* smem, const uint32_t* __restrict__ iw,
                                                 const uint32_t* __restrict__ iwp, LimbOf limb_of) {
#pragma unroll 1
    for (int mm = LOGN - 1; mm >= 0; mm--) {
        const int h = 1 << mm, t = N >> (mm + 1);
        for (int idx = threadIdx.x; idx < NPOLY * (N / 2); idx += blockDim.x) {
            const int p = idx >> (LOGN - 1);
            const int b = idx & (N / 2 - 1);
            const int i = b >> (LOGN - 1 - mm);
            const int j = b & (t - 1);
            const int l = limb_of(p);
            const uint32_t q = l ? Q1 : Q0, two_q = 2 * q;
            const uint32_t w = __ldg(iw + l * N + h + i), wp = __ldg(iwp + l * N + h + i);
            uint32_t* o = smem + p * N + 2 * t * i + j;
            uint32_t x = o[0], y = o[t];
            uint32_t tt = two_q - y + x;
            uint32_t cx = x + y - ((2 * x >= tt) ? two_q : 0);
            uint32_t ht = __umulhi(tt, wp);
            o[0] = (cx + ((tt & 1) ? q : 0)) >> 1;
            o[t] = w * tt - ht * q;
        }
        __syncthreads();
    }
    for (int idx = threadIdx.x; idx < NPOLY * N; idx += blockDim.x) {
        const int l = limb_of(idx >> LOGN);
        const uint32_t q = l ? Q1 : Q0;
        uint32_t v = smem[idx];
        v -= (v >= 2 * q) ? 2 * q : 0;
        v -= (v >= q) ? q : 0;
        smem[idx] = v;
    }
    __syncthreads();
}

// slot of the forward NTT output that evaluates at psi^e (e odd):  the
// Cooley-Tukey order with bit-reversed twiddles leaves slot s holding the
// evaluation at psi^(2*brv(s)+1).
__device__ __forceinline__ uint32_t slot_of_exponent(uint32_t e) {
    return __brev((e - 1) >> 1) >> (32 - LOGN);
}
__device__ __forceinline__ uint32_t exponent_of_slot(uint32_t s) {
    return 2 * (__brev(s) >> (32 - LOGN)) + 1;
}

// NTT-domain Galois automorphism x -> x^t as a slot permutation:
// NTT(a(x^t))[s] = NTT(a)[auto_src(t, s)]  (closed form of
// generate_automorph_tables_brute_force, src/pir/packing.rs:1423-1468)
__device__ __forceinline__ uint32_t auto_src(uint32_t t, uint32_t s) {
    return slot_of_exponent((t * exponent_of_slot(s)) & (2 * N - 1));
}

}  // namespace ipr
