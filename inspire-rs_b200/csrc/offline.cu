// offline.cu — the offline precomputation of the InspiRING packing on the GPU: from the
// encoded DB to a_hat, bold_t, bold_t_bar, bold_t_hat (the arrays respond() streams).
//
// Restates PirServer::perform_offline_precomputation_simplepir (rkdud007/inspire-rs
// src/pir/server/engine.rs:677-1042) for gamma = N: per packing instance I (DB columns
// I*N .. I*N + N)
//   a_j   = NTT(negacyclic_perm(hint column I*N + j))              prep_pack_lwes, packing.rs:1032-1062
//           hint column = INTT(sum_row NTT(DB chunk) * query_row)  multiply_with_db_ring, engine.rs:434-498
//   r_i   = sum_j NTT(+-x^(j g'_i mod 2N)) * a_j,  g'_i = 5^((N-i) mod N)   packing.rs:2627-2679
//   r_all[i] = automorph(N^-1 r_i, 5^i),  r_bar_all[i] likewise with -j g'_i and 2N - 5^i
//   collapse over i = 1022 .. 0 (gadget digits, NTT, MAC with the rotated W mask)  packing.rs:2683-2734
//
// B200 design.  The reference forms r_i by brute force (2048 x 2048 products per slot and
// instance).  With E[s][z] = sum_j a_j[s] psi_z^j, the negacyclic NTT over j of the slot-s
// sequence, the sum collapses to a gather:
//   r_all[i][z] = N^-1 E[tau_{5^i}(z)][z],   r_bar_all[i][z] = N^-1 E[tau_{-5^i}(z)][z]
// (tau_t = the NTT-domain automorphism slot map; 5^i g'_i = 1 mod 2N).  So the whole packing
// sum is one NTT per (instance, limb, slot).  And since negacyclic_perm is x -> x^-1, a_j
// itself is the slot permutation tau_{-1} of NTT(DB column) * query: the hint's INTT/NTT
// pair cancels.  Kernels, per limb:
//   k_off_hint     column NTTs of the DB, * query, tau_{-1}          -> act[l][I][j][s]
//   k_off_jntt     NTT over j of 8 slots per CTA, * N^-1             -> E[l][I][s][z]
//   k_off_gather   per 8-column tile of E, the two slot gathers        -> F[I][chain][i][l][z]
//   k_off_collapse one CTA per (instance, chain): 1023 sequential steps of register NTTs
//   k_off_finish   bold_t_hat and a_hat per instance
// All values leave canonical, so the outputs equal the reference's bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <vector>

#include "host_math.hpp"
#include "ipr_b200.h"
#include "ipr_device.cuh"
#include "kernels.cuh"
#include "ntt_regs.cuh"

namespace ipr {
void set_last_error(const char* msg);

namespace {

using nttr::eA;
using nttr::eD;
using nttr::EPT;
constexpr int HALF = N / 2;   // packing outputs per instance (num_to_pack_half)
constexpr int HCOLS = 4;      // DB columns per CTA in k_off_hint
constexpr int JS = 8;         // slots per CTA in k_off_jntt
constexpr int GZ = 8;         // z columns per CTA in k_off_gather
constexpr uint64_t MASK19 = (1ull << GADGET_BITS) - 1;

__device__ __forceinline__ uint32_t limb_q(int g) { return g ? Q1 : Q0; }
__device__ __forceinline__ uint64_t limb_br(int g) { return g ? BR1 : BR0; }

// 5^i mod 2N (gen_pows, packing.rs:1645-1652)
__device__ __forceinline__ uint32_t gen_pow(uint32_t i) {
    uint32_t r = 1, b = 5;
    for (; i; i >>= 1, b = (b * b) & (2 * N - 1))
        if (i & 1) r = (r * b) & (2 * N - 1);
    return r;
}

// act[l][c][s] = tau_{-1}-permuted NTT_l(DB column c) * query, for chunk-local columns c.
// 512 threads: group g = threadIdx.x / 256 transforms limb g; HCOLS columns per CTA.
__global__ void __launch_bounds__(512, 1)
    k_off_hint(const uint16_t* __restrict__ db, int64_t db_rows, int64_t col0, int64_t ncols,
               const uint32_t* __restrict__ query, const uint32_t* __restrict__ fw, const uint32_t* __restrict__ fwp,
               uint32_t* __restrict__ act) {
    extern __shared__ uint32_t hsm[];  // [2 groups][HCOLS][N]
    const int g = threadIdx.x >> 8, t = threadIdx.x & 255;
    const uint32_t q = limb_q(g);
    const uint64_t br = limb_br(g);
    uint32_t* xbuf = hsm + g * HCOLS * N;
    const int64_t c0 = (int64_t)blockIdx.x * HCOLS;
    const int polys = (int)(db_rows / N);
    uint32_t acc[HCOLS][EPT];  // canonical running sum over the column's row polynomials
#pragma unroll
    for (int p = 0; p < HCOLS; p++)
#pragma unroll
        for (int m = 0; m < EPT; m++) acc[p][m] = 0;
    for (int row = 0; row < polys; row++) {
        uint32_t v[HCOLS][EPT];
#pragma unroll
        for (int p = 0; p < HCOLS; p++) {
            const bool live = c0 + p < ncols;
            const uint16_t* col = db + (col0 + (live ? c0 + p : 0)) * db_rows + (int64_t)row * N;
#pragma unroll
            for (int m = 0; m < EPT; m++) v[p][m] = live ? (uint32_t)__ldg(col + eA(t, m)) : 0u;
        }
        nttr::forward<HCOLS>(v, t, xbuf, 1 + g, fw + g * N, fwp + g * N, q);  // layout D, canonical
        const uint32_t* qr = query + ((int64_t)row * 2 + g) * N;
#pragma unroll
        for (int p = 0; p < HCOLS; p++)
#pragma unroll
            for (int m = 0; m < EPT; m++) acc[p][m] = mod64((uint64_t)v[p][m] * __ldg(qr + eD(t, m)) + acc[p][m], q, br);
    }
    // slot w = eD(t, m) holds V[w]; the permuted polynomial has V[w] at tau_{-1}(w) (an involution)
    nttr::group_bar(1 + g);
#pragma unroll
    for (int p = 0; p < HCOLS; p++)
#pragma unroll
        for (int m = 0; m < EPT; m++) xbuf[p * N + auto_src(2 * N - 1, eD(t, m))] = acc[p][m];
    nttr::group_bar(1 + g);
#pragma unroll
    for (int p = 0; p < HCOLS; p++) {
        if (c0 + p >= ncols) break;
        uint32_t* dst = act + ((int64_t)g * ncols + c0 + p) * N;
#pragma unroll
        for (int m = 0; m < EPT; m++) dst[eA(t, m)] = xbuf[p * N + eA(t, m)];
    }
}

// E[l][I][s][z] = N^-1 * NTT over j of act[l][I][j][s], JS consecutive slots per CTA.
// grid (N / JS, instances, 2 limbs), 256 threads
__global__ void __launch_bounds__(256)
    k_off_jntt(const uint32_t* __restrict__ act, int64_t inst, const uint32_t* __restrict__ fw,
               const uint32_t* __restrict__ fwp, uint32_t* __restrict__ E) {
    __shared__ __align__(16) uint32_t xbuf[4 * N];
    const int t = threadIdx.x;
    const int s0 = blockIdx.x * JS, l = blockIdx.z;
    const int64_t base = ((int64_t)l * inst + blockIdx.y) * N * N;
    const uint32_t q = limb_q(l);
    const uint64_t br = limb_br(l);
    uint32_t v[JS][EPT];
#pragma unroll
    for (int m = 0; m < EPT; m++) {
        const uint4* src = reinterpret_cast<const uint4*>(act + base + (int64_t)eA(t, m) * N + s0);
        const uint4 a = __ldg(src), b = __ldg(src + 1);
        v[0][m] = a.x; v[1][m] = a.y; v[2][m] = a.z; v[3][m] = a.w;
        v[4][m] = b.x; v[5][m] = b.y; v[6][m] = b.z; v[7][m] = b.w;
    }
    nttr::forward<JS, 4>(v, t, xbuf, 1, fw + l * N, fwp + l * N, q);
    const uint32_t ninv = l ? (uint32_t)(Q1 - (Q1 - 1) / N) : (uint32_t)(Q0 - (Q0 - 1) / N);  // N^-1 mod q_l
#pragma unroll
    for (int p = 0; p < JS; p++) {
        uint32_t o[EPT];
#pragma unroll
        for (int k = 0; k < EPT; k++) o[k] = mod64((uint64_t)v[p][k] * ninv, q, br);
        uint4* dst = reinterpret_cast<uint4*>(E + base + (int64_t)(s0 + p) * N + eD(t, 0));
        dst[0] = make_uint4(o[0], o[1], o[2], o[3]);
        dst[1] = make_uint4(o[4], o[5], o[6], o[7]);
    }
}

// F[I][chain][i][l][z] = E[l][I][tau(z)][z], tau = tau_{5^i} (chain 0) or tau_{-5^i} (chain 1),
// for a tile of GZ columns z.  grid (N / GZ, instances, 2 limbs), 256 threads, 64 KB dynamic smem
__global__ void __launch_bounds__(256)
    k_off_gather(const uint32_t* __restrict__ E, int64_t inst, uint32_t* __restrict__ F) {
    extern __shared__ __align__(16) uint32_t tile[];  // [N][GZ]
    const int t = threadIdx.x;
    const int z0 = blockIdx.x * GZ, l = blockIdx.z;
    const int64_t I = blockIdx.y;
    const uint32_t* src = E + ((int64_t)l * inst + I) * N * N + z0;
    for (int s = t; s < N; s += 256) {
        const uint4* p = reinterpret_cast<const uint4*>(src + (int64_t)s * N);
        const uint4 a = __ldg(p), b = __ldg(p + 1);
        *reinterpret_cast<uint4*>(&tile[s * GZ]) = a;
        *reinterpret_cast<uint4*>(&tile[s * GZ + 4]) = b;
    }
    __syncthreads();
    for (int idx = t; idx < HALF * GZ; idx += 256) {
        const int i = idx / GZ, zz = idx % GZ;
        const uint32_t z = (uint32_t)(z0 + zz), gi = gen_pow((uint32_t)i);
        F[(((I * 2 + 0) * HALF + i) * 2 + l) * N + z] = tile[auto_src(gi, z) * GZ + zz];
        F[(((I * 2 + 1) * HALF + i) * 2 + l) * N + z] = tile[auto_src(2 * N - gi, z) * GZ + zz];
    }
}

// smem of the collapse / finish kernels
struct CollapseSmem {
    uint64_t x[N];               // raw value of the chain (canonical mod q)
    uint32_t wm[3][2][N];        // W mask (collapse) or V mask (finish), NTT domain
    uint32_t xb[2][3][N];        // per limb group: NTT exchange buffers / limb staging
};

// digits of x in layout A for group-local thread t: v[k][m] = bits [19k, 19k + 19) of x[eA(t, m)]
// (gadget_invert_transposed_into, packing.rs:2740-2768)
__device__ __forceinline__ void digits(const uint64_t* x, int t, uint32_t (&v)[3][EPT]) {
#pragma unroll
    for (int m = 0; m < EPT; m++) {
        const uint64_t e = x[eA(t, m)];
#pragma unroll
        for (int k = 0; k < 3; k++) v[k][m] = (uint32_t)((e >> (GADGET_BITS * k)) & MASK19);
    }
}

// y (layout D, canonical limb g) -> raw x = CRT of both limbs, through the staging buffers;
// all 512 threads take part
__device__ __forceinline__ void to_raw(CollapseSmem& sm, uint32_t (&y)[1][EPT], int g, int t,
                                       const uint32_t* __restrict__ iw, const uint32_t* __restrict__ iwp) {
    const uint32_t q = limb_q(g);
    nttr::inverse<1, 1>(y, t, &sm.xb[g][0][0], 1 + g, iw + g * N, iwp + g * N, q);  // layout A, canonical
    __syncthreads();  // both groups are done with their exchange buffers
#pragma unroll
    for (int m = 0; m < EPT; m++) sm.xb[g][1][eA(t, m)] = y[0][m];
    __syncthreads();
    for (int e = threadIdx.x; e < N; e += 512) sm.x[e] = crt2(sm.xb[0][1][e], sm.xb[1][1][e], Q0INV, BR1);
    __syncthreads();
}

// one CTA per (instance, chain); chain 0 folds r_all with W rotated by 5^i into bold_t,
// chain 1 folds r_bar_all with W rotated by -5^i into bold_t_bar.  Leaves the final
// NTT-domain r_all[0] (chain 0) or raw(r_bar_all[0]) (chain 1) for k_off_finish.
// With wrows non-null the W row of step i is read from wrows[chain][i][k][l][z] instead of
// being rotated out of the mask (the reference's collapse takes w_all / w_bar_all as arrays).
__global__ void __launch_bounds__(512, 1)
    k_off_collapse(const uint32_t* __restrict__ F, int64_t inst0, const uint32_t* __restrict__ wmask,
                   const uint32_t* __restrict__ fw, const uint32_t* __restrict__ fwp, const uint32_t* __restrict__ iw,
                   const uint32_t* __restrict__ iwp, uint64_t* __restrict__ bt, uint64_t* __restrict__ btb,
                   uint32_t* __restrict__ r0, uint64_t* __restrict__ xbar0, const uint32_t* __restrict__ wrows) {
    extern __shared__ __align__(16) uint8_t csm_raw[];
    CollapseSmem& sm = *reinterpret_cast<CollapseSmem*>(csm_raw);
    const int g = threadIdx.x >> 8, t = threadIdx.x & 255;
    const int64_t I = blockIdx.x;
    const int chain = blockIdx.y;
    const uint32_t q = limb_q(g);
    const uint64_t br = limb_br(g);
    const uint32_t* Fc = F + (I * 2 + chain) * (int64_t)HALF * 2 * N;  // [i][l][z]
    uint32_t* out = reinterpret_cast<uint32_t*>((chain ? btb : bt) + (inst0 + I) * (int64_t)NINNER * N);
    if (!wrows)
        for (int e = threadIdx.x; e < 3 * 2 * N; e += 512) (&sm.wm[0][0][0])[e] = __ldg(wmask + e);
    const uint32_t* wr = wrows ? wrows + (int64_t)chain * NROT * 3 * 2 * N : nullptr;
    // x = raw(r_all[1023]): r_all[1023] is never updated (packing.rs:2691)
    uint32_t y[1][EPT];
    {
        const uint4* p = reinterpret_cast<const uint4*>(Fc + ((int64_t)(HALF - 1) * 2 + g) * N + eD(t, 0));
        const uint4 a = __ldg(p), b = __ldg(p + 1);
        y[0][0] = a.x; y[0][1] = a.y; y[0][2] = a.z; y[0][3] = a.w;
        y[0][4] = b.x; y[0][5] = b.y; y[0][6] = b.z; y[0][7] = b.w;
    }
    to_raw(sm, y, g, t, iw, iwp);
    for (int i = HALF - 2; i >= 0; i--) {
        uint32_t f[EPT];
        {
            const uint4* p = reinterpret_cast<const uint4*>(Fc + ((int64_t)i * 2 + g) * N + eD(t, 0));
            const uint4 a = __ldg(p), b = __ldg(p + 1);
            f[0] = a.x; f[1] = a.y; f[2] = a.z; f[3] = a.w;
            f[4] = b.x; f[5] = b.y; f[6] = b.z; f[7] = b.w;
        }
        uint32_t v[3][EPT];
        digits(sm.x, t, v);
        nttr::forward<3, 3>(v, t, &sm.xb[g][0][0], 1 + g, fw + g * N, fwp + g * N, q);  // layout D, canonical
        // bold_t[i][k] condensed: limb 0 in the low word, limb 1 in the high word (condense_matrix)
#pragma unroll
        for (int k = 0; k < 3; k++)
#pragma unroll
            for (int m = 0; m < EPT; m++) out[(((int64_t)i * 3 + k) * N + eD(t, m)) * 2 + g] = v[k][m];
        const uint32_t gi = gen_pow((uint32_t)i), ti = chain ? 2 * N - gi : gi;
#pragma unroll
        for (int m = 0; m < EPT; m++) {
            const uint32_t z = (uint32_t)eD(t, m);
            const uint32_t src = auto_src(ti, z);  // W rotated by t_i (apply_automorph_ntt)
            uint64_t acc = (uint64_t)f[m];
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const uint32_t w = wr ? __ldg(wr + (((int64_t)i * 3 + k) * 2 + g) * N + z) : sm.wm[k][g][src];
                acc += (uint64_t)w * v[k][m];  // < 2^31 + 3 q^2
            }
            y[0][m] = mod64(acc, q, br);
        }
        if (i == 0 && chain == 0) {  // r_all[0] stays in the NTT domain for k_off_finish
            uint4* d = reinterpret_cast<uint4*>(r0 + (I * 2 + g) * N + eD(t, 0));
            d[0] = make_uint4(y[0][0], y[0][1], y[0][2], y[0][3]);
            d[1] = make_uint4(y[0][4], y[0][5], y[0][6], y[0][7]);
            break;
        }
        __syncthreads();  // every thread has read sm.x for its digits
        to_raw(sm, y, g, t, iw, iwp);
    }
    if (chain == 1)
        for (int e = threadIdx.x; e < N; e += 512) xbar0[I * N + e] = sm.x[e];
}

// per instance: bold_t_hat = NTT(digits(raw(r_bar_all[0]))), a_hat = raw(r_all[0] + V * bold_t_hat)
// (packing.rs:2721-2734)
__global__ void __launch_bounds__(512, 1)
    k_off_finish(const uint32_t* __restrict__ r0, const uint64_t* __restrict__ xbar0, int64_t inst0,
                 const uint32_t* __restrict__ vmask, const uint32_t* __restrict__ fw, const uint32_t* __restrict__ fwp,
                 const uint32_t* __restrict__ iw, const uint32_t* __restrict__ iwp, uint64_t* __restrict__ bth,
                 uint64_t* __restrict__ a_hat) {
    extern __shared__ __align__(16) uint8_t fsm_raw[];
    CollapseSmem& sm = *reinterpret_cast<CollapseSmem*>(fsm_raw);
    const int g = threadIdx.x >> 8, t = threadIdx.x & 255;
    const int64_t I = blockIdx.x;
    const uint32_t q = limb_q(g);
    const uint64_t br = limb_br(g);
    for (int e = threadIdx.x; e < 3 * 2 * N; e += 512) (&sm.wm[0][0][0])[e] = __ldg(vmask + e);
    for (int e = threadIdx.x; e < N; e += 512) sm.x[e] = xbar0[I * N + e];
    __syncthreads();
    uint32_t v[3][EPT];
    digits(sm.x, t, v);
    nttr::forward<3, 3>(v, t, &sm.xb[g][0][0], 1 + g, fw + g * N, fwp + g * N, q);
    uint32_t* out = reinterpret_cast<uint32_t*>(bth + (inst0 + I) * 3 * (int64_t)N);
    uint32_t y[1][EPT];
#pragma unroll
    for (int m = 0; m < EPT; m++) {
        const int z = eD(t, m);
        uint64_t acc = r0[(I * 2 + g) * N + z];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            out[((int64_t)k * N + z) * 2 + g] = v[k][m];
            acc += (uint64_t)sm.wm[k][g][z] * v[k][m];
        }
        y[0][m] = mod64(acc, q, br);
    }
    __syncthreads();
    to_raw(sm, y, g, t, iw, iwp);
    for (int e = threadIdx.x; e < N; e += 512) a_hat[(inst0 + I) * N + e] = sm.x[e];
}

// act[l][c][i][s] = NTT_l(negacyclic_perm(a-vector of LWE i of set c)) (prep_pack_lwes,
// packing.rs:1032-1062) for LWE matrices lwe[c][N + 1][N] (row j = coefficient j of the 2048
// a-vectors, row N = the b values).  negacyclic_perm keeps coefficient 0 and puts
// q - a[N - k] at k >= 1; modulo q_l (q = 0 mod q_l) that is -a[N - k].
__global__ void __launch_bounds__(512, 1)
    k_lwe_prep(const uint64_t* __restrict__ lwe, int64_t sets, const uint32_t* __restrict__ fw,
               const uint32_t* __restrict__ fwp, uint32_t* __restrict__ act) {
    extern __shared__ uint32_t lsm[];  // [2 groups][HCOLS][N]
    const int g = threadIdx.x >> 8, t = threadIdx.x & 255;
    const uint32_t q = limb_q(g);
    const uint64_t br = limb_br(g);
    const int i0 = blockIdx.x * HCOLS;
    const int64_t c = blockIdx.y;
    const uint64_t* L = lwe + c * (int64_t)(N + 1) * N;
    uint32_t v[HCOLS][EPT];
#pragma unroll
    for (int m = 0; m < EPT; m++) {
        const int k = eA(t, m);
        const uint64_t* row = L + (int64_t)(k ? N - k : 0) * N + i0;
#pragma unroll
        for (int p = 0; p < HCOLS; p++) {
            const uint32_t x = mod64(__ldg(row + p), q, br);
            v[p][m] = (k == 0 || x == 0) ? x : q - x;
        }
    }
    nttr::forward<HCOLS>(v, t, lsm + g * HCOLS * N, 1 + g, fw + g * N, fwp + g * N, q);  // layout D, canonical
#pragma unroll
    for (int p = 0; p < HCOLS; p++) {
        uint4* dst = reinterpret_cast<uint4*>(act + (((int64_t)g * sets + c) * N + i0 + p) * N + eD(t, 0));
        dst[0] = make_uint4(v[p][0], v[p][1], v[p][2], v[p][3]);
        dst[1] = make_uint4(v[p][4], v[p][5], v[p][6], v[p][7]);
    }
}

// packed RLWE of set c: row 0 = a_hat, row 1 = b + raw(sum), the sum not reduced (add_raw,
// packing.rs:3011-3016)
__global__ void k_inspiring_out(const uint64_t* __restrict__ a_hat, const uint64_t* __restrict__ R,
                                const uint64_t* __restrict__ lwe, int64_t sets, uint64_t* __restrict__ out) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < sets * N; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = e / N, k = e % N;
        out[c * 2 * N + k] = a_hat[e];
        out[c * 2 * N + N + k] = lwe[(c * (N + 1) + N) * N + k] + R[e];
    }
}

// F[c][chain][i][l][z] (u32) from the reference's r_all / r_bar_all ([c][i][l*N + z] u64, canonical)
__global__ void k_off_to_f(const uint64_t* __restrict__ r_all, const uint64_t* __restrict__ r_bar_all, int64_t cols,
                           uint32_t* __restrict__ F) {
    const int64_t n = cols * HALF * 2 * N;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = e / ((int64_t)HALF * 2 * N), rest = e % ((int64_t)HALF * 2 * N);
        F[(c * 2 + 0) * (int64_t)HALF * 2 * N + rest] = (uint32_t)r_all[e];
        F[(c * 2 + 1) * (int64_t)HALF * 2 * N + rest] = (uint32_t)r_bar_all[e];
    }
}

// u64 [n] -> u32 [n] (canonical residues)
__global__ void k_narrow(const uint64_t* __restrict__ in, int64_t n, uint32_t* __restrict__ out) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
        out[e] = (uint32_t)in[e];
}

int cuda_fail(cudaError_t e, const char* what) {
    static thread_local char buf[256];
    snprintf(buf, sizeof(buf), "offline precomputation: %s: %s", what, cudaGetErrorString(e));
    set_last_error(buf);
    return e == cudaErrorMemoryAllocation ? IPR_E_OOM : IPR_E_CUDA;
}

}  // namespace

// The collapse of `cols` columns from the reference's r_all / r_bar_all arrays with explicit W
// rows (wrows = [2][1023][3][2][N] u32: w_all then w_bar_all) and the V mask ([3][2][N] u32):
// bold_t / bold_t_bar [cols][3069][N], bold_t_hat [cols][3][N] condensed, a_hat [cols][N].
// Scratch: F (cols * 32 MB), r0 (cols * 16 KB), xb (cols * 16 KB).
cudaError_t offline_collapse_arrays(const uint64_t* r_all, const uint64_t* r_bar_all, int64_t cols,
                                    const uint32_t* wrows, const uint32_t* vmask, const uint32_t* tab /*fw fwp iw iwp*/,
                                    uint32_t* F, uint32_t* r0, uint64_t* xb, uint64_t* bt, uint64_t* btb, uint64_t* bth,
                                    uint64_t* a_hat, cudaStream_t st) {
    const int coll_smem = (int)sizeof(CollapseSmem);
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k_off_collapse, cudaFuncAttributeMaxDynamicSharedMemorySize, coll_smem)) ||
        (e = cudaFuncSetAttribute(k_off_finish, cudaFuncAttributeMaxDynamicSharedMemorySize, coll_smem)))
        return e;
    const uint32_t *fw = tab, *fwp = tab + 2 * N, *iw = tab + 4 * N, *iwp = tab + 6 * N;
    k_off_to_f<<<148 * 8, 256, 0, st>>>(r_all, r_bar_all, cols, F);
    k_off_collapse<<<dim3((unsigned)cols, 2), 512, coll_smem, st>>>(F, 0, nullptr, fw, fwp, iw, iwp, bt, btb, r0, xb,
                                                                   wrows);
    k_off_finish<<<(unsigned)cols, 512, coll_smem, st>>>(r0, xb, 0, vmask, fw, fwp, iw, iwp, bth, a_hat);
    return cudaGetLastError();
}

// E[l][I][s][z] = N^-1 * NTT over j of act[l][I][j][s] for `inst` instances
cudaError_t offline_jntt(const uint32_t* act, int64_t inst, const uint32_t* fw, const uint32_t* fwp, uint32_t* E,
                         cudaStream_t st) {
    k_off_jntt<<<dim3(N / JS, (unsigned)inst, 2), 256, 0, st>>>(act, inst, fw, fwp, E);
    return cudaGetLastError();
}

cudaError_t narrow_u64(const uint64_t* in, int64_t n, uint32_t* out, cudaStream_t st) {
    k_narrow<<<148 * 4, 256, 0, st>>>(in, n, out);
    return cudaGetLastError();
}

// scratch bytes per instance: act / F (32 MB) + E (32 MB) + the chain ends (32 KB)
constexpr uint64_t kOfflineScratchPerInstance = 2ull * 2 * N * N * 4 + 2ull * N * 4 + (uint64_t)N * 8;

int offline_precompute_device(const uint16_t* d_db, uint64_t db_rows, uint64_t instances, uint64_t* d_a_hat,
                              uint64_t* d_bt, uint64_t* d_btb, uint64_t* d_bth, uint64_t scratch_budget,
                              cudaStream_t st) {
    if (!d_db || !d_a_hat || !d_bt || !d_btb || !d_bth || !instances || !db_rows || db_rows % N ||
        db_rows > (1u << 20) || instances > (1u << 20)) {
        set_last_error("offline precomputation: db_rows must be a positive multiple of 2048, instances > 0");
        return IPR_E_ARGS;
    }
    HostParams hp;
    host_params_init(hp);
    std::vector<uint32_t> query, wmask, vmask;
    offline_host_inputs(hp, (unsigned)(db_rows / N), query, wmask, vmask);
    // chunk of instances per pass, bounded by the scratch budget (0 = 4 GiB)
    const uint64_t budget = scratch_budget ? scratch_budget : (4ull << 30);
    const uint64_t chunk = std::max<uint64_t>(1, std::min<uint64_t>(instances, budget / kOfflineScratchPerInstance));
    uint32_t *d_tab = nullptr, *d_query = nullptr, *d_wv = nullptr, *d_act = nullptr, *d_E = nullptr, *d_r0 = nullptr;
    uint64_t* d_xb = nullptr;
    auto release = [&]() {
        for (void* p : {(void*)d_tab, (void*)d_query, (void*)d_wv, (void*)d_act, (void*)d_E, (void*)d_r0, (void*)d_xb})
            if (p) cudaFree(p);
    };
    cudaError_t e;
    const size_t tb = 2 * N * sizeof(uint32_t);
    if ((e = cudaMalloc(&d_tab, 4 * tb)) != cudaSuccess || (e = cudaMalloc(&d_query, query.size() * 4)) != cudaSuccess ||
        (e = cudaMalloc(&d_wv, 2 * wmask.size() * 4)) != cudaSuccess ||
        (e = cudaMalloc(&d_act, chunk * 2ull * N * N * 4)) != cudaSuccess ||
        (e = cudaMalloc(&d_E, chunk * 2ull * N * N * 4)) != cudaSuccess ||
        (e = cudaMalloc(&d_r0, chunk * 2ull * N * 4)) != cudaSuccess ||
        (e = cudaMalloc(&d_xb, chunk * (uint64_t)N * 8)) != cudaSuccess) {
        release();
        return cuda_fail(e, "scratch allocation");
    }
    uint32_t *d_fw = d_tab, *d_fwp = d_tab + 2 * N, *d_iw = d_tab + 4 * N, *d_iwp = d_tab + 6 * N;
    uint32_t *d_wm = d_wv, *d_vm = d_wv + wmask.size();
    int status = IPR_OK;
    do {
        if ((e = cudaMemcpyAsync(d_fw, hp.fw.data(), tb, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
            (e = cudaMemcpyAsync(d_fwp, hp.fwp.data(), tb, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
            (e = cudaMemcpyAsync(d_iw, hp.iw.data(), tb, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
            (e = cudaMemcpyAsync(d_iwp, hp.iwp.data(), tb, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
            (e = cudaMemcpyAsync(d_query, query.data(), query.size() * 4, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
            (e = cudaMemcpyAsync(d_wm, wmask.data(), wmask.size() * 4, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
            (e = cudaMemcpyAsync(d_vm, vmask.data(), vmask.size() * 4, cudaMemcpyHostToDevice, st)) != cudaSuccess) {
            status = cuda_fail(e, "table upload");
            break;
        }
        const int hint_smem = 2 * HCOLS * N * 4, gather_smem = N * GZ * 4, coll_smem = (int)sizeof(CollapseSmem);
        if ((e = cudaFuncSetAttribute(k_off_hint, cudaFuncAttributeMaxDynamicSharedMemorySize, hint_smem)) ||
            (e = cudaFuncSetAttribute(k_off_gather, cudaFuncAttributeMaxDynamicSharedMemorySize, gather_smem)) ||
            (e = cudaFuncSetAttribute(k_off_collapse, cudaFuncAttributeMaxDynamicSharedMemorySize, coll_smem)) ||
            (e = cudaFuncSetAttribute(k_off_finish, cudaFuncAttributeMaxDynamicSharedMemorySize, coll_smem))) {
            status = cuda_fail(e, "kernel attributes");
            break;
        }
        for (uint64_t i0 = 0; i0 < instances && status == IPR_OK; i0 += chunk) {
            const int64_t c = (int64_t)std::min<uint64_t>(chunk, instances - i0);
            const int64_t ncols = c * N;
            k_off_hint<<<(unsigned)((ncols + HCOLS - 1) / HCOLS), 512, hint_smem, st>>>(
                d_db, (int64_t)db_rows, (int64_t)i0 * N, ncols, d_query, d_fw, d_fwp, d_act);
            k_off_jntt<<<dim3(N / JS, (unsigned)c, 2), 256, 0, st>>>(d_act, c, d_fw, d_fwp, d_E);
            k_off_gather<<<dim3(N / GZ, (unsigned)c, 2), 256, gather_smem, st>>>(d_E, c, d_act);  // F reuses act
            k_off_collapse<<<dim3((unsigned)c, 2), 512, coll_smem, st>>>(d_act, (int64_t)i0, d_wm, d_fw, d_fwp, d_iw,
                                                                       d_iwp, d_bt, d_btb, d_r0, d_xb, nullptr);
            k_off_finish<<<(unsigned)c, 512, coll_smem, st>>>(d_r0, d_xb, (int64_t)i0, d_vm, d_fw, d_fwp, d_iw, d_iwp,
                                                              d_bth, d_a_hat);
            if ((e = cudaGetLastError()) != cudaSuccess) status = cuda_fail(e, "launch");
        }
        if (status == IPR_OK && (e = cudaStreamSynchronize(st)) != cudaSuccess) status = cuda_fail(e, "run");
    } while (false);
    cudaStreamSynchronize(st);
    release();
    return status;
}

}  // namespace ipr

extern "C" int ipr_offline_precompute(int device, const uint16_t* d_db, uint64_t db_rows, uint64_t instances,
                                      uint64_t* d_a_hat, uint64_t* d_bold_t, uint64_t* d_bold_t_bar,
                                      uint64_t* d_bold_t_hat, uint64_t scratch_bytes, void* stream) {
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        ipr::set_last_error(cudaGetErrorString(e));
        return IPR_E_CUDA;
    }
    return ipr::offline_precompute_device(d_db, db_rows, instances, d_a_hat, d_bold_t, d_bold_t_bar, d_bold_t_hat,
                                          scratch_bytes, static_cast<cudaStream_t>(stream));
}

// ---------------------------------------------------------------------------
// InspiRING packing of LWE sets (packing_fully_online, packing.rs:3122-3162): the offline
// kernels above on the sets' own a-vectors, then the online packing sum and INTT of the
// respond() path (k_pack, k_intt_crt) with the caller's packing keys.
// ---------------------------------------------------------------------------
struct ipr_inspiring {
    int device = 0;
    int max_sets = 0;
    std::vector<void*> allocs;
    uint32_t *fw = nullptr, *fwp = nullptr, *iw = nullptr, *iwp = nullptr, *wm = nullptr, *vm = nullptr;
    uint32_t *act = nullptr, *E = nullptr, *r0 = nullptr, *S = nullptr;
    uint64_t *xb = nullptr, *a_hat = nullptr, *bt = nullptr, *btb = nullptr, *bth = nullptr, *R = nullptr;
    template <typename T>
    cudaError_t alloc(T** p, size_t bytes) {
        void* v = nullptr;
        cudaError_t e = cudaMalloc(&v, bytes);
        if (e == cudaSuccess) allocs.push_back(v), *p = static_cast<T*>(v);
        return e;
    }
};

extern "C" {

void ipr_inspiring_destroy(ipr_inspiring* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    for (void* p : ctx->allocs) cudaFree(p);
    delete ctx;
}

int ipr_inspiring_create(int device, int max_sets, ipr_inspiring** out) {
    if (!out || max_sets < 1 || max_sets > 1024) {
        ipr::set_last_error("ipr_inspiring_create: max_sets must be in [1, 1024]");
        return IPR_E_ARGS;
    }
    *out = nullptr;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return ipr::cuda_fail(e, "set device");
    auto* c = new ipr_inspiring();
    c->device = device;
    c->max_sets = max_sets;
    ipr::HostParams hp;
    ipr::host_params_init(hp);
    std::vector<uint32_t> query, wmask, vmask;
    ipr::offline_host_inputs(hp, 1, query, wmask, vmask);
    const size_t tb = 2 * ipr::N * 4, ms = (size_t)max_sets, NN = (size_t)ipr::N * ipr::N;
    if ((e = c->alloc(&c->fw, tb)) || (e = c->alloc(&c->fwp, tb)) || (e = c->alloc(&c->iw, tb)) ||
        (e = c->alloc(&c->iwp, tb)) || (e = c->alloc(&c->wm, wmask.size() * 4)) ||
        (e = c->alloc(&c->vm, vmask.size() * 4)) || (e = c->alloc(&c->act, ms * 2 * NN * 4)) ||
        (e = c->alloc(&c->E, ms * 2 * NN * 4)) || (e = c->alloc(&c->r0, ms * 2 * ipr::N * 4)) ||
        (e = c->alloc(&c->xb, ms * ipr::N * 8)) || (e = c->alloc(&c->a_hat, ms * ipr::N * 8)) ||
        (e = c->alloc(&c->bt, ms * ipr::NINNER * ipr::N * 8)) || (e = c->alloc(&c->btb, ms * ipr::NINNER * ipr::N * 8)) ||
        (e = c->alloc(&c->bth, ms * 3 * ipr::N * 8)) || (e = c->alloc(&c->S, ms * 2 * ipr::N * 4)) ||
        (e = c->alloc(&c->R, ms * ipr::N * 8)) ||
        (e = cudaMemcpy(c->fw, hp.fw.data(), tb, cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy(c->fwp, hp.fwp.data(), tb, cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy(c->iw, hp.iw.data(), tb, cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy(c->iwp, hp.iwp.data(), tb, cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy(c->wm, wmask.data(), wmask.size() * 4, cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy(c->vm, vmask.data(), vmask.size() * 4, cudaMemcpyHostToDevice)) ||
        (e = ipr::init_device_kernels()) || (e = ipr::set_constants(hp.barrett, hp.q0_inv_mod_q1)) ||
        (e = cudaFuncSetAttribute(ipr::k_lwe_prep, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * ipr::HCOLS * ipr::N * 4)) ||
        (e = cudaFuncSetAttribute(ipr::k_off_gather, cudaFuncAttributeMaxDynamicSharedMemorySize, ipr::N * ipr::GZ * 4)) ||
        (e = cudaFuncSetAttribute(ipr::k_off_collapse, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sizeof(ipr::CollapseSmem))) ||
        (e = cudaFuncSetAttribute(ipr::k_off_finish, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sizeof(ipr::CollapseSmem)))) {
        ipr_inspiring_destroy(c);
        return ipr::cuda_fail(e, "ipr_inspiring_create");
    }
    *out = c;
    return IPR_OK;
}

int ipr_inspiring_pack(ipr_inspiring* c, int sets, const uint64_t* d_lwe, const uint64_t* d_y_body,
                       const uint64_t* d_z_body, uint64_t* d_out, void* stream) {
    if (!c || !d_lwe || !d_y_body || !d_z_body || !d_out || sets < 1 || sets > c->max_sets) {
        ipr::set_last_error("ipr_inspiring_pack: null argument or sets outside [1, max_sets]");
        return IPR_E_ARGS;
    }
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return ipr::cuda_fail(e, "set device");
    using namespace ipr;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int coll_smem = (int)sizeof(CollapseSmem);
    k_lwe_prep<<<dim3(N / HCOLS, (unsigned)sets), 512, 2 * HCOLS * N * 4, st>>>(d_lwe, sets, c->fw, c->fwp, c->act);
    k_off_jntt<<<dim3(N / JS, (unsigned)sets, 2), 256, 0, st>>>(c->act, sets, c->fw, c->fwp, c->E);
    k_off_gather<<<dim3(N / GZ, (unsigned)sets, 2), 256, N * GZ * 4, st>>>(c->E, sets, c->act);
    k_off_collapse<<<dim3((unsigned)sets, 2), 512, coll_smem, st>>>(c->act, 0, c->wm, c->fw, c->fwp, c->iw, c->iwp,
                                                                   c->bt, c->btb, c->r0, c->xb, nullptr);
    k_off_finish<<<(unsigned)sets, 512, coll_smem, st>>>(c->r0, c->xb, 0, c->vm, c->fw, c->fwp, c->iw, c->iwp, c->bth,
                                                         c->a_hat);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "offline kernels");
    if ((e = launch_pack(c->bt, c->btb, c->bth, d_y_body, d_z_body, c->S, sets, st)) != cudaSuccess ||
        (e = launch_intt_crt(c->S, c->iw, c->iwp, c->R, sets, st)) != cudaSuccess)
        return cuda_fail(e, "online kernels");
    k_inspiring_out<<<148, 256, 0, st>>>(c->a_hat, c->R, d_lwe, sets, d_out);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "output");
    return IPR_OK;
}

}  // extern "C"
