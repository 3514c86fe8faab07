// client.cu — the keyword-PIR client on the GPU: query generation and response
// decryption of rkdud007/inspire-rs's KeywordClient (src/pir/client/keyword.rs).
//
// A query payload (serialize_keyword_query, src/protocol/wire.rs:542-615) holds
//   * the packing keys y_k, z_k (PackingKeys::init_full, src/pir/packing.rs:1895-1943;
//     generate_ksk_body, packing.rs:3272-3293): NTT(e + tau_g(s) 2^(19k)) - s * mask_k,
//     g = 5 with the W mask and g = 2N - 1 with the V mask;
//   * per sub-query the first-dimension row (generate_query_impl, client/online.rs:216-287,
//     scaled-Regev samples under the public seed, only their b values kept): the raw
//     polynomial s * a_r + e + Delta X^(row mod N) in the polynomial r = row / N;
//   * per sub-query 6 RGSW bodies (build_query_for_index, client/keyword.rs:137-191):
//     column 2j+1 encrypts sigma_j = +-2^(19j) X^(e mod N), column 2j encrypts s * sigma_j,
//     each NTT(e + msg) + s * a with a from RGSW_SEEDS (all equal, wire.rs:88-113).
// s * a for the public polynomials and -s * mask are fixed per client and computed at
// creation, so a payload costs 6 + 6 nq forward NTTs per limb on the device.
//
// Randomness is deterministic in the client's 32-byte seed: the ternary secret key (256
// coefficients +1 and 256 -1, gen_ternary_mat, client/base.rs:126-139) is placed by a
// Fisher-Yates shuffle driven by ChaCha20(seed, stream 1); noise coefficient g of a call
// with nonce n is a centered binomial sample with eta = 82 (variance 41, sigma 6.40, the
// width of the reference's discrete Gaussian, s = 16.042421 = 6.4 sqrt(2 pi)) from ChaCha20
// block g of stream 2 + n: popcount of 82 bits minus popcount of 82 others.
//
// Decryption (decrypt_response_values, client/keyword.rs:193-226): recover_how_many
// (pir/modulus_switch.rs:102-130) rescales the 28-bit row-0 and 20-bit row-1 fields back
// to q, then s * row0 + row1 (decrypt_matrix_reg, client/base.rs:525-527) and rescale to
// the plaintext modulus 65535 (decrypt_ct_reg_measured, client/online.rs:118-135).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "host_math.hpp"
#include "ipr_b200.h"
#include "ipr_device.cuh"

namespace ipr {
void set_last_error(const char* msg);
}

namespace {

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    ipr::set_last_error(buf);
    return code;
}

using ipr::N;
using ipr::Q0;
using ipr::Q1;
using ipr::QQ;

constexpr int KEY_POLYS = 6;     // y_0..2, z_0..2
constexpr int GSW_COLS = 6;      // 2 t_gsw
constexpr int HAMMING = 256;     // HAMMING_WEIGHT (client/base.rs:14)
constexpr int CBD_BITS = 82;     // eta: variance 41 = 6.40^2

__device__ __forceinline__ uint32_t rotl32(uint32_t x, int n) { return (x << n) | (x >> (32 - n)); }

// ChaCha20 block (RFC 8439 rounds) in rand_chacha's word layout: 64-bit block counter in
// words 12-13, 64-bit stream id in words 14-15
__device__ void chacha_block(const uint32_t* key, uint64_t counter, uint64_t stream, uint32_t out[16]) {
    uint32_t s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u, key[0], key[1], key[2], key[3],
                      key[4], key[5], key[6], key[7], (uint32_t)counter, (uint32_t)(counter >> 32),
                      (uint32_t)stream, (uint32_t)(stream >> 32)};
    uint32_t x[16];
#pragma unroll
    for (int i = 0; i < 16; i++) x[i] = s[i];
#define QR(a, b, c, d)                                \
    x[a] += x[b]; x[d] = rotl32(x[d] ^ x[a], 16);     \
    x[c] += x[d]; x[b] = rotl32(x[b] ^ x[c], 12);     \
    x[a] += x[b]; x[d] = rotl32(x[d] ^ x[a], 8);      \
    x[c] += x[d]; x[b] = rotl32(x[b] ^ x[c], 7);
#pragma unroll
    for (int r = 0; r < 10; r++) {
        QR(0, 4, 8, 12) QR(1, 5, 9, 13) QR(2, 6, 10, 14) QR(3, 7, 11, 15)
        QR(0, 5, 10, 15) QR(1, 6, 11, 12) QR(2, 7, 8, 13) QR(3, 4, 9, 14)
    }
#undef QR
#pragma unroll
    for (int i = 0; i < 16; i++) out[i] = x[i] + s[i];
}

// centered binomial noise coefficient g of stream `stream`: words 0, 1 and the low 18 bits of
// word 2 against words 3, 4 and the low 18 bits of word 5 of ChaCha20 block g
__device__ __forceinline__ int cbd_sample(const uint32_t* key, uint64_t stream, uint64_t g) {
    uint32_t w[16];
    chacha_block(key, g, stream, w);
    const uint32_t m = (1u << (CBD_BITS - 64)) - 1;
    return (__popc(w[0]) + __popc(w[1]) + __popc(w[2] & m)) - (__popc(w[3]) + __popc(w[4]) + __popc(w[5] & m));
}

__device__ __forceinline__ uint32_t signed_mod(int64_t v, uint32_t q) {
    int64_t r = v % (int64_t)q;
    return (uint32_t)(r < 0 ? r + q : r);
}

__device__ __forceinline__ uint32_t addmod(uint32_t a, uint32_t b, uint32_t q) {
    uint32_t s = a + b;
    return s >= q ? s - q : s;
}

__device__ __forceinline__ uint32_t mulmod32(uint32_t a, uint32_t b, uint32_t q, uint64_t br) {
    return ipr::mod64((uint64_t)a * b, q, br);
}

// rescale (src/core/arith.rs:436-452): round(a * out / inp) with the input centred in
// (-inp/2, inp/2] and the result taken mod out
__device__ __forceinline__ uint64_t rescale_any(uint64_t a, uint64_t inp, uint64_t out) {
    const uint64_t av = a % inp, half = inp / 2;
    const bool neg = av >= half;
    const uint64_t u = neg ? inp - av : av;
    const unsigned __int128 num = (unsigned __int128)u * out + half;
    const uint64_t r = (uint64_t)(num / inp), rm = r % out;
    return neg ? (rm ? out - rm : 0) : rm;
}

struct BuildArgs {
    const uint32_t* key;        // [8] ChaCha key (the client seed)
    uint64_t stream;            // 2 + nonce
    int n, rpolys, interp;      // sub-queries, db_rows / N, interpolation degree
    int64_t db_rows;
    const int8_t* s;            // [N] secret key
    const int8_t* tau;          // [2][N] tau_5(s), tau_{2N-1}(s)
    const uint32_t* sa_row;     // [rpolys][2][N] raw residues of s * a_r
    const int64_t* targets;     // [n][2] (row, sub-column)
    uint64_t* limb0;            // [6 + 6n][N] residues to transform, limb 0
    uint64_t* limb1;
    uint64_t* fields;           // 56-bit wire fields of the payload
};

// One thread per noise coefficient.  Noise polys: the 6 keys, then per sub-query its
// rpolys row polys and its 6 RGSW columns in the order 1, 0, 3, 2, 5, 4 (the reference
// encrypts sigma_j before s * sigma_j).
__global__ void k_client_build(BuildArgs a) {
    __shared__ uint32_t key[8];
    if (threadIdx.x < 8) key[threadIdx.x] = a.key[threadIdx.x];
    __syncthreads();
    const int per_q = a.rpolys + GSW_COLS;
    const int64_t total = (int64_t)(KEY_POLYS + a.n * per_q) * N;
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < total;
         g += (int64_t)gridDim.x * blockDim.x) {
        const int p = (int)(g / N), i = (int)(g % N);
        const int e = cbd_sample(key, a.stream, (uint64_t)g);
        int64_t term = 0;  // message term of coefficient i (a small multiple of a gadget power)
        int64_t dst = -1;  // transformed poly index, or -1 for a row poly
        int64_t field = -1;
        if (p < KEY_POLYS) {
            const int which = p / 3, k = p % 3;
            term = (int64_t)a.tau[which * N + i] * ((int64_t)1 << (ipr::GADGET_BITS * k));
            dst = p;
        } else {
            const int q = (p - KEY_POLYS) / per_q, r = (p - KEY_POLYS) % per_q;
            const int64_t row = a.targets[2 * q], sub = a.targets[2 * q + 1];
            if (r < a.rpolys) {
                const uint64_t m = (r == row / N && i == row % N) ? QQ / ipr::PT : 0;
                const uint32_t* sa = a.sa_row + (int64_t)r * 2 * N;
                const uint32_t v0 = addmod(addmod(sa[i], signed_mod(e, Q0), Q0), (uint32_t)(m % Q0), Q0);
                const uint32_t v1 = addmod(addmod(sa[N + i], signed_mod(e, Q1), Q1), (uint32_t)(m % Q1), Q1);
                field = KEY_POLYS * N + (int64_t)q * (a.db_rows + GSW_COLS * N) + (int64_t)r * N + i;
                a.fields[field] = (uint64_t)v0 | ((uint64_t)v1 << 28);
                continue;
            }
            const int col = (r - a.rpolys) ^ 1, j = col >> 1;
            const int ex = (int)((2 * N * sub / a.interp) % (2 * N));
            const int pos = ex % N;
            const int64_t sgn = ex < N ? 1 : -1, g2 = (int64_t)1 << (ipr::GADGET_BITS * j);
            if (col & 1) {
                term = i == pos ? sgn * g2 : 0;  // sigma_j
            } else {                             // s * sigma_j = +-2^(19j) X^pos s, negacyclic
                const int si = i >= pos ? a.s[i - pos] : -a.s[i - pos + N];
                term = sgn * g2 * si;
            }
            dst = KEY_POLYS + (int64_t)q * GSW_COLS + col;
        }
        a.limb0[dst * N + i] = signed_mod((int64_t)e + term, Q0);
        a.limb1[dst * N + i] = signed_mod((int64_t)e + term, Q1);
    }
}

// fields of the transformed polys: keys y_k / z_k (+ -s * mask), RGSW bodies (+ s * a)
__global__ void k_client_finish(const uint64_t* __restrict__ limb0, const uint64_t* __restrict__ limb1, int n,
                                int64_t db_rows, const uint32_t* __restrict__ neg_sm,
                                const uint32_t* __restrict__ sa_gsw, uint64_t* __restrict__ fields) {
    const int64_t total = (int64_t)(KEY_POLYS + GSW_COLS * n) * N;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int pp = (int)(t / N), z = (int)(t % N);
        const uint32_t* add;
        int64_t field;
        if (pp < KEY_POLYS) {
            const int which = pp / 3, k = pp % 3;
            add = neg_sm + ((int64_t)(which * 3 + k) * 2) * N;
            field = 2 * ((int64_t)k * N + z) + which;  // y and z interleaved per (column, slot)
        } else {
            const int q = (pp - KEY_POLYS) / GSW_COLS, c = (pp - KEY_POLYS) % GSW_COLS;
            add = sa_gsw;
            field = KEY_POLYS * N + (int64_t)q * (db_rows + GSW_COLS * N) + db_rows + (int64_t)c * N + z;
        }
        const uint32_t v0 = addmod((uint32_t)limb0[t], add[z], Q0);
        const uint32_t v1 = addmod((uint32_t)limb1[t], add[N + z], Q1);
        fields[field] = (uint64_t)v0 | ((uint64_t)v1 << 28);
    }
}

// 1 count byte, then every field as 7 little-endian bytes
__global__ void k_client_serialize(const uint64_t* __restrict__ fields, int64_t nfields, int n,
                                   uint8_t* __restrict__ out) {
    const int64_t f0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (f0 == 0) out[0] = (uint8_t)n;
    for (int64_t f = f0; f < nfields; f += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t v = fields[f];
#pragma unroll
        for (int b = 0; b < 7; b++) out[1 + 7 * f + b] = (uint8_t)(v >> (8 * b));
    }
}

__device__ __forceinline__ uint64_t read_bits_dev(const uint8_t* buf, int64_t bit, int nbits) {
    const int64_t byte = bit >> 3;
    const int sh = (int)(bit & 7), nbytes = (sh + nbits + 7) >> 3;  // at most 5 bytes, all inside the field
    uint64_t v = 0;
    for (int b = 0; b < nbytes; b++) v |= (uint64_t)buf[byte + b] << (8 * b);
    return (v >> sh) & ((1ull << nbits) - 1);
}

// recover_how_many: result r's row 0 (28-bit fields, rescaled from q'_2) goes to the limb
// arrays for the transform, row 1 (20-bit fields, from q'_1) is kept as residues
__global__ void k_client_unpack(const uint8_t* __restrict__ resp, const int64_t* __restrict__ offsets, int nres,
                                uint64_t* __restrict__ limb0, uint64_t* __restrict__ limb1,
                                uint32_t* __restrict__ row1) {
    const int64_t total = (int64_t)nres * N;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(t / N), i = (int)(t % N);
        const uint8_t* c = resp + offsets[r];
        const uint64_t v0 = rescale_any(read_bits_dev(c, 28LL * i, 28), ipr::QP2, QQ);
        const uint64_t v1 = rescale_any(read_bits_dev(c, 28LL * N + 20LL * i, 20), ipr::QP1, QQ);
        limb0[t] = v0 % Q0;
        limb1[t] = v0 % Q1;
        row1[(int64_t)r * 2 * N + i] = (uint32_t)(v1 % Q0);
        row1[(int64_t)r * 2 * N + N + i] = (uint32_t)(v1 % Q1);
    }
}

__global__ void k_client_mul_s(uint64_t* __restrict__ limb0, uint64_t* __restrict__ limb1, int nres,
                               const uint32_t* __restrict__ s_ntt) {
    const int64_t total = (int64_t)nres * N;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int z = (int)(t % N);
        limb0[t] = mulmod32((uint32_t)limb0[t], s_ntt[z], Q0, ipr::BR0);
        limb1[t] = mulmod32((uint32_t)limb1[t], s_ntt[N + z], Q1, ipr::BR1);
    }
}

// s * row0 (back in coefficients) + row1, CRT to [0, q), rescale to 65535
__global__ void k_client_decode(const uint64_t* __restrict__ limb0, const uint64_t* __restrict__ limb1,
                                const uint32_t* __restrict__ row1, int nres, uint16_t* __restrict__ out) {
    const int64_t total = (int64_t)nres * N;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(t / N), i = (int)(t % N);
        const uint32_t d0 = addmod((uint32_t)limb0[t], row1[(int64_t)r * 2 * N + i], Q0);
        const uint32_t d1 = addmod((uint32_t)limb1[t], row1[(int64_t)r * 2 * N + N + i], Q1);
        const uint64_t raw = ipr::crt2(d0, d1, ipr::Q0INV, ipr::BR1);
        out[t] = (uint16_t)rescale_any(raw, QQ, ipr::PT);
    }
}

unsigned grid_for(int64_t work) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>((work + 255) / 256, 148 * 16)); }

}  // namespace

struct ipr_client {
    int device = 0;
    cudaStream_t stream = nullptr;
    ipr_plan plan{};
    uint64_t per = 0, item_elems = 0;
    int rpolys = 0;
    uint32_t key[8];
    int8_t s[N];
    // device state fixed per client
    uint32_t* d_key = nullptr;
    int8_t* d_s = nullptr;        // [N]
    int8_t* d_tau = nullptr;      // [2][N]
    uint32_t* d_s_ntt = nullptr;  // [2][N]
    uint32_t* d_sa_row = nullptr; // [rpolys][2][N]
    uint32_t* d_sa_gsw = nullptr; // [2][N]
    uint32_t* d_neg_sm = nullptr; // [2][3][2][N]
    // scratch, grown on demand
    uint64_t* d_limb[2] = {nullptr, nullptr};
    size_t limb_polys = 0;
    uint64_t* d_fields = nullptr;
    size_t fields_cap = 0;
    uint8_t* d_bytes = nullptr;   // query bytes out / response bytes in
    size_t bytes_cap = 0;
    int64_t* d_aux = nullptr;     // targets / result offsets
    size_t aux_cap = 0;
    uint32_t* d_row1 = nullptr;
    size_t row1_cap = 0;
    uint16_t* d_vals = nullptr;
    size_t vals_cap = 0;
};

namespace {

template <class T>
int grow(T*& p, size_t& cap, size_t need) {
    if (need <= cap && p) return IPR_OK;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    if (cudaMalloc(&p, need * sizeof(T)) != cudaSuccess) {
        cudaGetLastError();
        return fail(IPR_E_OOM, "client scratch of %zu bytes", need * sizeof(T));
    }
    cap = need;
    return IPR_OK;
}

int ensure_limbs(ipr_client* c, size_t polys) {
    if (polys <= c->limb_polys && c->d_limb[0]) return IPR_OK;
    for (auto& p : c->d_limb) {
        if (p) cudaFree(p);
        p = nullptr;
    }
    c->limb_polys = 0;
    for (auto& p : c->d_limb)
        if (cudaMalloc(&p, polys * N * sizeof(uint64_t)) != cudaSuccess) {
            cudaGetLastError();
            return fail(IPR_E_OOM, "client transform buffers");
        }
    c->limb_polys = polys;
    return IPR_OK;
}

int cuda_ok(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return IPR_OK;
    return fail(e == cudaErrorMemoryAllocation ? IPR_E_OOM : IPR_E_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

template <class T>
int upload(T** d, const std::vector<T>& h, cudaStream_t st) {
    if (cudaMalloc(d, h.size() * sizeof(T)) != cudaSuccess) {
        cudaGetLastError();
        return fail(IPR_E_OOM, "client state");
    }
    return cuda_ok(cudaMemcpyAsync(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st), "client upload");
}

// x -> x^t on a raw ternary polynomial (automorph_alloc, src/core/poly.rs:806-834)
void automorph_ternary(const int8_t* s, uint32_t t, int8_t* out) {
    std::memset(out, 0, N);
    for (int i = 0; i < N; i++) {
        const uint32_t d = (uint32_t)(((uint64_t)i * t) % (2 * N));
        if (d < (uint32_t)N) out[d] = s[i];
        else out[d - N] = (int8_t)-s[i];
    }
}

}  // namespace

extern "C" {

int ipr_client_create(int device, const ipr_plan* plan, const uint8_t seed[32], ipr_client** out) {
    if (!plan || !seed || !out) return fail(IPR_E_ARGS, "null argument");
    *out = nullptr;
    if (plan->db_rows < (uint64_t)N || plan->db_rows % N || !plan->interp || !plan->c || !plan->num_items ||
        plan->num_items % plan->db_rows || plan->item_size_bits < 16 || plan->db_cols != plan->instances * N ||
        plan->instances != plan->interp * plan->c)
        return fail(IPR_E_ARGS, "implausible plan");
    if (cudaSetDevice(device) != cudaSuccess) return cuda_ok(cudaGetLastError(), "cudaSetDevice");
    auto* c = new ipr_client();
    c->device = device;
    c->plan = *plan;
    c->per = plan->num_items / plan->db_rows;
    c->item_elems = plan->item_size_bits / 16;
    c->rpolys = (int)(plan->db_rows / N);
    auto bail = [&](int st) {
        ipr_client_destroy(c);
        return st;
    };
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(cuda_ok(cudaGetLastError(), "stream"));

    ipr::HostParams hp;
    ipr::host_params_init(hp);
    // secret key: Fisher-Yates over [+1 x 256, -1 x 256, 0 ...] with ChaCha20(seed, stream 1)
    ipr::ChaCha kr = ipr::chacha_from_seed(seed, 1);
    std::memcpy(c->key, kr.key, sizeof(c->key));
    for (int i = 0; i < N; i++) c->s[i] = i < HAMMING ? 1 : (i < 2 * HAMMING ? -1 : 0);
    for (int i = N - 1; i > 0; i--) {
        const int j = (int)(((unsigned __int128)kr.next_u64() * (unsigned)(i + 1)) >> 64);
        std::swap(c->s[i], c->s[j]);
    }
    std::vector<int8_t> tau(2 * N);
    automorph_ternary(c->s, 5, tau.data());
    automorph_ternary(c->s, 2 * N - 1, tau.data() + N);
    // s in the NTT domain
    std::vector<uint64_t> sl(2 * N);
    for (int l = 0; l < 2; l++)
        for (int i = 0; i < N; i++) sl[l * N + i] = c->s[i] < 0 ? hp.q[l] - 1 : (uint64_t)c->s[i];
    ipr::forward_ntt_u64(hp, sl.data());
    std::vector<uint32_t> s_ntt(2 * N);
    for (int i = 0; i < 2 * N; i++) s_ntt[i] = (uint32_t)sl[i];
    // s * a_r of the public query polynomials (ChaCha20 of the all-zero seed, each a_r[i] =
    // next_u64 mod q), a sparse negacyclic product per limb
    uint8_t zero[32] = {0};
    ipr::ChaCha ar = ipr::chacha_from_seed(zero, 0);
    std::vector<uint32_t> sa_row((size_t)c->rpolys * 2 * N);
    std::vector<uint64_t> a(N);
    std::vector<int> supp;
    for (int j = 0; j < N; j++)
        if (c->s[j]) supp.push_back(j);
    for (int r = 0; r < c->rpolys; r++) {
        for (int i = 0; i < N; i++) a[i] = ar.next_u64() % hp.modulus;
        for (int l = 0; l < 2; l++) {
            const uint64_t q = hp.q[l];
            std::vector<uint64_t> acc(N, 0);
            for (int j : supp)
                for (int i = 0; i < N; i++) {
                    const uint64_t av = a[i] % q;
                    const int d = i + j;
                    const bool pos = (d < N) == (c->s[j] > 0);  // sign of the term after the wrap
                    uint64_t& slot = acc[d < N ? d : d - N];
                    slot = pos ? (slot + av) % q : (slot + q - av) % q;
                }
            for (int i = 0; i < N; i++) sa_row[((size_t)r * 2 + l) * N + i] = (uint32_t)acc[i];
        }
    }
    // s * a of the RGSW public polynomial in the NTT domain: a = q - row0 (row0 = NTT(-a))
    std::vector<uint32_t> sa_gsw(2 * N);
    for (int l = 0; l < 2; l++)
        for (int z = 0; z < N; z++) {
            const uint64_t q = hp.q[l], an = (q - hp.row0[l * N + z]) % q;
            sa_gsw[l * N + z] = (uint32_t)(((unsigned __int128)an * s_ntt[l * N + z]) % q);
        }
    // -s * mask for the W (y keys) and V (z keys) masks
    std::vector<uint32_t> hq, wm, vm;
    ipr::offline_host_inputs(hp, 0, hq, wm, vm);
    std::vector<uint32_t> neg_sm(2 * 3 * 2 * N);
    for (int which = 0; which < 2; which++)
        for (int k = 0; k < 3; k++)
            for (int l = 0; l < 2; l++)
                for (int z = 0; z < N; z++) {
                    const uint64_t q = hp.q[l];
                    const uint64_t m = (which ? vm : wm)[((size_t)k * 2 + l) * N + z];
                    const uint64_t p = ((unsigned __int128)m * s_ntt[l * N + z]) % q;
                    neg_sm[(((size_t)which * 3 + k) * 2 + l) * N + z] = (uint32_t)((q - p) % q);
                }
    std::vector<uint32_t> keyv(c->key, c->key + 8);
    std::vector<int8_t> sv(c->s, c->s + N);
    int st;
    if ((st = upload(&c->d_key, keyv, c->stream)) || (st = upload(&c->d_s, sv, c->stream)) ||
        (st = upload(&c->d_tau, tau, c->stream)) || (st = upload(&c->d_s_ntt, s_ntt, c->stream)) ||
        (st = upload(&c->d_sa_row, sa_row, c->stream)) || (st = upload(&c->d_sa_gsw, sa_gsw, c->stream)) ||
        (st = upload(&c->d_neg_sm, neg_sm, c->stream)) ||
        (st = cuda_ok(cudaStreamSynchronize(c->stream), "client setup")))
        return bail(st);
    *out = c;
    return IPR_OK;
}

int ipr_client_query(ipr_client* c, uint64_t nonce, unsigned n, const uint64_t* buckets, uint8_t* out, size_t cap,
                     size_t* out_len) {
    if (!c || (n && !buckets) || n > 255 || nonce >= (1ull << 62)) return fail(IPR_E_ARGS, "bad argument");
    const uint64_t need = ipr::query_bytes(c->plan.db_rows, n);
    if (out_len) *out_len = need;
    if (!out || cap < need) return fail(IPR_E_SPACE, "query needs %llu bytes", (unsigned long long)need);
    std::vector<int64_t> targets(2 * (size_t)n);
    for (unsigned q = 0; q < n; q++) {
        if (buckets[q] >= c->plan.num_items) return fail(IPR_E_ARGS, "bucket %llu out of range",
                                                             (unsigned long long)buckets[q]);
        const uint64_t col = (buckets[q] % c->per) * c->item_elems;  // build_query_for_index
        targets[2 * q] = (int64_t)(buckets[q] / c->per);
        targets[2 * q + 1] = (int64_t)((col % (c->plan.interp * N)) / N);
    }
    if (cudaSetDevice(c->device) != cudaSuccess) return cuda_ok(cudaGetLastError(), "cudaSetDevice");
    const int64_t nfields = (int64_t)(need - 1) / 7;
    int st;
    if ((st = ensure_limbs(c, KEY_POLYS + (size_t)GSW_COLS * n)) ||
        (st = grow(c->d_aux, c->aux_cap, std::max<size_t>(targets.size(), 1))) ||
        (st = grow(c->d_fields, c->fields_cap, (size_t)nfields)) || (st = grow(c->d_bytes, c->bytes_cap, need)))
        return st;
    if (n && (st = cuda_ok(cudaMemcpyAsync(c->d_aux, targets.data(), targets.size() * sizeof(int64_t),
                                           cudaMemcpyHostToDevice, c->stream), "targets")))
        return st;
    BuildArgs a{c->d_key, 2 + nonce, (int)n, c->rpolys, (int)c->plan.interp, (int64_t)c->plan.db_rows,
                c->d_s, c->d_tau, c->d_sa_row, c->d_aux, c->d_limb[0], c->d_limb[1], c->d_fields};
    const int64_t coeffs = (int64_t)(KEY_POLYS + n * (c->rpolys + GSW_COLS)) * N;
    k_client_build<<<grid_for(coeffs), 256, 0, c->stream>>>(a);
    if ((st = cuda_ok(cudaGetLastError(), "k_client_build"))) return st;
    const uint64_t tp = KEY_POLYS + (uint64_t)GSW_COLS * n;
    for (int l = 0; l < 2; l++)
        if ((st = ipr_ntt_batch(c->device, c->d_limb[l], tp, l, 0, c->stream))) return st;
    k_client_finish<<<grid_for((int64_t)tp * N), 256, 0, c->stream>>>(c->d_limb[0], c->d_limb[1], (int)n,
                                                                       (int64_t)c->plan.db_rows, c->d_neg_sm,
                                                                       c->d_sa_gsw, c->d_fields);
    k_client_serialize<<<grid_for(nfields), 256, 0, c->stream>>>(c->d_fields, nfields, (int)n, c->d_bytes);
    if ((st = cuda_ok(cudaGetLastError(), "client kernels")) ||
        (st = cuda_ok(cudaMemcpyAsync(out, c->d_bytes, need, cudaMemcpyDeviceToHost, c->stream), "query D2H")) ||
        (st = cuda_ok(cudaStreamSynchronize(c->stream), "client query")))
        return st;
    return IPR_OK;
}

int ipr_client_decrypt(ipr_client* c, const uint8_t* response, size_t len, uint16_t* values, size_t cap,
                       size_t* count) {
    if (!c || !response) return fail(IPR_E_ARGS, "null argument");
    // framing (serialize_keyword_response, wire.rs:708-726): u32 count, per response u32 length + bytes
    auto u32 = [&](size_t off, uint32_t* v) {
        if (off + 4 > len) return false;
        *v = (uint32_t)response[off] | ((uint32_t)response[off + 1] << 8) | ((uint32_t)response[off + 2] << 16) |
             ((uint32_t)response[off + 3] << 24);
        return true;
    };
    uint32_t nq = 0;
    if (!u32(0, &nq)) return fail(IPR_E_FORMAT, "short response");
    const uint64_t per_result = (uint64_t)ipr::RESULT_BYTES, c_groups = c->plan.c;
    std::vector<int64_t> offsets;
    size_t off = 4;
    for (uint32_t q = 0; q < nq; q++) {
        uint32_t n = 0;
        if (!u32(off, &n) || n != c_groups * per_result || off + 4 + n > len)
            return fail(IPR_E_FORMAT, "response %u: length does not match the plan", q);
        for (uint64_t w = 0; w < c_groups; w++) offsets.push_back((int64_t)(off + 4 + w * per_result));
        off += 4 + n;
    }
    const size_t nres = offsets.size(), nvals = nres * N;
    if (count) *count = nvals;
    if (!values || cap < nvals) return fail(IPR_E_SPACE, "decryption needs %zu values", nvals);
    if (!nres) return IPR_OK;
    if (cudaSetDevice(c->device) != cudaSuccess) return cuda_ok(cudaGetLastError(), "cudaSetDevice");
    int st;
    if ((st = ensure_limbs(c, nres)) || (st = grow(c->d_aux, c->aux_cap, nres)) ||
        (st = grow(c->d_bytes, c->bytes_cap, off)) || (st = grow(c->d_row1, c->row1_cap, nres * 2 * N)) ||
        (st = grow(c->d_vals, c->vals_cap, nres * N)))
        return st;
    if ((st = cuda_ok(cudaMemcpyAsync(c->d_bytes, response, off, cudaMemcpyHostToDevice, c->stream), "response")) ||
        (st = cuda_ok(cudaMemcpyAsync(c->d_aux, offsets.data(), nres * sizeof(int64_t), cudaMemcpyHostToDevice,
                                      c->stream), "offsets")))
        return st;
    const int64_t work = (int64_t)nres * N;
    k_client_unpack<<<grid_for(work), 256, 0, c->stream>>>(c->d_bytes, c->d_aux, (int)nres, c->d_limb[0],
                                                           c->d_limb[1], c->d_row1);
    if ((st = cuda_ok(cudaGetLastError(), "k_client_unpack"))) return st;
    for (int l = 0; l < 2; l++)
        if ((st = ipr_ntt_batch(c->device, c->d_limb[l], nres, l, 0, c->stream))) return st;
    k_client_mul_s<<<grid_for(work), 256, 0, c->stream>>>(c->d_limb[0], c->d_limb[1], (int)nres, c->d_s_ntt);
    if ((st = cuda_ok(cudaGetLastError(), "k_client_mul_s"))) return st;
    for (int l = 0; l < 2; l++)
        if ((st = ipr_ntt_batch(c->device, c->d_limb[l], nres, l, 1, c->stream))) return st;
    k_client_decode<<<grid_for(work), 256, 0, c->stream>>>(c->d_limb[0], c->d_limb[1], c->d_row1, (int)nres,
                                                           c->d_vals);
    if ((st = cuda_ok(cudaGetLastError(), "k_client_decode")) ||
        (st = cuda_ok(cudaMemcpyAsync(values, c->d_vals, nvals * sizeof(uint16_t), cudaMemcpyDeviceToHost,
                                      c->stream), "values D2H")) ||
        (st = cuda_ok(cudaStreamSynchronize(c->stream), "client decrypt")))
        return st;
    return IPR_OK;
}

// SipHash-2-4 (Aumasson and Bernstein) of `len` bytes under keys (k0, k1)
static uint64_t siphash24(uint64_t k0, uint64_t k1, const uint8_t* m, size_t len) {
    uint64_t v0 = k0 ^ 0x736f6d6570736575ull, v1 = k1 ^ 0x646f72616e646f6dull;
    uint64_t v2 = k0 ^ 0x6c7967656e657261ull, v3 = k1 ^ 0x7465646279746573ull;
    auto rotl = [](uint64_t x, int b) { return (x << b) | (x >> (64 - b)); };
    auto round = [&]() {
        v0 += v1; v1 = rotl(v1, 13); v1 ^= v0; v0 = rotl(v0, 32);
        v2 += v3; v3 = rotl(v3, 16); v3 ^= v2;
        v0 += v3; v3 = rotl(v3, 21); v3 ^= v0;
        v2 += v1; v1 = rotl(v1, 17); v1 ^= v2; v2 = rotl(v2, 32);
    };
    size_t i = 0;
    for (; i + 8 <= len; i += 8) {
        uint64_t w = 0;
        for (int b = 0; b < 8; b++) w |= (uint64_t)m[i + b] << (8 * b);
        v3 ^= w;
        round();
        round();
        v0 ^= w;
    }
    uint64_t last = (uint64_t)(len & 0xff) << 56;
    for (size_t b = 0; i + b < len; b++) last |= (uint64_t)m[i + b] << (8 * b);
    v3 ^= last;
    round();
    round();
    v0 ^= last;
    v2 ^= 0xff;
    for (int r = 0; r < 4; r++) round();
    return v0 ^ v1 ^ v2 ^ v3;
}

int ipr_cuckoo_positions(const uint8_t seed[16], uint64_t num_buckets, unsigned num_hashes, const uint8_t* key,
                         size_t key_len, uint64_t* out) {
    if (!seed || !out || (key_len && !key) || num_buckets < 2 || num_hashes < 1 || num_hashes > 255)
        return fail(IPR_E_ARGS, "bad argument");
    bool trivial = true;
    for (int i = 0; i < 16; i++) trivial = trivial && seed[i] == 0;
    uint64_t s0 = 0, s1 = 0;
    for (int b = 0; b < 8; b++) {
        s0 |= (uint64_t)seed[b] << (8 * b);
        s1 |= (uint64_t)seed[8 + b] << (8 * b);
    }
    for (unsigned h = 0; h < num_hashes; h++) {
        if (trivial) {  // identity: the last 8 key bytes, big-endian, into one half of the table
            uint64_t idx = 0;
            const size_t n = key_len < 8 ? key_len : 8, start = key_len - n;
            for (size_t b = 0; b < n; b++) idx |= (uint64_t)key[start + b] << (8 * (7 - b));
            const uint64_t half = num_buckets / 2;
            out[h] = h == 0 ? idx % half : half + idx % half;
        } else {
            out[h] = siphash24(s0 ^ h, s1 ^ ((uint64_t)h << 32), key, key_len) % num_buckets;
        }
    }
    return IPR_OK;
}

int ipr_client_secret_key(const ipr_client* c, int8_t* out) {
    if (!c || !out) return fail(IPR_E_ARGS, "null argument");
    std::memcpy(out, c->s, N);
    return IPR_OK;
}

void ipr_client_destroy(ipr_client* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    void* ps[] = {c->d_key, c->d_s, c->d_tau, c->d_s_ntt, c->d_sa_row, c->d_sa_gsw, c->d_neg_sm, c->d_limb[0],
                  c->d_limb[1], c->d_fields, c->d_bytes, c->d_aux, c->d_row1, c->d_vals};
    for (void* p : ps)
        if (p) cudaFree(p);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

}  // extern "C"
