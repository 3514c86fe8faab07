// dataset.cu — DatasetGenerator on the GPU: seeded ML-KEM public keys and their IDs.
//
// Restates (rkdud007/inspire-rs) DatasetGenerator::generate_record
// (src/dataset/generator.rs:171-193): record idx of a dataset with seed `seed` is
//   seed64 = ChaCha20Rng::seed_from_u64(seed) keystream at word position 16 * idx: one
//            64-byte ChaCha20 block, counter idx (rand_chacha: 64-bit counter in words
//            12-13, stream id 0 in words 14-15),
//   pk     = the encapsulation key of KemCore::generate_deterministic(d, z) with
//            d = seed64[0..32], z = seed64[32..64] (src/dataset/kem.rs:27-44): FIPS 203
//            ML-KEM.KeyGen_internal, whose ek = K-PKE.KeyGen(d).ek depends on d only,
//   id     = SHA3-256("pq-key:v1:" || kem_name || pk) (src/dataset/dataset.rs:36-46).
// Output rows are id (32 bytes) || pk (384 k + 32 bytes), the reference's flat record
// layout (generator.rs:101-118).  The ChaCha20 key (rand_core's seed_from_u64: PCG32 words)
// is derived on the host.  Keccak-f[1600] round constants and rotation offsets come from
// FIPS 202's definitions (the rc(t) LFSR, the (t+1)(t+2)/2 rho offsets).
//
// One thread per record: a record is ~45 Keccak-f permutations, six or eight 256-point
// NTTs mod 3329 and k^2 base-case products, small enough for local memory.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "ipr_b200.h"
#include "kernels.cuh"

namespace ipr {

namespace {

__constant__ uint64_t c_keccak_rc[24];
__constant__ int16_t c_zeta[128];   // 17^BitRev7(i) mod 3329
__constant__ int16_t c_gamma[128];  // 17^(2 BitRev7(i) + 1) mod 3329

constexpr int MQ = 3329;

__host__ __device__ constexpr int rho_offset(int x, int y) {  // FIPS 202 Algorithm 2
    if (x == 0 && y == 0) return 0;
    int cx = 1, cy = 0;
    for (int t = 0; t < 24; t++) {
        if (cx == x && cy == y) return ((t + 1) * (t + 2) / 2) % 64;
        const int nx = cy, ny = (2 * cx + 3 * cy) % 5;
        cx = nx;
        cy = ny;
    }
    return 0;
}

__device__ __forceinline__ uint64_t rotl64(uint64_t v, int n) { return n ? (v << n) | (v >> (64 - n)) : v; }

__device__ void keccakf(uint64_t (&a)[25]) {
#pragma unroll 1
    for (int ir = 0; ir < 24; ir++) {
        uint64_t c[5], d[5], b[25];
#pragma unroll
        for (int x = 0; x < 5; x++) c[x] = a[x] ^ a[x + 5] ^ a[x + 10] ^ a[x + 15] ^ a[x + 20];
#pragma unroll
        for (int x = 0; x < 5; x++) d[x] = c[(x + 4) % 5] ^ rotl64(c[(x + 1) % 5], 1);
#pragma unroll
        for (int i = 0; i < 25; i++) a[i] ^= d[i % 5];
#pragma unroll
        for (int x = 0; x < 5; x++)
#pragma unroll
            for (int y = 0; y < 5; y++) b[y + 5 * ((2 * x + 3 * y) % 5)] = rotl64(a[x + 5 * y], rho_offset(x, y));
#pragma unroll
        for (int x = 0; x < 5; x++)
#pragma unroll
            for (int y = 0; y < 5; y++)
                a[x + 5 * y] = b[x + 5 * y] ^ (~b[(x + 1) % 5 + 5 * y] & b[(x + 2) % 5 + 5 * y]);
        a[0] ^= c_keccak_rc[ir];
    }
}

// a Keccak sponge over one thread's state; rate in bytes
struct Sponge {
    uint64_t s[25];
    int rate, pos;
    __device__ void init(int r) {
#pragma unroll
        for (int i = 0; i < 25; i++) s[i] = 0;
        rate = r;
        pos = 0;
    }
    __device__ void absorb_byte(uint8_t v) {
        s[pos >> 3] ^= (uint64_t)v << (8 * (pos & 7));
        if (++pos == rate) {
            keccakf(s);
            pos = 0;
        }
    }
    __device__ void finish(uint8_t ds) {  // pad10*1 with the domain bits
        s[pos >> 3] ^= (uint64_t)ds << (8 * (pos & 7));
        s[(rate - 1) >> 3] ^= 0x80ull << (8 * ((rate - 1) & 7));
        keccakf(s);
        pos = 0;
    }
    __device__ uint8_t squeeze_byte() {
        if (pos == rate) {
            keccakf(s);
            pos = 0;
        }
        const uint8_t v = (uint8_t)(s[pos >> 3] >> (8 * (pos & 7)));
        pos++;
        return v;
    }
};

__device__ __forceinline__ uint32_t rotl32(uint32_t v, int n) { return (v << n) | (v >> (32 - n)); }

__device__ void chacha20_block(const uint32_t key[8], uint64_t counter, uint8_t out[64]) {
    uint32_t s[16], x[16];
    s[0] = 0x61707865u;
    s[1] = 0x3320646eu;
    s[2] = 0x79622d32u;
    s[3] = 0x6b206574u;
#pragma unroll
    for (int i = 0; i < 8; i++) s[4 + i] = key[i];
    s[12] = (uint32_t)counter;
    s[13] = (uint32_t)(counter >> 32);
    s[14] = 0;
    s[15] = 0;
#pragma unroll
    for (int i = 0; i < 16; i++) x[i] = s[i];
    auto qr = [&](int a, int b, int c, int d) {
        x[a] += x[b]; x[d] ^= x[a]; x[d] = rotl32(x[d], 16);
        x[c] += x[d]; x[b] ^= x[c]; x[b] = rotl32(x[b], 12);
        x[a] += x[b]; x[d] ^= x[a]; x[d] = rotl32(x[d], 8);
        x[c] += x[d]; x[b] ^= x[c]; x[b] = rotl32(x[b], 7);
    };
#pragma unroll 1
    for (int r = 0; r < 10; r++) {
        qr(0, 4, 8, 12); qr(1, 5, 9, 13); qr(2, 6, 10, 14); qr(3, 7, 11, 15);
        qr(0, 5, 10, 15); qr(1, 6, 11, 12); qr(2, 7, 8, 13); qr(3, 4, 9, 14);
    }
#pragma unroll
    for (int i = 0; i < 16; i++) {
        const uint32_t v = x[i] + s[i];
#pragma unroll
        for (int b = 0; b < 4; b++) out[4 * i + b] = (uint8_t)(v >> (8 * b));
    }
}

__device__ __forceinline__ int16_t red(int v) { return (int16_t)(v % MQ); }  // v >= 0

// FIPS 203 Algorithm 9 (NTT), coefficients in [0, q)
__device__ void mlkem_ntt(int16_t* f) {
    int i = 1;
#pragma unroll 1
    for (int len = 128; len >= 2; len >>= 1)
#pragma unroll 1
        for (int start = 0; start < 256; start += 2 * len) {
            const int zeta = c_zeta[i++];
#pragma unroll 4
            for (int j = start; j < start + len; j++) {
                const int t = zeta * f[j + len] % MQ;
                f[j + len] = red(f[j] - t + MQ);
                f[j] = red(f[j] + t);
            }
        }
}

// FIPS 203 Algorithm 8 with PRF_eta(sigma, n) = SHAKE256(sigma || n) (64 eta bytes)
__device__ void sample_cbd(const uint8_t sigma[32], int n, int eta, int16_t* f) {
    Sponge sp;
    sp.init(136);
    for (int i = 0; i < 32; i++) sp.absorb_byte(sigma[i]);
    sp.absorb_byte((uint8_t)n);
    sp.finish(0x1F);
    // eta = 2: one byte gives two coefficients; eta = 3: three bytes give four
    if (eta == 2) {
        for (int i = 0; i < 128; i++) {
            const uint32_t b = sp.squeeze_byte();
            const int x0 = (b & 1) + ((b >> 1) & 1), y0 = ((b >> 2) & 1) + ((b >> 3) & 1);
            const int x1 = ((b >> 4) & 1) + ((b >> 5) & 1), y1 = ((b >> 6) & 1) + ((b >> 7) & 1);
            f[2 * i] = red(x0 - y0 + MQ);
            f[2 * i + 1] = red(x1 - y1 + MQ);
        }
    } else {
        for (int i = 0; i < 64; i++) {
            const uint32_t b = sp.squeeze_byte() | ((uint32_t)sp.squeeze_byte() << 8) |
                               ((uint32_t)sp.squeeze_byte() << 16);
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const uint32_t w = b >> (6 * c);
                const int x = (w & 1) + ((w >> 1) & 1) + ((w >> 2) & 1);
                const int y = ((w >> 3) & 1) + ((w >> 4) & 1) + ((w >> 5) & 1);
                f[4 * i + c] = red(x - y + MQ);
            }
        }
    }
}

__global__ void __launch_bounds__(128) k_dataset(int k, uint4 key_lo, uint4 key_hi, uint64_t first, uint64_t count,
                                                 uint8_t* __restrict__ out) {
    const uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (r >= count) return;
    const int pk_len = 384 * k + 32;
    uint8_t* rec = out + r * (uint64_t)(32 + pk_len);
    uint8_t* pk = rec + 32;
    // record seed: ChaCha20 block number first + r
    const uint32_t key[8] = {key_lo.x, key_lo.y, key_lo.z, key_lo.w, key_hi.x, key_hi.y, key_hi.z, key_hi.w};
    uint8_t seed64[64];
    chacha20_block(key, first + r, seed64);
    // K-PKE.KeyGen (FIPS 203 Algorithm 13): (rho, sigma) = SHA3-512(d || k)
    uint8_t rho[32], sigma[32];
    {
        Sponge sp;
        sp.init(72);
        for (int i = 0; i < 32; i++) sp.absorb_byte(seed64[i]);
        sp.absorb_byte((uint8_t)k);
        sp.finish(0x06);
        for (int i = 0; i < 32; i++) rho[i] = sp.squeeze_byte();
        for (int i = 0; i < 32; i++) sigma[i] = sp.squeeze_byte();
    }
    const int eta1 = k == 2 ? 3 : 2;
    int16_t s[4][256], t[256];
    for (int i = 0; i < k; i++) {
        sample_cbd(sigma, i, eta1, s[i]);
        mlkem_ntt(s[i]);
    }
    for (int i = 0; i < k; i++) {
        sample_cbd(sigma, k + i, eta1, t);  // e[i]
        mlkem_ntt(t);
        for (int j = 0; j < k; j++) {
            // A_hat[i][j] = SampleNTT(SHAKE128(rho || j || i)) (Algorithm 7), consumed pairwise by
            // the base-case products (Algorithms 11, 12) as it is sampled
            Sponge sp;
            sp.init(168);
            for (int b = 0; b < 32; b++) sp.absorb_byte(rho[b]);
            sp.absorb_byte((uint8_t)j);
            sp.absorb_byte((uint8_t)i);
            sp.finish(0x1F);
            int have = 0, pend = 0;
            while (have < 256) {
                const int c0 = sp.squeeze_byte(), c1 = sp.squeeze_byte(), c2 = sp.squeeze_byte();
                const int dv[2] = {c0 + 256 * (c1 & 15), (c1 >> 4) + 16 * c2};
#pragma unroll
                for (int u = 0; u < 2; u++) {
                    if (dv[u] >= MQ || have >= 256) continue;
                    if (have & 1) {  // coefficients 2p, 2p + 1 complete: add A_p * s_j,p
                        const int p = have >> 1, a0 = pend, a1 = dv[u];
                        const int b0 = s[j][2 * p], b1 = s[j][2 * p + 1];
                        t[2 * p] = red(t[2 * p] + a0 * b0 % MQ + (a1 * b1 % MQ) * c_gamma[p] % MQ);
                        t[2 * p + 1] = red(t[2 * p + 1] + a0 * b1 % MQ + a1 * b0 % MQ);
                    } else {
                        pend = dv[u];
                    }
                    have++;
                }
            }
        }
        for (int p = 0; p < 128; p++) {  // ByteEncode_12 (Algorithm 5)
            const int c0 = t[2 * p], c1 = t[2 * p + 1];
            pk[384 * i + 3 * p] = (uint8_t)c0;
            pk[384 * i + 3 * p + 1] = (uint8_t)((c0 >> 8) | ((c1 & 15) << 4));
            pk[384 * i + 3 * p + 2] = (uint8_t)(c1 >> 4);
        }
    }
    for (int b = 0; b < 32; b++) pk[384 * k + b] = rho[b];
    // id = SHA3-256("pq-key:v1:" || kem_name || pk)
    {
        const char* name = k == 2 ? "ml-kem-512" : (k == 3 ? "ml-kem-768" : "ml-kem-1024");
        const char* dom = "pq-key:v1:";
        Sponge sp;
        sp.init(136);
        for (int i = 0; i < 10; i++) sp.absorb_byte((uint8_t)dom[i]);
        for (int i = 0; name[i]; i++) sp.absorb_byte((uint8_t)name[i]);
        for (int i = 0; i < pk_len; i++) sp.absorb_byte(pk[i]);
        sp.finish(0x06);
        for (int i = 0; i < 32; i++) rec[i] = sp.squeeze_byte();
    }
}

// host: FIPS 202 Algorithm 5, bit i of r holds R[i]
int rc_bit(int t) {
    if (t % 255 == 0) return 1;
    unsigned r = 1;
    for (int i = 1; i <= t % 255; i++) {
        r <<= 1;
        r ^= ((r >> 8) & 1) * 0x71u;
        r &= 0xFF;
    }
    return r & 1;
}

int brv7(int x) {
    int r = 0;
    for (int i = 0; i < 7; i++) r |= ((x >> i) & 1) << (6 - i);
    return r;
}

int pow17(int e) {
    int64_t r = 1, b = 17;
    while (e) {
        if (e & 1) r = r * b % MQ;
        b = b * b % MQ;
        e >>= 1;
    }
    return (int)r;
}

cudaError_t load_dataset_constants() {
    uint64_t rc[24];
    for (int ir = 0; ir < 24; ir++) {
        rc[ir] = 0;
        for (int j = 0; j <= 6; j++)
            if (rc_bit(j + 7 * ir)) rc[ir] |= 1ull << ((1 << j) - 1);
    }
    int16_t zeta[128], gamma[128];
    for (int i = 0; i < 128; i++) {
        zeta[i] = (int16_t)pow17(brv7(i));
        gamma[i] = (int16_t)pow17(2 * brv7(i) + 1);
    }
    cudaError_t e = cudaMemcpyToSymbol(c_keccak_rc, rc, sizeof(rc));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_zeta, zeta, sizeof(zeta));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_gamma, gamma, sizeof(gamma));
    return e;
}

// rand_core SeedableRng::seed_from_u64: PCG32 output words, little endian
void seed_from_u64(uint64_t state, uint32_t key[8]) {
    const uint64_t mul = 6364136223846793005ull, inc = 11634580027462260723ull;
    for (int w = 0; w < 8; w++) {
        state = state * mul + inc;
        const uint32_t xs = (uint32_t)(((state >> 18) ^ state) >> 27);
        const int rot = (int)(state >> 59);
        key[w] = rot ? (xs >> rot) | (xs << (32 - rot)) : xs;
    }
}

}  // namespace

void set_last_error(const char* msg);  // server.cu: the text ipr_last_error() returns

namespace {
int cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return IPR_OK;
    set_last_error(cudaGetErrorString(e));
    return IPR_E_CUDA;
}
}  // namespace

}  // namespace ipr

extern "C" int ipr_dataset_generate(int device, int kem, uint64_t seed, uint64_t first, uint64_t count,
                                    uint8_t* d_records, void* stream) {
    const int k = kem == 512 ? 2 : (kem == 768 ? 3 : (kem == 1024 ? 4 : 0));
    if (!k) {
        ipr::set_last_error("ipr_dataset_generate: kem must be 512, 768 or 1024");
        return IPR_E_ARGS;
    }
    if (count == 0) return IPR_OK;
    if (!d_records) {
        ipr::set_last_error("ipr_dataset_generate: null output");
        return IPR_E_ARGS;
    }
    int st = ipr::cuda_status(cudaSetDevice(device));
    if (st) return st;
    if ((st = ipr::cuda_status(ipr::load_dataset_constants()))) return st;
    uint32_t key[8];
    ipr::seed_from_u64(seed, key);
    const uint4 lo = make_uint4(key[0], key[1], key[2], key[3]), hi = make_uint4(key[4], key[5], key[6], key[7]);
    const uint64_t blocks = (count + 127) / 128;
    if (blocks > 0x7fffffffull) {
        ipr::set_last_error("ipr_dataset_generate: count too large for one call");
        return IPR_E_ARGS;
    }
    ipr::k_dataset<<<(unsigned)blocks, 128, 0, static_cast<cudaStream_t>(stream)>>>(k, lo, hi, first, count,
                                                                                   d_records);
    return ipr::cuda_status(cudaGetLastError());
}

// the same records into host memory: a device buffer of one batch (at most 65,536 records)
// is filled and copied back batch by batch
extern "C" int ipr_dataset_generate_host(int device, int kem, uint64_t seed, uint64_t first, uint64_t count,
                                         uint8_t* h_records) {
    const uint64_t pk_len = kem == 512 ? 800 : (kem == 768 ? 1184 : (kem == 1024 ? 1568 : 0));
    if (!pk_len) {
        ipr::set_last_error("ipr_dataset_generate_host: kem must be 512, 768 or 1024");
        return IPR_E_ARGS;
    }
    if (count == 0) return IPR_OK;
    if (!h_records) {
        ipr::set_last_error("ipr_dataset_generate_host: null output");
        return IPR_E_ARGS;
    }
    int st = ipr::cuda_status(cudaSetDevice(device));
    if (st) return st;
    const uint64_t rs = 32 + pk_len, batch = count < 65536 ? count : 65536;
    uint8_t* d = nullptr;
    if (cudaMalloc(&d, batch * rs) != cudaSuccess) {
        cudaGetLastError();
        ipr::set_last_error("ipr_dataset_generate_host: cudaMalloc failed");
        return IPR_E_OOM;
    }
    for (uint64_t c0 = 0; c0 < count && !st; c0 += batch) {
        const uint64_t n = count - c0 < batch ? count - c0 : batch;
        st = ipr_dataset_generate(device, kem, seed, first + c0, n, d, nullptr);
        if (!st) st = ipr::cuda_status(cudaMemcpy(h_records + c0 * rs, d, n * rs, cudaMemcpyDeviceToHost));
    }
    cudaFree(d);
    return st;
}
