/* ipr_dataset.c — CPU restatement of the reference's dataset generation (test
 * infrastructure only: the checker for the device generator in csrc/dataset.cu).
 *
 * DatasetGenerator (rkdud007/inspire-rs src/dataset/generator.rs:24-193): record idx of a
 * dataset with seed `seed` is
 *   seed64 = the 64 bytes of ChaCha20Rng::seed_from_u64(seed) at word position 16 * idx
 *            (generator.rs:171-175, 189-193: one keystream block per record),
 *   pk     = ML-KEM encapsulation key of KemCore::generate_deterministic(d = seed64[0..32],
 *            z = seed64[32..64]) (src/dataset/kem.rs:27-44),
 *   id     = SHA3-256("pq-key:v1:" || kem_name || pk) (src/dataset/dataset.rs:36-46).
 * The algorithms live in third-party crates absent from the reference tree; they are
 * restated here from their published specifications:
 *   rand_core 0.10.1   SeedableRng::seed_from_u64: PCG32 output words expand the u64 to the
 *                      32-byte key (the crate's documented default method)
 *   rand_chacha 0.10.0 ChaCha20 (the block function ipr_chacha20_block of ipr_oracle.c,
 *                      pinned to RFC 8439's vector), 64-bit block counter, stream id 0
 *   ml-kem 0.2.3       FIPS 203 ML-KEM.KeyGen_internal (Algorithms 13 and 16; the
 *                      encapsulation key depends on d only)
 *   sha3 0.11.0        FIPS 202 SHA3-256 / SHA3-512 / SHAKE128 / SHAKE256 (Keccak-f[1600])
 * The Keccak round constants and rotation offsets are computed from FIPS 202's own
 * definitions (rc(t) LFSR, Algorithm 5; the (t+1)(t+2)/2 offsets of rho, Algorithm 2). */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "ipr_oracle.h"

/* ---------------------------------------------------------------- Keccak (FIPS 202) */
static uint64_t kc_rc[24];
static int kc_rho[25];
static int kc_ready = 0;

static int rc_bit(int t) { /* FIPS 202 Algorithm 5; bit i of r holds R[i] */
    if (t % 255 == 0) return 1;
    unsigned r = 1; /* R = 10000000 */
    for (int i = 1; i <= t % 255; i++) {
        r <<= 1;                     /* R = 0 || R */
        r ^= ((r >> 8) & 1) * 0x71u; /* R[0], R[4], R[5], R[6] ^= R[8] */
        r &= 0xFF;                   /* Trunc8 */
    }
    return r & 1;
}

static void kc_init(void) {
    if (kc_ready) return;
    for (int ir = 0; ir < 24; ir++) {
        uint64_t rc = 0;
        for (int j = 0; j <= 6; j++)
            if (rc_bit(j + 7 * ir)) rc |= 1ull << ((1 << j) - 1);
        kc_rc[ir] = rc;
    }
    memset(kc_rho, 0, sizeof(kc_rho));
    int x = 1, y = 0;
    for (int t = 0; t < 24; t++) {
        kc_rho[x + 5 * y] = ((t + 1) * (t + 2) / 2) % 64;
        int nx = y, ny = (2 * x + 3 * y) % 5;
        x = nx;
        y = ny;
    }
    kc_ready = 1;
}

static uint64_t rotl64(uint64_t v, int n) { return n ? (v << n) | (v >> (64 - n)) : v; }

void ipr_keccakf(uint64_t a[25]) {
    kc_init();
    for (int ir = 0; ir < 24; ir++) {
        uint64_t c[5], d[5], b[25];
        for (int x = 0; x < 5; x++) c[x] = a[x] ^ a[x + 5] ^ a[x + 10] ^ a[x + 15] ^ a[x + 20];
        for (int x = 0; x < 5; x++) d[x] = c[(x + 4) % 5] ^ rotl64(c[(x + 1) % 5], 1);
        for (int i = 0; i < 25; i++) a[i] ^= d[i % 5];
        /* rho and pi: B[y, 2x + 3y] = ROT(A[x, y], rho[x, y]) */
        for (int x = 0; x < 5; x++)
            for (int y = 0; y < 5; y++) b[y + 5 * ((2 * x + 3 * y) % 5)] = rotl64(a[x + 5 * y], kc_rho[x + 5 * y]);
        for (int x = 0; x < 5; x++)
            for (int y = 0; y < 5; y++)
                a[x + 5 * y] = b[x + 5 * y] ^ (~b[(x + 1) % 5 + 5 * y] & b[(x + 2) % 5 + 5 * y]);
        a[0] ^= kc_rc[ir];
    }
}

typedef struct {
    uint64_t s[25];
    int rate, pos;
} sponge;

static void sp_init(sponge *sp, int rate) {
    memset(sp, 0, sizeof(*sp));
    sp->rate = rate;
}
static void sp_absorb(sponge *sp, const uint8_t *m, size_t n) {
    for (size_t i = 0; i < n; i++) {
        sp->s[sp->pos / 8] ^= (uint64_t)m[i] << (8 * (sp->pos % 8));
        if (++sp->pos == sp->rate) {
            ipr_keccakf(sp->s);
            sp->pos = 0;
        }
    }
}
static void sp_finish(sponge *sp, uint8_t dsbyte) { /* pad10*1 with the domain bits */
    sp->s[sp->pos / 8] ^= (uint64_t)dsbyte << (8 * (sp->pos % 8));
    sp->s[(sp->rate - 1) / 8] ^= 0x80ull << (8 * ((sp->rate - 1) % 8));
    ipr_keccakf(sp->s);
    sp->pos = 0;
}
static void sp_squeeze(sponge *sp, uint8_t *out, size_t n) {
    for (size_t i = 0; i < n; i++) {
        if (sp->pos == sp->rate) {
            ipr_keccakf(sp->s);
            sp->pos = 0;
        }
        out[i] = (uint8_t)(sp->s[sp->pos / 8] >> (8 * (sp->pos % 8)));
        sp->pos++;
    }
}

void ipr_sha3_256(const uint8_t *m, size_t n, uint8_t out[32]) {
    sponge sp;
    sp_init(&sp, 136);
    sp_absorb(&sp, m, n);
    sp_finish(&sp, 0x06);
    sp_squeeze(&sp, out, 32);
}
void ipr_sha3_512(const uint8_t *m, size_t n, uint8_t out[64]) {
    sponge sp;
    sp_init(&sp, 72);
    sp_absorb(&sp, m, n);
    sp_finish(&sp, 0x06);
    sp_squeeze(&sp, out, 64);
}
void ipr_shake128(const uint8_t *m, size_t n, uint8_t *out, size_t outlen) {
    sponge sp;
    sp_init(&sp, 168);
    sp_absorb(&sp, m, n);
    sp_finish(&sp, 0x1F);
    sp_squeeze(&sp, out, outlen);
}
void ipr_shake256(const uint8_t *m, size_t n, uint8_t *out, size_t outlen) {
    sponge sp;
    sp_init(&sp, 136);
    sp_absorb(&sp, m, n);
    sp_finish(&sp, 0x1F);
    sp_squeeze(&sp, out, outlen);
}

/* ---------------------------------------------------------------- ML-KEM (FIPS 203) */
#define MQ 3329

static int brv7(int x) {
    int r = 0;
    for (int i = 0; i < 7; i++) r |= ((x >> i) & 1) << (6 - i);
    return r;
}
static int powq(int b, int e) {
    int64_t r = 1, x = b;
    while (e) {
        if (e & 1) r = r * x % MQ;
        x = x * x % MQ;
        e >>= 1;
    }
    return (int)r;
}

/* Algorithm 9: NTT with zeta = 17 */
static void mlkem_ntt(int16_t f[256]) {
    int i = 1;
    for (int len = 128; len >= 2; len /= 2)
        for (int start = 0; start < 256; start += 2 * len) {
            const int zeta = powq(17, brv7(i++));
            for (int j = start; j < start + len; j++) {
                const int t = zeta * f[j + len] % MQ;
                f[j + len] = (int16_t)((f[j] - t + MQ) % MQ);
                f[j] = (int16_t)((f[j] + t) % MQ);
            }
        }
}

/* Algorithm 7: SampleNTT from SHAKE128(rho || j || i) */
static void sample_ntt(const uint8_t rho[32], uint8_t jj, uint8_t ii, int16_t a[256]) {
    uint8_t in[34];
    memcpy(in, rho, 32);
    in[32] = jj;
    in[33] = ii;
    sponge sp;
    sp_init(&sp, 168);
    sp_absorb(&sp, in, 34);
    sp_finish(&sp, 0x1F);
    int j = 0;
    while (j < 256) {
        uint8_t c[3];
        sp_squeeze(&sp, c, 3);
        const int d1 = c[0] + 256 * (c[1] & 15), d2 = (c[1] >> 4) + 16 * c[2];
        if (d1 < MQ) a[j++] = (int16_t)d1;
        if (d2 < MQ && j < 256) a[j++] = (int16_t)d2;
    }
}

/* Algorithm 8: SamplePolyCBD_eta from PRF_eta(sigma, n) = SHAKE256(sigma || n, 64 eta bytes) */
static void sample_cbd(const uint8_t sigma[32], uint8_t n, int eta, int16_t f[256]) {
    uint8_t in[33], b[192];
    memcpy(in, sigma, 32);
    in[32] = n;
    ipr_shake256(in, 33, b, (size_t)64 * eta);
    for (int i = 0; i < 256; i++) {
        int x = 0, y = 0;
        for (int j = 0; j < eta; j++) {
            const int bx = 2 * i * eta + j, by = 2 * i * eta + eta + j;
            x += (b[bx >> 3] >> (bx & 7)) & 1;
            y += (b[by >> 3] >> (by & 7)) & 1;
        }
        f[i] = (int16_t)((x - y + MQ) % MQ);
    }
}

/* K-PKE.KeyGen (Algorithm 13) -> ek = ByteEncode12(t_hat) || rho; ML-KEM.KeyGen_internal
 * (Algorithm 16) returns it unchanged as the encapsulation key.  k = 2, 3, 4; eta1 = 3, 2, 2. */
void ipr_mlkem_ek(int k, const uint8_t d[32], uint8_t *ek) {
    const int eta1 = k == 2 ? 3 : 2;
    uint8_t g_in[33], g[64];
    memcpy(g_in, d, 32);
    g_in[32] = (uint8_t)k;
    ipr_sha3_512(g_in, 33, g);
    const uint8_t *rho = g, *sigma = g + 32;
    int16_t s[4][256], e[4][256], a[256];
    uint8_t nctr = 0;
    for (int i = 0; i < k; i++) sample_cbd(sigma, nctr++, eta1, s[i]);
    for (int i = 0; i < k; i++) sample_cbd(sigma, nctr++, eta1, e[i]);
    for (int i = 0; i < k; i++) {
        mlkem_ntt(s[i]);
        mlkem_ntt(e[i]);
    }
    for (int i = 0; i < k; i++) {
        int32_t t[256];
        for (int z = 0; z < 256; z++) t[z] = e[i][z];
        for (int j = 0; j < k; j++) {
            sample_ntt(rho, (uint8_t)j, (uint8_t)i, a); /* A_hat[i][j] (Algorithm 13 line 4) */
            for (int p = 0; p < 128; p++) { /* MultiplyNTTs / BaseCaseMultiply (Algorithms 11, 12) */
                const int gam = powq(17, 2 * brv7(p) + 1);
                const int a0 = a[2 * p], a1 = a[2 * p + 1], b0 = s[j][2 * p], b1 = s[j][2 * p + 1];
                t[2 * p] = (t[2 * p] + a0 * b0 % MQ + (a1 * b1 % MQ) * gam % MQ) % MQ;
                t[2 * p + 1] = (t[2 * p + 1] + a0 * b1 % MQ + a1 * b0 % MQ) % MQ;
            }
        }
        for (int p = 0; p < 128; p++) { /* ByteEncode_12 (Algorithm 5) */
            const int c0 = t[2 * p], c1 = t[2 * p + 1];
            ek[384 * i + 3 * p] = (uint8_t)c0;
            ek[384 * i + 3 * p + 1] = (uint8_t)((c0 >> 8) | ((c1 & 15) << 4));
            ek[384 * i + 3 * p + 2] = (uint8_t)(c1 >> 4);
        }
    }
    memcpy(ek + 384 * k, rho, 32);
}

/* ---------------------------------------------------------------- seeds (rand_core / rand_chacha) */
void ipr_seed_from_u64(uint64_t state, uint8_t key[32]) {
    const uint64_t mul = 6364136223846793005ull, inc = 11634580027462260723ull;
    for (int w = 0; w < 8; w++) {
        state = state * mul + inc;
        const uint32_t xs = (uint32_t)(((state >> 18) ^ state) >> 27);
        const int rot = (int)(state >> 59);
        const uint32_t x = rot ? (xs >> rot) | (xs << (32 - rot)) : xs;
        for (int b = 0; b < 4; b++) key[4 * w + b] = (uint8_t)(x >> (8 * b));
    }
}

/* one dataset record: out = id (32 bytes) || pk (384 k + 32 bytes); kem_k = 2, 3 or 4 */
void ipr_dataset_record(int kem_k, uint64_t seed, uint64_t idx, uint8_t *out) {
    static const char *names[5] = {0, 0, "ml-kem-512", "ml-kem-768", "ml-kem-1024"};
    uint8_t key[32], seed64[64];
    uint32_t kw[8], blk[16];
    ipr_seed_from_u64(seed, key);
    for (int i = 0; i < 8; i++)
        kw[i] = (uint32_t)key[4 * i] | ((uint32_t)key[4 * i + 1] << 8) | ((uint32_t)key[4 * i + 2] << 16) |
                ((uint32_t)key[4 * i + 3] << 24);
    ipr_chacha20_block(kw, idx, 0, blk); /* block idx = words 16 idx .. 16 idx + 15 */
    for (int i = 0; i < 16; i++)
        for (int b = 0; b < 4; b++) seed64[4 * i + b] = (uint8_t)(blk[i] >> (8 * b));
    uint8_t *pk = out + 32;
    ipr_mlkem_ek(kem_k, seed64, pk);
    const size_t pk_len = 384 * (size_t)kem_k + 32, nl = strlen(names[kem_k]);
    uint8_t *msg = malloc(10 + nl + pk_len);
    memcpy(msg, "pq-key:v1:", 10);
    memcpy(msg + 10, names[kem_k], nl);
    memcpy(msg + 10 + nl, pk, pk_len);
    ipr_sha3_256(msg, 10 + nl + pk_len, out);
    free(msg);
}
