/*
 * ipr_oracle.c — CPU restatement of the InsPIRe keyword-PIR respond() path.
 * TEST INFRASTRUCTURE ONLY (the checker); never linked by the product.
 * See ipr_oracle.h for the pinning strategy.  Citations are to files of
 * rkdud007/inspire-rs.
 */
#include "ipr_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef unsigned __int128 u128;

/* ------------------------------------------------------------------ */
/* arithmetic                                                          */
/* ------------------------------------------------------------------ */

static uint64_t mulmod(uint64_t a, uint64_t b, uint64_t m) { /* arith.rs:5-7 */
    return (uint64_t)(((u128)a * b) % m);
}

static uint64_t powmod(uint64_t b, uint64_t e, uint64_t m) { /* arith.rs:52-78 */
    uint64_t r = 1 % m;
    b %= m;
    while (e) {
        if (e & 1) r = mulmod(r, b, m);
        b = mulmod(b, b, m);
        e >>= 1;
    }
    return r;
}

uint64_t ipr_reverse_bits(uint64_t x, unsigned bits) { /* arith.rs:80-87 */
    if (bits == 0) return 0;
    uint64_t r = 0;
    for (unsigned i = 0; i < bits; i++) r |= ((x >> i) & 1ULL) << (bits - 1 - i);
    return r;
}

uint64_t ipr_div2_uint_mod(uint64_t x, uint64_t m) { /* arith.rs:89-100 */
    if (x & 1) {
        u128 s = (u128)x + m;
        return (uint64_t)(s >> 1);
    }
    return x >> 1;
}

/* floor(2^128 / modulus) split into (low, high) words: get_barrett_crs arith.rs:117-122 */
void ipr_get_barrett_crs(uint64_t modulus, uint64_t *cr0, uint64_t *cr1) {
    /* long division of 2^128 by a 64-bit modulus */
    u128 hi_num = ((u128)1 << 64);          /* 2^128 / 2^64 */
    u128 qhi = hi_num / modulus;            /* quotient of the upper 64+1 bits */
    u128 rem = hi_num % modulus;
    u128 lo_part = (rem << 64);             /* rem < modulus < 2^64 */
    u128 qlo = lo_part / modulus;
    /* 2^128 / m = qhi * 2^64 + qlo */
    *cr0 = (uint64_t)qlo;
    *cr1 = (uint64_t)qhi;
}

uint64_t ipr_barrett_raw_u64(uint64_t in, uint64_t cr1, uint64_t modulus) { /* arith.rs:133-141 */
    uint64_t tmp = (uint64_t)(((u128)in * cr1) >> 64);
    uint64_t res = in - tmp * modulus;
    return res >= modulus ? res - modulus : res;
}

/* barrett_raw_u128 + one conditional subtraction, arith.rs:172-209 */
uint64_t ipr_barrett_reduction_u128_raw(uint64_t modulus, uint64_t cr0, uint64_t cr1, uint64_t zx,
                                        uint64_t zy) {
    uint64_t carry = (uint64_t)(((u128)zx * cr0) >> 64);
    u128 t2 = (u128)zx * cr1;
    uint64_t t2x = (uint64_t)t2, t2y = (uint64_t)(t2 >> 64);
    uint64_t tmp1 = t2x + carry;
    uint64_t tmp3 = t2y + (tmp1 < t2x);
    t2 = (u128)zy * cr0;
    t2x = (uint64_t)t2;
    t2y = (uint64_t)(t2 >> 64);
    uint64_t old = tmp1;
    tmp1 = old + t2x;
    carry = t2y + (tmp1 < old);
    tmp1 = zy * cr1 + tmp3 + carry;
    uint64_t r = zx - tmp1 * modulus;
    if (r >= modulus) r -= modulus;
    return r;
}

uint64_t ipr_invert_uint_mod(uint64_t v, uint64_t m) { /* number_theory.rs:57-96 */
    if (v == 0) return 0;
    int64_t prev_a = 1, a = 0;
    uint64_t x = v, y = m;
    while (y != 0) {
        uint64_t q = x / y, t = x % y;
        x = y;
        y = t;
        int64_t tmp = a;
        a = prev_a - (int64_t)q * a;
        prev_a = tmp;
    }
    if (x != 1) return 0;
    return prev_a < 0 ? (uint64_t)prev_a + m : (uint64_t)prev_a;
}

/* get_minimal_primitive_root number_theory.rs:41-55: the smallest primitive
 * `degree`-th root of unity (the minimum over all odd powers of any one). */
uint64_t ipr_minimal_primitive_root(uint64_t degree, uint64_t modulus) {
    uint64_t g = 0;
    for (uint64_t r = 2; r < modulus; r++) {
        uint64_t c = powmod(r, (modulus - 1) / degree, modulus);
        if (c != 0 && powmod(c, degree >> 1, modulus) == modulus - 1) {
            g = c;
            break;
        }
    }
    uint64_t best = g, cur = g, g2 = mulmod(g, g, modulus);
    for (uint64_t i = 0; i < degree; i++) {
        if (cur < best) best = cur;
        cur = mulmod(cur, g2, modulus);
    }
    return best;
}

/* crt_compose_2 core/params.rs:203-215 */
uint64_t ipr_crt_compose(const ipr_params *p, uint64_t x, uint64_t y) {
    u128 v = (u128)x * p->mod1_inv_mod0 + (u128)y * p->mod0_inv_mod1;
    return ipr_barrett_reduction_u128_raw(p->modulus, p->cr0_mod, p->cr1_mod, (uint64_t)v,
                                          (uint64_t)(v >> 64));
}

/* rescale arith.rs:436-452 (round half away from zero, centred input) */
uint64_t ipr_rescale(uint64_t a, uint64_t inp_mod, uint64_t out_mod) {
    int64_t inp_mod_i = (int64_t)inp_mod;
    __int128 out_mod_i = (__int128)out_mod;
    int64_t inp_val = (int64_t)(a % inp_mod);
    if (inp_val >= inp_mod_i / 2) inp_val -= inp_mod_i;
    int64_t sign = inp_val >= 0 ? 1 : -1;
    __int128 val = (__int128)inp_val * (__int128)out_mod;
    __int128 result = (val + (__int128)(sign * (inp_mod_i / 2))) / (__int128)inp_mod;
    result = (result + (__int128)((inp_mod / out_mod) * out_mod) + 2 * out_mod_i) % out_mod_i;
    return (uint64_t)((result + out_mod_i) % out_mod_i);
}

/* ------------------------------------------------------------------ */
/* Params + NTT tables                                                  */
/* ------------------------------------------------------------------ */

/* powers_of_primitive_root ntt.rs:6-17 */
static void powers_of_root(uint64_t root, uint64_t m, uint64_t *out) {
    uint64_t power = root;
    for (uint64_t i = 1; i < IPR_N; i++) {
        out[ipr_reverse_bits(i, IPR_LOGN)] = power;
        power = mulmod(power, root, m);
    }
    out[0] = 1;
}

/* scale_powers_u32 ntt.rs:29-37 */
static void scale_u32(uint64_t m, const uint64_t *in, uint64_t *out) {
    for (int i = 0; i < IPR_N; i++) out[i] = (uint64_t)(uint32_t)((in[i] << 32) / m);
}

void ipr_params_init(ipr_params *p) { /* Params::init core/params.rs:225-301 */
    memset(p, 0, sizeof(*p));
    p->q[0] = IPR_Q0;
    p->q[1] = IPR_Q1;
    p->modulus = IPR_Q0 * IPR_Q1;
    p->modulus_log2 = (uint64_t)ceil(log2((double)p->modulus));
    for (int i = 0; i < 2; i++) ipr_get_barrett_crs(p->q[i], &p->barrett_cr0[i], &p->barrett_cr1[i]);
    ipr_get_barrett_crs(p->modulus, &p->cr0_mod, &p->cr1_mod);
    p->mod0_inv_mod1 = IPR_Q0 * ipr_invert_uint_mod(IPR_Q0, IPR_Q1);
    p->mod1_inv_mod0 = IPR_Q1 * ipr_invert_uint_mod(IPR_Q1, IPR_Q0);
    for (int l = 0; l < 2; l++) { /* build_ntt_tables ntt.rs:74-108 */
        uint64_t m = p->q[l];
        uint64_t root = ipr_minimal_primitive_root(2 * IPR_N, m);
        p->root[l] = root;
        uint64_t inv_root = ipr_invert_uint_mod(root, m);
        powers_of_root(root, m, p->ntt[l][0]);
        scale_u32(m, p->ntt[l][0], p->ntt[l][1]);
        powers_of_root(inv_root, m, p->ntt[l][2]);
        for (int i = 0; i < IPR_N; i++) p->ntt[l][2][i] = ipr_div2_uint_mod(p->ntt[l][2][i], m);
        scale_u32(m, p->ntt[l][2], p->ntt[l][3]);
    }
}

/* ntt_forward, scalar Harvey butterfly, ntt.rs:111-160 */
void ipr_ntt_forward(const ipr_params *p, uint64_t *data) {
    for (int l = 0; l < 2; l++) {
        uint64_t *op = data + l * IPR_N;
        const uint64_t *w_tab = p->ntt[l][0], *wp_tab = p->ntt[l][1];
        uint32_t q = (uint32_t)p->q[l], two_q = 2 * q;
        for (int mm = 0; mm < IPR_LOGN; mm++) {
            int m = 1 << mm, t = IPR_N >> (mm + 1);
            for (int i = 0; i < m; i++) {
                uint64_t w = w_tab[m + i], wp = wp_tab[m + i];
                uint64_t *o = op + 2 * t * i;
                for (int j = 0; j < t; j++) {
                    uint32_t x = (uint32_t)o[j], y = (uint32_t)o[t + j];
                    uint32_t cx = x - two_q * (uint32_t)(x >= two_q);
                    uint64_t qt = ((uint64_t)y * wp) >> 32;
                    uint64_t qn = w * (uint64_t)y - qt * (uint64_t)q;
                    o[j] = (uint64_t)cx + qn;
                    o[t + j] = (uint64_t)cx + ((uint64_t)two_q - qn);
                }
            }
        }
        for (int i = 0; i < IPR_N; i++) {
            op[i] -= (uint64_t)(op[i] >= two_q) * two_q;
            op[i] -= (uint64_t)(op[i] >= q) * q;
        }
    }
}

/* ntt_inverse, scalar Gentleman-Sande with halved twiddles, ntt.rs:731-780 */
void ipr_ntt_inverse(const ipr_params *p, uint64_t *data) {
    for (int l = 0; l < 2; l++) {
        uint64_t *op = data + l * IPR_N;
        const uint64_t *w_tab = p->ntt[l][2], *wp_tab = p->ntt[l][3];
        uint64_t q = p->q[l], two_q = 2 * q;
        for (int mm = IPR_LOGN - 1; mm >= 0; mm--) {
            int h = 1 << mm, t = IPR_N >> (mm + 1);
            for (int i = 0; i < h; i++) {
                uint64_t w = w_tab[h + i], wp = wp_tab[h + i];
                uint64_t *o = op + 2 * t * i;
                for (int j = 0; j < t; j++) {
                    uint64_t x = o[j], y = o[t + j];
                    uint64_t tt = two_q - y + x;
                    uint64_t cx = x + y - two_q * (uint64_t)((x << 1) >= tt);
                    uint64_t ht = (tt * wp) >> 32;
                    o[j] = (cx + q * (tt & 1)) >> 1;
                    o[t + j] = w * tt - ht * q;
                }
            }
        }
        for (int i = 0; i < IPR_N; i++) {
            op[i] -= (uint64_t)(op[i] >= two_q) * two_q;
            op[i] -= (uint64_t)(op[i] >= q) * q;
        }
    }
}

void ipr_to_ntt(const ipr_params *p, const uint64_t *raw, uint64_t *out) {
    for (int l = 0; l < 2; l++)
        for (int z = 0; z < IPR_N; z++)
            out[l * IPR_N + z] = ipr_barrett_raw_u64(raw[z], p->barrett_cr1[l], p->q[l]);
    ipr_ntt_forward(p, out);
}

void ipr_from_ntt(const ipr_params *p, const uint64_t *in, uint64_t *raw) {
    uint64_t s[2 * IPR_N];
    memcpy(s, in, sizeof(s));
    ipr_ntt_inverse(p, s);
    for (int z = 0; z < IPR_N; z++) raw[z] = ipr_crt_compose(p, s[z], s[IPR_N + z]);
}

/* gadget_invert_rdim with rdim = 2, mx = 6 (gadget.rs:3-9, 35-61) */
void ipr_gadget_invert_2(const ipr_params *p, const uint64_t *in2, uint64_t *out6) {
    const unsigned num_elems = 3;
    unsigned bits_per = (unsigned)floor((double)p->modulus_log2 / (double)num_elems) + 1; /* 19 */
    uint64_t mask = (1ULL << bits_per) - 1;
    for (int j = 0; j < 2; j++)
        for (int z = 0; z < IPR_N; z++) {
            uint64_t v = in2[j * IPR_N + z];
            for (unsigned k = 0; k < num_elems; k++) {
                unsigned off = k * bits_per;
                out6[(j + k * 2) * IPR_N + z] = off >= 64 ? 0 : (v >> off) & mask;
            }
        }
}

/* gadget_invert_rdim (gadget.rs:35-61) for any mx = rows * num_elems:
 * out row j + k*rows holds bits [k*bits_per, (k+1)*bits_per) of input row j */
void ipr_gadget_invert_general(const ipr_params *p, const uint64_t *in, unsigned rows, unsigned num_elems,
                               uint64_t *out) {
    unsigned bits_per = (num_elems == p->modulus_log2)
                            ? 1
                            : (unsigned)floor((double)p->modulus_log2 / (double)num_elems) + 1;
    uint64_t mask = (1ULL << bits_per) - 1;
    for (unsigned j = 0; j < rows; j++)
        for (int z = 0; z < IPR_N; z++) {
            uint64_t v = in[(size_t)j * IPR_N + z];
            for (unsigned k = 0; k < num_elems; k++) {
                unsigned off = k * bits_per;
                out[((size_t)j + (size_t)k * rows) * IPR_N + z] = off >= 64 ? 0 : (v >> off) & mask;
            }
        }
}

/* ------------------------------------------------------------------ */
/* automorphisms                                                        */
/* ------------------------------------------------------------------ */

void ipr_automorph_poly(const ipr_params *p, const uint64_t *a, uint64_t *res, uint64_t t) {
    for (uint64_t i = 0; i < IPR_N; i++) { /* poly.rs:531-543 */
        uint64_t num = (i * t) / IPR_N, rem = (i * t) % IPR_N;
        res[rem] = (num % 2 == 0) ? a[i] : p->modulus - a[i];
    }
}

/* Closed form of generate_automorph_tables_brute_force (packing.rs:1423-1468):
 * forward-NTT slot s evaluates at psi^(2*brv(s)+1), so NTT(a(x^t))[s] =
 * NTT(a)[slot of t*(2*brv(s)+1) mod 2N]. */
void ipr_automorph_table(uint64_t t, uint32_t *table) {
    for (uint64_t s = 0; s < IPR_N; s++) {
        uint64_t e = 2 * ipr_reverse_bits(s, IPR_LOGN) + 1;
        uint64_t e2 = (t * e) % (2 * IPR_N);
        table[s] = (uint32_t)ipr_reverse_bits((e2 - 1) / 2, IPR_LOGN);
    }
}

uint64_t ipr_synth(uint64_t seed, uint64_t stream, uint64_t idx);

/* Brute-force definition, restated: for a random poly a, table[j] = i such
 * that NTT(a)[i] == NTT(auto_t(a))[j] (limb 0), unique.  Returns 0 on success,
 * 1 if a value collision made the match ambiguous. */
int ipr_automorph_table_bruteforce(const ipr_params *p, uint64_t t, uint32_t *table, uint64_t seed) {
    uint64_t *a = malloc(sizeof(uint64_t) * IPR_N), *b = malloc(sizeof(uint64_t) * IPR_N);
    uint64_t *an = malloc(sizeof(uint64_t) * 2 * IPR_N), *bn = malloc(sizeof(uint64_t) * 2 * IPR_N);
    for (int i = 0; i < IPR_N; i++) a[i] = ipr_synth(seed, 77, (uint64_t)i) % p->modulus;
    ipr_automorph_poly(p, a, b, t);
    ipr_to_ntt(p, a, an);
    ipr_to_ntt(p, b, bn);
    int bad = 0;
    for (int i = 0; i < IPR_N && !bad; i++) {
        int total = 0, found = -1;
        for (int j = 0; j < IPR_N; j++)
            if (an[i] == bn[j]) {
                total++;
                found = j;
            }
        if (total != 1) bad = 1;
        else table[found] = (uint32_t)i;
    }
    free(a); free(b); free(an); free(bn);
    return bad;
}

uint64_t ipr_gen_pow(unsigned i) { return powmod(5, i, 2 * IPR_N); }

/* ------------------------------------------------------------------ */
/* bits (util.rs:289-321), little-endian byte order                     */
/* ------------------------------------------------------------------ */

uint64_t ipr_read_bits(const uint8_t *data, size_t bit_offs, unsigned num_bits) {
    uint64_t v = 0;
    for (unsigned i = 0; i < num_bits; i++) {
        size_t b = bit_offs + i;
        v |= (uint64_t)((data[b >> 3] >> (b & 7)) & 1) << i;
    }
    return v;
}

void ipr_write_bits(uint8_t *data, uint64_t val, size_t bit_offs, unsigned num_bits) {
    for (unsigned i = 0; i < num_bits; i++) {
        size_t b = bit_offs + i;
        uint8_t bit = (uint8_t)((val >> i) & 1);
        data[b >> 3] = (uint8_t)((data[b >> 3] & ~(1u << (b & 7))) | (bit << (b & 7)));
    }
}

/* ------------------------------------------------------------------ */
/* ChaCha20                                                             */
/* ------------------------------------------------------------------ */

#define ROTL(x, n) (((x) << (n)) | ((x) >> (32 - (n))))
#define QR(a, b, c, d)                                                                          \
    a += b; d ^= a; d = ROTL(d, 16); c += d; b ^= c; b = ROTL(b, 12);                         \
    a += b; d ^= a; d = ROTL(d, 8);  c += d; b ^= c; b = ROTL(b, 7);

static void chacha_core(const uint32_t in[16], uint32_t out[16]) {
    uint32_t x[16];
    memcpy(x, in, sizeof(x));
    for (int r = 0; r < 10; r++) {
        QR(x[0], x[4], x[8], x[12]) QR(x[1], x[5], x[9], x[13])
        QR(x[2], x[6], x[10], x[14]) QR(x[3], x[7], x[11], x[15])
        QR(x[0], x[5], x[10], x[15]) QR(x[1], x[6], x[11], x[12])
        QR(x[2], x[7], x[8], x[13]) QR(x[3], x[4], x[9], x[14])
    }
    for (int i = 0; i < 16; i++) out[i] = x[i] + in[i];
}

static const uint32_t SIGMA[4] = {0x61707865, 0x3320646e, 0x79622d32, 0x6b206574};

/* rand_chacha layout: words 12-13 = 64-bit block counter, 14-15 = 64-bit stream id */
void ipr_chacha20_block(const uint32_t key[8], uint64_t counter, uint64_t stream, uint32_t out[16]) {
    uint32_t s[16];
    memcpy(s, SIGMA, 16);
    memcpy(s + 4, key, 32);
    s[12] = (uint32_t)counter;
    s[13] = (uint32_t)(counter >> 32);
    s[14] = (uint32_t)stream;
    s[15] = (uint32_t)(stream >> 32);
    chacha_core(s, out);
}

/* RFC 8439 layout (32-bit counter, 96-bit nonce) for the published test vector */
void ipr_chacha20_rfc8439_block(const uint32_t key[8], uint32_t counter, const uint32_t nonce[3],
                                uint32_t out[16]) {
    uint32_t s[16];
    memcpy(s, SIGMA, 16);
    memcpy(s + 4, key, 32);
    s[12] = counter;
    s[13] = nonce[0];
    s[14] = nonce[1];
    s[15] = nonce[2];
    chacha_core(s, out);
}

void ipr_chacha_seed(ipr_chacha_rng *r, const uint8_t seed[32]) {
    for (int i = 0; i < 8; i++)
        r->key[i] = (uint32_t)seed[4 * i] | ((uint32_t)seed[4 * i + 1] << 8) |
                    ((uint32_t)seed[4 * i + 2] << 16) | ((uint32_t)seed[4 * i + 3] << 24);
    r->counter = 0;
    r->idx = 64; /* empty buffer: 4 blocks generated per refill */
}

uint64_t ipr_chacha_next_u64(ipr_chacha_rng *r) {
    if (r->idx + 2 > 64) {
        for (int b = 0; b < 4; b++) ipr_chacha20_block(r->key, r->counter + b, 0, r->buf + 16 * b);
        r->counter += 4;
        r->idx = 0;
    }
    uint64_t lo = r->buf[r->idx], hi = r->buf[r->idx + 1];
    r->idx += 2;
    return lo | (hi << 32);
}

/* keyword.rs:546-555: ct_gsw row 0, column i = NTT(-a_i), a_i = random_rng(ChaCha20(RGSW_SEEDS[i]))
 * (poly.rs:211-231: StandardUniform u64 % modulus).  All six RGSW_SEEDS are [7;32]
 * (wire.rs:88-113), so one polynomial serves every column. */
void ipr_rgsw_row0(const ipr_params *p, uint64_t out[2 * IPR_N]) {
    uint8_t seed[32];
    memset(seed, 7, 32);
    ipr_chacha_rng r;
    ipr_chacha_seed(&r, seed);
    uint64_t a[IPR_N];
    for (int i = 0; i < IPR_N; i++) a[i] = p->modulus - ipr_chacha_next_u64(&r) % p->modulus;
    ipr_to_ntt(p, a, out);
}

/* PolyMatrixRaw::random_rng (poly.rs:211-231): `count` coefficients, each one ChaCha20Rng u64
 * reduced mod q, from a generator seeded with `seed`.  The test client draws with it the public
 * `a` polynomials of its query ciphertexts (get_seed(SEED_0), client/online.rs:164-168, 216-250)
 * and of its RGSW ciphertexts (RGSW_SEEDS, client/keyword.rs:168-181). */
void ipr_oracle_random_raw(const ipr_params *p, const uint8_t seed[32], uint64_t count, uint64_t *out) {
    ipr_chacha_rng r;
    ipr_chacha_seed(&r, seed);
    for (uint64_t i = 0; i < count; i++) out[i] = ipr_chacha_next_u64(&r) % p->modulus;
}

/* `count` ChaCha20 blocks of stream `stream` from block counter `first`, key = the 32-byte
 * seed read as little-endian words (rand_chacha's layout): the test model of the device
 * client draws its key shuffle and its centered binomial noise from these */
void ipr_oracle_chacha_blocks(const uint8_t seed[32], uint64_t stream, uint64_t first, uint64_t count,
                              uint32_t *out) {
    uint32_t key[8];
    for (int i = 0; i < 8; i++)
        key[i] = (uint32_t)seed[4 * i] | ((uint32_t)seed[4 * i + 1] << 8) | ((uint32_t)seed[4 * i + 2] << 16) |
                 ((uint32_t)seed[4 * i + 3] << 24);
#pragma omp parallel for schedule(static)
    for (int64_t b = 0; b < (int64_t)count; b++) ipr_chacha20_block(key, first + (uint64_t)b, stream, out + 16 * b);
}

/* rescale (arith.rs:436-452) over an array */
void ipr_oracle_rescale_many(const uint64_t *in, uint64_t n, uint64_t inp_mod, uint64_t out_mod, uint64_t *out) {
    for (uint64_t i = 0; i < n; i++) out[i] = ipr_rescale(in[i], inp_mod, out_mod);
}

/* ------------------------------------------------------------------ */
/* shape plan                                                           */
/* ------------------------------------------------------------------ */

static uint64_t next_pow2(uint64_t x) {
    uint64_t r = 1;
    while (r < x) r <<= 1;
    return r;
}

/* max_interpolate_degree wire.rs:386-412 */
static uint64_t max_interp_degree(double modulus, double d0, double p, double t_exp, double t_rgsw,
                                  double poly_len) {
    double sigma_x = 6.4;
    double modulus_len = log2(modulus);
    double z1 = pow(2.0, (int)ceil(modulus_len / t_exp));
    double z2 = pow(2.0, (int)ceil(modulus_len / t_rgsw));
    double term1 = d0 * (p * p) * (sigma_x * sigma_x);
    double term2 = t_exp * (poly_len * poly_len) * (z1 * z1) * (sigma_x * sigma_x) / 4.0;
    double term3 = t_rgsw * poly_len * (z2 * z2) * (sigma_x * sigma_x) / 2.0;
    double total = log2(sqrt(term1 + term2 + term3));
    double ub = log2(modulus / (2. * 2. * p)) - log2(sqrt(2.0 * 41.0 * log(2.0)));
    double mx = 2. * (ub - total);
    if (mx < 0) return 0;
    uint64_t m = (uint64_t)floor(pow(2.0, mx));
    return m < (uint64_t)poly_len ? m : (uint64_t)poly_len;
}

/* params_rgswpir_given_input_size_and_dim0 wire.rs:414-477 -> (instances, interp, db_rows) */
static int rgswpir_params(uint64_t num_items, uint64_t item_bits, uint64_t dim0, uint64_t *instances,
                          uint64_t *interp_out, uint64_t *db_rows_out) {
    const double poly_len = 2048, log_p = 16;
    double modulus = (double)(IPR_Q0 * IPR_Q1);
    uint64_t mx = max_interp_degree(modulus, (double)dim0, 65535.0, 3.0, 3.0, poly_len);
    if (mx <= 1) return IPR_E_ARGS;
    double bits_per_poly = poly_len * log_p;
    uint64_t factor = (uint64_t)floor(bits_per_poly / (double)item_bits);
    if (factor == 0) factor = 1;
    uint64_t n_items = (uint64_t)ceil((double)num_items / (double)factor);
    uint64_t item_sz = item_bits * factor;
    uint64_t padded_bits = (uint64_t)ceil((double)item_sz / bits_per_poly) * (uint64_t)bits_per_poly;
    uint64_t padded_pts = (uint64_t)ceil((double)padded_bits / log_p);
    uint64_t lower = padded_pts * (uint64_t)ceil((double)n_items / (double)dim0);
    uint64_t cur = padded_pts, interp = 1;
    while (cur < lower) {
        interp *= 2;
        cur *= 2;
        if (2 * interp > mx) break;
    }
    uint64_t new_pts = (uint64_t)ceil((double)lower / (double)cur) * cur; /* round_up_to_multiple_of */
    uint64_t db_rows = dim0 >= 8 ? dim0 : 8;
    *instances = (uint64_t)ceil((double)new_pts / poly_len);
    *interp_out = interp;
    *db_rows_out = db_rows;
    return IPR_OK;
}

/* KeywordServerSetupPlan::from_shape keyword.rs:145-233 + estimate keyword.rs:105-141 */
int ipr_plan_from_shape(uint64_t record_count, uint64_t key_size, uint64_t value_size,
                        uint64_t buckets, uint64_t dim0, ipr_plan *out) {
    if (record_count == 0 || key_size == 0 || value_size == 0) return IPR_E_ARGS;
    uint64_t rc = record_count < 512 ? 512 : record_count;
    uint64_t num_items = buckets ? buckets : next_pow2(rc * 2);
    if (num_items < record_count) return IPR_E_ARGS;
    uint64_t entry = key_size + value_size, bits = entry * 8;
    if (bits % 16 != 0) return IPR_E_ARGS;
    uint64_t inst, interp, rows;
    if (!dim0) {
        uint64_t d = num_items >= 256000000ULL ? 32768 : 2048;
        if (rgswpir_params(num_items, bits, d, &inst, &interp, &rows)) return IPR_E_ARGS;
        dim0 = rows;
    }
    if (rgswpir_params(num_items, bits, dim0, &inst, &interp, &rows)) return IPR_E_ARGS;
    uint64_t nr = next_pow2(rows);
    if (nr < IPR_N) return IPR_E_ARGS; /* db_dim_1 would underflow */
    out->num_items = num_items;
    out->entry_size = entry;
    out->item_size_bits = bits;
    out->dim0 = dim0;
    out->db_rows = nr;
    out->instances = inst;
    out->db_cols = inst * IPR_N;
    out->interp = interp;
    out->c = inst / interp;
    if (num_items < out->db_rows) return IPR_E_ARGS;
    uint64_t nph = IPR_N / 2;
    uint64_t db_bytes = out->db_rows * out->db_cols * 2;
    uint64_t prep = out->db_cols * 2 * IPR_N * 8;
    uint64_t rbuf = 2 * inst * nph * 2 * IPR_N * 8;
    uint64_t bt = 2 * inst * (nph - 1) * IPR_T * IPR_N * 8;
    out->peak_bytes = db_bytes + prep + rbuf + bt;
    return IPR_OK;
}

/* ------------------------------------------------------------------ */
/* respond() steps                                                      */
/* ------------------------------------------------------------------ */

int ipr_oracle_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* gemv_kernel.cu:46-103 / kernel.rs:139-237: c[j] = CRT(sum_k a_lo D, sum_k a_hi D) */
void ipr_oracle_gemv(const ipr_params *p, const ipr_oracle_db *db, const uint64_t *a, uint64_t *c) {
    int64_t cols = (int64_t)db->db_cols;
    uint64_t rows = db->db_rows;
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < cols; j++) {
        const uint16_t *col = db->db + (uint64_t)j * rows;
        u128 s0 = 0, s1 = 0;
        for (uint64_t k = 0; k < rows; k++) {
            s0 += (uint64_t)(uint32_t)a[k] * col[k];
            s1 += (a[k] >> 32) * col[k];
        }
        uint64_t r0 = (uint64_t)(s0 % p->q[0]), r1 = (uint64_t)(s1 % p->q[1]);
        c[j] = ipr_crt_compose(p, r0, r1);
    }
}

/* generate_rotations_double packing.rs:1756-1785 / rotation_kernel.cu:21-59:
 * y_all[i][k][z] = y[k][tab_{g_i}[z]], y_bar_all[i][k][z] = y[k][tab_{2N-g_i}[z]] */
void ipr_oracle_rotations(const uint64_t *y_body, uint64_t *y_all, uint64_t *y_bar_all) {
    uint32_t *t1 = malloc(sizeof(uint32_t) * IPR_N), *t2 = malloc(sizeof(uint32_t) * IPR_N);
    for (unsigned i = 0; i < IPR_NROT; i++) {
        uint64_t g = ipr_gen_pow(i);
        ipr_automorph_table(g, t1);
        ipr_automorph_table(2 * IPR_N - g, t2);
        for (int k = 0; k < IPR_T; k++)
            for (int z = 0; z < IPR_N; z++) {
                size_t o = ((size_t)i * IPR_T + k) * IPR_N + z;
                y_all[o] = y_body[k * IPR_N + t1[z]];
                y_bar_all[o] = y_body[k * IPR_N + t2[z]];
            }
    }
    free(t1);
    free(t2);
}

/* packing_online_kernel.cu:18-92 / full_packing_with_preprocessing_online packing.rs:2941-3012:
 * S[j][l][z] = sum_{i,k} y_l[i,k][z] T_l[j][i,k][z] + ybar T_bar + sum_k z_l[k][z] T_hat_l[j][k][z] mod q_l */
void ipr_oracle_packing_sum(const ipr_params *p, const ipr_oracle_db *db, const uint64_t *y_body,
                            const uint64_t *z_body, uint64_t *S) {
    size_t ysz = (size_t)IPR_NINNER * IPR_N;
    uint64_t *y_all = malloc(sizeof(uint64_t) * ysz), *yb_all = malloc(sizeof(uint64_t) * ysz);
    ipr_oracle_rotations(y_body, y_all, yb_all);
    int64_t nout = (int64_t)db->num_outputs;
#pragma omp parallel for schedule(dynamic)
    for (int64_t j = 0; j < nout; j++) {
        const uint64_t *T = db->bold_t + (size_t)j * ysz;
        const uint64_t *Tb = db->bold_t_bar + (size_t)j * ysz;
        const uint64_t *Th = db->bold_t_hat + (size_t)j * IPR_T * IPR_N;
        u128 *acc = calloc(2 * IPR_N, sizeof(u128));
        for (size_t r = 0; r < IPR_NINNER; r++) {
            const uint64_t *yr = y_all + r * IPR_N, *ybr = yb_all + r * IPR_N;
            const uint64_t *tr = T + r * IPR_N, *tbr = Tb + r * IPR_N;
            for (int z = 0; z < IPR_N; z++) {
                acc[z] += (u128)((uint64_t)(uint32_t)yr[z] * (uint32_t)tr[z]) +
                          (uint64_t)(uint32_t)ybr[z] * (uint32_t)tbr[z];
                acc[IPR_N + z] += (u128)((yr[z] >> 32) * (tr[z] >> 32)) + (ybr[z] >> 32) * (tbr[z] >> 32);
            }
        }
        for (int k = 0; k < IPR_T; k++)
            for (int z = 0; z < IPR_N; z++) {
                uint64_t zv = z_body[k * IPR_N + z], tv = Th[k * IPR_N + z];
                acc[z] += (uint64_t)(uint32_t)zv * (uint32_t)tv;
                acc[IPR_N + z] += (zv >> 32) * (tv >> 32);
            }
        for (int z = 0; z < IPR_N; z++) {
            S[(size_t)j * 2 * IPR_N + z] = (uint64_t)(acc[z] % p->q[0]);
            S[(size_t)j * 2 * IPR_N + IPR_N + z] = (uint64_t)(acc[IPR_N + z] % p->q[1]);
        }
        free(acc);
    }
    free(y_all);
    free(yb_all);
}

/* packing_online.rs:359-397: packed_j = (a_hat_j, INTT(S_j) + b_poly_j), sum not reduced.
 * gamma = poly_len, so group_size = 1 and b_poly_j[k] = b_values[j*N + k]. */
void ipr_oracle_postprocess(const ipr_params *p, const ipr_oracle_db *db, const uint64_t *S,
                            const uint64_t *b_values, uint64_t *packed) {
    int64_t nout = (int64_t)db->num_outputs;
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < nout; j++) {
        uint64_t raw[IPR_N];
        ipr_from_ntt(p, S + (size_t)j * 2 * IPR_N, raw);
        uint64_t *dst = packed + (size_t)j * 2 * IPR_N;
        memcpy(dst, db->a_hat + (size_t)j * IPR_N, sizeof(uint64_t) * IPR_N);
        for (int k = 0; k < IPR_N; k++) dst[IPR_N + k] = b_values[(size_t)j * IPR_N + k] + raw[k];
    }
}

/* RGSW fold keyword.rs:543-574: for each group wp, s = 0; for i = interp-1 .. 0:
 *   s = from_ntt(CT_gsw * to_ntt(G^-1(s))) + packed[wp*interp + i]  (mod q)
 * CT_gsw = [row0: NTT(-a) in all 6 columns; row1: ct_gsw_body columns 0..5] (multiply poly.rs:613-634). */
void ipr_oracle_fold(const ipr_params *p, const ipr_oracle_db *db, const uint64_t *row0,
                     const uint64_t *body, const uint64_t *packed, uint64_t *results) {
    int64_t c = (int64_t)db->c;
    uint64_t interp = db->interp;
#pragma omp parallel for schedule(dynamic)
    for (int64_t wp = 0; wp < c; wp++) {
        uint64_t *sum = calloc(2 * IPR_N, sizeof(uint64_t));
        uint64_t *g = malloc(sizeof(uint64_t) * 6 * IPR_N);
        uint64_t *gn = malloc(sizeof(uint64_t) * 6 * 2 * IPR_N);
        uint64_t *prod = malloc(sizeof(uint64_t) * 2 * 2 * IPR_N);
        for (int64_t i = (int64_t)interp - 1; i >= 0; i--) {
            ipr_gadget_invert_2(p, sum, g);
            for (int r = 0; r < 6; r++) ipr_to_ntt(p, g + r * IPR_N, gn + r * 2 * IPR_N);
            for (int row = 0; row < 2; row++)
                for (int l = 0; l < 2; l++)
                    for (int z = 0; z < IPR_N; z++) {
                        u128 acc = 0;
                        for (int k = 0; k < 6; k++) {
                            uint64_t a = row == 0 ? row0[l * IPR_N + z]
                                                  : body[(size_t)k * 2 * IPR_N + l * IPR_N + z];
                            acc += (u128)a * gn[k * 2 * IPR_N + l * IPR_N + z];
                        }
                        prod[row * 2 * IPR_N + l * IPR_N + z] = (uint64_t)(acc % p->q[l]);
                    }
            const uint64_t *pk = packed + (size_t)(wp * (int64_t)interp + i) * 2 * IPR_N;
            for (int row = 0; row < 2; row++) {
                uint64_t raw[IPR_N];
                ipr_from_ntt(p, prod + row * 2 * IPR_N, raw);
                for (int z = 0; z < IPR_N; z++)
                    sum[row * IPR_N + z] = (raw[z] + pk[row * IPR_N + z]) % p->modulus;
            }
        }
        memcpy(results + (size_t)wp * 2 * IPR_N, sum, sizeof(uint64_t) * 2 * IPR_N);
        free(sum); free(g); free(gn); free(prod);
    }
}

/* switch_and_keep modulus_switch.rs:45-73 with q1' = 2^20, q2' = 268369921, keep N */
void ipr_oracle_switch(const ipr_params *p, const uint64_t *result, uint8_t *out) {
    memset(out, 0, IPR_RESULT_BYTES);
    size_t bo = 0;
    for (int z = 0; z < IPR_N; z++, bo += 28)
        ipr_write_bits(out, ipr_rescale(result[z], p->modulus, IPR_QP2), bo, 28);
    for (int z = 0; z < IPR_N; z++, bo += 20)
        ipr_write_bits(out, ipr_rescale(result[IPR_N + z], p->modulus, IPR_QP1), bo, 20);
}

/* ------------------------------------------------------------------ */
/* wire                                                                 */
/* ------------------------------------------------------------------ */

size_t ipr_query_bytes(uint64_t db_rows, unsigned nq) { /* serialize_keyword_query wire.rs:542-615 */
    uint64_t nvals = (uint64_t)IPR_T * IPR_N * 2 + (uint64_t)nq * (db_rows + 2 * IPR_T * IPR_N);
    return (size_t)((8 + nvals * 56 + 7) / 8);
}

/* deserialize_keyword_query wire.rs:618-705.  Output layouts:
 * y_body,z_body [3][N] condensed; query_rows [nq][db_rows] condensed;
 * gsw_bodies [nq][6][2][N] (limb-major per poly). */
int ipr_oracle_parse_query(const uint8_t *buf, size_t len, uint64_t db_rows, unsigned *num_queries,
                           uint64_t *y_body, uint64_t *z_body, uint64_t *query_rows,
                           uint64_t *gsw_bodies, unsigned max_queries) {
    if (len < 1) return IPR_E_FORMAT;
    unsigned nq = buf[0];
    *num_queries = nq;
    if (len < ipr_query_bytes(db_rows, nq)) return IPR_E_FORMAT;
    if (nq > max_queries) return IPR_E_SPACE;
    const uint64_t m28 = (1ULL << 28) - 1;
    size_t bo = 8;
    for (int i = 0; i < IPR_T; i++)
        for (int k = 0; k < IPR_N; k++) {
            uint64_t v = ipr_read_bits(buf, bo, 56); bo += 56;
            y_body[i * IPR_N + k] = (v & m28) | (((v >> 28) & m28) << 32);
            v = ipr_read_bits(buf, bo, 56); bo += 56;
            z_body[i * IPR_N + k] = (v & m28) | (((v >> 28) & m28) << 32);
        }
    for (unsigned q = 0; q < nq; q++) {
        for (uint64_t r = 0; r < db_rows; r++) {
            uint64_t v = ipr_read_bits(buf, bo, 56); bo += 56;
            query_rows[q * db_rows + r] = (v & m28) | (((v >> 28) & m28) << 32);
        }
        for (int c = 0; c < 2 * IPR_T; c++)
            for (int z = 0; z < IPR_N; z++) {
                uint64_t v = ipr_read_bits(buf, bo, 56); bo += 56;
                uint64_t *poly = gsw_bodies + ((size_t)q * 6 + c) * 2 * IPR_N;
                poly[z] = v & m28;
                poly[IPR_N + z] = (v >> 28) & m28;
            }
    }
    return IPR_OK;
}

size_t ipr_response_bytes(const ipr_oracle_db *db, unsigned nq) { /* wire.rs:708-726 */
    return 4 + (size_t)nq * (4 + db->c * IPR_RESULT_BYTES) + 4 +
           db->stash_count * (4 + db->stash_entry_bytes);
}

static void put_u32(uint8_t *o, uint32_t v) {
    o[0] = (uint8_t)v; o[1] = (uint8_t)(v >> 8); o[2] = (uint8_t)(v >> 16); o[3] = (uint8_t)(v >> 24);
}

/* KeywordServer::respond keyword.rs:534-628 + respond_to_serialized_query :636-640 */
int ipr_oracle_respond(const ipr_params *p, const ipr_oracle_db *db, const uint8_t *query, size_t len,
                       uint8_t *out, size_t cap, size_t *out_len) {
    if (!query || len < 1) return IPR_E_FORMAT;
    unsigned nq = query[0];
    size_t need = ipr_response_bytes(db, nq);
    if (out_len) *out_len = need;
    if (len < ipr_query_bytes(db->db_rows, nq)) return IPR_E_FORMAT;
    if (cap < need) return IPR_E_SPACE;
    uint64_t *y = malloc(8 * 3 * IPR_N), *zb = malloc(8 * 3 * IPR_N);
    uint64_t *rows = malloc(8 * (nq ? nq : 1) * db->db_rows);
    uint64_t *gsw = malloc(8 * (nq ? nq : 1) * 12 * IPR_N);
    unsigned got;
    int st = ipr_oracle_parse_query(query, len, db->db_rows, &got, y, zb, rows, gsw, 255);
    if (st) { free(y); free(zb); free(rows); free(gsw); return st; }
    uint64_t no = db->num_outputs;
    uint64_t *S = malloc(8 * no * 2 * IPR_N);
    uint64_t *cvec = malloc(8 * db->db_cols);
    uint64_t *packed = malloc(8 * no * 2 * IPR_N);
    uint64_t *res = malloc(8 * db->c * 2 * IPR_N);
    uint64_t row0[2 * IPR_N];
    ipr_rgsw_row0(p, row0);
    /* the packing inner product depends only on the keys: computed once per payload
     * (the reference recomputes it per query with an identical result, keyword.rs:583-604) */
    ipr_oracle_packing_sum(p, db, y, zb, S);
    size_t o = 0;
    put_u32(out + o, nq); o += 4;
    for (unsigned q = 0; q < nq; q++) {
        ipr_oracle_gemv(p, db, rows + (size_t)q * db->db_rows, cvec);
        ipr_oracle_postprocess(p, db, S, cvec, packed);
        ipr_oracle_fold(p, db, row0, gsw + (size_t)q * 12 * IPR_N, packed, res);
        put_u32(out + o, (uint32_t)(db->c * IPR_RESULT_BYTES)); o += 4;
        for (uint64_t w = 0; w < db->c; w++, o += IPR_RESULT_BYTES)
            ipr_oracle_switch(p, res + w * 2 * IPR_N, out + o);
    }
    put_u32(out + o, (uint32_t)db->stash_count); o += 4;
    for (uint64_t s = 0; s < db->stash_count; s++) {
        put_u32(out + o, (uint32_t)db->stash_entry_bytes); o += 4;
        memcpy(out + o, db->stash + s * db->stash_entry_bytes, db->stash_entry_bytes);
        o += db->stash_entry_bytes;
    }
    free(y); free(zb); free(rows); free(gsw); free(S); free(cvec); free(packed); free(res);
    return IPR_OK;
}

/* ------------------------------------------------------------------ */
/* seeded synthetic data                                                */
/* ------------------------------------------------------------------ */

uint64_t ipr_synth(uint64_t seed, uint64_t stream, uint64_t idx) {
    uint64_t x = seed ^ (stream * 0x9E3779B97F4A7C15ULL) ^ (idx * 0xD1B54A32D192ED03ULL);
    x ^= x >> 30; x *= 0xBF58476D1CE4E5B9ULL;
    x ^= x >> 27; x *= 0x94D049BB133111EBULL;
    x ^= x >> 31;
    x += 0x9E3779B97F4A7C15ULL;
    x ^= x >> 29; x *= 0xBF58476D1CE4E5B9ULL;
    x ^= x >> 32;
    return x;
}

static uint64_t synth_condensed(uint64_t seed, uint64_t stream, uint64_t idx) {
    uint64_t x = ipr_synth(seed, stream, idx);
    return ((x & 0xffffffffULL) % IPR_Q0) | (((x >> 32) % IPR_Q1) << 32);
}

void ipr_synth_db(uint64_t seed, uint64_t db_rows, uint64_t db_cols, uint16_t *db) {
    int64_t n = (int64_t)(db_rows * db_cols);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) db[i] = (uint16_t)(ipr_synth(seed, 1, (uint64_t)i) % IPR_PT);
}

void ipr_synth_precomp(uint64_t seed, uint64_t no, uint64_t *a_hat, uint64_t *bt, uint64_t *btb,
                       uint64_t *bth) {
    const uint64_t q = IPR_Q0 * IPR_Q1;
    for (uint64_t i = 0; i < no * IPR_N; i++) a_hat[i] = ipr_synth(seed, 2, i) % q;
    int64_t n = (int64_t)(no * IPR_NINNER * IPR_N);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) {
        bt[i] = synth_condensed(seed, 3, (uint64_t)i);
        btb[i] = synth_condensed(seed, 4, (uint64_t)i);
    }
    for (uint64_t i = 0; i < no * IPR_T * IPR_N; i++) bth[i] = synth_condensed(seed, 5, i);
}

/* the slice of ipr_synth_db + ipr_synth_precomp belonging to instances
 * [first, first + count) of a server with `db_rows` rows: the same global element
 * indices, so a fold-group shard of a large synthetic server is generated alone */
void ipr_synth_shard(uint64_t seed, uint64_t db_rows, uint64_t first, uint64_t count, uint16_t *db,
                     uint64_t *a_hat, uint64_t *bt, uint64_t *btb, uint64_t *bth) {
    const uint64_t q = IPR_Q0 * IPR_Q1;
    const int64_t ndb = (int64_t)(count * IPR_N * db_rows);
    const uint64_t db0 = first * IPR_N * db_rows;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < ndb; i++) db[i] = (uint16_t)(ipr_synth(seed, 1, db0 + (uint64_t)i) % IPR_PT);
    for (uint64_t i = 0; i < count * IPR_N; i++) a_hat[i] = ipr_synth(seed, 2, first * IPR_N + i) % q;
    const int64_t n = (int64_t)(count * IPR_NINNER * IPR_N);
    const uint64_t b0 = first * IPR_NINNER * IPR_N;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) {
        bt[i] = synth_condensed(seed, 3, b0 + (uint64_t)i);
        btb[i] = synth_condensed(seed, 4, b0 + (uint64_t)i);
    }
    for (uint64_t i = 0; i < count * IPR_T * IPR_N; i++) bth[i] = synth_condensed(seed, 5, first * IPR_T * IPR_N + i);
}

/* a well-formed query payload with canonical limbs (serialize_keyword_query layout) */
int ipr_synth_query(uint64_t seed, uint64_t db_rows, unsigned nq, uint8_t *out, size_t cap,
                    size_t *out_len) {
    size_t need = ipr_query_bytes(db_rows, nq);
    *out_len = need;
    if (cap < need) return IPR_E_SPACE;
    memset(out, 0, need);
    out[0] = (uint8_t)nq;
    size_t bo = 8;
    uint64_t idx = 0;
    for (int i = 0; i < IPR_T; i++)
        for (int k = 0; k < IPR_N; k++)
            for (int yz = 0; yz < 2; yz++) {
                uint64_t v = synth_condensed(seed, 10, idx++);
                ipr_write_bits(out, (v & 0xffffffffULL) | ((v >> 32) << 28), bo, 56);
                bo += 56;
            }
    for (unsigned q = 0; q < nq; q++) {
        for (uint64_t r = 0; r < db_rows; r++) {
            uint64_t v = synth_condensed(seed, 11 + q, r);
            ipr_write_bits(out, (v & 0xffffffffULL) | ((v >> 32) << 28), bo, 56);
            bo += 56;
        }
        for (uint64_t r = 0; r < 6 * IPR_N; r++) {
            uint64_t v = synth_condensed(seed, 300 + q, r);
            ipr_write_bits(out, (v & 0xffffffffULL) | ((v >> 32) << 28), bo, 56);
            bo += 56;
        }
    }
    return IPR_OK;
}

/* ---- setup-time DB layout and encode ----------------------------------------------------- */

/* KeywordCuckooTable::to_raw_db (src/pir/keyword/cuckoo.rs:314-353): raw[(item*ise + j) *
 * db_rows + row] = big-endian u16 of entry bytes (2j, 2j+1) of bucket row*per + item, zero
 * for empty buckets and buckets past the table; ise = entry_size / 2 u16 elements. */
void ipr_oracle_raw_db(const uint8_t *entries, const uint8_t *occupied, uint64_t num_buckets,
                       uint64_t entry_size, uint64_t db_rows, uint64_t db_cols, uint64_t per,
                       uint16_t *raw) {
    const uint64_t ise = entry_size / 2;
    memset(raw, 0, db_rows * db_cols * sizeof(uint16_t));
    for (uint64_t item = 0; item < per; item++)
        for (uint64_t row = 0; row < db_rows; row++) {
            const uint64_t b = row * per + item;
            if (b >= num_buckets || !occupied[b]) continue;
            const uint8_t *e = entries + b * entry_size;
            for (uint64_t j = 0; j < ise; j++)
                raw[(item * ise + j) * db_rows + row] = (uint16_t)(((uint16_t)e[2 * j] << 8) | e[2 * j + 1]);
        }
}

/* sums mod p = 65535 (the plaintext modulus, 2^16 - 1): fold the carry back in */
static uint32_t fold65535(uint32_t x) {
    uint32_t r = (x & 0xFFFFu) + (x >> 16);
    r = (r & 0xFFFFu) + (r >> 16);
    return r >= 65535u ? r - 65535u : r;
}

/* The DB encode of gpu_encode_db (native/cuda/encode_kernel.cu:18-228, 264-386):
 * per DB row and fold group wp, the interp polynomials of columns wp*interp*N + j*N + k are
 * interpolated by a radix-2 Cooley-Tukey pass over Z_65535[X]/(X^N + 1) whose twiddles are
 * monomials: inputs in bit-reversed order, level L pairs (even, odd) at distance 2^L and
 * adds / subtracts odd * X^e with e = (2N - 2N*i/2^(L+1)) mod 2N for the i-th pair of a
 * group; the results are scaled by interp^-1 mod 65535 and stored in natural order. */
int ipr_oracle_encode_db(const uint16_t *raw, uint16_t *out, uint64_t db_rows, uint64_t db_cols,
                         uint64_t interp) {
    const uint64_t n = IPR_N, two_n = 2 * IPR_N;
    if (!interp || (interp & (interp - 1)) || db_cols % (interp * n)) return IPR_E_ARGS;
    const uint64_t c = db_cols / (interp * n);
    unsigned logi = 0;
    while ((1ull << logi) < interp) logi++;
    uint32_t inv = 1; /* interp^-1 mod 65535 (interp is a power of two, 2^16 = 1 mod 65535) */
    for (unsigned b = 0; b < (16 - logi) % 16; b++) inv = fold65535(inv * 2);
    const uint64_t unit = interp * n;
    int err = 0;
#pragma omp parallel
    {
        uint32_t *a = (uint32_t *)malloc(unit * sizeof(uint32_t));
        uint32_t *b = (uint32_t *)malloc(unit * sizeof(uint32_t));
        if (!a || !b) {
#pragma omp atomic write
            err = 1;
        } else {
#pragma omp for schedule(static) collapse(2)
            for (int64_t row = 0; row < (int64_t)db_rows; row++)
                for (int64_t wp = 0; wp < (int64_t)c; wp++) {
                    for (uint64_t j = 0; j < interp; j++) {
                        uint64_t r = 0;
                        for (unsigned t = 0; t < logi; t++) r |= ((j >> t) & 1) << (logi - 1 - t);
                        for (uint64_t k = 0; k < n; k++)
                            a[r * n + k] = raw[((uint64_t)wp * unit + j * n + k) * db_rows + (uint64_t)row];
                    }
                    for (unsigned lv = 0; lv < logi; lv++) {
                        const uint64_t gs = 2ull << lv, half = 1ull << lv;
                        for (uint64_t g = 0; g < interp / gs; g++)
                            for (uint64_t i = 0; i < half; i++) {
                                const uint64_t ev = g * gs + i, od = ev + half;
                                const uint64_t e = (two_n - two_n * i / gs) % two_n;
                                for (uint64_t k = 0; k < n; k++) {
                                    const uint64_t src = (k + two_n - e) % two_n;
                                    const uint32_t o = a[od * n + (src % n)];
                                    const uint32_t tw = src < n ? o : 65535u - o;  /* X^N = -1 */
                                    b[ev * n + k] = fold65535(a[ev * n + k] + tw);
                                    b[od * n + k] = fold65535(a[ev * n + k] + 65535u - tw);
                                }
                            }
                        uint32_t *tmp = a;
                        a = b;
                        b = tmp;
                    }
                    for (uint64_t j = 0; j < interp; j++)
                        for (uint64_t k = 0; k < n; k++)
                            out[((uint64_t)wp * unit + j * n + k) * db_rows + (uint64_t)row] =
                                (uint16_t)fold65535(a[j * n + k] * inv);
                }
        }
        free(a);
        free(b);
    }
    return err ? IPR_E_SPACE : IPR_OK;
}
