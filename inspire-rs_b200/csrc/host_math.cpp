// host_math.cpp — see host_math.hpp for the restated reference functions.
#include "host_math.hpp"

#include <cmath>
#include <cstring>

#include "ipr_status.h"

namespace ipr {

namespace {

constexpr int kN = 2048, kLogN = 11;
using u128 = unsigned __int128;

uint64_t mulmod(uint64_t a, uint64_t b, uint64_t m) { return (uint64_t)(((u128)a * b) % m); }

uint64_t powmod(uint64_t b, uint64_t e, uint64_t m) {
    uint64_t r = 1 % m;
    b %= m;
    for (; e; e >>= 1) {
        if (e & 1) r = mulmod(r, b, m);
        b = mulmod(b, b, m);
    }
    return r;
}

uint64_t inverse(uint64_t v, uint64_t m) {  // extended Euclid
    int64_t a0 = 1, a1 = 0;
    uint64_t x = v, y = m;
    while (y) {
        uint64_t qq = x / y, t = x % y;
        x = y;
        y = t;
        int64_t tmp = a1;
        a1 = a0 - (int64_t)qq * a1;
        a0 = tmp;
    }
    return a0 < 0 ? (uint64_t)a0 + m : (uint64_t)a0;
}

uint32_t brv(uint32_t x, int bits) {
    uint32_t r = 0;
    for (int i = 0; i < bits; i++) r |= ((x >> i) & 1u) << (bits - 1 - i);
    return r;
}

// smallest primitive 2N-th root of unity mod m (minimum over the odd powers of any one)
uint64_t min_primitive_root(uint64_t degree, uint64_t m) {
    uint64_t g = 0;
    for (uint64_t r = 2; r < m; r++) {
        uint64_t c = powmod(r, (m - 1) / degree, m);
        if (c && powmod(c, degree / 2, m) == m - 1) {
            g = c;
            break;
        }
    }
    uint64_t best = g, cur = g, g2 = mulmod(g, g, m);
    for (uint64_t i = 0; i < degree; i++) {
        if (cur < best) best = cur;
        cur = mulmod(cur, g2, m);
    }
    return best;
}

void root_powers(uint64_t root, uint64_t m, uint64_t* out) {
    uint64_t pw = root;
    for (uint32_t i = 1; i < (uint32_t)kN; i++) {
        out[brv(i, kLogN)] = pw;
        pw = mulmod(pw, root, m);
    }
    out[0] = 1;
}

uint64_t half_mod(uint64_t x, uint64_t m) { return (x & 1) ? (uint64_t)(((u128)x + m) >> 1) : x >> 1; }

}  // namespace

// ChaCha20 keystream in rand_chacha's layout: 64-bit block counter in words 12-13,
// 64-bit stream id in words 14-15; a u64 is two consecutive words, low first
uint32_t ChaCha::rotl(uint32_t x, int n) { return (x << n) | (x >> (32 - n)); }

void ChaCha::block() {
    static const uint32_t sigma[4] = {0x61707865, 0x3320646e, 0x79622d32, 0x6b206574};
    uint32_t s[16], x[16];
    std::memcpy(s, sigma, 16);
    std::memcpy(s + 4, key, 32);
    s[12] = (uint32_t)counter;
    s[13] = (uint32_t)(counter >> 32);
    s[14] = (uint32_t)stream;
    s[15] = (uint32_t)(stream >> 32);
    std::memcpy(x, s, sizeof(x));
    auto qr = [&](int a, int b, int c, int d) {
        x[a] += x[b]; x[d] ^= x[a]; x[d] = rotl(x[d], 16);
        x[c] += x[d]; x[b] ^= x[c]; x[b] = rotl(x[b], 12);
        x[a] += x[b]; x[d] ^= x[a]; x[d] = rotl(x[d], 8);
        x[c] += x[d]; x[b] ^= x[c]; x[b] = rotl(x[b], 7);
    };
    for (int r = 0; r < 10; r++) {
        qr(0, 4, 8, 12); qr(1, 5, 9, 13); qr(2, 6, 10, 14); qr(3, 7, 11, 15);
        qr(0, 5, 10, 15); qr(1, 6, 11, 12); qr(2, 7, 8, 13); qr(3, 4, 9, 14);
    }
    for (int i = 0; i < 16; i++) buf[i] = x[i] + s[i];
    counter++;
    idx = 0;
}

uint64_t ChaCha::next_u64() {
    if (idx + 2 > 16) block();
    uint64_t lo = buf[idx], hi = buf[idx + 1];
    idx += 2;
    return lo | (hi << 32);
}

ChaCha chacha_from_seed(const uint8_t seed[32], uint64_t stream) {
    ChaCha rng;
    for (int i = 0; i < 8; i++)
        rng.key[i] = (uint32_t)seed[4 * i] | ((uint32_t)seed[4 * i + 1] << 8) | ((uint32_t)seed[4 * i + 2] << 16) |
                     ((uint32_t)seed[4 * i + 3] << 24);
    rng.stream = stream;
    return rng;
}

void forward_ntt_u64(const HostParams& p, uint64_t* a) {  // exact reference-order forward NTT
    for (int l = 0; l < 2; l++) {
        uint64_t m = p.q[l];
        uint64_t* op = a + l * kN;
        for (int mm = 0; mm < kLogN; mm++) {
            int mcount = 1 << mm, t = kN >> (mm + 1);
            for (int i = 0; i < mcount; i++) {
                uint64_t w = p.fw[l * kN + mcount + i];
                for (int j = 0; j < t; j++) {
                    uint64_t x = op[2 * t * i + j], y = mulmod(op[2 * t * i + j + t], w, m);
                    op[2 * t * i + j] = (x + y) % m;
                    op[2 * t * i + j + t] = (x + m - y) % m;
                }
            }
        }
    }
}

namespace {

// params_rgswpir_given_input_size_and_dim0 -> (instances, interp, db_rows)
int rgswpir(uint64_t num_items, uint64_t item_bits, uint64_t dim0, uint64_t& inst, uint64_t& interp,
            uint64_t& rows) {
    const double poly_len = 2048, log_p = 16, p = 65535;
    const double modulus = (double)(268369921ull * 249561089ull);
    // max_interpolate_degree (wire.rs:386-412)
    const double sigma = 6.4, t_exp = 3, t_rgsw = 3;
    const double mlen = std::log2(modulus);
    const double z1 = std::pow(2.0, (int)std::ceil(mlen / t_exp));
    const double z2 = std::pow(2.0, (int)std::ceil(mlen / t_rgsw));
    const double v1 = (double)dim0 * (p * p) * (sigma * sigma);
    const double v2 = t_exp * (poly_len * poly_len) * (z1 * z1) * (sigma * sigma) / 4.0;
    const double v3 = t_rgsw * poly_len * (z2 * z2) * (sigma * sigma) / 2.0;
    const double total = std::log2(std::sqrt(v1 + v2 + v3));
    const double ub = std::log2(modulus / (2. * 2. * p)) - std::log2(std::sqrt(2.0 * 41.0 * std::log(2.0)));
    const double mx_log = 2. * (ub - total);
    if (mx_log < 0) return IPR_E_ARGS;
    uint64_t mx = (uint64_t)std::floor(std::pow(2.0, mx_log));
    if (mx > 2048) mx = 2048;
    if (mx <= 1) return IPR_E_ARGS;
    const double bits_per_poly = poly_len * log_p;
    uint64_t factor = (uint64_t)std::floor(bits_per_poly / (double)item_bits);
    if (!factor) factor = 1;
    const uint64_t n = (uint64_t)std::ceil((double)num_items / (double)factor);
    const uint64_t isz = item_bits * factor;
    const uint64_t pbits = (uint64_t)std::ceil((double)isz / bits_per_poly) * (uint64_t)bits_per_poly;
    const uint64_t ppts = (uint64_t)std::ceil((double)pbits / log_p);
    const uint64_t lower = ppts * (uint64_t)std::ceil((double)n / (double)dim0);
    uint64_t cur = ppts;
    interp = 1;
    while (cur < lower) {
        interp *= 2;
        cur *= 2;
        if (2 * interp > mx) break;
    }
    const uint64_t npts = (uint64_t)std::ceil((double)lower / (double)cur) * cur;
    rows = dim0 >= 8 ? dim0 : 8;
    inst = (uint64_t)std::ceil((double)npts / poly_len);
    return IPR_OK;
}

uint64_t next_pow2(uint64_t x) {
    uint64_t r = 1;
    while (r < x) r <<= 1;
    return r;
}

}  // namespace

void host_params_init(HostParams& p) {
    p.q[0] = 268369921ull;
    p.q[1] = 249561089ull;
    p.modulus = p.q[0] * p.q[1];
    for (int l = 0; l < 2; l++) p.barrett[l] = (uint64_t)((((u128)1) << 64) / p.q[l]);
    p.q0_inv_mod_q1 = (uint32_t)inverse(p.q[0] % p.q[1], p.q[1]);
    p.fw.assign(2 * kN, 0);
    p.fwp.assign(2 * kN, 0);
    p.iw.assign(2 * kN, 0);
    p.iwp.assign(2 * kN, 0);
    std::vector<uint64_t> tmp(kN);
    for (int l = 0; l < 2; l++) {
        const uint64_t m = p.q[l];
        const uint64_t root = min_primitive_root(2 * kN, m);
        root_powers(root, m, tmp.data());
        for (int i = 0; i < kN; i++) {
            p.fw[l * kN + i] = (uint32_t)tmp[i];
            p.fwp[l * kN + i] = (uint32_t)((tmp[i] << 32) / m);
        }
        root_powers(inverse(root, m), m, tmp.data());
        for (int i = 0; i < kN; i++) {
            const uint64_t h = half_mod(tmp[i], m);
            p.iw[l * kN + i] = (uint32_t)h;
            p.iwp[l * kN + i] = (uint32_t)((h << 32) / m);
        }
    }
    // RGSW row 0: NTT(-a), a = random_rng(ChaCha20Rng::from_seed([7;32])) mod q
    ChaCha rng;
    uint8_t seed[32];
    std::memset(seed, 7, 32);
    for (int i = 0; i < 8; i++)
        rng.key[i] = (uint32_t)seed[4 * i] | ((uint32_t)seed[4 * i + 1] << 8) | ((uint32_t)seed[4 * i + 2] << 16) |
                     ((uint32_t)seed[4 * i + 3] << 24);
    std::vector<uint64_t> a(2 * kN);
    for (int z = 0; z < kN; z++) {
        const uint64_t v = p.modulus - rng.next_u64() % p.modulus;  // -a, may equal q
        a[z] = v % p.q[0];
        a[kN + z] = v % p.q[1];
    }
    forward_ntt_u64(p, a.data());
    p.row0.resize(2 * kN);
    for (int i = 0; i < 2 * kN; i++) p.row0[i] = (uint32_t)a[i];
    p.iwu.assign(2 * kN, 0);
    p.iwup.assign(2 * kN, 0);
    p.row0s.assign(2 * kN, 0);
    p.row0m.assign(2 * kN, 0);
    for (int l = 0; l < 2; l++) {
        const uint64_t m = p.q[l], ninv = inverse(kN, m);
        p.ninv[2 * l] = (uint32_t)ninv;
        p.ninv[2 * l + 1] = (uint32_t)((ninv << 32) / m);
        const uint64_t ninvr = mulmod(ninv, (1ull << 32) % m, m);
        p.ninvr[2 * l] = (uint32_t)ninvr;
        p.ninvr[2 * l + 1] = (uint32_t)((ninvr << 32) / m);
        for (int i = 0; i < kN; i++) p.row0m[l * kN + i] = (uint32_t)mulmod(p.row0[l * kN + i], ninvr, m);
        for (int i = 0; i < kN; i++) {
            const uint64_t w = (2 * (uint64_t)p.iw[l * kN + i]) % m;
            p.iwu[l * kN + i] = (uint32_t)w;
            p.iwup[l * kN + i] = (uint32_t)((w << 32) / m);
            p.row0s[l * kN + i] = (uint32_t)mulmod(p.row0[l * kN + i], ninv, m);
        }
    }
    p.fwi.assign(4 * kN, 0);
    p.iwi.assign(4 * kN, 0);
    for (int i = 0; i < 2 * kN; i++) {
        p.fwi[2 * i] = p.fw[i];
        p.fwi[2 * i + 1] = p.fwp[i];
        p.iwi[2 * i] = p.iwu[i];
        p.iwi[2 * i + 1] = p.iwup[i];
    }
}

namespace {

// PolyMatrixNTT::random_rng(params, 1, 3, ChaCha20Rng::from_seed(seed)) (poly.rs:418-440):
// column c, limb l, coefficient j <- next_u64 % q_l
void random_ntt_3(const HostParams& p, const uint8_t seed[32], std::vector<uint32_t>& out) {
    ChaCha rng = chacha_from_seed(seed);
    out.assign(3 * 2 * kN, 0);
    for (int c = 0; c < 3; c++)
        for (int l = 0; l < 2; l++)
            for (int j = 0; j < kN; j++) out[(c * 2 + l) * kN + j] = (uint32_t)(rng.next_u64() % p.q[l]);
}
}  // namespace

void offline_host_inputs(const HostParams& p, unsigned polys, std::vector<uint32_t>& query,
                         std::vector<uint32_t>& w_mask, std::vector<uint32_t>& v_mask) {
    // generate_pseudorandom_query(SEED_0) (engine.rs:500-534): ChaCha20Rng from get_seed(0), the
    // all-zero seed (client/online.rs:164-168); poly r is a_r = random_rng mod q, the query keeps
    // ct.raw() row 0 = -a_r mod q (client/base.rs:438-457), negacyclic_perm(., 0, q)
    // (utils.rs:5-21) maps c(X) to c(X^-1): coefficient 0 stays, coefficient i >= 1 is
    // -c[N - i] = a_r[N - i]; then to_ntt
    uint8_t zero[32];
    std::memset(zero, 0, sizeof(zero));
    ChaCha rng = chacha_from_seed(zero);
    query.assign((size_t)polys * 2 * kN, 0);
    std::vector<uint64_t> a(kN), t(2 * kN);
    for (unsigned r = 0; r < polys; r++) {
        for (int i = 0; i < kN; i++) a[i] = rng.next_u64() % p.modulus;
        for (int i = 0; i < kN; i++) {
            const uint64_t c = i == 0 ? (a[0] ? p.modulus - a[0] : 0) : a[kN - i];
            t[i] = c % p.q[0];
            t[kN + i] = c % p.q[1];
        }
        forward_ntt_u64(p, t.data());
        for (int i = 0; i < 2 * kN; i++) query[(size_t)r * 2 * kN + i] = (uint32_t)t[i];
    }
    // OfflinePackingKeys::init_full (packing.rs:1843-1870) with W_SEED / V_SEED (scheme.rs:46-51)
    uint8_t ws[32], vs[32];
    std::memset(ws, 7, 32);
    std::memset(vs, 7, 32);
    vs[0] = vs[1] = 8;
    random_ntt_3(p, ws, w_mask);
    random_ntt_3(p, vs, v_mask);
}

void host_moduli_constants(uint64_t barrett[2], uint32_t* q0_inv_mod_q1) {
    const uint64_t q0 = 268369921ull, q1 = 249561089ull;
    barrett[0] = (uint64_t)((((u128)1) << 64) / q0);
    barrett[1] = (uint64_t)((((u128)1) << 64) / q1);
    *q0_inv_mod_q1 = (uint32_t)inverse(q0 % q1, q1);
}

int plan_from_shape(uint64_t record_count, uint64_t key_size, uint64_t value_size, uint64_t buckets,
                    uint64_t dim0, Plan& out) {
    if (!record_count || !key_size || !value_size) return IPR_E_ARGS;
    const uint64_t rc = record_count < 512 ? 512 : record_count;
    const uint64_t num_items = buckets ? buckets : next_pow2(rc * 2);  // default_bucket_count keyword.rs:29-31
    if (num_items < record_count) return IPR_E_ARGS;
    const uint64_t entry = key_size + value_size, bits = entry * 8;
    if (bits % 16) return IPR_E_ARGS;
    uint64_t inst, interp, rows;
    if (!dim0) {
        if (rgswpir(num_items, bits, num_items >= 256000000ull ? 32768 : 2048, inst, interp, rows)) return IPR_E_ARGS;
        dim0 = rows;
    }
    if (rgswpir(num_items, bits, dim0, inst, interp, rows)) return IPR_E_ARGS;
    const uint64_t db_rows = next_pow2(rows);
    if (db_rows < (uint64_t)kN || num_items < db_rows) return IPR_E_ARGS;
    out.num_items = num_items;
    out.entry_size = entry;
    out.item_size_bits = bits;
    out.dim0 = dim0;
    out.db_rows = db_rows;
    out.instances = inst;
    out.db_cols = inst * kN;
    out.interp = interp;
    out.c = inst / interp;
    const uint64_t nph = kN / 2;
    out.peak_bytes = out.db_rows * out.db_cols * 2 + out.db_cols * 2 * kN * 8 + 2 * inst * nph * 2 * kN * 8 +
                     2 * inst * (nph - 1) * 3 * kN * 8;
    return IPR_OK;
}

uint64_t query_bytes(uint64_t db_rows, unsigned nq) {
    const uint64_t nvals = 3ull * kN * 2 + (uint64_t)nq * (db_rows + 6ull * kN);
    return (8 + nvals * 56 + 7) / 8;
}

}  // namespace ipr
