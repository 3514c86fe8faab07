/*
 * ipr_offline.c — CPU restatement of the reference's offline precomputation for
 * the InspiRING second-level packing (rkdud007/inspire-rs), the setup step whose
 * outputs (a_hat, bold_t, bold_t_bar, bold_t_hat) respond() streams.  TEST
 * INFRASTRUCTURE ONLY, like the rest of this directory: the product library never
 * links or calls it.
 *
 * Pipeline (PirServer::perform_offline_precomputation_simplepir, CPU branches,
 * src/pir/server/engine.rs:677-1042), per packing instance (2048 DB columns):
 *   hint query   generate_pseudorandom_query(SEED_0)      engine.rs:500-534
 *   hint         multiply_with_db_ring                    engine.rs:434-498
 *   a_ct_tilde   prep_pack_many_lwes / prep_pack_lwes     src/pir/packing.rs:1032-1105
 *   keys         OfflinePackingKeys::init_full            packing.rs:1843-1870
 *   r, r_bar     full_packing_with_preprocessing_offline  packing.rs:2627-2679 (CPU branch)
 *   collapse     same function                            packing.rs:2683-2734
 * Every value here is an exact residue; the functions follow the reference's
 * loops (including its brute-force O(N^2)-per-slot packing sum) so that they are
 * the definition the device's faster algorithm is checked against.
 */
#include <stdlib.h>
#include <string.h>

#include "ipr_oracle.h"

typedef unsigned __int128 u128;

/* W_SEED / V_SEED, src/pir/scheme.rs:46-51 */
static const uint8_t kWSeed[32] = {7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7,
                                   7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7};
static const uint8_t kVSeed[32] = {8, 8, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7,
                                   7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7, 7};

static uint64_t barrett_coeff(const ipr_params *p, uint64_t v, int l) { /* arith.rs:147-149 */
    return ipr_barrett_raw_u64(v, p->barrett_cr1[l], p->q[l]);
}

/* fast_barrett_raw_u64 (packing.rs:643-650): Barrett without the final subtraction */
static uint64_t fast_barrett(const ipr_params *p, uint64_t v, int l) {
    uint64_t tmp = (uint64_t)(((u128)v * p->barrett_cr1[l]) >> 64);
    return v - tmp * p->q[l];
}

/* negacyclic_perm(a, 0, modulus) (src/pir/utils.rs:5-21) */
static void negacyclic_perm0(const uint64_t *a, uint64_t modulus, uint64_t *out) {
    out[0] = a[0];
    for (int i = 1; i < IPR_N; i++) {
        uint64_t v = modulus - (a[IPR_N - i] % modulus);
        out[i] = v == modulus ? 0 : v;
    }
}

void ipr_oracle_hint_query(const ipr_params *p, unsigned polys, uint64_t *out) {
    /* get_seed(SEED_0) (client/online.rs:164-168): STATIC_PUBLIC_SEED with byte 0 = 0 */
    uint8_t seed[32];
    memset(seed, 0, sizeof(seed));
    ipr_chacha_rng rng;
    ipr_chacha_seed(&rng, seed);
    uint64_t a[IPR_N], neg[IPR_N], perm[IPR_N];
    for (unsigned r = 0; r < polys; r++) {
        /* get_scaled_regev_sample (client/base.rs:438-457): a = random_rng(rng_pub), row 0 of
         * the ciphertext is NTT(-a); generate_query_impl keeps ct.raw() row 0 = -a mod q */
        for (int i = 0; i < IPR_N; i++) a[i] = ipr_chacha_next_u64(&rng) % p->modulus;
        for (int i = 0; i < IPR_N; i++) neg[i] = a[i] ? p->modulus - a[i] : 0;
        negacyclic_perm0(neg, p->modulus, perm);
        ipr_to_ntt(p, perm, out + (size_t)r * 2 * IPR_N);
    }
}

void ipr_oracle_prep_pack(const ipr_params *p, const uint16_t *db, uint64_t db_rows, uint64_t inst,
                          const uint64_t *query, uint64_t *a_ct) {
    const uint64_t polys = db_rows / IPR_N;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < IPR_N; j++) {
        uint64_t col = inst * IPR_N + (uint64_t)j;
        uint64_t sum[2 * IPR_N], prod[2 * IPR_N], elem[IPR_N], dn[2 * IPR_N], raw[IPR_N], perm[IPR_N];
        memset(sum, 0, sizeof(sum));
        /* multiply_with_db_ring (engine.rs:456-485): sum over the column's row polynomials of
         * NTT(db chunk) * query[row]; add_into_no_reduce except for the last row (add_into) */
        for (uint64_t row = 0; row < polys; row++) {
            for (int z = 0; z < IPR_N; z++) elem[z] = db[col * db_rows + row * IPR_N + (uint64_t)z];
            ipr_to_ntt(p, elem, dn);
            for (int l = 0; l < 2; l++) /* multiply (poly.rs:613-634): multiply_modular per limb */
                for (int z = 0; z < IPR_N; z++) {
                    int idx = l * IPR_N + z;
                    prod[idx] = barrett_coeff(p, dn[idx] * query[row * 2 * IPR_N + idx], l);
                }
            if (row == polys - 1)
                for (int l = 0; l < 2; l++)
                    for (int z = 0; z < IPR_N; z++) {
                        int idx = l * IPR_N + z;
                        sum[idx] = barrett_coeff(p, sum[idx] + prod[idx], l);
                    }
            else
                for (int idx = 0; idx < 2 * IPR_N; idx++) sum[idx] += prod[idx];
        }
        ipr_from_ntt(p, sum, raw); /* sum.raw(); SimplePIR keeps it (no SEED_0 permutation) */
        /* prep_pack_lwes (packing.rs:1032-1062): the hint column in negacyclic order, to NTT */
        negacyclic_perm0(raw, p->modulus, perm);
        ipr_to_ntt(p, perm, a_ct + (size_t)j * 2 * IPR_N);
    }
}

void ipr_oracle_prep_pack_lwes(const ipr_params *p, const uint64_t *lwe, uint64_t *a_ct) {
    /* prep_pack_lwes (packing.rs:1032-1062): LWE i's a-vector is column i of rows 0..N-1
     * (row N holds the b values, skipped); to negacyclic order, then to NTT */
#pragma omp parallel for schedule(static)
    for (int i = 0; i < IPR_N; i++) {
        uint64_t poly[IPR_N], perm[IPR_N];
        for (int j = 0; j < IPR_N; j++) poly[j] = lwe[(size_t)j * IPR_N + (size_t)i];
        negacyclic_perm0(poly, p->modulus, perm);
        ipr_to_ntt(p, perm, a_ct + (size_t)i * 2 * IPR_N);
    }
}

/* PolyMatrixNTT::random_rng(params, 1, 3, ChaCha20Rng::from_seed(seed)) (poly.rs:418-440):
 * column c, limb l, coefficient j <- next_u64 % q_l */
static void random_ntt_3(const ipr_params *p, const uint8_t seed[32], uint64_t *out) {
    ipr_chacha_rng rng;
    ipr_chacha_seed(&rng, seed);
    for (int c = 0; c < IPR_T; c++)
        for (int l = 0; l < 2; l++)
            for (int j = 0; j < IPR_N; j++)
                out[(size_t)c * 2 * IPR_N + l * IPR_N + j] = ipr_chacha_next_u64(&rng) % p->q[l];
}

/* apply_automorph_ntt_raw (packing.rs:1500-1516) on each limb: out[s] = in[table[s]] */
static void automorph_ntt(const uint64_t *in, uint64_t *out, uint64_t t) {
    uint32_t table[IPR_N];
    ipr_automorph_table(t, table);
    for (int l = 0; l < 2; l++)
        for (int s = 0; s < IPR_N; s++) out[l * IPR_N + s] = in[l * IPR_N + table[s]];
}

void ipr_oracle_offline_keys(const ipr_params *p, uint64_t *w_mask, uint64_t *v_mask, uint64_t *w_all,
                             uint64_t *w_bar_all) {
    random_ntt_3(p, kWSeed, w_mask);
    random_ntt_3(p, kVSeed, v_mask);
    /* generate_rotations_double (packing.rs:1758-1785): row i < 1023 = w_mask under gen_pows[i] / 2N - gen_pows[i] */
#pragma omp parallel for schedule(static)
    for (int i = 0; i < IPR_NROT; i++) {
        uint64_t g = ipr_gen_pow((unsigned)i);
        for (int k = 0; k < IPR_T; k++) {
            size_t o = ((size_t)i * IPR_T + (size_t)k) * 2 * IPR_N;
            automorph_ntt(w_mask + (size_t)k * 2 * IPR_N, w_all + o, g);
            automorph_ntt(w_mask + (size_t)k * 2 * IPR_N, w_bar_all + o, 2 * IPR_N - g);
        }
    }
}

void ipr_oracle_pack_r(const ipr_params *p, const uint64_t *a_ct, uint64_t *r_all, uint64_t *r_bar_all) {
    const int half = IPR_N / 2;
    /* PackParams::new (packing.rs:1635-1670): monomial_ntts[j] = NTT(x^j), neg = -NTT(x^j);
     * mod_inv_poly = NTT of the constant N^-1 mod q */
    uint64_t *mono = malloc(sizeof(uint64_t) * 2 * IPR_N * 2 * IPR_N);
#pragma omp parallel for schedule(static)
    for (int e = 0; e < IPR_N; e++) {
        uint64_t raw[IPR_N];
        memset(raw, 0, sizeof(raw));
        raw[e] = 1;
        uint64_t *m = mono + (size_t)e * 2 * IPR_N, *nm = mono + ((size_t)IPR_N + e) * 2 * IPR_N;
        ipr_to_ntt(p, raw, m);
        for (int l = 0; l < 2; l++) /* -&PolyMatrixNTT: (q - v) % q per limb */
            for (int z = 0; z < IPR_N; z++) {
                uint64_t v = m[l * IPR_N + z];
                nm[l * IPR_N + z] = v ? p->q[l] - v : 0;
            }
    }
    uint64_t inv_raw[IPR_N], inv_ntt[2 * IPR_N];
    memset(inv_raw, 0, sizeof(inv_raw));
    inv_raw[0] = ipr_invert_uint_mod(IPR_N, p->modulus);
    ipr_to_ntt(p, inv_raw, inv_ntt);
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < half; i++) {
        uint64_t r[2 * IPR_N], rb[2 * IPR_N], tmp[2 * IPR_N];
        memset(r, 0, sizeof(r));
        memset(rb, 0, sizeof(rb));
        const uint64_t gp = ipr_gen_pow((unsigned)((IPR_N - i) % IPR_N));
        for (int j = 0; j < IPR_N; j++) {
            const uint64_t *pol2 = a_ct + (size_t)j * 2 * IPR_N;
            uint64_t index = ((uint64_t)j * gp) % (2 * IPR_N);
            uint64_t index_bar = (2 * IPR_N - ((uint64_t)j * gp) % (2 * IPR_N)) % (2 * IPR_N);
            /* index < N: monomial_ntts[index]; else neg_monomial_ntts[index % N] */
            const uint64_t *pol1 = mono + (size_t)(index < IPR_N ? index : IPR_N + index % IPR_N) * 2 * IPR_N;
            const uint64_t *pol1b =
                mono + (size_t)(index_bar < IPR_N ? index_bar : IPR_N + index_bar % IPR_N) * 2 * IPR_N;
            for (int l = 0; l < 2; l++) /* multiply_add_poly (poly.rs:474-481) */
                for (int z = 0; z < IPR_N; z++) {
                    int idx = l * IPR_N + z;
                    r[idx] = barrett_coeff(p, pol1[idx] * pol2[idx] + r[idx], l);
                    rb[idx] = barrett_coeff(p, pol1b[idx] * pol2[idx] + rb[idx], l);
                }
        }
        /* fast_reduce is the identity on canonical values; scalar_multiply by mod_inv_poly
         * (poly.rs:829-843, multiply_poly), then apply_automorph_ntt by gen_pows[i] and
         * 2N - gen_pows[i] */
        const uint64_t g = ipr_gen_pow((unsigned)i);
        for (int l = 0; l < 2; l++)
            for (int z = 0; z < IPR_N; z++) tmp[l * IPR_N + z] = barrett_coeff(p, r[l * IPR_N + z] * inv_ntt[l * IPR_N + z], l);
        automorph_ntt(tmp, r_all + (size_t)i * 2 * IPR_N, g);
        for (int l = 0; l < 2; l++)
            for (int z = 0; z < IPR_N; z++) tmp[l * IPR_N + z] = barrett_coeff(p, rb[l * IPR_N + z] * inv_ntt[l * IPR_N + z], l);
        automorph_ntt(tmp, r_bar_all + (size_t)i * 2 * IPR_N, 2 * IPR_N - g);
    }
    free(mono);
}

/* gadget_invert_transposed_into (packing.rs:2740-2768) of raw(x), then .ntt(): the three
 * 19-bit digit polynomials of the canonical raw value, each to the NTT domain */
static void digits_ntt(const ipr_params *p, const uint64_t *x_ntt, uint64_t *dig /* [3][2N] */) {
    uint64_t raw[IPR_N], d[IPR_T * IPR_N];
    ipr_from_ntt(p, x_ntt, raw);
    ipr_gadget_invert_general(p, raw, 1, IPR_T, d);
    for (int k = 0; k < IPR_T; k++) ipr_to_ntt(p, d + (size_t)k * IPR_N, dig + (size_t)k * 2 * IPR_N);
}

/* condense_matrix (packing.rs:867-884): limb 0 in the low word, limb 1 in the high word */
static void condense(const uint64_t *x, uint64_t *out) {
    for (int z = 0; z < IPR_N; z++) out[z] = x[z] | (x[IPR_N + z] << 32);
}

/* res = sum_k w[k] * t[k] (multiply_add_poly from zero), then fast_add_into(acc, res) */
static void mac3_fast_add(const ipr_params *p, const uint64_t *w, const uint64_t *t, uint64_t *acc) {
    uint64_t res[2 * IPR_N];
    memset(res, 0, sizeof(res));
    for (int k = 0; k < IPR_T; k++)
        for (int l = 0; l < 2; l++)
            for (int z = 0; z < IPR_N; z++) {
                int idx = l * IPR_N + z;
                res[idx] = barrett_coeff(p, w[(size_t)k * 2 * IPR_N + idx] * t[(size_t)k * 2 * IPR_N + idx] + res[idx], l);
            }
    for (int l = 0; l < 2; l++) /* fast_add_into (packing.rs:652-676) */
        for (int z = 0; z < IPR_N; z++) {
            int idx = l * IPR_N + z;
            acc[idx] = fast_barrett(p, acc[idx] + res[idx], l);
        }
}

void ipr_oracle_collapse(const ipr_params *p, uint64_t *r_all, uint64_t *r_bar_all, const uint64_t *w_all,
                         const uint64_t *w_bar_all, const uint64_t *v_mask, uint64_t *a_hat, uint64_t *bold_t,
                         uint64_t *bold_t_bar, uint64_t *bold_t_hat) {
    uint64_t dig[IPR_T * 2 * IPR_N];
    for (int i = IPR_N / 2 - 2; i >= 0; i--) { /* packing.rs:2691-2719 */
        digits_ntt(p, r_all + (size_t)(i + 1) * 2 * IPR_N, dig);
        for (int k = 0; k < IPR_T; k++)
            condense(dig + (size_t)k * 2 * IPR_N, bold_t + ((size_t)i * IPR_T + (size_t)k) * IPR_N);
        mac3_fast_add(p, w_all + (size_t)i * IPR_T * 2 * IPR_N, dig, r_all + (size_t)i * 2 * IPR_N);

        digits_ntt(p, r_bar_all + (size_t)(i + 1) * 2 * IPR_N, dig);
        for (int k = 0; k < IPR_T; k++)
            condense(dig + (size_t)k * 2 * IPR_N, bold_t_bar + ((size_t)i * IPR_T + (size_t)k) * IPR_N);
        mac3_fast_add(p, w_bar_all + (size_t)i * IPR_T * 2 * IPR_N, dig, r_bar_all + (size_t)i * 2 * IPR_N);
    }
    digits_ntt(p, r_bar_all, dig); /* packing.rs:2721-2732 */
    for (int k = 0; k < IPR_T; k++) condense(dig + (size_t)k * 2 * IPR_N, bold_t_hat + (size_t)k * IPR_N);
    mac3_fast_add(p, v_mask, dig, r_all);
    ipr_from_ntt(p, r_all, a_hat);
}

int ipr_oracle_offline_instance(const ipr_params *p, const uint16_t *db, uint64_t db_rows, uint64_t inst,
                                const uint64_t *query, const uint64_t *w_all, const uint64_t *w_bar_all,
                                const uint64_t *v_mask, uint64_t *a_hat, uint64_t *bold_t, uint64_t *bold_t_bar,
                                uint64_t *bold_t_hat) {
    if (!db_rows || db_rows % IPR_N) return IPR_E_ARGS;
    uint64_t *a_ct = malloc(sizeof(uint64_t) * (size_t)IPR_N * 2 * IPR_N);
    uint64_t *r = malloc(sizeof(uint64_t) * (size_t)(IPR_N / 2) * 2 * IPR_N);
    uint64_t *rb = malloc(sizeof(uint64_t) * (size_t)(IPR_N / 2) * 2 * IPR_N);
    ipr_oracle_prep_pack(p, db, db_rows, inst, query, a_ct);
    ipr_oracle_pack_r(p, a_ct, r, rb);
    ipr_oracle_collapse(p, r, rb, w_all, w_bar_all, v_mask, a_hat, bold_t, bold_t_bar, bold_t_hat);
    free(a_ct);
    free(r);
    free(rb);
    return IPR_OK;
}
