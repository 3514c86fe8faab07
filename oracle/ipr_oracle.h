/*
 * ipr_oracle.h — CPU restatement of the InsPIRe keyword-PIR server respond()
 * path (rkdud007/inspire-rs).  TEST INFRASTRUCTURE ONLY: this library is the
 * checker used by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg.  The product library (inspire-rs_b200/csrc) never links or calls it.
 *
 * Every function cites the reference file:line whose behaviour it restates.
 * Parity pins: the reference's own known-answer tests (src/core/ntt.rs:797-840,
 * src/core/arith.rs:463-528, src/core/gadget.rs:80-96, src/pir/packing.rs:3943-3985,
 * src/core/util.rs:411-427) are re-run against this code in tests/test_oracle_kat.py;
 * the GEMV / rotation / packing kernels are additionally cross-checked against the
 * reference's own CUDA kernels (the native/cuda kernel sources, built into oracle/_ref/) on a GPU.
 * Third-party stream semantics (rand_chacha 0.10 ChaCha20Rng, used only for the
 * RGSW mask polynomials) are restated from RFC 8439 and pinned to its test vector.
 */
#ifndef IPR_ORACLE_H
#define IPR_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IPR_N 2048          /* ring dimension, src/pir/wire.rs:419-420 */
#define IPR_LOGN 11
#define IPR_T 3             /* t_exp_left = t_gsw, wire.rs:424 */
#define IPR_NROT 1023       /* poly_len/2 - 1 rotations, packing.rs:1766 */
#define IPR_NINNER (IPR_NROT * IPR_T) /* 3069 */
#define IPR_Q0 268369921ULL /* src/pir/params.rs:8 */
#define IPR_Q1 249561089ULL
#define IPR_PT 65535ULL     /* wire.rs:421 */
#define IPR_QP1 (1ULL << 20)       /* params.rs:346-348 */
#define IPR_QP2 268369921ULL       /* Q2_VALUES[28], core/params.rs:37 */
#define IPR_RESULT_BYTES 12288     /* (28*2048 + 20*2048)/8, modulus_switch.rs:51-53 */

/* status codes (shared with the product's C-ABI) */
#define IPR_OK 0
#define IPR_E_ARGS -1
#define IPR_E_FORMAT -5
#define IPR_E_SPACE -6

typedef struct {
    uint64_t q[2];
    uint64_t modulus;          /* q0*q1 */
    uint64_t barrett_cr0[2];   /* floor(2^128/q_i) low word  (get_barrett, arith.rs:124-131) */
    uint64_t barrett_cr1[2];   /* floor(2^128/q_i) high word = floor(2^64/q_i) */
    uint64_t cr0_mod, cr1_mod; /* floor(2^128/q) split (get_barrett_crs(modulus)) */
    uint64_t mod0_inv_mod1;    /* q0 * (q0^-1 mod q1), core/params.rs:268 */
    uint64_t mod1_inv_mod0;    /* q1 * (q1^-1 mod q0), core/params.rs:269 */
    uint64_t modulus_log2;     /* ceil(log2 q) = 56 */
    uint64_t root[2];          /* minimal primitive 2N-th root per prime */
    uint64_t ntt[2][4][IPR_N]; /* fwd, fwd', inv(halved), inv' (build_ntt_tables ntt.rs:74-108) */
} ipr_params;

/* ---- arithmetic (src/core/arith.rs, number_theory.rs) ---- */
void ipr_params_init(ipr_params *p);
void ipr_get_barrett_crs(uint64_t modulus, uint64_t *cr0, uint64_t *cr1);
uint64_t ipr_barrett_raw_u64(uint64_t in, uint64_t cr1, uint64_t modulus);
uint64_t ipr_barrett_reduction_u128_raw(uint64_t modulus, uint64_t cr0, uint64_t cr1,
                                        uint64_t lo, uint64_t hi);
uint64_t ipr_div2_uint_mod(uint64_t x, uint64_t m);
uint64_t ipr_invert_uint_mod(uint64_t v, uint64_t m);
uint64_t ipr_crt_compose(const ipr_params *p, uint64_t x, uint64_t y);
uint64_t ipr_rescale(uint64_t a, uint64_t inp_mod, uint64_t out_mod);
uint64_t ipr_reverse_bits(uint64_t x, unsigned bits);
uint64_t ipr_minimal_primitive_root(uint64_t degree, uint64_t modulus);

/* ---- NTT (ntt.rs:111-160 forward, ntt.rs:731-780 inverse), data = [limb0 N | limb1 N] ---- */
void ipr_ntt_forward(const ipr_params *p, uint64_t *data);
void ipr_ntt_inverse(const ipr_params *p, uint64_t *data);
/* to_ntt (poly.rs:857-876): reduce raw coefficients mod each q_i, then forward NTT */
void ipr_to_ntt(const ipr_params *p, const uint64_t *raw, uint64_t *ntt_out);
/* from_ntt (poly.rs:900-918): inverse NTT, CRT compose -> raw mod q */
void ipr_from_ntt(const ipr_params *p, const uint64_t *ntt_in, uint64_t *raw_out);

/* ---- gadget (gadget.rs:35-65): 2x1 raw -> 6x1 raw, row j + k*2 ---- */
void ipr_gadget_invert_2(const ipr_params *p, const uint64_t *in2, uint64_t *out6);
void ipr_gadget_invert_general(const ipr_params *p, const uint64_t *in, unsigned rows, unsigned num_elems,
                               uint64_t *out);

/* ---- automorphisms (poly.rs:531-543, packing.rs:1423-1516) ---- */
void ipr_automorph_poly(const ipr_params *p, const uint64_t *a, uint64_t *res, uint64_t t);
void ipr_automorph_table(uint64_t t, uint32_t *table);  /* closed form */
int ipr_automorph_table_bruteforce(const ipr_params *p, uint64_t t, uint32_t *table, uint64_t seed);
uint64_t ipr_gen_pow(unsigned i); /* 5^i mod 2N, packing.rs:1645-1652 */

/* ---- bits (util.rs:289-321) ---- */
uint64_t ipr_read_bits(const uint8_t *data, size_t bit_offs, unsigned num_bits);
void ipr_write_bits(uint8_t *data, uint64_t val, size_t bit_offs, unsigned num_bits);

/* ---- ChaCha20 (RFC 8439 block; rand_chacha ChaCha20Rng stream, nonce 0) ---- */
void ipr_chacha20_block(const uint32_t key[8], uint64_t counter, uint64_t stream, uint32_t out[16]);
void ipr_chacha20_rfc8439_block(const uint32_t key[8], uint32_t counter, const uint32_t nonce[3],
                                uint32_t out[16]);
typedef struct {
    uint32_t key[8];
    uint64_t counter;
    uint32_t buf[64];
    unsigned idx;
} ipr_chacha_rng;
void ipr_chacha_seed(ipr_chacha_rng *r, const uint8_t seed[32]);
uint64_t ipr_chacha_next_u64(ipr_chacha_rng *r);
/* NTT(-a) with a = PolyMatrixRaw::random_rng(ChaCha20(RGSW_SEEDS[i])) (keyword.rs:546-555) */
void ipr_rgsw_row0(const ipr_params *p, uint64_t out[2 * IPR_N]);
void ipr_oracle_random_raw(const ipr_params *p, const uint8_t seed[32], uint64_t count, uint64_t *out);
void ipr_oracle_chacha_blocks(const uint8_t seed[32], uint64_t stream, uint64_t first, uint64_t count,
                              uint32_t *out);
void ipr_oracle_rescale_many(const uint64_t *in, uint64_t n, uint64_t inp_mod, uint64_t out_mod, uint64_t *out);

/* ---- shape plan (keyword.rs:29-31,145-233; wire.rs:386-477) ---- */
typedef struct {
    uint64_t num_items, entry_size, item_size_bits, dim0;
    uint64_t db_rows, db_cols, instances, interp, c;
    uint64_t peak_bytes; /* KeywordServerGpuMemoryEstimate::from_plan keyword.rs:105-141 */
} ipr_plan;
int ipr_plan_from_shape(uint64_t record_count, uint64_t key_size, uint64_t value_size,
                        uint64_t buckets, uint64_t dim0, ipr_plan *out);

/* ---- server state for the oracle ---- */
typedef struct {
    uint64_t db_rows, db_cols, num_outputs, interp, c;
    const uint16_t *db;        /* [db_cols][db_rows], column-major (gemv_kernel.cu:63) */
    const uint64_t *a_hat;     /* [num_outputs][N] raw mod q */
    const uint64_t *bold_t;    /* [num_outputs][3069][N] condensed */
    const uint64_t *bold_t_bar;
    const uint64_t *bold_t_hat;/* [num_outputs][3][N] condensed */
    const uint8_t *stash;      /* stash_count * stash_entry_bytes */
    uint64_t stash_count, stash_entry_bytes;
} ipr_oracle_db;

/* step functions */
void ipr_oracle_gemv(const ipr_params *p, const ipr_oracle_db *db, const uint64_t *a, uint64_t *c);
void ipr_oracle_rotations(const uint64_t *y_body, uint64_t *y_all, uint64_t *y_bar_all);
void ipr_oracle_packing_sum(const ipr_params *p, const ipr_oracle_db *db, const uint64_t *y_body,
                            const uint64_t *z_body, uint64_t *S);
void ipr_oracle_postprocess(const ipr_params *p, const ipr_oracle_db *db, const uint64_t *S,
                            const uint64_t *b_values, uint64_t *packed);
void ipr_oracle_fold(const ipr_params *p, const ipr_oracle_db *db, const uint64_t *row0,
                     const uint64_t *ct_gsw_body, const uint64_t *packed, uint64_t *results);
void ipr_oracle_switch(const ipr_params *p, const uint64_t *result, uint8_t *out);

/* wire (wire.rs:618-726) */
size_t ipr_query_bytes(uint64_t db_rows, unsigned num_queries);
int ipr_oracle_parse_query(const uint8_t *buf, size_t len, uint64_t db_rows, unsigned *num_queries,
                           uint64_t *y_body, uint64_t *z_body, uint64_t *query_rows,
                           uint64_t *gsw_bodies, unsigned max_queries);
size_t ipr_response_bytes(const ipr_oracle_db *db, unsigned num_queries);
int ipr_oracle_respond(const ipr_params *p, const ipr_oracle_db *db, const uint8_t *query,
                       size_t len, uint8_t *out, size_t cap, size_t *out_len);

/* ---- seeded synthetic data (shared definition with the device generator) ---- */
uint64_t ipr_synth(uint64_t seed, uint64_t stream, uint64_t idx);
void ipr_synth_db(uint64_t seed, uint64_t db_rows, uint64_t db_cols, uint16_t *db);
void ipr_synth_precomp(uint64_t seed, uint64_t num_outputs, uint64_t *a_hat, uint64_t *bold_t,
                       uint64_t *bold_t_bar, uint64_t *bold_t_hat);
void ipr_synth_shard(uint64_t seed, uint64_t db_rows, uint64_t first, uint64_t count, uint16_t *db,
                     uint64_t *a_hat, uint64_t *bt, uint64_t *btb, uint64_t *bth);
void ipr_oracle_raw_db(const uint8_t *entries, const uint8_t *occupied, uint64_t num_buckets,
                       uint64_t entry_size, uint64_t db_rows, uint64_t db_cols, uint64_t per,
                       uint16_t *raw);
int ipr_oracle_encode_db(const uint16_t *raw, uint16_t *out, uint64_t db_rows, uint64_t db_cols,
                         uint64_t interp);
int ipr_synth_query(uint64_t seed, uint64_t db_rows, unsigned num_queries, uint8_t *out,
                    size_t cap, size_t *out_len);

/* ---- offline precomputation (ipr_offline.c; engine.rs:677-1042, packing.rs) ---- */
/* generate_pseudorandom_query(SEED_0) engine.rs:500-534: `polys` = db_rows/2048 NTT polys [polys][2N] */
void ipr_oracle_hint_query(const ipr_params *p, unsigned polys, uint64_t *out);
/* a_ct_tilde of instance `inst` (hint columns inst*2048 .. +2048): [2048][2N] NTT */
void ipr_oracle_prep_pack(const ipr_params *p, const uint16_t *db, uint64_t db_rows, uint64_t inst,
                          const uint64_t *query, uint64_t *a_ct);
/* prep_pack_lwes (packing.rs:1032-1062): lwe [N+1][N] (row j = coefficient j of the 2048
 * LWE a-vectors, row N = the b values) -> a_ct [N][2N] NTT */
void ipr_oracle_prep_pack_lwes(const ipr_params *p, const uint64_t *lwe, uint64_t *a_ct);
/* OfflinePackingKeys::init_full: w_mask, v_mask [3][2N]; w_all, w_bar_all [1023][3][2N] */
void ipr_oracle_offline_keys(const ipr_params *p, uint64_t *w_mask, uint64_t *v_mask, uint64_t *w_all,
                             uint64_t *w_bar_all);
/* packing sums (brute force, CPU branch packing.rs:2627-2679): r_all, r_bar_all [1024][2N] */
void ipr_oracle_pack_r(const ipr_params *p, const uint64_t *a_ct, uint64_t *r_all, uint64_t *r_bar_all);
/* collapse (packing.rs:2683-2734); r_all / r_bar_all are updated in place.  a_hat [N] raw,
 * bold_t / bold_t_bar [1023*3][N] condensed, bold_t_hat [3][N] condensed */
void ipr_oracle_collapse(const ipr_params *p, uint64_t *r_all, uint64_t *r_bar_all, const uint64_t *w_all,
                         const uint64_t *w_bar_all, const uint64_t *v_mask, uint64_t *a_hat, uint64_t *bold_t,
                         uint64_t *bold_t_bar, uint64_t *bold_t_hat);
int ipr_oracle_offline_instance(const ipr_params *p, const uint16_t *db, uint64_t db_rows, uint64_t inst,
                                const uint64_t *query, const uint64_t *w_all, const uint64_t *w_bar_all,
                                const uint64_t *v_mask, uint64_t *a_hat, uint64_t *bold_t, uint64_t *bold_t_bar,
                                uint64_t *bold_t_hat);

int ipr_oracle_threads(void);

/* dataset generation (ipr_dataset.c): FIPS 202 hashes, FIPS 203 encapsulation keys, the
 * rand_core record-seed key and one DatasetGenerator record (id || pk) */
void ipr_keccakf(uint64_t a[25]);
void ipr_sha3_256(const uint8_t *m, size_t n, uint8_t out[32]);
void ipr_sha3_512(const uint8_t *m, size_t n, uint8_t out[64]);
void ipr_shake128(const uint8_t *m, size_t n, uint8_t *out, size_t outlen);
void ipr_shake256(const uint8_t *m, size_t n, uint8_t *out, size_t outlen);
void ipr_mlkem_ek(int k, const uint8_t d[32], uint8_t *ek);
void ipr_seed_from_u64(uint64_t state, uint8_t key[32]);
void ipr_dataset_record(int kem_k, uint64_t seed, uint64_t idx, uint8_t *out);

#ifdef __cplusplus
}
#endif
#endif
