/*
 * ipr_b200.h — C ABI of the B200-native InsPIRe keyword-PIR respond() path.
 *
 * Drop-in boundary for rkdud007/inspire-rs: the Rust KeywordServer
 * (src/pir/server/keyword.rs) keeps setup / public_params / respond and the
 * client wire format; the device work behind respond() is this library.
 * Plain pointers and sizes only; every call returns an int status
 * (IPR_OK = 0, negative on error) and never aborts; ipr_last_error() gives the
 * message of the calling thread's last failure.
 *
 * The reference-named entry points the Rust crate already declares
 * (src/pir/gpu/gemv.rs:5-25, encode.rs:3-32, packing_online.rs:11-92) are in
 * ipr_b200_compat.h.
 */
#ifndef IPR_B200_H
#define IPR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IPR_OK 0
#define IPR_E_ARGS -1     /* bad argument or shape */
#define IPR_E_OOM -2      /* device or host allocation failed, or HBM budget exceeded */
#define IPR_E_CUDA -3     /* CUDA runtime error (message in ipr_last_error) */
#define IPR_E_TIMEOUT -4  /* a bounded wait ran out */
#define IPR_E_FORMAT -5   /* malformed query bytes or state file */
#define IPR_E_SPACE -6    /* output buffer too small (required size reported) */
#define IPR_E_STATE -7    /* call made in the wrong state */
#define IPR_E_BUSY -8     /* request queue full (serving loop admission) */
#define IPR_E_IO -9       /* file read/write failed (state files) */
#define IPR_PENDING 1     /* request accepted, result not ready yet */

#define IPR_POLY_LEN 2048
#define IPR_RESULT_BYTES 12288 /* one switched RLWE result: 2048x28 + 2048x20 bits */

/* Shape plan of a keyword server.
 * Replaces KeywordServerSetupPlan::from_shape (src/pir/server/keyword.rs:145-233)
 * and KeywordServerGpuMemoryEstimate::from_plan (keyword.rs:105-141);
 * buckets = 0 / dim0 = 0 select the reference defaults (keyword.rs:29-31, 191-200). */
typedef struct ipr_plan {
    uint64_t num_items;      /* cuckoo buckets */
    uint64_t entry_size;     /* key + value bytes */
    uint64_t item_size_bits;
    uint64_t dim0;
    uint64_t db_rows;        /* first dimension (query row length) */
    uint64_t db_cols;        /* instances * 2048 */
    uint64_t instances;      /* packing outputs per query */
    uint64_t interp;         /* interpolation degree (fold depth) */
    uint64_t c;              /* fold groups = result polys per query */
    uint64_t peak_bytes;     /* the reference's setup peak estimate */
} ipr_plan;

int ipr_plan_from_shape(uint64_t record_count, uint64_t key_size, uint64_t value_size, uint64_t buckets,
                        uint64_t dim0, ipr_plan *out);

/* Serialized sizes: deserialize_keyword_query (src/protocol/wire.rs:618-705) and
 * serialize_keyword_response (wire.rs:708-726). */
uint64_t ipr_query_bytes(uint64_t db_rows, unsigned num_queries);

/* Fold-group sharding over several GPUs (no reference counterpart; the
 * partition follows the independence of the fold groups in
 * KeywordServer::respond, keyword.rs:558-574).  Shard k of S gets a
 * contiguous run of the plan's c fold groups (c / S, the first c % S shards
 * one more): instances [first_instance, first_instance + out->instances),
 * i.e. DB columns first_instance*2048 .. and the matching precomputation
 * rows.  Each shard's server answers the same query bytes with its groups'
 * results; ipr_response_merge concatenates the parts' results per query in
 * shard order and keeps the first part's stash block, which gives exactly the
 * unsharded server's response. */
int ipr_plan_shard(const ipr_plan *full, int num_shards, int shard, ipr_plan *out, uint64_t *first_instance);
int ipr_response_merge(const uint8_t *const *parts, const size_t *lens, int num_parts, uint8_t *out, size_t cap,
                       size_t *out_len);

typedef struct ipr_server ipr_server;

/* Host copies of the server state produced by setup (encode + offline
 * precomputation).  Layouts follow the reference:
 *   db          [db_cols][db_rows] u16, column-major (native/cuda/gemv_kernel.cu:63)
 *   a_hat       [instances][2048] u64 mod q           (PrecompInsPIR::a_hat, packing.rs:1718-1723)
 *   bold_t      [instances][3069][2048] u64 condensed (lo32 = mod q0, hi32 = mod q1)
 *   bold_t_bar  same layout
 *   bold_t_hat  [instances][3][2048] u64 condensed
 *   stash       stash_count entries of stash_entry_bytes (echoed in every response)
 * The public-parameter fields feed ipr_server_public_params_json. */
typedef struct ipr_server_data {
    const uint16_t *db;
    const uint64_t *a_hat;
    const uint64_t *bold_t;
    const uint64_t *bold_t_bar;
    const uint64_t *bold_t_hat;
    const uint8_t *stash;
    uint64_t stash_count;
    uint64_t stash_entry_bytes;
    uint64_t key_size, value_size, num_records;
    uint8_t cuckoo_seed[16];
} ipr_server_data;

/* Upload server state to device `device` and build the per-request pipeline.
 * Replaces gpu_gemv_upload_db + gpu_packing_online_upload_precomp +
 * gpu_rotation_upload_tables (gemv_kernel.cu:116-141, packing_online_kernel.cu:110-142,
 * rotation_kernel.cu:71-94).  Fails with IPR_E_OOM if it does not fit. */
int ipr_server_create(int device, const ipr_plan *plan, const ipr_server_data *data, ipr_server **out);

/* Same, with data->db the RAW database (KeywordCuckooTable::to_raw_db layout,
 * src/pir/keyword/cuckoo.rs:314-353): the server encodes it on the device
 * (ipr_encode_db) instead of the caller running gpu_encode_db first. */
int ipr_server_create_from_raw(int device, const ipr_plan *plan, const ipr_server_data *data, ipr_server **out);

/* KeywordServer::setup on the device (keyword.rs:366-468 with the GPU branches of
 * perform_offline_precomputation_simplepir): data->db is the DB (the RAW to_raw_db layout
 * when db_is_raw, else already encoded); the encode and the whole offline precomputation
 * run on `device` (ipr_encode_db, ipr_offline_precompute), so data->a_hat, bold_t,
 * bold_t_bar and bold_t_hat are ignored (may be NULL).  Stash and public parameters as
 * in ipr_server_create. */
int ipr_server_setup(int device, const ipr_plan *plan, const ipr_server_data *data, int db_is_raw, ipr_server **out);

/* Same, with seeded synthetic DB / precomputation generated on the device
 * (uniform u16 < 65535, uniform residues), the timing mode the reference
 * itself uses (online_only, src/pir/server/engine.rs:693-729). */
int ipr_server_create_synthetic(int device, const ipr_plan *plan, uint64_t seed, ipr_server **out);
/* Shard `shard` of `num_shards` (ipr_plan_shard) of the synthetic server that
 * ipr_server_create_synthetic(full, seed) builds: the same elements of DB and
 * precomputation, generated alone, so the shards' merged responses equal the full
 * server's. */
int ipr_server_create_synthetic_shard(int device, const ipr_plan *full, int num_shards, int shard, uint64_t seed,
                                      ipr_server **out);

void ipr_server_destroy(ipr_server *srv);

/* KeywordServer::public_params (keyword.rs:511-532), serde JSON form of PublicParams. */
int ipr_server_public_params_json(const ipr_server *srv, char *out, size_t cap, size_t *out_len);

uint64_t ipr_server_query_bytes(const ipr_server *srv, unsigned num_queries);
uint64_t ipr_server_response_bytes(const ipr_server *srv, unsigned num_queries);
int ipr_server_hbm_bytes(const ipr_server *srv, uint64_t *out);
int ipr_server_plan(const ipr_server *srv, ipr_plan *out);

/* KeywordServer::respond_to_serialized_query (keyword.rs:636-640): serialized
 * KeywordQueryPayload in, serialized KeywordResponsePayload out, host buffers.
 * On IPR_E_SPACE *out_len holds the required size.  Thread safe (serialised
 * per server). */
int ipr_server_respond(ipr_server *srv, const uint8_t *query, size_t len, uint8_t *out, size_t cap,
                       size_t *out_len);

/* n payloads; statuses[i] receives each payload's status.  Payloads carrying
 * the usual two cuckoo queries are answered together, up to 64 per pass, on
 * the tensor-core batch path (byte-split INT8 tcgen05 GEMMs for the first
 * dimension and for the InspiRING packing of all clients at once); results
 * are identical to answering them one at a time. */
int ipr_server_respond_batch(ipr_server *srv, int n, const uint8_t *const *queries, const size_t *lens,
                             uint8_t *const *outs, const size_t *caps, size_t *out_lens, int *statuses);

/* Build the batch-path state ahead of the first batch (the slot-indexed
 * packing precomputation, instances x 2 x 2048 x 128 x 6144 / 32 bytes, and
 * scratch for max_payloads <= 64 payloads). */
int ipr_server_prepare_batch(ipr_server *srv, int max_payloads);

/* Device-resident batch: n (1..64) two-query payloads packed back to back in
 * device memory (stride ipr_server_query_bytes(srv, 2)), responses written back
 * to back (stride ipr_server_response_bytes(srv, 2)).  Enqueued on the server
 * stream; returns without waiting. */
int ipr_server_respond_batch_device(ipr_server *srv, int n, const uint8_t *d_queries, uint8_t *d_out);

/* Device-resident variant: query and response already in device memory of
 * the server's device.  Enqueued on the server stream and returns without
 * waiting; `len` must be the exact query size for the payload's query count. */
int ipr_server_respond_device(ipr_server *srv, const uint8_t *d_query, size_t len, uint8_t *d_out, size_t cap,
                              size_t *out_len);
int ipr_server_stream(ipr_server *srv, void **cuda_stream);
int ipr_server_sync(ipr_server *srv);

/* Per-stage CUDA-event timing on the server stream (stages below), summed
 * over the calls since profiling was enabled.  IPR_STAGE_POST is the step between
 * the packing sum and the fold: the scaling pass of the fused fold (default), or the
 * INTT + CRT pass of the separate form (IPR_OPT_FOLD_REGISTER_NTT 0 or 1). */
#define IPR_STAGE_PARSE 0
#define IPR_STAGE_GEMV 1
#define IPR_STAGE_PACK 2
#define IPR_STAGE_POST 3
#define IPR_STAGE_FOLD 4
#define IPR_NSTAGES 5
int ipr_server_set_profiling(ipr_server *srv, int on);

/* Execution options.  IPR_OPT_TENSOR_GEMV: 1 = first-dimension GEMV on the
 * tensor cores over DB byte planes (default where db_rows <= 32768), 0 = the
 * CUDA-core kernel on the u16 DB.  Both give identical results. */
#define IPR_OPT_TENSOR_GEMV 1
/* IPR_OPT_FOLD_REGISTER_NTT: the form of the RGSW fold.  3 (default) = register-
 * resident NTTs with the packing post-process (INTT + CRT + b add) fused into the
 * fold's own inverse transforms, one chain per CTA, chosen per call between two CTAs
 * per SM (the query's RGSW bodies staged through shared memory) and three per SM (the
 * bodies read from L2 where they are used) by the rounds each needs for the call's
 * chains; 4 = always three per SM; 5 = always two per SM; 2 = the same fused fold on two chains of one
 * query per CTA sharing the bodies in shared memory (an odd fold-group count leaves
 * half a CTA idle); 1 = register-resident NTTs after a separate INTT + CRT pass;
 * 0 = shared-memory NTTs after that pass (single-payload calls only; batches then
 * use form 1).  Identical results. */
#define IPR_OPT_FOLD_REGISTER_NTT 2
/* IPR_OPT_PACK_CTA_PAIR: 1 = the batch path's packing GEMM runs on CTA pairs
 * (tcgen05 cta_group::2, M = 256 across two SMs); 0 = one CTA per unit;
 * 2 (default) = pairs from 48 payloads per batch up, where they are faster.
 * Identical results. */
#define IPR_OPT_PACK_CTA_PAIR 3
/* IPR_OPT_GEMV_TILE: cap on the first-dimension GEMM's query-byte tile height
 * (16, 32, 64, 128 or 256; 0 = 256, the default).  A query takes 7 byte rows (the bytes
 * of its CRT-composed value), so the tile height N of each MMA is the smallest multiple of
 * 16 that holds the call's queries, at most 224 (32 queries), and under a cap of 128 or
 * more the largest multiple of 112 (16 queries) within it.  Up to 128 the two accumulators
 * of a tile are double-buffered in TMEM. */
#define IPR_OPT_GEMV_TILE 4
/* IPR_OPT_GEMV_FORM: form of the CUDA-core first-dimension GEMV (IPR_OPT_TENSOR_GEMV 0)
 * for two queries: 0 / 1 / 2 = 8 / 4 / 2 DB columns per warp loaded into
 * registers (fewer columns, fewer partial sums per thread, more warps per SM); 3 = 8 columns
 * per warp streamed through a 4-stage shared-memory ring by cp.async; 4 = form 0 with the
 * products on the FP64 pipe (exact: every partial sum is an integer below 2^53); 5 = form
 * 3's shared-memory ring with the products on the FP64 pipe, the query residues converted to
 * doubles once per CTA and the DB entries turned into doubles by integer operations (up to
 * 4,096 DB rows; above, form 4); 6 (default) = a lane per DB column in 16 warps, the DB and
 * the query residues brought into shared memory in stages by TMA, the products on the FP64
 * pipe (any number of DB rows that is a multiple of 256).  Forms 4 and 5 run as form 0 above
 * 16,384 DB rows.  Identical results. */
#define IPR_OPT_GEMV_FORM 5
int ipr_server_set_option(ipr_server *srv, int option, int64_t value);

/* Autotuner for the batch path: runs `reps` timed batches of `payloads` synthetic payloads,
 * and as many of payloads / 4 (from 4 payloads up), after one warm-up each, under every
 * candidate of IPR_OPT_PACK_CTA_PAIR {2 (automatic), 0, 1} x IPR_OPT_GEMV_TILE {256, 128},
 * timed with CUDA events on the server's stream, round-robin.  It leaves the server set
 * to the candidate with the least device time per payload summed over the two sizes, so a
 * choice that only suits full batches does not slow the smaller ones a serving loop also
 * runs.  Every candidate gives identical responses.  On an error the options are restored. */
#define IPR_AUTOTUNE_MAX 8
typedef struct {
    int candidates;                    /* how many were timed */
    int pack_cta_pair[IPR_AUTOTUNE_MAX];
    int gemv_tile[IPR_AUTOTUNE_MAX];
    double ms[IPR_AUTOTUNE_MAX];       /* mean device time per batch of `payloads` */
    int chosen;                        /* index of the candidate now in force */
    int small_payloads;                /* the second batch size timed (0: none) */
    double ms_small[IPR_AUTOTUNE_MAX]; /* mean device time per batch of small_payloads */
} ipr_autotune_result;
int ipr_server_autotune(ipr_server *srv, int payloads, int reps, ipr_autotune_result *out);
int ipr_server_stage_times(ipr_server *srv, double *ms_sum, uint64_t *calls);

const char *ipr_last_error(void);
const char *ipr_version(void);

/* First-dimension GEMV query that allocates no device memory.  No counterpart
 * in the reference: it is gpu_gemv_query (ipr_b200_compat.h) for callers that
 * cannot call cudaMalloc, e.g. a process whose framework has reserved all free
 * HBM for its own pool, or a request path that cannot take cudaMalloc's
 * device-wide synchronisation.  Same arguments and result as gpu_gemv_query
 * (h_a: db_rows condensed query values; h_c: b_cols results mod q; d_db: the
 * column-major u16 DB on the current device), but the query row and result
 * are staged in a fixed 8.5 MiB device array inside this library (at most
 * 65,536 rows and 1,048,576 columns; larger shapes return IPR_E_ARGS, and so
 * does a query entry that is not reduced, lo32 >= q0 or hi32 >= q1).  Every
 * GPU that loads the library holds that array until the process exits.  All
 * calls share it, so calls that overlap on the GPU race; issue them one at a
 * time.  The first call on a device resolves the array's address and loads
 * constants for that device; make it before any stream capture there.
 * Returns IPR_OK or a negative status (message in ipr_last_error()). */
int ipr_gemv_query_noalloc(uint64_t *h_c, const uint64_t *h_a, const uint16_t *d_db, int db_rows, int b_cols);

/* Kernel-level building blocks over device buffers (no reference counterpart as
 * entry points: the reference runs them inside respond()).  Polynomials are
 * 2048 u64 coefficients of one CRT limb (canonical residues mod q_limb).
 * ipr_ntt_batch: in place, the negacyclic NTT of ntt_forward / ntt_inverse
 * (src/core/ntt.rs:111-160, 731-780) for `count` polynomials of limb 0 or 1.
 * ipr_automorph_batch: out[j][p] = the NTT-domain image of in[p] under
 * x -> x^ks[j] (ks odd, < 4096; the rotation gather of
 * native/cuda/rotation_kernel.cu:21-59), out holding nk * count polynomials.
 * Both are enqueued on `stream` (a cudaStream_t, NULL = legacy default). */
int ipr_ntt_batch(int device, uint64_t *d_polys, uint64_t count, int limb, int inverse, void *stream);
int ipr_automorph_batch(int device, const uint64_t *d_in, uint64_t count, const uint32_t *d_ks, int nk,
                        uint64_t *d_out, void *stream);

/* Offline precomputation on the GPU: PirServer::perform_offline_precomputation_simplepir
 * (src/pir/server/engine.rs:677-1042; hint, prep_pack, packing sums, automorphisms and
 * the 1023-step collapse of full_packing_with_preprocessing_offline, packing.rs:2440-2734)
 * for the encoded column-major DB d_db ([instances * 2048][db_rows] u16, db_rows a
 * multiple of 2048).  Writes the arrays of ipr_server_data on the device:
 * d_a_hat [instances][2048] u64 mod q, d_bold_t / d_bold_t_bar [instances][3069][2048]
 * condensed, d_bold_t_hat [instances][3][2048] condensed.  Replaces the reference's
 * gpu_hint_*, gpu_prep_pack_*, gpu_packing_* and gpu_collapse_* sequence.  Scratch is
 * allocated inside, at most scratch_bytes (0 = 4 GiB; 64 MiB per instance processed
 * together); the call returns when the outputs are complete. */
int ipr_offline_precompute(int device, const uint16_t *d_db, uint64_t db_rows, uint64_t instances,
                           uint64_t *d_a_hat, uint64_t *d_bold_t, uint64_t *d_bold_t_bar, uint64_t *d_bold_t_hat,
                           uint64_t scratch_bytes, void *stream);

/* InspiRING packing of LWE ciphertexts into RLWE ciphertexts on the GPU:
 * packing_fully_online (src/pir/packing.rs:3122-3162) for sets of 2048 LWEs each —
 * the offline precomputation of full_packing_with_preprocessing_offline on the
 * sets' a-vectors (as in ipr_offline_precompute) followed by
 * full_packing_with_preprocessing_online (packing.rs:2941-3021) with the packing
 * keys.  d_lwe [sets][2049][2048] u64: row j < 2048 holds coefficient j of the
 * 2048 a-vectors (LWE i in column i), row 2048 the b values; d_y_body / d_z_body:
 * the packing keys' y_body / z_body, condensed [3][2048] (lo32 = mod q0, hi32 =
 * mod q1).  d_out [sets][2][2048] u64: row 0 = a_hat mod q, row 1 = b + the packed
 * sum mod q (not reduced, < 2q, as add_raw leaves it).  The context holds the
 * tables, the W / V masks and scratch for up to max_sets sets (about 150 MB each);
 * calls on one context must not overlap on the GPU. */
typedef struct ipr_inspiring ipr_inspiring;
int ipr_inspiring_create(int device, int max_sets, ipr_inspiring **out);
int ipr_inspiring_pack(ipr_inspiring *ctx, int sets, const uint64_t *d_lwe, const uint64_t *d_y_body,
                       const uint64_t *d_z_body, uint64_t *d_out, void *stream);
void ipr_inspiring_destroy(ipr_inspiring *ctx);

/* Server state file (no reference counterpart: the reference reruns encode and the
 * offline precomputation on every start, keyword.rs:366-457).  ipr_server_save writes
 * the setup outputs the server was built from (the arrays of ipr_server_data: encoded
 * DB, a_hat, bold_t, bold_t_bar, bold_t_hat, stash) with the plan and public
 * parameters; ipr_server_load rebuilds a server from such a file on `device`, answering
 * byte for byte like the saved one, without the caller holding the arrays in host memory.
 * Format: a 4096-byte header (magic "IPRSTATE", version 1, the ipr_plan fields, key /
 * value sizes, record count, cuckoo seed, stash shape, one {offset, bytes, checksum}
 * entry per section, a header checksum), then the six sections in that order, each
 * starting on a 4096-byte boundary, the file ending on one.  Checksums are
 * sum_i mix64(w_i + i * 0x9E3779B97F4A7C15) mod 2^64 over the section's little-endian
 * 64-bit words w_i (last word zero-padded), mix64 the splitmix64 finaliser.  A file
 * whose header, section table, size or checksums disagree is refused with IPR_E_FORMAT;
 * I/O failures return IPR_E_IO.  ipr_state_file_plan reads only the header (no GPU). */
int ipr_server_save(ipr_server *srv, const char *path);
int ipr_server_load(int device, const char *path, ipr_server **out);
int ipr_state_file_plan(const char *path, ipr_plan *out);

/* ---- keyword-PIR client on the GPU (KeywordClient, src/pir/client/keyword.rs) ----------
 * Query generation and response decryption for a server plan.  The secret key (ternary,
 * 256 coefficients +1 and 256 -1, gen_ternary_mat, client/base.rs:126-139) and all noise are
 * drawn deterministically from `seed` with ChaCha20: key placement from stream 1, the noise
 * of a query from stream 2 + nonce (centered binomial, eta = 82: sigma 6.40, the width of the
 * reference's discrete Gaussian).  A nonce must not be reused under one seed.  A client
 * handle keeps per-call scratch: use it from one thread at a time (one handle per thread). */
typedef struct ipr_client ipr_client;

/* KeywordClient::setup_from_public_params (keyword.rs:60-115) for `plan` */
int ipr_client_create(int device, const ipr_plan *plan, const uint8_t seed[32], ipr_client **out);
/* build_query_payload + serialize_query (keyword.rs:193-214, wire.rs:542-615): one payload
 * whose n sub-queries ask for the given buckets (cuckoo positions); writes
 * ipr_query_bytes(db_rows, n) bytes (IPR_E_SPACE when `cap` is smaller; *out_len is set). */
int ipr_client_query(ipr_client *c, uint64_t nonce, unsigned n, const uint64_t *buckets, uint8_t *out,
                     size_t cap, size_t *out_len);
/* decrypt_response_values (keyword.rs:216-245) of every response of a serialized
 * KeywordResponsePayload: values[q][w][z] (u16 plaintexts mod 65535, fold group w, slot z),
 * *count = responses x c x 2048.  The stash block is not read. */
int ipr_client_decrypt(ipr_client *c, const uint8_t *response, size_t len, uint16_t *values, size_t cap,
                       size_t *count);
/* CuckooHash::all_positions (src/pir/keyword/cuckoo.rs:105-131): the num_hashes bucket
 * positions of a keyword under the server's 16-byte cuckoo seed.  Hash i is SipHash-2-4
 * with keys (seed[0..8] LE ^ i, seed[8..16] LE ^ (i << 32)) mod num_buckets; the all-zero
 * seed is the identity layout (last 8 key bytes big-endian, hash 0 into the first half of the
 * table, hash 1 into the second).  Host only. */
int ipr_cuckoo_positions(const uint8_t seed[16], uint64_t num_buckets, unsigned num_hashes, const uint8_t *key,
                         size_t key_len, uint64_t *out);
/* the client's secret key, 2048 coefficients in {-1, 0, 1} (for tests) */
int ipr_client_secret_key(const ipr_client *c, int8_t *out);
void ipr_client_destroy(ipr_client *c);

/* Fault injection for tests (process-wide): the next `after` device allocations of servers
 * succeed and the one after fails as an out-of-memory would (IPR_E_OOM from the call that
 * needed it); the hook then switches itself off.  after < 0 switches it off at once. */
int ipr_debug_fail_allocation(int64_t after);

/* The compute capability the library's device code was compiled for, as the CUDA runtime
 * reports it for one of its kernels on `device` (100 for sm_100a), without reading the
 * binary. */
int ipr_device_binary_version(int device, int *binary_version);

/* Failure detection self-test: launches one CTA that waits, with the bounded wait every
 * tensor-core kernel of this library uses on its mbarriers, on a barrier nothing arrives
 * on.  The wait gives up after limit_us microseconds of GPU global time (1 .. 1,000,000,
 * else IPR_E_ARGS); the call returns IPR_E_TIMEOUT (the status a server call returns when
 * one of its kernels' waits runs out, after 100 ms there) and the device stays usable. */
int ipr_selftest_bounded_wait(int device, uint32_t limit_us);

/* Bounds-checked debug build (libipr_b200_dbg.so, built with -DIPR_BOUNDS_CHECK by
 * `make -C inspire-rs_b200 debug`).  ipr_bounds_checked_build returns 1 in that build and
 * 0 in the release library.  In the debug build every launch of the respond() path first
 * checks each buffer argument's byte range, computed from the launch's parameters, against
 * the device allocation holding it (a launch outside fails with IPR_E_CUDA), and the fold
 * and its scaling pass check every global index against the extents they are given,
 * skipping the access and recording a site id instead of faulting.  ipr_bounds_report
 * synchronises the current device, writes one line per failure since the last report
 * (NUL-terminated, truncated to cap) and returns their count; 0 in the release build. */
int ipr_bounds_checked_build(void);
int ipr_bounds_report(char *out, size_t cap);
/* Debug build only (IPR_E_STATE in the release library): ipr_debug_check_extent runs the
 * launch-argument check on [d_ptr, d_ptr + bytes) (IPR_OK inside one device allocation,
 * IPR_E_ARGS outside, recorded for ipr_bounds_report); ipr_debug_cut_fold_extent(words)
 * makes every later fold launch believe its packing-output buffer is `words` words shorter
 * than it is, so that the fold's own index checks trip on allocated memory (0 restores). */
int ipr_debug_check_extent(const void *d_ptr, uint64_t bytes);
int ipr_debug_cut_fold_extent(int64_t words);

/* Dataset generation on the GPU: DatasetGenerator::generate_record (src/dataset/generator.rs:
 * 171-193) for records first .. first + count - 1 of the dataset with `seed` and KEM
 * ML-KEM-`kem` (512, 768 or 1024).  Record i is id (32 bytes) || pk (800 / 1184 / 1568
 * bytes), written to d_records + i * (32 + pk_len): pk the FIPS 203 encapsulation key from
 * d = the ChaCha20Rng::seed_from_u64(seed) keystream block number first + i (kem.rs:27-44),
 * id = SHA3-256("pq-key:v1:" || "ml-kem-<kem>" || pk) (dataset.rs:36-46).  Enqueued on
 * `stream` (a cudaStream_t, NULL = legacy default). */
int ipr_dataset_generate(int device, int kem, uint64_t seed, uint64_t first, uint64_t count, uint8_t *d_records,
                         void *stream);
/* The same records into host memory h_records (count * (32 + pk_len) bytes), generated in
 * device batches of up to 65,536 records; returns when they are copied. */
int ipr_dataset_generate_host(int device, int kem, uint64_t seed, uint64_t first, uint64_t count, uint8_t *h_records);

/* Setup-time database layout and encode on device buffers.
 * ipr_cuckoo_to_raw_db: KeywordCuckooTable::to_raw_db (cuckoo.rs:314-353) — bucket
 * entries (num_buckets x entry_size bytes, row-major) and occupancy flags (one byte
 * per bucket) -> the column-major u16 raw DB [db_cols][db_rows], per = buckets per
 * DB row, entry bytes (2j, 2j+1) big-endian into column item * entry_size/2 + j.
 * ipr_encode_db: gpu_encode_db (native/cuda/encode_kernel.cu:264-386) — the
 * interpolation of each fold group's interp polynomials over Z_65535[X]/(X^2048+1),
 * raw -> encoded ([db_cols][db_rows] u16 both; interp a power of two <= 32,
 * db_rows a multiple of 32; input and output distinct, 16-byte aligned). */
int ipr_cuckoo_to_raw_db(int device, const uint8_t *d_entries, const uint8_t *d_occupied, uint64_t num_buckets,
                         uint64_t entry_size, uint64_t db_rows, uint64_t db_cols, uint64_t per, uint16_t *d_raw,
                         void *stream);
int ipr_encode_db(int device, const uint16_t *d_raw, uint16_t *d_encoded, uint64_t db_rows, uint64_t db_cols,
                  uint64_t interp, void *stream);

/* ---------------------------------------------------------------------------
 * Serving loop with continuous batching (no reference counterpart: the
 * reference answers one payload at a time, keyword.rs:534-640).  One
 * scheduler thread per service; requests are queued per database (index into
 * `servers`); whenever a device slot of a database frees, everything pending
 * for it (up to the admitted batch size) is launched as one tensor-core batch,
 * so batches grow with the load.  Two-query payloads take the batch path;
 * other query counts are answered alone, in arrival order.  Responses are
 * byte-identical to ipr_server_respond.
 *
 * Admission: the batch size is the largest B <= max_batch (<= 64) whose
 * batch-path device memory over all databases fits hbm_budget_bytes (0 = the
 * free HBM at creation minus 2 GiB); creation fails with IPR_E_OOM if even
 * B = 1 does not fit.  At most max_pending requests wait (0 = 4096); beyond
 * that ipr_service_submit returns IPR_E_BUSY.  The servers must outlive the
 * service; direct calls on them stay legal and are serialised with it.
 * -------------------------------------------------------------------------- */
typedef struct ipr_service ipr_service;

typedef struct ipr_service_config {
    int max_batch;
    int max_pending;
    uint64_t hbm_budget_bytes;
} ipr_service_config;

typedef struct ipr_service_stats {
    uint64_t submitted, completed, rejected, failed;
    uint64_t batches, batched_payloads; /* device batch passes and the payloads they carried */
    uint64_t pending, in_flight;        /* queued / submitted but not yet collected */
    int max_batch;                      /* admitted batch size */
    uint64_t hbm_bytes;                 /* device bytes the batch path and the I/O slots hold */
    double p50_us, p99_us, mean_us, max_us; /* submit -> completion, completed requests since the last reset */
    uint64_t latency_samples;
    double batch_ms_mean, batch_ms_max;     /* device time per batch (its start to its responses on the host) */
    double queue_ms_mean, queue_ms_max;     /* submit -> launch of the request's batch */
} ipr_service_stats;

int ipr_service_create(ipr_server *const *servers, int num_servers, const ipr_service_config *cfg,
                       ipr_service **out);
/* Admit one more database to a running service (up to 64 in all): its batch size is the
 * largest B <= max_batch whose batch-path memory and I/O slots fit what the earlier
 * databases left of the HBM budget (IPR_E_OOM if even B = 1 does not fit); *db is its
 * index for submit.  The databases already served keep running meanwhile. */
int ipr_service_add_database(ipr_service *svc, ipr_server *server, int *db);
/* Queue one serialized KeywordQueryPayload for database `db`; *ticket names it. */
int ipr_service_submit(ipr_service *svc, int db, const uint8_t *query, size_t len, uint64_t *ticket);
/* n payloads queued atomically (all or none: IPR_E_BUSY if the queue cannot take all,
 * IPR_E_FORMAT if any is malformed), so the dispatcher sees them together and fills whole
 * batches at once, e.g. for a frontend forwarding a burst.  tickets[i] for queries[i]. */
int ipr_service_submit_batch(ipr_service *svc, int db, int n, const uint8_t *const *queries, const size_t *lens,
                             uint64_t *tickets);
/* IPR_PENDING while running; otherwise the request's status, with the serialized
 * response copied to out (IPR_E_SPACE and *out_len = size if cap is short; the
 * result is kept for a retry).  A collected ticket is released. */
int ipr_service_poll(ipr_service *svc, uint64_t ticket, uint8_t *out, size_t cap, size_t *out_len);
/* As poll, blocking up to timeout_ms (< 0: no limit); IPR_PENDING on timeout. */
int ipr_service_wait(ipr_service *svc, uint64_t ticket, int timeout_ms, uint8_t *out, size_t cap, size_t *out_len);
int ipr_service_get_stats(ipr_service *svc, ipr_service_stats *out);
/* The most recent batches (up to 4096 kept), oldest first: times in ms since the
 * service was created — launch (enqueued), start (device free for it), ready
 * (responses on the host) — and the longest submit -> launch wait in it. */
typedef struct ipr_service_batch {
    int db, payloads;
    double launch_ms, start_ms, ready_ms, queue_ms_max;
} ipr_service_batch;
int ipr_service_batch_log(ipr_service *svc, ipr_service_batch *out, int cap, int *n);
int ipr_service_reset_stats(ipr_service *svc);
/* A text snapshot of every database lane for diagnosing a stalled service: queued
 * requests, busy I/O slots, and whether each slot's upload and compute events and the
 * lane's server and download streams have completed (CUDA queries, no waiting).
 * NUL-terminated, truncated to cap bytes. */
int ipr_service_diagnose(ipr_service *svc, char *out, size_t cap);
/* Finishes the batches in flight, drops queued and uncollected requests. */
void ipr_service_destroy(ipr_service *svc);

#ifdef __cplusplus
}
#endif
#endif
