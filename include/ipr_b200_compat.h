/*
 * ipr_b200_compat.h — the respond-path symbols the reference's Rust crate
 * already declares, exported with identical names, argument meaning and
 * (void) error behaviour, implemented on this library's sm_100a kernels.
 * Linking these in place of native/cuda/{gemv,rotation,packing_online,encode,hint,
 * prep_pack,packing,collapse}_kernel.cu lets the unmodified Rust glue drive the new
 * kernels, setup included.  Errors are printed to
 * stderr and recorded for ipr_last_error(), then the call returns, as in the
 * reference (CHECK_CUDA_TAG, native/cuda/common.h:16-23).
 *
 * Global state mirrors the reference: one resident DB per process, one set of
 * packing buffers, all work on one high-priority query stream.
 */
#ifndef IPR_B200_COMPAT_H
#define IPR_B200_COMPAT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* src/pir/gpu/encode.rs:3-8 (native/cuda/encode_kernel.cu:233-262) */
void gpu_init_memory_pool(void);
void gpu_trim_memory_pool(void);
uint64_t gpu_available_memory_bytes(void);

/* src/pir/gpu/encode.rs:7-20 (native/cuda/encode_kernel.cu:264-480): encode the host raw
 * DB and keep the encoded DB on the device (h_db_out is not written, as in the
 * reference); modulus must be 65535 and num_inv interp^-1 mod 65535. */
void gpu_encode_db(uint16_t *d_db_in, uint16_t *d_db_out, int db_rows, int db_cols, int interp_degree, int gamma,
                   int c, uint32_t modulus, uint32_t num_inv);
void gpu_encode_db_from_host(const uint16_t *h_db_in, uint16_t *h_db_out, int db_rows, int db_cols,
                             int interp_degree, int gamma, int c, uint32_t modulus, uint32_t num_inv);
const uint16_t *gpu_encode_get_device_db(void);
void gpu_encode_free_device_db(void);
/* src/pir/gpu/encode.rs:20-31 (native/cuda/encode_kernel.cu:452-516): encode a new host DB
 * into a secondary device slot (uploaded in 256 MB pieces on the per-thread stream) while
 * the primary keeps serving; get its pointer; free the primary and promote the secondary. */
void gpu_encode_db_from_host_fold(const uint16_t *h_db_in, int db_rows, int db_cols, int interp_degree, int gamma,
                                  int c, uint32_t modulus, uint32_t num_inv);
const uint16_t *gpu_encode_get_device_db_fold(void);
void gpu_encode_swap_primary(void);

/* src/pir/gpu/gemv.rs:5-25 (native/cuda/gemv_kernel.cu:106-194) */
void gpu_gemv_upload_db(const uint16_t *h_db, uint16_t **d_db_out, size_t db_size_bytes);
void gpu_gemv_set_device_db(uint16_t **d_db_out, const uint16_t *d_db_in, size_t db_size_bytes);
void gpu_gemv_free_db(uint16_t *d_db);
void gpu_gemv_query(uint64_t *h_c, const uint64_t *h_a, const uint16_t *d_db, int db_rows, int b_cols,
                    uint64_t mod0, uint64_t mod1, uint64_t cr0, uint64_t cr1, uint64_t mod0_inv_mod1,
                    uint64_t mod1_inv_mod0, uint64_t modulus, uint64_t barrett_cr0_mod,
                    uint64_t barrett_cr1_mod);

/* src/pir/gpu/packing_online.rs:11-92 (native/cuda/rotation_kernel.cu:71-144,
 * native/cuda/packing_online_kernel.cu:110-333) */
void gpu_rotation_upload_tables(const uint32_t *h_tables, const uint32_t *h_gen_pows, int num_tables,
                                int num_rotations, int poly_len);
void gpu_rotation_expand_keys(uint64_t *d_y_all_out, uint64_t *d_y_bar_all_out, const uint64_t *h_y_body,
                              int num_rotations, int t_exp_left, int poly_len);
void gpu_rotation_free(void);
void gpu_packing_online_ensure_key_buffers(int n_inner, int t_exp_left, int poly_len);
uint64_t *gpu_packing_online_get_d_y_all(void);
uint64_t *gpu_packing_online_get_d_y_bar_all(void);
void gpu_packing_online_upload_z_body(const uint64_t *h_z_body, int t_exp_left, int poly_len);
void gpu_packing_online_upload_precomp(const uint64_t *h_bold_t, const uint64_t *h_bold_t_bar,
                                       const uint64_t *h_bold_t_hat, int num_outputs, int n_inner,
                                       int t_exp_left, int poly_len);
void gpu_packing_online_upload_keys(const uint64_t *h_y_all, const uint64_t *h_y_bar_all,
                                    const uint64_t *h_z_body, int n_inner, int t_exp_left, int poly_len);
void gpu_packing_online_compute(uint64_t *h_output, int num_outputs, int nphalf_minus_1, int t_exp_left,
                                int poly_len, int addition_capacity, uint64_t mod0, uint64_t mod1, uint64_t cr0,
                                uint64_t cr1);
void gpu_packing_online_adopt_precomp(uint64_t *d_bold_t, uint64_t *d_bold_t_bar, uint64_t *d_bold_t_hat,
                                      int num_outputs, int n_inner, int t_exp_left, int poly_len);
void gpu_packing_online_swap_precomp(uint64_t *new_bt, uint64_t *new_bt_bar, uint64_t *new_bt_hat,
                                     int num_outputs, int n_inner, int t_exp_left, int poly_len);
void gpu_packing_online_free(void);

/* ---- offline precomputation (csrc/compat_offline.cu) ----
 * src/pir/gpu/hint.rs:6-71 (native/cuda/hint_kernel.cu:270-420): tables [2][4][2048] u64
 * (fwd, fwd', inv, inv' per limb), query [db_rows_poly][2][2048] NTT, hint output
 * [2048][db_cols] u64 raw mod q (transposed: coefficient z of column c at z * db_cols + c). */
void gpu_hint_upload_tables(const uint64_t *h_ntt_tables, int poly_len);
void gpu_hint_upload_query_ffi(const uint64_t *h_query, int db_rows_poly, int poly_len);
void gpu_hint_compute(const uint16_t *d_db, uint64_t *h_output, int db_rows, int db_rows_poly, int db_cols,
                      uint32_t mod0, uint32_t mod1, uint64_t barrett_cr1_0, uint64_t barrett_cr1_1,
                      uint64_t mod0_inv_mod1, uint64_t mod1_inv_mod0, uint64_t modulus, uint64_t barrett_cr0_mod,
                      uint64_t barrett_cr1_mod);
void gpu_hint_compute_from_host(const uint16_t *h_db, uint64_t *h_output, int db_rows, int db_rows_poly,
                                int db_cols, uint32_t mod0, uint32_t mod1, uint64_t barrett_cr1_0,
                                uint64_t barrett_cr1_1, uint64_t mod0_inv_mod1, uint64_t mod1_inv_mod0,
                                uint64_t modulus, uint64_t barrett_cr0_mod, uint64_t barrett_cr1_mod);
void gpu_hint_compute_no_d2h(const uint16_t *d_db, int db_rows, int db_rows_poly, int db_cols, uint32_t mod0,
                             uint32_t mod1, uint64_t barrett_cr1_0, uint64_t barrett_cr1_1, uint64_t mod0_inv_mod1,
                             uint64_t mod1_inv_mod0, uint64_t modulus, uint64_t barrett_cr0_mod,
                             uint64_t barrett_cr1_mod);
void gpu_hint_free(void);
void gpu_hint_free_query_only(void);
void gpu_hint_free_output_and_tables(void);
const uint64_t *gpu_hint_get_device_output(void);
const uint64_t *gpu_hint_get_ntt_tables(void);
int gpu_hint_get_db_cols(void);

/* src/pir/gpu/prep_pack.rs:12-24 (native/cuda/prep_pack_kernel.cu:125-167): output
 * [db_cols][2][2048] NTT of each hint column in negacyclic order */
void gpu_prep_pack_compute(const uint64_t *d_hint_output, const uint64_t *d_ntt_tables, int db_cols, uint32_t mod0,
                           uint32_t mod1, uint64_t modulus);
const uint64_t *gpu_prep_pack_get_output(void);
void gpu_prep_pack_free(void);

/* src/pir/gpu/packing.rs:9-80 (native/cuda/packing_kernel.cu:134-806): packing sums
 * r / r_bar [nphalf][2 * 2048] before the automorphisms, times mod_inv */
void gpu_packing_precomp(const uint64_t *h_mono_table, const uint64_t *h_a_ct, const int *h_idx, const int *h_idx_bar,
                         const uint64_t *h_mod_inv, uint64_t *h_r_out, uint64_t *h_r_bar_out, int num_to_pack_half,
                         int non_zeros, int poly_len, int crt_count, uint64_t mod0, uint64_t mod1,
                         uint64_t barrett_cr0, uint64_t barrett_cr1);
void gpu_packing_setup(const uint64_t *h_mono_table, const int *h_idx, const int *h_idx_bar, const uint64_t *h_mod_inv,
                       int num_to_pack_half, int non_zeros, int poly_len, int crt_count, uint64_t mod0, uint64_t mod1,
                       uint64_t barrett_cr0, uint64_t barrett_cr1);
void gpu_packing_precomp_fast(const uint64_t *h_a_ct, uint64_t *h_r_out, uint64_t *h_r_bar_out);
void gpu_packing_precomp_fast_device(const uint64_t *d_a_ct_device, uint64_t *h_r_out, uint64_t *h_r_bar_out);
void gpu_packing_precomp_fast_device_no_d2h(const uint64_t *d_a_ct_device);
void gpu_packing_teardown(void);
void gpu_packing_precomp_batched(const uint64_t *h_mono_table, const uint64_t *h_a_ct_batch, const int *h_idx,
                                 const int *h_idx_bar, const uint64_t *h_mod_inv, uint64_t *h_r_out,
                                 uint64_t *h_r_bar_out, int batch_count, int num_to_pack_half, int non_zeros,
                                 int poly_len, int crt_count, uint64_t mod0, uint64_t mod1, uint64_t barrett_cr0,
                                 uint64_t barrett_cr1);
void gpu_packing_batched_fused(uint64_t *d_r_all, uint64_t *d_r_bar_all, const uint64_t *d_prepacked, int num_cols);
uint64_t *gpu_packing_get_s_r_out(void);
uint64_t *gpu_packing_get_s_r_bar_out(void);
int gpu_packing_get_coeff_count(void);
int gpu_packing_get_nphalf(void);

/* src/pir/gpu/collapse.rs:10-132 (native/cuda/collapse_kernel.cu:603-975): r_all / r_bar_all
 * [num_cols][nphalf][2 * 2048], W rows [nphalf - 1][3][2 * 2048], V [3][2 * 2048]; outputs
 * bold_t / bold_t_bar [num_cols][3069][2048] condensed, bold_t_hat [num_cols][3][2048],
 * a_hat [num_cols][2048].  The _fold / _new set fills a second set of outputs, and
 * gpu_collapse_swap_bold_t exchanges the two. */
void gpu_collapse_alloc_r(int num_cols, int nphalf, int coeff_count);
uint64_t *gpu_collapse_get_r_all_col(int col, int nphalf, int coeff_count);
uint64_t *gpu_collapse_get_r_bar_all_col(int col, int nphalf, int coeff_count);
uint64_t *gpu_collapse_get_r_all(void);
uint64_t *gpu_collapse_get_r_bar_all(void);
void gpu_collapse_automorph_column(const uint64_t *d_r_flat, const uint64_t *d_r_bar_flat, int col, int nphalf,
                                   int coeff_count, int poly_len, int crt_count, const uint32_t *d_tables,
                                   const uint32_t *d_gen_pows, int num_tables);
void gpu_collapse_batched_automorphism(const uint32_t *d_tables, const uint32_t *d_gen_pows, int num_cols, int nphalf,
                                       int poly_len, int crt_count);
void gpu_collapse_setup(const uint64_t *h_w_all, const uint64_t *h_w_bar_all, const uint64_t *h_v_mask,
                        const uint64_t *h_ntt_tables, int num_cols, int nphalf, int t_exp, int coeff_count);
void gpu_collapse_run(int num_cols, int nphalf, int t_exp, int bits_per, uint32_t mod0, uint32_t mod1,
                      uint64_t barrett_cr1_0, uint64_t barrett_cr1_1, uint64_t mod0_inv_mod1, uint64_t mod1_inv_mod0,
                      uint64_t crt_modulus, uint64_t barrett_cr0_mod, uint64_t barrett_cr1_mod);
void gpu_collapse_download_a_hat(uint64_t *h_a_hat, int num_cols);
uint64_t *gpu_collapse_get_bold_t(void);
uint64_t *gpu_collapse_get_bold_t_bar(void);
uint64_t *gpu_collapse_get_bold_t_hat(void);
void gpu_collapse_setup_fold(const uint64_t *h_w_all, const uint64_t *h_w_bar_all, const uint64_t *h_v_mask,
                             const uint64_t *h_ntt_tables, int num_cols, int nphalf, int t_exp, int coeff_count);
void gpu_collapse_run_fold(int num_cols, int nphalf, int t_exp, int bits_per, uint32_t mod0, uint32_t mod1,
                           uint64_t barrett_cr1_0, uint64_t barrett_cr1_1, uint64_t mod0_inv_mod1,
                           uint64_t mod1_inv_mod0, uint64_t crt_modulus, uint64_t barrett_cr0_mod,
                           uint64_t barrett_cr1_mod);
void gpu_collapse_download_a_hat_new(uint64_t *h_a_hat, int num_cols);
uint64_t *gpu_collapse_get_bold_t_new(void);
uint64_t *gpu_collapse_get_bold_t_bar_new(void);
uint64_t *gpu_collapse_get_bold_t_hat_new(void);
void gpu_collapse_swap_bold_t(void);
void gpu_collapse_free_working(void);
void gpu_collapse_free_all(void);

#ifdef __cplusplus
}
#endif
#endif
