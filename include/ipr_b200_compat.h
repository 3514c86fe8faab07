/*
 * ipr_b200_compat.h — the respond-path symbols the reference's Rust crate
 * already declares, exported with identical names, argument meaning and
 * (void) error behaviour, implemented on this library's sm_100a kernels.
 * Linking these in place of native/cuda/{gemv,rotation,packing_online}_kernel.cu
 * lets the unmodified Rust glue drive the new kernels.  Errors are printed to
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

#ifdef __cplusplus
}
#endif
#endif
