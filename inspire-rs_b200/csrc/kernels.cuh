// kernels.cuh — host-side launch wrappers for the respond() kernels (kernels.cu)
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace ipr {

cudaError_t set_constants(const uint64_t br[2], uint32_t q0inv);
cudaError_t init_device_kernels();

// qbytes (optional): tensor-core GEMM operand [(query*2 + limb)*4 + byte][db_rows] u8,
// this payload's queries starting at global query index qbase
cudaError_t launch_parse_query(const uint8_t* qb, int nq, int db_rows, uint64_t* y, uint64_t* z,
                               uint32_t* a_il, uint32_t* gsw, uint8_t* qbytes, int qbase, cudaStream_t st);
// nq must be 1 or 2; a_il points at the pair group, c at [nq][db_cols]; form of the two-query
// kernel: 0 / 1 / 2 = 8 / 4 / 2 DB columns per warp loaded into registers, 3 = 8 columns per
// warp staged through shared memory by cp.async, 4 / 5 = forms 0 / 3 with FP64-pipe products,
// 6 = a lane per column with TMA-fed stages and FP64-pipe products (needs err_flag and
// db_rows a multiple of 256, at most 2^18; otherwise form 5 runs, or form 0 above 16,384
// rows).  One query always takes 16 columns per warp.
cudaError_t launch_gemv(const uint16_t* db, int db_rows, int64_t db_cols, int nq, const uint32_t* a_il,
                        uint64_t* c, int sm_count, cudaStream_t st, int form = 0, int* err_flag = nullptr);
// 2D tensor map over the column-major u16 DB ([db_cols][db_rows]), boxes of box_rows x box_cols
// with the 32-byte swizzle (box_rows = 16)
cudaError_t make_u16_col_map(CUtensorMap* map, const uint16_t* db, int db_rows, int64_t db_cols, uint32_t box_rows,
                             uint32_t box_cols);
cudaError_t launch_pack(const uint64_t* bt, const uint64_t* btb, const uint64_t* bth, const uint64_t* y,
                        const uint64_t* z, uint32_t* S, int num_outputs, cudaStream_t st);
// R = from_ntt(S) per (client, output) polynomial pair; with z_bodies non-null the
// z_body x That term of client f / instances is added to S first
cudaError_t launch_intt_crt(const uint32_t* S, const uint32_t* iw, const uint32_t* iwp, uint64_t* R,
                            int num_outputs, cudaStream_t st, const uint64_t* z_bodies = nullptr,
                            const uint64_t* bth = nullptr, int instances = 1);
cudaError_t launch_fold_switch(const uint32_t* row0, const uint32_t* gsw, const uint64_t* a_hat,
                               const uint64_t* R, const uint64_t* cvec, const uint32_t* fw,
                               const uint32_t* fwp, const uint32_t* iw, const uint32_t* iwp, int interp,
                               int c_groups, int nq, int64_t db_cols, uint8_t* resp,
                               int64_t resp_query_stride, cudaStream_t st);
cudaError_t launch_response_frame(uint8_t* resp, int nq, int64_t per_query, const uint8_t* stash,
                                  int64_t stash_count, int64_t stash_entry, cudaStream_t st, int npay = 1,
                                  int64_t pstride = 0);
// npay payloads of nq queries each, pstride bytes apart, into per-payload key / body slots
cudaError_t launch_parse_batch(const uint8_t* qb, int npay, int64_t pstride, int nq, int db_rows, uint64_t* y,
                               uint64_t* z, uint32_t* gsw, uint8_t* qbytes, cudaStream_t st);
// batched packing on tcgen05 (pack_tc.cu)
int pack_mma_nt(int clients);
uint64_t tpp_bytes(int instances);
cudaError_t init_pack_mma_kernel();
cudaError_t launch_relayout_tpp(const uint64_t* bt, const uint64_t* btb, uint8_t* tpp, int instances,
                                cudaStream_t st);
cudaError_t launch_build_y8(const uint64_t* y_bodies, uint8_t* y8, int clients, int np, cudaStream_t st);
// S[c][j][l][z] without the z_body x That term (added by launch_intt_crt when given z_bodies)
// the CTA-pair form: tm_y_half has boxes of pack_mma_nt(clients)/2 rows
cudaError_t init_pack_pair_kernel();
cudaError_t launch_pack_mma_pair(const CUtensorMap* tm_t, const CUtensorMap* tm_y_half, int instances, int clients,
                                 int np, uint32_t* S, int* err_flag, int sm_count, cudaStream_t st);
cudaError_t launch_pack_mma(const CUtensorMap* tm_t, const CUtensorMap* tm_y, int instances, int clients, int np,
                            uint32_t* S, int* err_flag, int sm_count, cudaStream_t st);
cudaError_t launch_rotations(const uint64_t* y_body, uint64_t* y_all, uint64_t* y_bar_all, int num_rotations,
                             cudaStream_t st);
cudaError_t launch_pack_materialized(const uint64_t* bt, const uint64_t* btb, const uint64_t* bth,
                                     const uint64_t* y_all, const uint64_t* y_bar_all, const uint64_t* z,
                                     int num_outputs, int n_rot, uint64_t* out, cudaStream_t st);
cudaError_t launch_ntt_batch(uint64_t* data, int npairs, int forward, const uint32_t* w, const uint32_t* wp,
                             cudaStream_t st);
// seeded synthetic arrays; element i is element idx0 + i of the whole array
cudaError_t launch_synth_db(uint16_t* db, int64_t n, uint64_t seed, cudaStream_t st, uint64_t idx0 = 0);
cudaError_t launch_synth_condensed(uint64_t* out, int64_t n, uint64_t seed, uint64_t stream, cudaStream_t st,
                                   uint64_t idx0 = 0);
cudaError_t launch_synth_modq(uint64_t* out, int64_t n, uint64_t seed, uint64_t stream, cudaStream_t st,
                              uint64_t idx0 = 0);

// tensor-core first-dimension GEMM (gemm_tc.cu)
cudaError_t make_u8_tile_map(CUtensorMap* map, const void* base, uint64_t row_bytes, uint64_t rows, uint32_t box_rows);
cudaError_t init_gemm1_kernel();
cudaError_t launch_db_to_planes(const uint16_t* db, uint8_t* planes, int64_t n, cudaStream_t st);
// nt: query-byte columns per tile (16..256, multiple of 16); db_rows <= 32768
cudaError_t launch_gemm1(const CUtensorMap* tm_db, const CUtensorMap* tm_qb, int db_rows, int64_t db_cols, int nt,
                         int n_tiles, int num_queries, uint64_t* c, int* err_flag, int sm_count, cudaStream_t st);

// register-resident-NTT fold + switch (fold.cu); queries grouped qpp per payload
cudaError_t init_fold2_kernel();
cudaError_t launch_fold2(const uint32_t* row0, const uint32_t* gsw, const uint64_t* a_hat, const uint64_t* R,
                         int64_t r_payload_stride, const uint64_t* cvec, const uint32_t* fw, const uint32_t* fwp,
                         const uint32_t* iw, const uint32_t* iwp, int interp, int c_groups, int num_queries,
                         int64_t db_cols, int qpp, uint8_t* resp, int64_t resp_payload_stride,
                         int64_t resp_query_stride, cudaStream_t st);

// fold with the packing post-process fused in (fold3.cu).  ninv = {N^-1 mod q0, its Shoup
// companion, N^-1 mod q1, companion}.  launch_fold_prep turns the packing outputs S
// ([count][2][N] u32) in place into (S + z_body x That) * N^-1 (zb null: the scaling alone;
// zb / bth indexed by f / instances and f % instances); launch_fold3 then folds with the forward
// twiddles fwi and the plain inverse twiddles iwi, both [limb][N] pairs (w, Shoup companion),
// and row0s = row 0 x N^-1, S of payload p at S + p * s_payload_stride.  With gsw non-null,
// launch_fold_prep also scales the RGSW bodies of gsw_queries parsed queries in place by
// ninv_bodies (N^-1 x 2^32 with its Shoup companion, per limb; the one-chain fold's
// Montgomery form), as launch_fold4 expects them, and launch_fold4 takes row 0 x N^-1 x 2^32.
cudaError_t init_fold3_kernel();
cudaError_t launch_fold_prep(uint32_t* S, int64_t count, const uint64_t* zb, const uint64_t* bth, int instances,
                             const uint32_t ninv[4], int sm_count, cudaStream_t st, uint32_t* gsw = nullptr,
                             int gsw_queries = 0, const uint32_t* ninv_bodies = nullptr);
cudaError_t launch_fold3(const uint32_t* row0s, const uint32_t* gsw, const uint64_t* a_hat, const uint32_t* S,
                         int64_t s_payload_stride, const uint64_t* cvec, const uint32_t* fwi, const uint32_t* iwi,
                         const uint32_t ninv[4], int interp, int c_groups,
                         int num_queries, int64_t db_cols, int qpp, uint8_t* resp, int64_t resp_payload_stride,
                         int64_t resp_query_stride, cudaStream_t st);
// The extents (in elements of each buffer's type, from its base pointer) of the buffers the
// one-chain fold reads and writes: checked against the allocations before the launch and
// against every index inside the kernel in the bounds-checked debug build (bounds.cuh).
struct FoldExtents {
    int64_t s_words;     // u32 packing outputs
    int64_t gsw_words;   // u32 RGSW bodies, scaled by N^-1
    int64_t ahat_words;  // u64 a_hat rows
    int64_t c_words;     // u64 first-dimension outputs
    int64_t resp_bytes;  // response bytes
};
cudaError_t launch_fold4(const uint32_t* row0s, const uint32_t* gsw_scaled, const uint64_t* a_hat, const uint32_t* S,
                         int64_t s_payload_stride, const uint64_t* cvec, const uint32_t* fwi, const uint32_t* iwi,
                         int interp, int c_groups, int num_queries, int64_t db_cols, int qpp, uint8_t* resp,
                         int64_t resp_payload_stride, int64_t resp_query_stride, const FoldExtents& ext,
                         cudaStream_t st, bool staged = true);

}  // namespace ipr
