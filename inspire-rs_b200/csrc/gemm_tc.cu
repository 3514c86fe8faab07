// gemm_tc.cu — first-dimension GEMM on the 5th-generation tensor cores.
//
// c[q][j] = CRT( sum_k a_q,0[k] D[j][k] mod q0 , sum_k a_q,1[k] D[j][k] mod q1 )
// (native/cuda/gemv_kernel.cu:46-103 of rkdud007/inspire-rs, for many queries).
// Exact split precision: the DB is kept as two byte planes D = D_0 + 256 D_1
// ([plane][db_cols][db_rows] u8).  A query value arrives as its two residues (a_0 mod q0,
// a_1 mod q1); the parse composes them by the CRT into X < q0 q1 < 2^56, with X = a_l mod
// q_l, and stores the 7 bytes X = sum_b 256^b X_b, so the dot products are sums of u8 x u8
// products:
//   sum_k D[j][k] X[k] = sum_{p,b} 256^(p+b) P_pb[j],  P_pb[j] = sum_k D_p[j][k] X_b[k]
// and sum_k D[j][k] a_l[k] = (sum_k D[j][k] X[k]) mod q_l.  Seven bytes per query instead of
// four per residue take 2 x 7 byte products per DB entry and query, not 2 x 8.
// Each P_pb is one column of a u8 x u8 -> 32-bit tcgen05.mma (kind::i8) GEMM;
// P_pb < 255^2 * db_rows < 2^31 for db_rows <= 32768, so accumulation is exact.  The
// recombination splits at byte 4: W0 = sum_{b<4} 256^b S_b < 2^64 and
// W1 = sum_{b>=4} 256^(b-4) S_b < 2^56 with S_b = P_0b + 256 P_1b, and the sum is
// W0 + 2^32 W1, reduced mod q_l by two Montgomery steps.
//
// Query-byte layout: row 7 q + b holds byte b of query q's values.  A tile of NT rows (N of
// the MMA, a multiple of 16) carries floor(NT / 7) whole queries and starts at row
// 7 floor(NT / 7) n; its last NT mod 7 rows are the next queries' bytes, ignored.
//
// Kernel shape: persistent CTAs of 10 warps.  Warp 0 issues TMA loads into a
// multi-stage shared-memory ring (128-byte swizzle); one stage holds the same
// [128 rows x 128 bytes] K-slice of both DB planes and one [NT x 128 bytes]
// query-byte tile, so each query tile feeds two MMAs; warp 1 issues the MMAs
// (M = 128 DB columns, N = NT query-byte columns, K = 32 bytes each) into
// TMEM accumulators, one per plane, double buffered when they fit; warps 2-5
// read the accumulators, recombine, reduce mod q0 / q1 and CRT-compose.
// Sixteen epilogue warps (four per TMEM lane quarter) keep the drain short while
// both accumulators of a tile occupy all of TMEM.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "bounds.cuh"
#include "ipr_device.cuh"
#include "kernels.cuh"
#include "umma.cuh"

namespace ipr {

namespace {

constexpr int G1_THREADS = 576;  // producer, MMA, 16 epilogue warps
constexpr int G1_EPI_WARPS = 16;
constexpr int TILE_M = 128;
constexpr int TILE_K = 128;  // bytes per stage along K (one 128-byte swizzle row)
constexpr int A_STAGE_BYTES = TILE_M * TILE_K;
constexpr int MAX_STAGES = 8;

struct G1Smem {
    uint64_t full[MAX_STAGES], empty[MAX_STAGES], acc_full[2], acc_empty[2];
    uint32_t tmem_base;
    int err;
};

}  // namespace

// One octet of queries of an accumulator tile (octet 2 sg + ODD: local queries
// 16 sg + 8 ODD .. + 8, columns 112 sg + 56 ODD .. + 56, inside column groups 7 sg + 3 ODD ..
// 7 sg + 3 ODD + 3): each thread recombines its DB column's byte sums of the 8 queries and
// writes their CRT-composed residue pairs.
template <int ODD>
__device__ __forceinline__ void epilogue_octet(uint32_t acc0, uint32_t acc1, int sg, int nt, int qpt, int q0,
                                               int num_queries, uint64_t* __restrict__ c, int64_t db_cols,
                                               int64_t j) {
    uint64_t w0[8], w1[8];
#pragma unroll
    for (int i = 0; i < 8; i++) w0[i] = w1[i] = 0;
#pragma unroll
    for (int g = 3 * ODD; g < 3 * ODD + 4; g++) {
        const int col0 = sg * 112 + g * 16;
        if (col0 >= nt) break;
        uint32_t p0[16], p1[16];
        umma::tmem_ld16(acc0 + (uint32_t)col0, p0);
        umma::tmem_ld16(acc1 + (uint32_t)col0, p1);
        umma::tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 16; i++) {
            const int cl = g * 16 + i, ql = cl / 7 - 8 * ODD, b = cl % 7;
            if (ql >= 0 && ql < 8) {
                const uint64_t sb = (uint64_t)p0[i] + ((uint64_t)p1[i] << 8);
                if (b < 4) w0[ql] += sb << (8 * b);
                else w1[ql] += sb << (8 * (b - 4));
            }
        }
    }
#pragma unroll
    for (int ql = 0; ql < 8; ql++) {
        const int qloc = sg * 16 + 8 * ODD + ql, q = q0 + qloc;
        if (qloc < qpt && q < num_queries) {
            c[(int64_t)q * db_cols + j] = crt2m(mod96m(w0[ql], w1[ql], Q0), mod96m(w0[ql], w1[ql], Q1));
        }
    }
}

__global__ void __launch_bounds__(G1_THREADS, 1)
    k_gemm1(const __grid_constant__ CUtensorMap tm_db, const __grid_constant__ CUtensorMap tm_qb, int db_rows,
            int64_t db_cols, int nt, int n_tiles, int num_queries, int stages, uint64_t* __restrict__ c,
            int* __restrict__ err_flag) {
    extern __shared__ uint8_t smem_raw[];
    // 1024-byte aligned tile area (128-byte swizzle atoms)
    uint8_t* base = smem_raw + ((1024 - (umma::smem_addr(smem_raw) & 1023)) & 1023);
    G1Smem* sh = reinterpret_cast<G1Smem*>(base);
    volatile int* err = &sh->err;
    uint8_t* tiles = base + 1024;
    const int b_stage_bytes = nt * TILE_K;
    uint8_t* a_tiles = tiles;  // [stage][plane][128 x 128]
    uint8_t* b_tiles = tiles + stages * 2 * A_STAGE_BYTES;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nbuf = (4 * nt <= 512) ? 2 : 1;
    uint32_t ncols = 32;
    while (ncols < (uint32_t)(nbuf * 2 * nt)) ncols <<= 1;

    if (threadIdx.x == 0) {
        for (int s = 0; s < stages; s++) {
            umma::mbar_init(&sh->full[s], 1);
            umma::mbar_init(&sh->empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            umma::mbar_init(&sh->acc_full[b], 1);
            umma::mbar_init(&sh->acc_empty[b], G1_EPI_WARPS);
        }
        *err = 0;
        umma::fence_mbar_init();
    }
    if (warp == 1) umma::tmem_alloc(&sh->tmem_base, ncols);
    umma::fence_before();
    __syncthreads();
    umma::fence_after();
    const uint32_t tmem = sh->tmem_base;

    const int ks_total = db_rows / TILE_K;  // stages per tile (both planes in each)
    const int64_t m_tiles = db_cols / TILE_M;
    const int64_t total = m_tiles * n_tiles;

    if (warp == 0) {
        if (lane == 0) {  // TMA producer
            int stage = 0;
            uint32_t phase = 0;
            int last_phase[MAX_STAGES];
            for (int s = 0; s < MAX_STAGES; s++) last_phase[s] = -1;
            for (int64_t t = blockIdx.x; t < total && !*err; t += gridDim.x) {
                const int64_t m = t / n_tiles;
                const int n = (int)(t % n_tiles);
                for (int ks = 0; ks < ks_total; ks++) {
                    if (!umma::mbar_wait(&sh->empty[stage], phase ^ 1)) {
                        *err = 1;
                        break;
                    }
                    umma::mbar_expect_tx(&sh->full[stage], 2 * A_STAGE_BYTES + b_stage_bytes);
                    uint8_t* at = a_tiles + stage * 2 * A_STAGE_BYTES;
                    umma::tma_load_2d(at, &tm_db, ks * TILE_K, (int)(m * TILE_M), &sh->full[stage]);
                    umma::tma_load_2d(at + A_STAGE_BYTES, &tm_db, ks * TILE_K, (int)(db_cols + m * TILE_M),
                                      &sh->full[stage]);
                    umma::tma_load_2d(b_tiles + stage * b_stage_bytes, &tm_qb, ks * TILE_K, n * (nt / 7) * 7,
                                      &sh->full[stage]);
                    last_phase[stage] = (int)phase;
                    if (++stage == stages) {
                        stage = 0;
                        phase ^= 1;
                    }
                }
            }
            // every tile load issued has landed before the CTA may exit
            for (int s = 0; s < stages; s++)
                if (last_phase[s] >= 0) umma::mbar_wait(&sh->full[s], (uint32_t)last_phase[s], umma::kDrainLimitNs);
        }
    } else if (warp == 1) {
        if (lane == 0) {  // MMA issuer
            const uint32_t idesc = umma::idesc_u8(TILE_M, nt);
            int stage = 0, buf = 0, last_stage = -1;
            uint32_t phase = 0, acc_phase = 0, last_parity = 0;
            for (int64_t t = blockIdx.x; t < total && !*err; t += gridDim.x) {
                if (!umma::mbar_wait(&sh->acc_empty[buf], acc_phase ^ 1)) {
                    *err = 2;
                    break;
                }
                umma::fence_after();
                bool ok = true;
                for (int ks = 0; ks < ks_total; ks++) {
                    if (!umma::mbar_wait(&sh->full[stage], phase)) {
                        *err = 3;
                        ok = false;
                        break;
                    }
                    umma::fence_after();
                    const uint32_t d0 = tmem + (uint32_t)(buf * 2 * nt), d1 = d0 + (uint32_t)nt;
                    const uint32_t sa = umma::smem_addr(a_tiles + stage * 2 * A_STAGE_BYTES);
                    const uint32_t sb = umma::smem_addr(b_tiles + stage * b_stage_bytes);
#pragma unroll
                    for (int k4 = 0; k4 < TILE_K / 32; k4++) {
                        const uint64_t db = umma::desc_sw128(sb + 32 * k4);
                        const uint32_t acc = (ks == 0 && k4 == 0) ? 0u : 1u;
                        umma::mma_u8(d0, umma::desc_sw128(sa + 32 * k4), db, idesc, acc);
                        umma::mma_u8(d1, umma::desc_sw128(sa + A_STAGE_BYTES + 32 * k4), db, idesc, acc);
                    }
                    umma::commit(&sh->empty[stage]);  // frees the smem stage when these MMAs finish
                    last_stage = stage;
                    last_parity = phase;
                    if (++stage == stages) {
                        stage = 0;
                        phase ^= 1;
                    }
                }
                if (!ok) break;
                umma::commit(&sh->acc_full[buf]);
                if (nbuf == 2) {
                    buf ^= 1;
                    if (buf == 0) acc_phase ^= 1;
                } else {
                    acc_phase ^= 1;
                }
            }
            // the last MMAs have completed before TMEM can be released
            if (last_stage >= 0) umma::mbar_wait(&sh->empty[last_stage], last_parity, umma::kDrainLimitNs);
        }
    } else {
        // epilogue: warps 2..17 -> TMEM lane quarters 2,3,0,1 (four times); the four warps of a
        // quarter split the accumulator's query octets between them
        const int quarter = warp & 3;
        const int sub = (warp - 2) >> 2;  // 0..3: the octets sub, sub + 4, ...
        const int row = quarter * 32 + lane;
        int buf = 0;
        uint32_t acc_phase = 0;
        for (int64_t t = blockIdx.x; t < total; t += gridDim.x) {
            if (!umma::mbar_wait(&sh->acc_full[buf], acc_phase)) {
                if (lane == 0) *err = 4;
                break;
            }
            umma::fence_after();
            const int64_t m = t / n_tiles;
            const int n_tile = (int)(t % n_tiles);
            const int64_t j = m * TILE_M + row;
            const uint32_t lane_off = (uint32_t)(quarter * 32) << 16;
            // queries in octets (8 queries = 56 columns); warps with sub even take even octets,
            // the others odd ones, so the column -> (query, byte) map is known at compile time
            const int qpt = nt / 7;
            const uint32_t acc0 = tmem + lane_off + (uint32_t)(buf * 2 * nt), acc1 = acc0 + (uint32_t)nt;
            const int q0 = n_tile * qpt;
            for (int o = sub; o < (qpt + 7) / 8; o += G1_EPI_WARPS / 4) {
                if (sub & 1) epilogue_octet<1>(acc0, acc1, o >> 1, nt, qpt, q0, num_queries, c, db_cols, j);
                else epilogue_octet<0>(acc0, acc1, o >> 1, nt, qpt, q0, num_queries, c, db_cols, j);
            }
            umma::fence_before();
            __syncwarp();
            if (lane == 0) umma::mbar_arrive(&sh->acc_empty[buf]);
            if (nbuf == 2) {
                buf ^= 1;
                if (buf == 0) acc_phase ^= 1;
            } else {
                acc_phase ^= 1;
            }
        }
    }
    umma::fence_before();
    __syncthreads();
    if (warp == 1) umma::tmem_dealloc(tmem, ncols);
    if (threadIdx.x == 0 && *err) atomicExch(err_flag, *err);
}

// [plane][db_cols][db_rows] byte planes of the column-major u16 DB
__global__ void k_db_to_planes(const uint16_t* __restrict__ db, uint8_t* __restrict__ planes, int64_t n) {
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) * 8; i < n;
         i += (int64_t)gridDim.x * blockDim.x * 8) {
        const uint4 v = *reinterpret_cast<const uint4*>(db + i);  // 8 values, 2 per word
        uint2 lo, hi;
        lo.x = __byte_perm(v.x, v.y, 0x6420);
        lo.y = __byte_perm(v.z, v.w, 0x6420);
        hi.x = __byte_perm(v.x, v.y, 0x7531);
        hi.y = __byte_perm(v.z, v.w, 0x7531);
        *reinterpret_cast<uint2*>(planes + i) = lo;
        *reinterpret_cast<uint2*>(planes + n + i) = hi;
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace {
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn g_encode = nullptr;
}  // namespace

cudaError_t make_u8_tile_map(CUtensorMap* map, const void* base, uint64_t row_bytes, uint64_t rows, uint32_t box_rows) {
    if (!g_encode) {
        cudaDriverEntryPointQueryResult q;
        cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", (void**)&g_encode, cudaEnableDefault, &q);
        if (e != cudaSuccess) return e;
        if (!g_encode || q != cudaDriverEntryPointSuccess) return cudaErrorNotSupported;
    }
    if ((reinterpret_cast<uintptr_t>(base) & 15) || (row_bytes & 15) || box_rows == 0 || box_rows > 256)
        return cudaErrorInvalidValue;
    cuuint64_t dims[2] = {row_bytes, rows};
    cuuint64_t strides[1] = {row_bytes};
    cuuint32_t box[2] = {128, box_rows};
    cuuint32_t elem[2] = {1, 1};
    CUresult r = g_encode(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(base), dims, strides, box, elem,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

cudaError_t make_u16_col_map(CUtensorMap* map, const uint16_t* db, int db_rows, int64_t db_cols, uint32_t box_rows,
                             uint32_t box_cols) {
    if (!g_encode) {
        cudaDriverEntryPointQueryResult q;
        cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", (void**)&g_encode, cudaEnableDefault, &q);
        if (e != cudaSuccess) return e;
        if (!g_encode || q != cudaDriverEntryPointSuccess) return cudaErrorNotSupported;
    }
    if ((reinterpret_cast<uintptr_t>(db) & 15) || (db_rows & 7) || box_rows * 2 != 32 || box_cols == 0 ||
        box_cols > 256)
        return cudaErrorInvalidValue;
    cuuint64_t dims[2] = {(cuuint64_t)db_rows, (cuuint64_t)db_cols};
    cuuint64_t strides[1] = {(cuuint64_t)db_rows * 2};
    cuuint32_t box[2] = {box_rows, box_cols};
    cuuint32_t elem[2] = {1, 1};
    CUresult r = g_encode(map, CU_TENSOR_MAP_DATA_TYPE_UINT16, 2, const_cast<uint16_t*>(db), dims, strides, box, elem,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

int gemm1_stages(int nt) {
    const int per = 2 * A_STAGE_BYTES + nt * TILE_K;
    int s = (210 * 1024) / per;
    return s > 8 ? 8 : (s < 2 ? 2 : s);
}

size_t gemm1_smem_bytes(int nt) { return 2048 + (size_t)gemm1_stages(nt) * (2 * A_STAGE_BYTES + nt * TILE_K); }

cudaError_t init_gemm1_kernel() {
    size_t mx = 0;  // the largest footprint over every tile height the launcher can pick
    for (int nt = 16; nt <= 256; nt += 16) mx = gemm1_smem_bytes(nt) > mx ? gemm1_smem_bytes(nt) : mx;
    return cudaFuncSetAttribute(k_gemm1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mx);
}

cudaError_t launch_db_to_planes(const uint16_t* db, uint8_t* planes, int64_t n, cudaStream_t st) {
    if (n % 8) return cudaErrorInvalidValue;
    k_db_to_planes<<<148 * 8, 256, 0, st>>>(db, planes, n);
    return cudaGetLastError();
}

cudaError_t launch_gemm1(const CUtensorMap* tm_db, const CUtensorMap* tm_qb, int db_rows, int64_t db_cols, int nt,
                         int n_tiles, int num_queries, uint64_t* c, int* err_flag, int sm_count, cudaStream_t st) {
    if (nt < 16 || nt > 256 || (nt & 15) || (db_rows % TILE_K) || db_rows > 32768 || (db_cols % TILE_M))
        return cudaErrorInvalidValue;
    cudaError_t e = check_extent(c, (uint64_t)num_queries * db_cols * 8, "first dimension: outputs");
    if (e != cudaSuccess) return e;
    const int stages = gemm1_stages(nt);
    const int64_t total = (db_cols / TILE_M) * n_tiles;
    const int grid = (int)(total < sm_count ? total : sm_count);
    k_gemm1<<<grid, G1_THREADS, gemm1_smem_bytes(nt), st>>>(*tm_db, *tm_qb, db_rows, db_cols, nt, n_tiles,
                                                            num_queries, stages, c, err_flag);
    return cudaGetLastError();
}

}  // namespace ipr
