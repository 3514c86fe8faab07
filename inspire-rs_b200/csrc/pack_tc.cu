// pack_tc.cu — the InspiRING packing inner product for a batch of clients on
// the 5th-generation tensor cores.
//
// For output j, NTT slot z, limb l (packing_online_kernel.cu:18-92 /
// full_packing_with_preprocessing_online, src/pir/packing.rs:2941-3012):
//   S[c][j][l][z] = sum_{i<1023,k<3} y_c[k][rot_i(z)] T[j][i,k][z] + y_c[k][rotbar_i(z)] Tbar[j][i,k][z]
//                 + sum_k z_c[k][z] That[j][k][z]                          (mod q_l)
// The rotated slots rot_i(z) = auto_src(5^i, z) and rotbar_i(z) = auto_src(2N - 5^i, z)
// are distinct for every (i, kind) at a fixed z (5 generates a subgroup of the
// odd residues mod 2N that excludes -1), so re-indexing the precomputation by
// the slot it multiplies turns the client side into a z-independent matrix:
//   S[c][j][l][z] = sum_{k, s} Y_l[c][k*N + s] * Tpp_{z,l}[j][k*N + s]   (+ the z_body term,
//                   which k_intt_crt adds before its inverse NTT)
//   Y_l[c][k*N + s]      = y_c[k][s] (limb l)
//   Tpp_{z,l}[j][k*N+s]  = T[j][i,k][z] if s = rot_i(z), Tbar[j][i,k][z] if s = rotbar_i(z), else 0
// Tpp is built once at setup.  Both operands are split into bytes (28-bit
// residues = 4 bytes) so every term is a u8 x u8 product:
//   S = sum_{a,b} 256^(a+b) P_ab,  P_ab = sum_K Y_l,a[c][K] * Tpp_{z,l},b[j][K]
// with P_ab < 255^2 * 6144 < 2^29 exact in a 32-bit accumulator.
//
// GEMM per (z, l, tile of 32 outputs): M = 128 rows = 4 bytes b x 32 outputs,
// N = 4 bytes a x clients (<= 256), K = 6144.  Persistent CTAs of 10 warps:
// TMA producer, MMA issuer, 2 x 4 epilogue warps; each unit is two slots that
// share the client operand.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "bounds.cuh"
#include "ipr_device.cuh"
#include "kernels.cuh"
#include "umma.cuh"

namespace ipr {

namespace {

constexpr int P_THREADS = 320;
constexpr int Q_THREADS = 192;  // CTA-pair form: producer, MMA, 4 epilogue warps
constexpr int P_TILE_M = 128;
constexpr int P_TILE_K = 128;
constexpr int P_K = 3 * N;  // 6144
constexpr int P_A_STAGE = P_TILE_M * P_TILE_K;
constexpr int P_MAX_STAGES = 8;

struct PSmem {
    uint64_t full[P_MAX_STAGES], empty[P_MAX_STAGES], acc_full[2], acc_empty[2];
    uint32_t tmem_base;
    int err;
    int ep_fail[2];  // written only by epilogue group t's warps, read after their named barrier
};

__device__ __forceinline__ uint32_t pow5(uint32_t i) {  // 5^i mod 2N
    uint32_t r = 1, b = 5;
    while (i) {
        if (i & 1) r = (r * b) & (2 * N - 1);
        b = (b * b) & (2 * N - 1);
        i >>= 1;
    }
    return r;
}

}  // namespace

// discrete logarithm base 5 of the odd residues mod 2N: entry (t - 1) / 2 = i for t = 5^i,
// i | 0x400 for t = 2N - 5^i (i < N / 2; the two cosets cover every odd t)
__device__ uint16_t g_dlog5[N];

__global__ void k_init_dlog5() {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N / 2) return;
    const uint32_t g = pow5((uint32_t)i);
    g_dlog5[(g - 1) / 2] = (uint16_t)i;
    g_dlog5[(2 * N - g - 1) / 2] = (uint16_t)(i | 0x400);
}

// Tpp rows ((z*2 + l)*mt_count + mt)*128 + b*32 + jl, columns k*N + s.  Entry (row, k*N + s)
// is byte b of limb l of (kind ? bold_t_bar : bold_t)[j = mt*32 + jl][i*3 + k][z] where
// x -> x^t with t = 5^i (kind 0) or 2N - 5^i (kind 1) carries slot z to slot s, i.e.
// t = exponent(s) / exponent(z) mod 2N; i = 1023 (no such row) and j >= instances give 0.
// One CTA assembles a 256-row x 256-column byte tile (rows (l, b, jl), slots s0 .. s0 + 255)
// of one (z, mt, k) in shared memory and writes it as contiguous row segments; its reads
// are single 8-byte words of the precomputation.  grid (N / 256, N, mt_count * 3)
__global__ void __launch_bounds__(256)
    k_relayout_tpp(const uint64_t* __restrict__ bt, const uint64_t* __restrict__ btb, uint8_t* __restrict__ tpp,
                   int instances, int mt_count) {
    extern __shared__ __align__(16) uint8_t rtile[];  // [256 rows][256 bytes]
    const int s0 = blockIdx.x * 256, z = blockIdx.y, mt = blockIdx.z / T_EXP, k = blockIdx.z % T_EXP;
    const int t = threadIdx.x, s = s0 + t;
    // exponent(z)^-1 mod 2N by Newton's iteration (x * x = 1 mod 8 for odd x)
    const uint32_t ez = exponent_of_slot((uint32_t)z);
    uint32_t iz = ez;
#pragma unroll
    for (int it = 0; it < 3; it++) iz = (iz * (2u - ez * iz)) & (2 * N - 1);
    const uint32_t tt = (exponent_of_slot((uint32_t)s) * iz) & (2 * N - 1);
    const uint32_t dl = g_dlog5[(tt - 1) / 2];
    const int i = (int)(dl & 0x3FF);
    const uint64_t* src = (dl & 0x400) ? btb : bt;
    const bool row_ok = i < NROT;
#pragma unroll 8
    for (int jl = 0; jl < 32; jl++) {
        const int j = mt * 32 + jl;
        const uint64_t v = (row_ok && j < instances) ? __ldg(src + ((int64_t)j * NINNER + i * T_EXP + k) * N + z) : 0;
#pragma unroll
        for (int l = 0; l < 2; l++) {
            const uint32_t limb = (uint32_t)(l ? (v >> 32) : v);
#pragma unroll
            for (int b = 0; b < 4; b++) rtile[(l * P_TILE_M + b * 32 + jl) * 256 + t] = (uint8_t)(limb >> (8 * b));
        }
    }
    __syncthreads();
    for (int c = t; c < 256 * 16; c += 256) {
        const int r = c >> 4, seg = c & 15;
        const int l = r / P_TILE_M, rb = r % P_TILE_M;  // rb = b*32 + jl
        const int64_t row = (((int64_t)z * 2 + l) * mt_count + mt) * P_TILE_M + rb;
        *reinterpret_cast<uint4*>(tpp + row * P_K + k * N + s0 + seg * 16) =
            *reinterpret_cast<const uint4*>(rtile + r * 256 + seg * 16);
    }
}

// Y8[l][c*4 + a][k*N + s] = byte a of y_c[k][s] (limb l); rows c >= clients stay as zeroed
__global__ void k_build_y8(const uint64_t* __restrict__ y_bodies, uint8_t* __restrict__ y8, int clients, int np) {
    const int64_t total = (int64_t)clients * T_EXP * N;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int c = (int)(idx / (T_EXP * N));
        const int ks = (int)(idx % (T_EXP * N));  // k*N + s
        const uint64_t v = y_bodies[idx];
#pragma unroll
        for (int l = 0; l < 2; l++) {
            const uint32_t limb = (uint32_t)(l ? (v >> 32) : v);
#pragma unroll
            for (int a = 0; a < 4; a++) y8[((int64_t)l * np + c * 4 + a) * P_K + ks] = (uint8_t)(limb >> (8 * a));
        }
    }
}

// Each unit is a pair of slots (z0 = 2 zp, z1 = z0 + 1) of one (limb, output tile):
// both M tiles multiply the same Y_l K-slice, so every B stage feeds two MMAs
// and the client operand crosses L2 once per slot pair instead of once per slot.
// Accumulators: tile t at TMEM columns [buf * 2 nt + t nt, + nt).
// Warps: 0 TMA producer, 1 MMA issuer, 2..5 epilogue of tile 0, 6..9 epilogue of tile 1.
__global__ void __launch_bounds__(P_THREADS, 1)
    k_pack_mma(const __grid_constant__ CUtensorMap tm_t, const __grid_constant__ CUtensorMap tm_y, int instances,
               int mt_count, int clients, int np, int nt, int stages, uint32_t* __restrict__ S,
               int* __restrict__ err_flag) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* base = smem_raw + ((1024 - (umma::smem_addr(smem_raw) & 1023)) & 1023);
    PSmem* sh = reinterpret_cast<PSmem*>(base);
    volatile int* err = &sh->err;
    uint8_t* a_tiles = base + 1024;  // [stage][tile][128 x 128]
    const int b_stage = nt * P_TILE_K;
    uint8_t* b_tiles = a_tiles + stages * 2 * P_A_STAGE;
    uint32_t* xch_all = reinterpret_cast<uint32_t*>(b_tiles + stages * b_stage);  // [tile][16 clients][4][32]

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
            umma::mbar_init(&sh->acc_empty[b], 8);
        }
        *err = 0;
        sh->ep_fail[0] = sh->ep_fail[1] = 0;
        umma::fence_mbar_init();
    }
    if (warp == 1) umma::tmem_alloc(&sh->tmem_base, ncols);
    umma::fence_before();
    __syncthreads();
    umma::fence_after();
    const uint32_t tmem = sh->tmem_base;

    const int ks_total = P_K / P_TILE_K;              // 48
    const int64_t total = (int64_t)2 * mt_count * (N / 2);  // units (l, mt, zp), zp fastest

    if (warp == 0) {
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            int last_phase[P_MAX_STAGES];
            for (int s = 0; s < P_MAX_STAGES; s++) last_phase[s] = -1;
            for (int64_t u = blockIdx.x; u < total && !*err; u += gridDim.x) {
                const int z0 = (int)(u & (N / 2 - 1)) * 2;
                const int lm = (int)(u >> (LOGN - 1));
                const int l = lm / mt_count, mt = lm % mt_count;
                const int arow0 = (int)(((int64_t)(z0 * 2 + l) * mt_count + mt) * P_TILE_M);
                const int arow1 = arow0 + 2 * mt_count * P_TILE_M;  // slot z0 + 1
                for (int ks = 0; ks < ks_total; ks++) {
                    if (!umma::mbar_wait(&sh->empty[stage], phase ^ 1)) {
                        *err = 11;
                        break;
                    }
                    uint8_t* at = a_tiles + stage * 2 * P_A_STAGE;
                    umma::mbar_expect_tx(&sh->full[stage], 2 * P_A_STAGE + b_stage);
                    umma::tma_load_2d(at, &tm_t, ks * P_TILE_K, arow0, &sh->full[stage]);
                    umma::tma_load_2d(at + P_A_STAGE, &tm_t, ks * P_TILE_K, arow1, &sh->full[stage]);
                    umma::tma_load_2d(b_tiles + stage * b_stage, &tm_y, ks * P_TILE_K, l * np, &sh->full[stage]);
                    last_phase[stage] = (int)phase;
                    if (++stage == stages) {
                        stage = 0;
                        phase ^= 1;
                    }
                }
            }
            for (int s = 0; s < stages; s++)
                if (last_phase[s] >= 0) umma::mbar_wait(&sh->full[s], (uint32_t)last_phase[s], umma::kDrainLimitNs);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = umma::idesc_u8(P_TILE_M, nt);
            int stage = 0, buf = 0, last_stage = -1;
            uint32_t phase = 0, acc_phase = 0, last_parity = 0;
            for (int64_t u = blockIdx.x; u < total && !*err; u += gridDim.x) {
                if (!umma::mbar_wait(&sh->acc_empty[buf], acc_phase ^ 1)) {
                    *err = 12;
                    break;
                }
                umma::fence_after();
                bool ok = true;
                const uint32_t d0 = tmem + (uint32_t)(buf * 2 * nt), d1 = d0 + (uint32_t)nt;
                for (int ks = 0; ks < ks_total; ks++) {
                    if (!umma::mbar_wait(&sh->full[stage], phase)) {
                        *err = 13;
                        ok = false;
                        break;
                    }
                    umma::fence_after();
                    const uint32_t sa = umma::smem_addr(a_tiles + stage * 2 * P_A_STAGE);
                    const uint32_t sb = umma::smem_addr(b_tiles + stage * b_stage);
#pragma unroll
                    for (int k4 = 0; k4 < P_TILE_K / 32; k4++) {
                        const uint64_t db = umma::desc_sw128(sb + 32 * k4);
                        const uint32_t acc = (ks == 0 && k4 == 0) ? 0u : 1u;
                        umma::mma_u8(d0, umma::desc_sw128(sa + 32 * k4), db, idesc, acc);
                        umma::mma_u8(d1, umma::desc_sw128(sa + P_A_STAGE + 32 * k4), db, idesc, acc);
                    }
                    umma::commit(&sh->empty[stage]);
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
            if (last_stage >= 0) umma::mbar_wait(&sh->empty[last_stage], last_parity, umma::kDrainLimitNs);
        }
    } else {
        // epilogue group t (warps 2+4t .. 5+4t) drains tile t (slot z0 + t).  Warp w reads TMEM
        // lanes 32 (w % 4) .. +31 = byte b = w % 4 of outputs mt*32 + lane.
        const int t = (warp - 2) >> 2;
        const int b = warp & 3;
        const int gbar = 1 + t;
        uint32_t* xch = xch_all + t * (16 * 4 * 32);
        volatile int* ep_fail = &sh->ep_fail[t];
        int buf = 0;
        uint32_t acc_phase = 0;
        const int chunks = (clients + 15) / 16;
        for (int64_t u = blockIdx.x; u < total; u += gridDim.x) {
            // the group's four warps leave together: the decision uses a flag only they write
            if (!umma::mbar_wait(&sh->acc_full[buf], acc_phase) && lane == 0) *ep_fail = 1;
            umma::named_bar(gbar, 128);
            if (*ep_fail) {
                if (b == 0 && lane == 0) *err = 14;
                break;
            }
            umma::fence_after();
            const int z = (int)(u & (N / 2 - 1)) * 2 + t;
            const int lm = (int)(u >> (LOGN - 1));
            const int l = lm / mt_count, mt = lm % mt_count;
            const uint32_t q = l ? Q1 : Q0;
            const uint32_t lane_off = (uint32_t)(b * 32) << 16;
            const uint32_t col0 = (uint32_t)(buf * 2 * nt + t * nt);
            const int j = mt * 32 + lane;
            for (int ch = 0; ch < chunks; ch++) {
                for (int g = ch * 4; g < ch * 4 + 4 && g < nt / 16; g++) {
                    uint32_t d[16];
                    umma::tmem_ld16(tmem + lane_off + col0 + (uint32_t)(g * 16), d);
                    umma::tmem_wait_ld();
#pragma unroll
                    for (int ci = 0; ci < 4; ci++) {
                        uint64_t v = 0;
#pragma unroll
                        for (int a = 0; a < 4; a++) v += (uint64_t)d[ci * 4 + a] << (8 * a);
                        const uint32_t r = mod64m(v, q);
                        xch[(((g - ch * 4) * 4 + ci) * 4 + b) * 32 + lane] = r;  // r < q: shifted by byte b below
                    }
                }
                if (ch == chunks - 1) {  // every TMEM read of this unit is done: free the buffer
                    umma::fence_before();
                    __syncwarp();
                    if (lane == 0) umma::mbar_arrive(&sh->acc_empty[buf]);
                }
                umma::named_bar(gbar, 128);
                // combine the 4 byte rows; thread (b, lane) owns clients c = b mod 4 of the chunk.
                // The z_body x That term is added by the inverse-NTT kernel that consumes S.
                if (j < instances) {
                    for (int cl = b; cl < 16; cl += 4) {
                        const int c = ch * 16 + cl;
                        if (c >= clients) break;
                        // sum_b 256^b r_b < 2^28 * (1 + 2^8 + 2^16 + 2^24) < 2^53: one reduction
                        const uint64_t tot = (uint64_t)xch[(cl * 4 + 0) * 32 + lane] +
                                             ((uint64_t)xch[(cl * 4 + 1) * 32 + lane] << 8) +
                                             ((uint64_t)xch[(cl * 4 + 2) * 32 + lane] << 16) +
                                             ((uint64_t)xch[(cl * 4 + 3) * 32 + lane] << 24);
                        S[(((int64_t)c * instances + j) * 2 + l) * N + z] = mod64m(tot, q);
                    }
                }
                umma::named_bar(gbar, 128);
            }
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

// ---------------------------------------------------------------------------
// CTA-pair form: a cluster of 2 CTAs issues M = 256 MMAs (tcgen05 cta_group::2).
// CTA r of the pair holds slot z0 + r of the unit (its 128 precomputation rows)
// and client rows r*nt/2 .. of Y, so each SM stages 16 KB + nt*64 bytes per
// k-step (half of the single-CTA form), and each CTA's TMEM holds only its own
// nt-column accumulator: double buffered, so the epilogue of one unit overlaps
// the MMAs of the next.
// Warps: 0 TMA producer (both CTAs), 1 MMA issuer (CTA 0), 2..5 epilogue (both).
// Barriers: full[] used in CTA 0 (both CTAs' loads complete on it), empty[] and
// acc_full[] in both (CTA 0's MMA commits to each), acc_empty[] in CTA 0
// (8 arrivals: the epilogue warps of both CTAs).
// ---------------------------------------------------------------------------
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(Q_THREADS, 1)
    k_pack_mma_pair(const __grid_constant__ CUtensorMap tm_t, const __grid_constant__ CUtensorMap tm_y, int instances,
                    int mt_count, int clients, int np, int nt, int stages, uint32_t* __restrict__ S,
                    int* __restrict__ err_flag) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* base = smem_raw + ((1024 - (umma::smem_addr(smem_raw) & 1023)) & 1023);
    PSmem* sh = reinterpret_cast<PSmem*>(base);
    volatile int* err = &sh->err;
    const int half = nt / 2;
    const int b_stage = half * P_TILE_K;
    uint8_t* a_tiles = base + 1024;                                           // [stage][128 x 128]
    uint8_t* b_tiles = a_tiles + stages * P_A_STAGE;                          // [stage][nt/2 x 128]
    uint32_t* xch = reinterpret_cast<uint32_t*>(b_tiles + stages * b_stage);  // [16 clients][4][32]

    const uint32_t rank = umma::cluster_rank();
    const bool leader = rank == 0;
    const int pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t ncols = 32;
    while (ncols < (uint32_t)(2 * nt)) ncols <<= 1;

    if (threadIdx.x == 0) {
        for (int s = 0; s < stages; s++) {
            umma::mbar_init(&sh->full[s], 1);
            umma::mbar_init(&sh->empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            umma::mbar_init(&sh->acc_full[b], 1);
            umma::mbar_init(&sh->acc_empty[b], 8);
        }
        *err = 0;
        sh->ep_fail[0] = sh->ep_fail[1] = 0;
        umma::fence_mbar_init();
    }
    if (warp == 1) umma::tmem_alloc_pair(&sh->tmem_base, ncols);
    umma::fence_before();
    umma::cluster_sync();  // barriers of both CTAs initialised before any cross-CTA arrive
    umma::fence_after();
    const uint32_t tmem = sh->tmem_base;

    const int ks_total = P_K / P_TILE_K;                    // 48
    const int64_t total = (int64_t)2 * mt_count * (N / 2);  // units (l, mt, zp), zp fastest

    if (warp == 0) {
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            int last_phase[P_MAX_STAGES];
            for (int s = 0; s < P_MAX_STAGES; s++) last_phase[s] = -1;
            const uint32_t tx = 2u * (uint32_t)(P_A_STAGE + b_stage);  // both CTAs' bytes land on CTA 0's barrier
            for (int64_t u = pair; u < total && !*err; u += npairs) {
                const int z = (int)(u & (N / 2 - 1)) * 2 + (int)rank;
                const int lm = (int)(u >> (LOGN - 1));
                const int l = lm / mt_count, mt = lm % mt_count;
                const int arow = (int)(((int64_t)(z * 2 + l) * mt_count + mt) * P_TILE_M);
                const int brow = l * np + (int)rank * half;
                for (int ks = 0; ks < ks_total; ks++) {
                    if (!umma::mbar_wait(&sh->empty[stage], phase ^ 1)) {
                        *err = 21;
                        break;
                    }
                    if (leader) umma::mbar_expect_tx(&sh->full[stage], tx);
                    const uint32_t fb = umma::map_to_rank(&sh->full[stage], 0);
                    umma::tma_load_2d_pair(a_tiles + stage * P_A_STAGE, &tm_t, ks * P_TILE_K, arow, fb);
                    umma::tma_load_2d_pair(b_tiles + stage * b_stage, &tm_y, ks * P_TILE_K, brow, fb);
                    last_phase[stage] = (int)phase;
                    if (++stage == stages) {
                        stage = 0;
                        phase ^= 1;
                    }
                }
            }
            if (leader)  // every load of either CTA has landed before the pair may exit
                for (int s = 0; s < stages; s++)
                    if (last_phase[s] >= 0) umma::mbar_wait(&sh->full[s], (uint32_t)last_phase[s], umma::kDrainLimitNs);
        }
    } else if (warp == 1) {
        if (leader && lane == 0) {
            const uint32_t idesc = umma::idesc_u8(2 * P_TILE_M, nt);
            int stage = 0, buf = 0, last_stage = -1;
            uint32_t phase = 0, acc_phase = 0, last_parity = 0;
            for (int64_t u = pair; u < total && !*err; u += npairs) {
                if (!umma::mbar_wait(&sh->acc_empty[buf], acc_phase ^ 1)) {
                    *err = 22;
                    break;
                }
                umma::fence_after();
                bool ok = true;
                const uint32_t d = tmem + (uint32_t)(buf * nt);
                for (int ks = 0; ks < ks_total; ks++) {
                    if (!umma::mbar_wait(&sh->full[stage], phase)) {
                        *err = 23;
                        ok = false;
                        break;
                    }
                    umma::fence_after();
                    const uint32_t sa = umma::smem_addr(a_tiles + stage * P_A_STAGE);
                    const uint32_t sb = umma::smem_addr(b_tiles + stage * b_stage);
#pragma unroll
                    for (int k4 = 0; k4 < P_TILE_K / 32; k4++)
                        umma::mma_u8_pair(d, umma::desc_sw128(sa + 32 * k4), umma::desc_sw128(sb + 32 * k4), idesc,
                                          (ks == 0 && k4 == 0) ? 0u : 1u);
                    umma::commit_pair(umma::map_to_rank(&sh->empty[stage], 0));
                    umma::commit_pair(umma::map_to_rank(&sh->empty[stage], 1));
                    last_stage = stage;
                    last_parity = phase;
                    if (++stage == stages) {
                        stage = 0;
                        phase ^= 1;
                    }
                }
                if (!ok) break;
                umma::commit_pair(umma::map_to_rank(&sh->acc_full[buf], 0));
                umma::commit_pair(umma::map_to_rank(&sh->acc_full[buf], 1));
                buf ^= 1;
                if (buf == 0) acc_phase ^= 1;
            }
            if (last_stage >= 0) umma::mbar_wait(&sh->empty[last_stage], last_parity, umma::kDrainLimitNs);
        }
    } else {
        // epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31 = byte b of outputs mt*32 + lane, slot z0 + rank
        const int b = warp & 3;
        volatile int* ep_fail = &sh->ep_fail[0];
        const uint32_t acc_empty0 = umma::map_to_rank(&sh->acc_empty[0], 0);
        const uint32_t acc_empty1 = umma::map_to_rank(&sh->acc_empty[1], 0);
        int buf = 0;
        uint32_t acc_phase = 0;
        const int chunks = (clients + 15) / 16;
        for (int64_t u = pair; u < total; u += npairs) {
            // the four warps leave together: the decision uses a flag only they write
            if (!umma::mbar_wait(&sh->acc_full[buf], acc_phase) && lane == 0) *ep_fail = 1;
            umma::named_bar(1, 128);
            if (*ep_fail) {
                if (b == 0 && lane == 0) *err = 24;
                break;
            }
            umma::fence_after();
            const int z = (int)(u & (N / 2 - 1)) * 2 + (int)rank;
            const int lm = (int)(u >> (LOGN - 1));
            const int l = lm / mt_count, mt = lm % mt_count;
            const uint32_t q = l ? Q1 : Q0;
            const uint32_t lane_off = (uint32_t)(b * 32) << 16;
            const uint32_t col0 = (uint32_t)(buf * nt);
            const int j = mt * 32 + lane;
            for (int ch = 0; ch < chunks; ch++) {
                for (int g = ch * 4; g < ch * 4 + 4 && g < nt / 16; g++) {
                    uint32_t d[16];
                    umma::tmem_ld16(tmem + lane_off + col0 + (uint32_t)(g * 16), d);
                    umma::tmem_wait_ld();
#pragma unroll
                    for (int ci = 0; ci < 4; ci++) {
                        uint64_t v = 0;
#pragma unroll
                        for (int a = 0; a < 4; a++) v += (uint64_t)d[ci * 4 + a] << (8 * a);
                        xch[(((g - ch * 4) * 4 + ci) * 4 + b) * 32 + lane] = mod64m(v, q);
                    }
                }
                if (ch == chunks - 1) {  // every TMEM read of this unit is done: free the buffer
                    umma::fence_before();
                    __syncwarp();
                    if (lane == 0) umma::mbar_arrive_remote(buf ? acc_empty1 : acc_empty0);
                }
                umma::named_bar(1, 128);
                if (j < instances) {
                    for (int cl = b; cl < 16; cl += 4) {
                        const int c = ch * 16 + cl;
                        if (c >= clients) break;
                        // sum_b 256^b r_b < 2^28 * (1 + 2^8 + 2^16 + 2^24) < 2^53: one reduction
                        const uint64_t tot = (uint64_t)xch[(cl * 4 + 0) * 32 + lane] +
                                             ((uint64_t)xch[(cl * 4 + 1) * 32 + lane] << 8) +
                                             ((uint64_t)xch[(cl * 4 + 2) * 32 + lane] << 16) +
                                             ((uint64_t)xch[(cl * 4 + 3) * 32 + lane] << 24);
                        S[(((int64_t)c * instances + j) * 2 + l) * N + z] = mod64m(tot, q);
                    }
                }
                umma::named_bar(1, 128);
            }
            buf ^= 1;
            if (buf == 0) acc_phase ^= 1;
        }
    }
    umma::fence_before();
    __syncthreads();
    umma::cluster_sync();  // the pair's MMAs and cross-CTA arrivals are complete in both CTAs
    if (warp == 1) umma::tmem_dealloc_pair(tmem, ncols);
    if (threadIdx.x == 0 && *err) atomicExch(err_flag, *err);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
int pack_mma_nt(int clients) {
    int n = (4 * clients + 15) / 16 * 16;
    return n < 16 ? 16 : n;
}

constexpr int P_XCH_BYTES = 2 * 16 * 4 * 32 * 4;  // two epilogue groups x 16 clients x 4 bytes x 32 outputs

int pack_mma_stages(int nt) {
    const int per = 2 * P_A_STAGE + nt * P_TILE_K;
    int s = (210 * 1024 - P_XCH_BYTES) / per;
    return s > P_MAX_STAGES ? P_MAX_STAGES : (s < 2 ? 2 : s);
}

size_t pack_mma_smem(int nt) {
    return 2048 + (size_t)pack_mma_stages(nt) * (2 * P_A_STAGE + nt * P_TILE_K) + P_XCH_BYTES;
}

cudaError_t init_pack_mma_kernel() {
    size_t mx = 0;  // the largest footprint over every client count the launcher can pick
    for (int nt = 16; nt <= 256; nt += 16) mx = pack_mma_smem(nt) > mx ? pack_mma_smem(nt) : mx;
    return cudaFuncSetAttribute(k_pack_mma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mx);
}

constexpr int Q_XCH_BYTES = 16 * 4 * 32 * 4;

int pack_pair_stages(int nt) {
    const int per = P_A_STAGE + (nt / 2) * P_TILE_K;
    int s = (210 * 1024 - Q_XCH_BYTES) / per;
    return s > P_MAX_STAGES ? P_MAX_STAGES : (s < 2 ? 2 : s);
}

size_t pack_pair_smem(int nt) {
    return 2048 + (size_t)pack_pair_stages(nt) * (P_A_STAGE + (nt / 2) * P_TILE_K) + Q_XCH_BYTES;
}

cudaError_t init_pack_pair_kernel() {
    size_t mx = 0;
    for (int nt = 16; nt <= 256; nt += 16) mx = pack_pair_smem(nt) > mx ? pack_pair_smem(nt) : mx;
    return cudaFuncSetAttribute(k_pack_mma_pair, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mx);
}

// CTA pairs that can be resident at once (a pair needs two SMs of one GPC).  The kernel is
// persistent, so the grid is exactly that many pairs.
int pack_pair_resident(int nt, int sm_count) {
    static int cached[17] = {0};
    const int key = nt / 16;
    if (!cached[key]) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)(sm_count & ~1));
        cfg.blockDim = dim3(Q_THREADS);
        cfg.dynamicSmemBytes = pack_pair_smem(nt);
        cudaLaunchAttribute attr;
        attr.id = cudaLaunchAttributeClusterDimension;
        attr.val.clusterDim.x = 2;
        attr.val.clusterDim.y = 1;
        attr.val.clusterDim.z = 1;
        cfg.attrs = &attr;
        cfg.numAttrs = 1;
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, (void*)k_pack_mma_pair, &cfg) != cudaSuccess || n < 1) {
            cudaGetLastError();
            n = sm_count / 2;
        }
        cached[key] = n < sm_count / 2 ? n : sm_count / 2;
    }
    return cached[key];
}

cudaError_t launch_pack_mma_pair(const CUtensorMap* tm_t, const CUtensorMap* tm_y_half, int instances, int clients,
                                 int np, uint32_t* S, int* err_flag, int sm_count, cudaStream_t st) {
    const int nt = pack_mma_nt(clients);
    if (clients < 1 || clients > 64 || np < nt) return cudaErrorInvalidValue;
    cudaError_t e = check_extent(S, (uint64_t)clients * instances * 2 * N * 4, "packing: outputs");
    if (e != cudaSuccess) return e;
    const int mt_count = (instances + 31) / 32;
    const int grid = 2 * pack_pair_resident(nt, sm_count);
    k_pack_mma_pair<<<grid, Q_THREADS, pack_pair_smem(nt), st>>>(*tm_t, *tm_y_half, instances, mt_count, clients, np,
                                                                 nt, pack_pair_stages(nt), S, err_flag);
    return cudaGetLastError();
}

uint64_t tpp_bytes(int instances) {
    const uint64_t mt = (uint64_t)(instances + 31) / 32;
    return (uint64_t)N * 2 * mt * P_TILE_M * P_K;
}

cudaError_t launch_relayout_tpp(const uint64_t* bt, const uint64_t* btb, uint8_t* tpp, int instances,
                                cudaStream_t st) {
    const int mt_count = (instances + 31) / 32;
    cudaError_t e = cudaFuncSetAttribute(k_relayout_tpp, cudaFuncAttributeMaxDynamicSharedMemorySize, 256 * 256);
    if (e != cudaSuccess) return e;
    k_init_dlog5<<<N / 2 / 256, 256, 0, st>>>();
    k_relayout_tpp<<<dim3(N / 256, N, mt_count * T_EXP), 256, 256 * 256, st>>>(bt, btb, tpp, instances, mt_count);
    return cudaGetLastError();
}

cudaError_t launch_build_y8(const uint64_t* y_bodies, uint8_t* y8, int clients, int np, cudaStream_t st) {
    cudaError_t e;
    if ((e = check_extent(y_bodies, (uint64_t)clients * T_EXP * N * 8, "client operand: y bodies")) != cudaSuccess ||
        (e = check_extent(y8, (uint64_t)2 * np * P_K, "client operand: byte rows")) != cudaSuccess)
        return e;
    e = cudaMemsetAsync(y8, 0, (size_t)2 * np * P_K, st);
    if (e != cudaSuccess) return e;
    k_build_y8<<<148 * 4, 256, 0, st>>>(y_bodies, y8, clients, np);
    return cudaGetLastError();
}

cudaError_t launch_pack_mma(const CUtensorMap* tm_t, const CUtensorMap* tm_y, int instances, int clients, int np,
                            uint32_t* S, int* err_flag, int sm_count, cudaStream_t st) {
    const int nt = pack_mma_nt(clients);
    if (clients < 1 || clients > 64 || np < nt) return cudaErrorInvalidValue;
    cudaError_t e = check_extent(S, (uint64_t)clients * instances * 2 * N * 4, "packing: outputs");
    if (e != cudaSuccess) return e;
    const int mt_count = (instances + 31) / 32;
    const int stages = pack_mma_stages(nt);
    k_pack_mma<<<sm_count, P_THREADS, pack_mma_smem(nt), st>>>(*tm_t, *tm_y, instances, mt_count, clients, np, nt,
                                                                stages, S, err_flag);
    return cudaGetLastError();
}

}  // namespace ipr
