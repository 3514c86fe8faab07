// kernels.cu — sm_100a kernels of the InsPIRe keyword-PIR respond() path.
//
// Step map (rkdud007/inspire-rs, src/pir/server/keyword.rs:534-628):
//   k_parse_query    deserialize_keyword_query (src/protocol/wire.rs:618-705)
//   k_gemv           first-dimension GEMV (native/cuda/gemv_kernel.cu:46-103),
//                    both queries of a payload in one pass over the DB
//   k_pack           InspiRING key-switch inner product with the Galois
//                    rotations of the client key fused in (rotation_kernel.cu:21-59
//                    + packing_online_kernel.cu:18-92), once per payload
//   k_intt_crt       from_ntt of the packing sums (src/pir/gpu/packing_online.rs:359-375)
//   k_fold_switch    RGSW interpolation fold (keyword.rs:543-574) fused with
//                    switch_and_keep (src/pir/modulus_switch.rs:45-73)
//   k_response_frame serialize_keyword_response framing (wire.rs:708-726)
#include <cuda_runtime.h>

#include <cstdint>

#include "bounds.cuh"
#include "ipr_device.cuh"
#include "kernels.cuh"
#include "ntt_regs.cuh"
#include "umma.cuh"

namespace ipr {

__constant__ uint64_t c_br[2];      // floor(2^64 / q_l)
__constant__ uint32_t c_q0inv;      // q0^-1 mod q1

__host__ cudaError_t set_constants(const uint64_t br[2], uint32_t q0inv) {
    cudaError_t e = cudaMemcpyToSymbol(c_br, br, sizeof(uint64_t) * 2);
    if (e != cudaSuccess) return e;
    return cudaMemcpyToSymbol(c_q0inv, &q0inv, sizeof(uint32_t));
}

__device__ __forceinline__ uint32_t modq(uint64_t x, int l) {
    return mod64(x, l ? Q1 : Q0, c_br[l]);
}

// ---------------------------------------------------------------------------
// query parse: 56-bit fields start at bit 8 (byte 1) and are byte aligned
// (7 bytes each), little-endian.  Field layout (serialize_keyword_query,
// wire.rs:542-615): keys y/z interleaved per (i<3, k<N); then per query the
// db_rows packed query row values followed by 6 raw-CRT RGSW body polys.
// ---------------------------------------------------------------------------
// npay payloads of nq queries each, `pstride` bytes apart; payload p writes its
// keys at y_body/z_body + p*3N, its RGSW bodies at gsw + p*nq*12N and its
// query bytes at global query index qbase + p*nq.  a_il is the CUDA-core GEMV
// operand (single payload only; may be null).
__global__ void k_parse_query(const uint8_t* __restrict__ qb_all, int nq, int db_rows,
                              uint64_t* __restrict__ y_all, uint64_t* __restrict__ z_all,
                              uint32_t* __restrict__ a_il, uint32_t* __restrict__ gsw_all,
                              uint8_t* __restrict__ qbytes, int qbase0, int npay, int64_t pstride) {
    const int64_t keys = 2LL * T_EXP * N;
    const int64_t per_q = (int64_t)db_rows + 2LL * T_EXP * N;
    const int64_t fpp = keys + (int64_t)nq * per_q;  // fields per payload
    const int64_t total_all = fpp * npay;
    const uint64_t m28 = (1ull << 28) - 1;
    for (int64_t fa = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; fa < total_all;
         fa += (int64_t)gridDim.x * blockDim.x) {
        const int pay = (int)(fa / fpp);
        const int64_t f = fa - (int64_t)pay * fpp;
        const uint8_t* qb = qb_all + (int64_t)pay * pstride;
        uint64_t* y_body = y_all + (int64_t)pay * T_EXP * N;
        uint64_t* z_body = z_all + (int64_t)pay * T_EXP * N;
        uint32_t* gsw = gsw_all + (int64_t)pay * nq * 12 * N;
        const int qbase = qbase0 + pay * nq;
        const uint8_t* p = qb + 1 + 7 * f;
        uint64_t v = 0;
#pragma unroll
        for (int b = 0; b < 7; b++) v |= (uint64_t)p[b] << (8 * b);
        const uint32_t lo = (uint32_t)(v & m28), hi = (uint32_t)((v >> 28) & m28);
        if (f < keys) {
            const int64_t ik = f >> 1;
            const uint64_t cond = (uint64_t)lo | ((uint64_t)hi << 32);
            if (f & 1) z_body[ik] = cond;
            else y_body[ik] = cond;
        } else {
            const int64_t g = f - keys;
            const int q = (int)(g / per_q);
            const int64_t r = g - (int64_t)q * per_q;
            if (r < db_rows) {
                // GEMV operand, queries grouped in pairs: a_il[g][k][qq][l], g = q/2
                const int g2 = q >> 1, qq = q & 1, ng = (nq - 2 * g2) < 2 ? (nq - 2 * g2) : 2;
                if (a_il) {
                    uint32_t* dst = a_il + (int64_t)g2 * db_rows * 4 + (r * ng + qq) * 2;
                    dst[0] = lo;
                    dst[1] = hi;
                }
                if (qbytes) {  // tensor-core operand: row query*7 + byte of X, column r, where
                    // X = crt(lo, hi) < q0 q1 < 2^56 is congruent to lo mod q0 and to hi mod q1
                    // (for any lo, hi below 2^28)
                    const uint64_t x = crt2m(lo, hi);
                    uint8_t* qrow = qbytes + (int64_t)(qbase + q) * 7 * db_rows + r;
#pragma unroll
                    for (int b = 0; b < 7; b++) qrow[(int64_t)b * db_rows] = (uint8_t)(x >> (8 * b));
                }
            } else {
                const int64_t rr = r - db_rows;  // poly c = rr / N, coeff z = rr % N
                const int c = (int)(rr >> LOGN), z = (int)(rr & (N - 1));
                uint32_t* poly = gsw + ((int64_t)q * 2 * T_EXP + c) * 2 * N;
                poly[z] = lo;
                poly[N + z] = hi;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// First-dimension GEMV for NQ queries in one pass over the DB:
//   c[q][j] = CRT( sum_k a_q,0[k] D[j][k] mod q0 , sum_k a_q,1[k] D[j][k] mod q1 )
// D is column-major [db_cols][db_rows] u16 (the reference layout).  A warp owns
// COLS consecutive columns; lane l reads 16 B (8 rows) of each column per
// 256-row stripe, so every load instruction covers 512 contiguous bytes.
// Per-lane u64 partial sums (NV = COLS * NQ * 2 of them) are folded across lane
// groups down to NV lanes and combined by a transpose-reduce.  Fewer columns per
// warp mean fewer accumulators, so more warps fit on an SM (MINB CTAs of 256) to
// keep loads in flight.
// ---------------------------------------------------------------------------
//
// FP selects the pipe of the products: 0 = u64 integer multiply-adds (IMAD.WIDE), 1 = the
// FP64 pipe (fused multiply-adds of doubles).  The FP64 products
// are exact integer arithmetic: a DB entry (< 2^16) and a residue (< 2^28) are converted
// exactly (2^52 + x, less 2^52), each product is below 2^44 and a lane sums db_rows / 32 of
// them, below 2^53 while db_rows <= 16384, so every partial sum is an exactly represented
// integer, converted exactly to u64 before the cross-lane reduction.
__device__ __forceinline__ double exact_dbl(uint32_t x) {  // x as a double, exactly, on the FP64 pipe
    return __hiloint2double(0x43300000, (int)x) - 4503599627370496.0;
}

template <int NQ, int COLS, int MINB = 1, int FP = 0>
__global__ void __launch_bounds__(256, MINB) k_gemv(const uint16_t* __restrict__ db, int db_rows,
                                                    int64_t db_cols, const uint32_t* __restrict__ a_il,
                                                    uint64_t* __restrict__ c) {
    constexpr int NV = COLS * NQ * 2;  // values reduced per warp task
    auto on_fp = [](int) { return FP == 1; };
    static_assert(NV == 8 || NV == 16 || NV == 32, "8, 16 or 32 values per lane");
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t ntasks = db_cols / COLS;
    const int stripes = db_rows >> 8;
    for (int64_t task = warp; task < ntasks; task += nwarps) {
        const int64_t col0 = task * COLS;
        uint64_t acc[NV];
        double accd[NV];
#pragma unroll
        for (int v = 0; v < NV; v++) {
            acc[v] = 0;
            accd[v] = 0.0;
        }
        for (int it = 0; it < stripes; it++) {
            const int k0 = it * 256 + lane * 8;
            uint4 d[COLS];
#pragma unroll
            for (int cc = 0; cc < COLS; cc++) {
                const uint4* src =
                    reinterpret_cast<const uint4*>(db + (col0 + cc) * (int64_t)db_rows + k0);
                asm volatile("ld.global.nc.L1::no_allocate.v4.u32 {%0,%1,%2,%3}, [%4];"
                             : "=r"(d[cc].x), "=r"(d[cc].y), "=r"(d[cc].z), "=r"(d[cc].w)
                             : "l"(src));
            }
#pragma unroll
            for (int kk = 0; kk < 8; kk++) {
                uint32_t av[NQ * 2];
                if constexpr (NQ == 2) {
                    uint4 t = __ldg(reinterpret_cast<const uint4*>(a_il) + (k0 + kk));
                    av[0] = t.x; av[1] = t.y; av[2] = t.z; av[3] = t.w;
                } else {
                    uint2 t = __ldg(reinterpret_cast<const uint2*>(a_il) + (k0 + kk));
                    av[0] = t.x; av[1] = t.y;
                }
                double ad[NQ * 2];
#pragma unroll
                for (int v = 0; v < NQ * 2; v++) ad[v] = on_fp(v) ? exact_dbl(av[v]) : 0.0;
#pragma unroll
                for (int cc = 0; cc < COLS; cc++) {
                    const uint32_t w = (&d[cc].x)[kk >> 1];
                    const uint32_t dv = (kk & 1) ? (w >> 16) : (w & 0xffffu);
                    const double dd = FP ? exact_dbl(dv) : 0.0;
#pragma unroll
                    for (int v = 0; v < NQ * 2; v++) {
                        if (on_fp(v)) accd[cc * NQ * 2 + v] = fma(ad[v], dd, accd[cc * NQ * 2 + v]);
                        else acc[cc * NQ * 2 + v] += (uint64_t)av[v] * dv;
                    }
                }
            }
        }
        if (FP) {  // exact integers below 2^53 (see above)
#pragma unroll
            for (int v = 0; v < NV; v++)
                if (on_fp(v % (NQ * 2))) acc[v] = (uint64_t)__double2ull_rn(accd[v]);
        }
        // fold lane groups down to NV lanes, then transpose-reduce: lane v (< NV) ends with the
        // warp-wide sum of value v (lanes v + NV, v + 2 NV, ... hold copies)
#pragma unroll
        for (int s = 16; s >= NV; s >>= 1)
#pragma unroll
            for (int i = 0; i < NV; i++) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], s);
#pragma unroll
        for (int s = NV / 2; s >= 1; s >>= 1) {
            const bool upper = lane & s;
#pragma unroll
            for (int i = 0; i < s; i++) {
                const uint64_t send = upper ? acc[i] : acc[i + s];
                const uint64_t keep = upper ? acc[i + s] : acc[i];
                acc[i] = keep + __shfl_xor_sync(0xffffffffu, send, s);
            }
        }
        // value v = cc*(NQ*2) + q*2 + l ; limb partner is lane ^ 1
        const int l = lane & 1;
        const uint32_t r = modq(acc[0], l);
        const uint32_t other = __shfl_xor_sync(0xffffffffu, r, 1);
        if (l == 0 && lane < NV) {
            const int q = (lane >> 1) % NQ, cc = lane / (NQ * 2);
            c[(int64_t)q * db_cols + col0 + cc] = crt2(r, other, c_q0inv, c_br[1]);
        }
    }
}

constexpr int GF_MAX_ROWS = 4096;  // rows of query residues the FP64 staged form converts into shared memory

// The two-query GEMV with each warp's DB stripes staged through shared memory: a warp owns 8
// consecutive columns per task (as k_gemv<2, 8>) and streams its (task, stripe) sequence
// through a private ring of STAGES stripes with 16-byte cp.async copies, so the HBM reads of
// the next STAGES - 1 stripes are in flight while one is multiplied.  Each lane reads back only
// the slots it copied itself, so the ring needs no warp synchronisation.
constexpr int GS_COLS = 8, GS_WARPS = 8;

__device__ __forceinline__ void gs_cp16(void* smem, const void* gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(smem)),
                 "l"(gmem)
                 : "memory");
}

template <int STAGES>
__global__ void __launch_bounds__(GS_WARPS * 32, 1)
    k_gemv_staged(const uint16_t* __restrict__ db, int db_rows, int64_t db_cols, const uint32_t* __restrict__ a_il,
                  uint64_t* __restrict__ c) {
    constexpr int NQ = 2, NV = GS_COLS * NQ * 2;  // 32 values per lane
    extern __shared__ uint4 gs_ring[];              // [warp][stage][column][lane]
    const int lane = threadIdx.x & 31;
    uint4* ring = gs_ring + (threadIdx.x >> 5) * STAGES * GS_COLS * 32;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t ntasks = db_cols / GS_COLS;
    const int stripes = db_rows >> 8;
    const int64_t my_tasks = warp < ntasks ? (ntasks - 1 - warp) / nwarps + 1 : 0;
    const int64_t items = my_tasks * stripes;  // (task, stripe) pairs of this warp, in order
    auto issue = [&](int64_t u) {
        if (u < items) {
            const int64_t col0 = (warp + (u / stripes) * nwarps) * GS_COLS;
            const int k0 = (int)(u % stripes) * 256 + lane * 8;
            uint4* dst = ring + (int)(u % STAGES) * GS_COLS * 32 + lane;
#pragma unroll
            for (int cc = 0; cc < GS_COLS; cc++) gs_cp16(dst + cc * 32, db + (col0 + cc) * (int64_t)db_rows + k0);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");  // one group per item, empty past the end
    };
#pragma unroll
    for (int u = 0; u < STAGES - 1; u++) issue(u);
    uint64_t acc[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) acc[v] = 0;
    for (int64_t u = 0; u < items; u++) {
        asm volatile("cp.async.wait_group %0;" ::"n"(STAGES - 2) : "memory");  // item u has landed
        const uint4* src = ring + (int)(u % STAGES) * GS_COLS * 32 + lane;
        uint4 d[GS_COLS];
#pragma unroll
        for (int cc = 0; cc < GS_COLS; cc++) d[cc] = src[cc * 32];
        issue(u + STAGES - 1);  // into the stage item u - 1 used, already read
        const int it = (int)(u % stripes);
        const int k0 = it * 256 + lane * 8;
#pragma unroll
        for (int kk = 0; kk < 8; kk++) {
            const uint4 t = __ldg(reinterpret_cast<const uint4*>(a_il) + (k0 + kk));
            const uint32_t av[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
            for (int cc = 0; cc < GS_COLS; cc++) {
                const uint32_t w = (&d[cc].x)[kk >> 1];
                const uint32_t dv = (kk & 1) ? (w >> 16) : (w & 0xffffu);
#pragma unroll
                for (int v = 0; v < 4; v++) acc[cc * 4 + v] += (uint64_t)av[v] * dv;
            }
        }
        if (it == stripes - 1) {  // the task's last stripe: reduce across the warp and write
#pragma unroll
            for (int s = 16; s >= 1; s >>= 1) {
                const bool upper = lane & s;
#pragma unroll
                for (int i = 0; i < s; i++) {
                    const uint64_t send = upper ? acc[i] : acc[i + s];
                    const uint64_t keep = upper ? acc[i + s] : acc[i];
                    acc[i] = keep + __shfl_xor_sync(0xffffffffu, send, s);
                }
            }
            const int l = lane & 1;
            const uint32_t r = modq(acc[0], l);
            const uint32_t other = __shfl_xor_sync(0xffffffffu, r, 1);
            if (l == 0) {
                const int q = (lane >> 1) % NQ, cc = lane / (NQ * 2);
                const int64_t col0 = (warp + (u / stripes) * nwarps) * GS_COLS;
                c[(int64_t)q * db_cols + col0 + cc] = crt2(r, other, c_q0inv, c_br[1]);
            }
#pragma unroll
            for (int v = 0; v < NV; v++) acc[v] = 0;
        }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
}
constexpr int GS_STAGES = 4;
constexpr int GS_SMEM = GS_WARPS * GS_STAGES * GS_COLS * 32 * 16;  // 128 KB

// k_gemv_staged with the products on the FP64 pipe.  The ring of DB stripes in shared memory
// as above is followed by the query residues, converted to doubles once per CTA
// ([stripe][kk][lane][4]: value v of row k = 256 stripe + 8 lane + kk, so that a warp's 32
// lanes read 32 consecutive 32-byte groups, no bank conflicts; db_rows <= GF_MAX_ROWS).  Each
// DB entry becomes the double 2^16 + d by integer operations alone (its 16 bits placed in the
// mantissa under the exponent of 2^16), so a product is one fused multiply-add.  The offset
// adds 2^16 x (sum of the lane's residues) to each partial sum; every thread computes that
// sum once, exactly, and takes it off after the conversion to u64.  Bounds: a product is
// below 2^28 x 2^17 = 2^45 and a lane sums db_rows / 32 <= 128 of them, below 2^53, so every
// partial sum is an exact integer.
template <int STAGES>
__global__ void __launch_bounds__(GS_WARPS * 32, 1)
    k_gemv_staged_f64(const uint16_t* __restrict__ db, int db_rows, int64_t db_cols,
                      const uint32_t* __restrict__ a_il, uint64_t* __restrict__ c) {
    constexpr int NV = GS_COLS * 4;  // 32 values per lane
    extern __shared__ uint4 gs_ring[];  // [warp][stage][column][lane], then the residues
    double* gf_a = reinterpret_cast<double*>(gs_ring + GS_WARPS * STAGES * GS_COLS * 32);
    for (int i = threadIdx.x; i < db_rows * 4; i += blockDim.x) {
        const int k = i >> 2, v = i & 3;
        gf_a[(((k >> 8) * 8 + (k & 7)) * 32 + ((k >> 3) & 31)) * 4 + v] = (double)__ldg(a_il + i);
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    uint4* ring = gs_ring + (threadIdx.x >> 5) * STAGES * GS_COLS * 32;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t ntasks = db_cols / GS_COLS;
    const int stripes = db_rows >> 8;
    uint64_t asum[4] = {0, 0, 0, 0};
    for (int it = 0; it < stripes; it++)
#pragma unroll
        for (int kk = 0; kk < 8; kk++) {
            const uint4 t = __ldg(reinterpret_cast<const uint4*>(a_il) + (it * 256 + lane * 8 + kk));
            asum[0] += t.x; asum[1] += t.y; asum[2] += t.z; asum[3] += t.w;
        }
    const int64_t my_tasks = warp < ntasks ? (ntasks - 1 - warp) / nwarps + 1 : 0;
    const int64_t items = my_tasks * stripes;
    auto issue = [&](int64_t u) {
        if (u < items) {
            const int64_t col0 = (warp + (u / stripes) * nwarps) * GS_COLS;
            const int k0 = (int)(u % stripes) * 256 + lane * 8;
            uint4* dst = ring + (int)(u % STAGES) * GS_COLS * 32 + lane;
#pragma unroll
            for (int cc = 0; cc < GS_COLS; cc++) gs_cp16(dst + cc * 32, db + (col0 + cc) * (int64_t)db_rows + k0);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
#pragma unroll
    for (int u = 0; u < STAGES - 1; u++) issue(u);
    double accd[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) accd[v] = 0.0;
    for (int64_t u = 0; u < items; u++) {
        asm volatile("cp.async.wait_group %0;" ::"n"(STAGES - 2) : "memory");
        const uint4* src = ring + (int)(u % STAGES) * GS_COLS * 32 + lane;
        uint4 d[GS_COLS];
#pragma unroll
        for (int cc = 0; cc < GS_COLS; cc++) d[cc] = src[cc * 32];
        issue(u + STAGES - 1);
        const int it = (int)(u % stripes);
#pragma unroll
        for (int kk = 0; kk < 8; kk++) {
            const double* ar = gf_a + ((it * 8 + kk) * 32 + lane) * 4;
            const double2 a01 = *reinterpret_cast<const double2*>(ar);
            const double2 a23 = *reinterpret_cast<const double2*>(ar + 2);
            const double ad[4] = {a01.x, a01.y, a23.x, a23.y};
#pragma unroll
            for (int cc = 0; cc < GS_COLS; cc++) {
                const uint32_t w = (&d[cc].x)[kk >> 1];
                const uint32_t m = (kk & 1) ? ((w >> 12) & 0xffff0u) : ((w << 4) & 0xffff0u);
                const double dd = __hiloint2double((int)(0x40f00000u | m), 0);
#pragma unroll
                for (int v = 0; v < 4; v++) accd[cc * 4 + v] = fma(ad[v], dd, accd[cc * 4 + v]);
            }
        }
        if (it == stripes - 1) {
            uint64_t acc[NV];
#pragma unroll
            for (int v = 0; v < NV; v++) acc[v] = (uint64_t)__double2ull_rn(accd[v]) - (asum[v & 3] << 16);
#pragma unroll
            for (int s = 16; s >= 1; s >>= 1) {
                const bool upper = lane & s;
#pragma unroll
                for (int i = 0; i < s; i++) {
                    const uint64_t send = upper ? acc[i] : acc[i + s];
                    const uint64_t keep = upper ? acc[i + s] : acc[i];
                    acc[i] = keep + __shfl_xor_sync(0xffffffffu, send, s);
                }
            }
            const int l = lane & 1;
            const uint32_t r = modq(acc[0], l);
            const uint32_t other = __shfl_xor_sync(0xffffffffu, r, 1);
            if (l == 0) {
                const int q = (lane >> 1) & 1, cc = lane >> 2;
                const int64_t col0 = (warp + (u / stripes) * nwarps) * GS_COLS;
                c[(int64_t)q * db_cols + col0 + cc] = crt2(r, other, c_q0inv, c_br[1]);
            }
#pragma unroll
            for (int v = 0; v < NV; v++) accd[v] = 0.0;
        }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
}
constexpr int GSF_STAGES = 3;  // 96 KB of ring + up to 128 KB of residues
constexpr int gsf_smem(int db_rows) { return GS_WARPS * GSF_STAGES * GS_COLS * 32 * 16 + db_rows * 4 * 8; }

// The two-query GEMV with a lane per DB column and TMA-fed stages (form 6).  A CTA owns a tile
// of GT_COLS = 128 consecutive columns (a contiguous 128 x db_rows x 2-byte block of the
// column-major DB) and its 16 warps split the tile's rows: in stage s warp w takes rows
// 256 s + 16 w .. + 16 of all 128 columns, one 2D TMA box ({16 rows, 128 columns}, 32-byte
// swizzle) plus a 256-byte bulk copy of those rows' query residues, through a private ring
// of GT_STAGES stages and one mbarrier per stage.  Lane l owns columns l, l + 32, l + 64,
// l + 96, so the residues of a row are the same for all lanes (broadcast reads, converted to
// doubles once per stage by the warp) and each residue read serves 4 columns x 4 values;
// the swizzle puts the 16-byte row chunks of 8 consecutive columns in 8 distinct bank groups.
// Products run on the FP64 pipe as in k_gemv_staged_f64 (a DB entry is the double 2^16 + d,
// built by integer operations; a product is below 2^45) and a lane's double accumulators
// are flushed after at most 16 stages (256 rows, below 2^53: exact) into 64-bit integer
// sums in shared memory by atomic adds.  At the tile's end the 16 warps meet at a named
// barrier and each of the first 256 threads finishes one (column, query) output: the offset
// 2^16 x (sum of the limb's residues over all rows) is taken off, then the Barrett
// reductions and the CRT.  The sums use two buffers (alternating tiles), so one barrier per
// tile suffices.  Sixteen warps of 122 registers fill the register file; more warps per SM,
// not deeper rings, is what shortened this kernel (0.85 ms at 1M against 0.92-0.95 ms for
// 8 warps with 5-stage rings).  A stage wait is bounded by time: after a failed wait the
// warp stops waiting and issuing, the kernel reports code 31 through err_flag and drains
// its own copies before it returns.
constexpr int GT_WARPS = 16, GT_ROWS = 16, GT_COLS = 128, GT_STAGES = 2;
constexpr int GT_DB_BYTES = GT_ROWS * GT_COLS * 2;  // 4 KB of DB per stage
constexpr int GT_RES_BYTES = GT_ROWS * 16;          // the stage rows' 4 u32 residues each
constexpr int gt_smem() {
    return 1024 + GT_WARPS * GT_STAGES * (GT_DB_BYTES + GT_RES_BYTES + GT_RES_BYTES * 2) + 2 * GT_COLS * 4 * 8 +
           GT_WARPS * GT_STAGES * 8 + 64;
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* mbar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     umma::smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(umma::smem_addr(mbar))
                 : "memory");
}

__global__ void __launch_bounds__(GT_WARPS * 32, 1)
    k_gemv_tma_f64(const __grid_constant__ CUtensorMap tm_db, int db_rows, int64_t db_cols,
                   const uint32_t* __restrict__ a_il, uint64_t* __restrict__ c, int* __restrict__ err_flag) {
    extern __shared__ uint8_t gt_raw[];
    uint8_t* base = gt_raw + ((1024 - (umma::smem_addr(gt_raw) & 1023)) & 1023);
    uint8_t* ring_db = base;                                                  // [warp][stage][4 KB]
    uint32_t* ring_ru = reinterpret_cast<uint32_t*>(base + GT_WARPS * GT_STAGES * GT_DB_BYTES);  // [warp][stage][64]
    double* ring_rd = reinterpret_cast<double*>(ring_ru + GT_WARPS * GT_STAGES * GT_ROWS * 4);    // [warp][stage][64]
    uint64_t* red = reinterpret_cast<uint64_t*>(ring_rd + GT_WARPS * GT_STAGES * GT_ROWS * 4);   // [2][128][4]
    uint64_t* bars = red + 2 * GT_COLS * 4;                                                      // [warp][stage]
    uint64_t* asum_sh = bars + GT_WARPS * GT_STAGES;                                             // [4]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < 2 * GT_COLS * 4; i += blockDim.x) red[i] = 0;
    if (threadIdx.x < 4) asum_sh[threadIdx.x] = 0;
    if (lane == 0)
        for (int s = 0; s < GT_STAGES; s++) umma::mbar_init(&bars[warp * GT_STAGES + s], 1);
    umma::fence_mbar_init();
    __syncthreads();
    {  // the offset: 2^16 x the sum of each limb's residues over all rows
        uint64_t a4[4] = {0, 0, 0, 0};
        for (int r = threadIdx.x; r < db_rows; r += blockDim.x) {
            const uint4 t = __ldg(reinterpret_cast<const uint4*>(a_il) + r);
            a4[0] += t.x; a4[1] += t.y; a4[2] += t.z; a4[3] += t.w;
        }
#pragma unroll
        for (int v = 0; v < 4; v++) {
#pragma unroll
            for (int s = 16; s >= 1; s >>= 1) a4[v] += __shfl_xor_sync(0xffffffffu, a4[v], s);
            if (lane == 0) atomicAdd(reinterpret_cast<unsigned long long*>(&asum_sh[v]), (unsigned long long)a4[v]);
        }
    }
    __syncthreads();
    const int oq = (threadIdx.x >> 7) & 1;  // the query of this thread's output (threads below 256)
    const uint64_t off = asum_sh[oq * 2] << 16, off1 = asum_sh[oq * 2 + 1] << 16;
    const int nst = db_rows / (GT_WARPS * GT_ROWS);  // stages per tile
    const int64_t ntiles = (db_cols + GT_COLS - 1) / GT_COLS;
    const int my_tiles = blockIdx.x < ntiles ? (int)((ntiles - 1 - blockIdx.x) / gridDim.x + 1) : 0;
    const int items = my_tiles * nst;  // (tile, stage) items of every warp of this CTA, in order
    uint8_t* my_db = ring_db + warp * GT_STAGES * GT_DB_BYTES;
    uint32_t* my_ru = ring_ru + warp * GT_STAGES * GT_ROWS * 4;
    double* my_rd = ring_rd + warp * GT_STAGES * GT_ROWS * 4;
    uint64_t* my_bars = bars + warp * GT_STAGES;
    int i_next = 0, i_st = 0, i_slot = 0;  // lane 0's issue position: item, its stage, its slot
    int64_t i_tile = blockIdx.x;
    auto issue = [&]() {  // lane 0: the next item into its slot, if any
        if (i_next < items) {
            const int row0 = i_st * (GT_WARPS * GT_ROWS) + warp * GT_ROWS;
            uint64_t* bar = &my_bars[i_slot];
            umma::mbar_expect_tx(bar, GT_DB_BYTES + GT_RES_BYTES);
            umma::tma_load_2d(my_db + i_slot * GT_DB_BYTES, &tm_db, row0, (int)(i_tile * GT_COLS), bar);
            bulk_load(my_ru + i_slot * GT_ROWS * 4, a_il + (int64_t)row0 * 4, GT_RES_BYTES, bar);
            i_next++;
            if (++i_slot == GT_STAGES) i_slot = 0;
            if (++i_st == nst) {
                i_st = 0;
                i_tile += gridDim.x;
            }
        }
    };
    if (lane == 0)
        for (int u = 0; u < GT_STAGES; u++) issue();
    double acc[16];
#pragma unroll
    for (int v = 0; v < 16; v++) acc[v] = 0.0;
    bool ok = true;
    int failed_at = -1, slot = 0, st = 0, b = 0;
    uint32_t phase = 0;
    int64_t tile = blockIdx.x;
    for (int u = 0; u < items; u++) {
        if (ok) {
            const bool got = umma::mbar_wait(&my_bars[slot], phase);
            if (!__all_sync(0xffffffffu, got)) {  // the warp stops together
                ok = false;
                failed_at = u;
                if (lane == 0) atomicExch(err_flag, 31);
            }
        }
        if (ok) {
            const uint32_t* ru = my_ru + slot * GT_ROWS * 4;
            double* rd = my_rd + slot * GT_ROWS * 4;
            rd[lane] = (double)ru[lane];
            rd[lane + 32] = (double)ru[lane + 32];
            const uint8_t* sb = my_db + slot * GT_DB_BYTES;
            uint4 d[4][2];
#pragma unroll
            for (int p = 0; p < 4; p++) {
                const int col = p * 32 + lane;
#pragma unroll
                for (int j = 0; j < 2; j++)  // 32-byte swizzle: chunk j of column col at chunk j ^ bit 2 of col
                    d[p][j] = *reinterpret_cast<const uint4*>(sb + col * 32 + ((j ^ ((col >> 2) & 1)) << 4));
            }
            __syncwarp();
#pragma unroll
            for (int i = 0; i < GT_ROWS; i++) {
                const double2 a01 = *reinterpret_cast<const double2*>(rd + i * 4);
                const double2 a23 = *reinterpret_cast<const double2*>(rd + i * 4 + 2);
                const double ad[4] = {a01.x, a01.y, a23.x, a23.y};
#pragma unroll
                for (int p = 0; p < 4; p++) {
                    const uint32_t w = (&d[p][i >> 3].x)[(i & 7) >> 1];
                    const uint32_t m = (i & 1) ? ((w >> 12) & 0xffff0u) : ((w << 4) & 0xffff0u);
                    const double dd = __hiloint2double((int)(0x40f00000u | m), 0);
#pragma unroll
                    for (int v = 0; v < 4; v++) acc[p * 4 + v] = fma(ad[v], dd, acc[p * 4 + v]);
                }
            }
        }
        __syncwarp();
        if (ok && lane == 0) issue();  // item u + GT_STAGES into the slot every lane has finished reading
        if ((st & 15) == 15 || st == nst - 1) {  // flush: at most 256 rows per accumulator
#pragma unroll
            for (int p = 0; p < 4; p++)
#pragma unroll
                for (int v = 0; v < 4; v++) {
                    atomicAdd(reinterpret_cast<unsigned long long*>(&red[(b * GT_COLS + p * 32 + lane) * 4 + v]),
                              (unsigned long long)__double2ull_rn(acc[p * 4 + v]));
                    acc[p * 4 + v] = 0.0;
                }
        }
        if (st == nst - 1) {  // the tile's last stage: every warp has added its sums
            umma::named_bar(1, GT_WARPS * 32);
            if (threadIdx.x < 2 * GT_COLS) {
                const int col = threadIdx.x & (GT_COLS - 1);
                uint64_t* sp = &red[(b * GT_COLS + col) * 4 + 2 * oq];
                const uint64_t s0 = sp[0] - off, s1 = sp[1] - off1;
                sp[0] = 0;
                sp[1] = 0;
                const int64_t gcol = tile * GT_COLS + col;
                if (gcol < db_cols)
                    c[(int64_t)oq * db_cols + gcol] = crt2(modq(s0, 0), modq(s1, 1), c_q0inv, c_br[1]);
            }
        }
        if (++slot == GT_STAGES) {
            slot = 0;
            phase ^= 1;
        }
        if (++st == nst) {
            st = 0;
            b ^= 1;
            tile += gridDim.x;
        }
    }
    if (!ok && lane == 0) {  // drain the copies this warp issued and did not consume
        const int end = failed_at + GT_STAGES < items ? failed_at + GT_STAGES : items;
        for (int v = failed_at; v < end; v++)
            umma::mbar_wait(&my_bars[v % GT_STAGES], (uint32_t)((v / GT_STAGES) & 1), umma::kDrainLimitNs);
    }
}

// ---------------------------------------------------------------------------
// Packing inner product, rotations fused.  For output j, NTT slot z, limb l:
//   S[j][l][z] = sum_{i<1023,k<3} y_l[k][rot_i(z)] T_l[j][i,k][z]
//              + y_l[k][rotbar_i(z)] Tbar_l[j][i,k][z] + sum_k z_l[k][z] That_l[j][k][z]
// with rot_i = auto_src(5^i mod 2N, .), rotbar_i = auto_src(2N - 5^i, .).
// The client key y_body stays in shared memory; the precomputed bold_t stream
// (the dominant HBM traffic) is read once per payload with 16-byte
// non-allocating loads, two adjacent slots per thread.  Slots z and z+1 (z even)
// rotate to the slot pair {s, s^1}, so each gather is one 16-byte smem load.
// ---------------------------------------------------------------------------
constexpr int PACK_THREADS = 128;
constexpr int PACK_ZB = 2 * PACK_THREADS;  // slots per CTA

__device__ __forceinline__ void ldg_nc_v2(const uint64_t* p, uint64_t& a, uint64_t& b) {
    asm volatile("ld.global.nc.L1::no_allocate.v2.u64 {%0,%1}, [%2];" : "=l"(a), "=l"(b) : "l"(p));
}

__global__ void __launch_bounds__(PACK_THREADS) k_pack(const uint64_t* __restrict__ bt,
                                                       const uint64_t* __restrict__ btb,
                                                       const uint64_t* __restrict__ bth,
                                                       const uint64_t* __restrict__ y_body,
                                                       const uint64_t* __restrict__ z_body,
                                                       uint32_t* __restrict__ S) {
    extern __shared__ uint64_t ys[];  // [3][N] condensed
    for (int i = threadIdx.x; i < T_EXP * N; i += blockDim.x) ys[i] = y_body[i];
    __syncthreads();
    const int j = blockIdx.y;
    const int z = blockIdx.x * PACK_ZB + 2 * threadIdx.x;
    const uint32_t ez = exponent_of_slot(z);
    const uint64_t* T = bt + (int64_t)j * NINNER * N + z;
    const uint64_t* Tb = btb + (int64_t)j * NINNER * N + z;
    uint64_t a00 = 0, a01 = 0, a10 = 0, a11 = 0;  // a{limb}{slot}
    uint32_t g = 1;                               // 5^i mod 2N
    for (int i0 = 0; i0 < NROT; i0 += 32) {
        const int iend = i0 + 32 < NROT ? i0 + 32 : NROT;
#pragma unroll 2
        for (int i = i0; i < iend; i++) {
            const uint32_t s1 = slot_of_exponent((g * ez) & (2 * N - 1));
            const uint32_t s2 = slot_of_exponent(((2 * N - g) * ez) & (2 * N - 1));
            uint64_t tv[3][2], tbv[3][2];
#pragma unroll
            for (int k = 0; k < T_EXP; k++) {
                ldg_nc_v2(T + (int64_t)(i * T_EXP + k) * N, tv[k][0], tv[k][1]);
                ldg_nc_v2(Tb + (int64_t)(i * T_EXP + k) * N, tbv[k][0], tbv[k][1]);
            }
#pragma unroll
            for (int k = 0; k < T_EXP; k++) {
                const ulonglong2 yp = *reinterpret_cast<const ulonglong2*>(ys + k * N + (s1 & ~1u));
                const ulonglong2 bp = *reinterpret_cast<const ulonglong2*>(ys + k * N + (s2 & ~1u));
                const uint64_t y0 = (s1 & 1) ? yp.y : yp.x, y1 = (s1 & 1) ? yp.x : yp.y;
                const uint64_t b0 = (s2 & 1) ? bp.y : bp.x, b1 = (s2 & 1) ? bp.x : bp.y;
                a00 += (uint64_t)(uint32_t)y0 * (uint32_t)tv[k][0] + (uint64_t)(uint32_t)b0 * (uint32_t)tbv[k][0];
                a01 += (uint64_t)(uint32_t)y1 * (uint32_t)tv[k][1] + (uint64_t)(uint32_t)b1 * (uint32_t)tbv[k][1];
                a10 += (y0 >> 32) * (tv[k][0] >> 32) + (b0 >> 32) * (tbv[k][0] >> 32);
                a11 += (y1 >> 32) * (tv[k][1] >> 32) + (b1 >> 32) * (tbv[k][1] >> 32);
            }
            g = (g * 5) & (2 * N - 1);
        }
        // <= 192 products of two 28-bit values plus a residue: no overflow
        a00 = modq(a00, 0); a01 = modq(a01, 0);
        a10 = modq(a10, 1); a11 = modq(a11, 1);
    }
    const uint64_t* Th = bth + (int64_t)j * T_EXP * N + z;
#pragma unroll
    for (int k = 0; k < T_EXP; k++) {
        const uint64_t t0 = Th[k * N], t1 = Th[k * N + 1];
        const uint64_t z0 = z_body[k * N + z], z1 = z_body[k * N + z + 1];
        a00 += (uint64_t)(uint32_t)z0 * (uint32_t)t0;
        a01 += (uint64_t)(uint32_t)z1 * (uint32_t)t1;
        a10 += (z0 >> 32) * (t0 >> 32);
        a11 += (z1 >> 32) * (t1 >> 32);
    }
    uint32_t* Sj = S + (int64_t)j * 2 * N;
    *reinterpret_cast<uint2*>(Sj + z) = make_uint2(modq(a00, 0), modq(a01, 0));
    *reinterpret_cast<uint2*>(Sj + N + z) = make_uint2(modq(a10, 1), modq(a11, 1));
}

// ---------------------------------------------------------------------------
// R[j] = from_ntt(S[j]) : inverse NTT per limb + CRT compose (one CTA per output)
// ---------------------------------------------------------------------------
// One CTA of 512 threads per pair of outputs (j0, j0 + 1): group g (256 threads) runs the
// inverse NTTs of limb g of both in registers (ntt_regs.cuh, one twiddle load per two
// butterflies); the limbs meet at the CRT compose.
constexpr int INTT_P = 2;

__global__ void __launch_bounds__(512) k_intt_crt(const uint32_t* __restrict__ S,
                                                  const uint32_t* __restrict__ iw,
                                                  const uint32_t* __restrict__ iwp,
                                                  uint64_t* __restrict__ R, int num_outputs,
                                                  const uint64_t* __restrict__ z_bodies,
                                                  const uint64_t* __restrict__ bth, int instances) {
    __shared__ uint32_t sm[2][INTT_P][N];  // [limb][output][slot]
    const int j0 = blockIdx.x * INTT_P;
    const int g = threadIdx.x >> 8, t = threadIdx.x & 255;
    const uint32_t q = g ? Q1 : Q0;
    uint32_t v[INTT_P][nttr::EPT];
    // layout D: thread t holds the 8 consecutive slots z0 .. z0 + 7 (16-byte loads)
    const int z0 = nttr::eD(t, 0);
#pragma unroll
    for (int p = 0; p < INTT_P; p++) {
        const int j = j0 + p < num_outputs ? j0 + p : num_outputs - 1;  // an odd count repeats the last
        const uint4* Sj = reinterpret_cast<const uint4*>(S + ((int64_t)j * 2 + g) * N + z0);
        const uint4 s0 = __ldg(Sj), s1 = __ldg(Sj + 1);
        const uint32_t sv[8] = {s0.x, s0.y, s0.z, s0.w, s1.x, s1.y, s1.z, s1.w};
        if (z_bodies) {  // + sum_k z_c[k][z] That[j'][k][z] per limb (packing_online_kernel.cu:76-83)
            const int c = j / instances, jj = j % instances;
            const uint64_t* zc = z_bodies + (int64_t)c * T_EXP * N + z0;
            const uint64_t* th = bth + (int64_t)jj * T_EXP * N + z0;
            const int sh = 32 * g;
            uint64_t acc[8];
#pragma unroll
            for (int m = 0; m < 8; m++) acc[m] = sv[m];
#pragma unroll
            for (int k = 0; k < T_EXP; k++) {
                const ulonglong2* zp = reinterpret_cast<const ulonglong2*>(zc + k * N);
                const ulonglong2* tp = reinterpret_cast<const ulonglong2*>(th + k * N);
#pragma unroll
                for (int h = 0; h < 4; h++) {
                    const ulonglong2 zv = __ldg(zp + h), tv = __ldg(tp + h);
                    acc[2 * h] += (uint64_t)(uint32_t)(zv.x >> sh) * (uint32_t)(tv.x >> sh);
                    acc[2 * h + 1] += (uint64_t)(uint32_t)(zv.y >> sh) * (uint32_t)(tv.y >> sh);
                }
            }
#pragma unroll
            for (int m = 0; m < 8; m++) v[p][m] = mod64(acc[m], q, g ? BR1 : BR0);
        } else {
#pragma unroll
            for (int m = 0; m < 8; m++) v[p][m] = sv[m];
        }
    }
    nttr::inverse<INTT_P>(v, t, &sm[g][0][0], 1 + g, iw + g * N, iwp + g * N, q);
#pragma unroll
    for (int p = 0; p < INTT_P; p++)
#pragma unroll
        for (int m = 0; m < nttr::EPT; m++) sm[g][p][nttr::eA(t, m)] = v[p][m];
    __syncthreads();
#pragma unroll
    for (int p = 0; p < INTT_P; p++) {
        if (j0 + p >= num_outputs) break;
        for (int z = threadIdx.x; z < N; z += blockDim.x)
            R[(int64_t)(j0 + p) * N + z] = crt2(sm[0][p][z], sm[1][p][z], Q0INV, BR1);
    }
}

// ---------------------------------------------------------------------------
// RGSW fold + modulus switch.  One CTA per (query, fold group wp):
//   s = 0; for i = interp-1 .. 0:
//     s = from_ntt(CT * to_ntt(G^-1(s))) + packed[wp*interp + i]  (mod q)
// packed[j] = (a_hat[j], c[j*N + z] + R[j][z]) (packing_online.rs:376-396).
// CT row 0 = NTT(-a) in every column (RGSW_SEEDS are all equal, wire.rs:88-113),
// CT row 1 = the query's 6 RGSW body polys.  The first step has s = 0, so
// G^-1(s) = 0 and the product vanishes: it reduces to s = packed[.] mod q.
// The final s is rescaled to (q'2, q'1) and bit-packed LSB-first into the
// response: 2048 x 28 bits then 2048 x 20 bits (12288 bytes).
// ---------------------------------------------------------------------------
constexpr int FOLD_THREADS = 1024;

__device__ __forceinline__ uint64_t rescale_dev(uint64_t v, uint64_t out_mod) {
    // rescale (src/core/arith.rs:436-452) of a canonical v in [0, q)
    const uint64_t half = QQ / 2;
    const bool neg = v >= half;
    const uint64_t u = neg ? QQ - v : v;
    const unsigned __int128 num = (unsigned __int128)u * out_mod + half;
    const uint64_t r = (uint64_t)(num / QQ);
    const uint64_t rm = r % out_mod;
    return neg ? (rm ? out_mod - rm : 0) : rm;
}

__global__ void __launch_bounds__(FOLD_THREADS) k_fold_switch(
    const uint32_t* __restrict__ row0,    // [2][N] NTT(-a)
    const uint32_t* __restrict__ gsw,     // [nq][6][2][N]
    const uint64_t* __restrict__ a_hat,   // [outputs][N]
    const uint64_t* __restrict__ R,       // [outputs][N]
    const uint64_t* __restrict__ cvec,    // [nq][db_cols]
    const uint32_t* __restrict__ fw, const uint32_t* __restrict__ fwp,
    const uint32_t* __restrict__ iw, const uint32_t* __restrict__ iwp,
    int interp, int c_groups, int64_t db_cols, uint8_t* __restrict__ resp, int64_t resp_query_stride) {
    extern __shared__ uint32_t G[];  // [6][2][N] digits in NTT form; reused for products
    const int wp = blockIdx.x, q = blockIdx.y;
    const uint32_t* body = gsw + (int64_t)q * 2 * T_EXP * 2 * N;
    const uint64_t* cq = cvec + (int64_t)q * db_cols;
    uint64_t s[2][2];  // [row][which of my two slots]
    const int z0 = threadIdx.x, z1 = threadIdx.x + FOLD_THREADS;
    const uint64_t mask = (1ull << GADGET_BITS) - 1;
    for (int step = interp - 1; step >= 0; step--) {
        const int j = wp * interp + step;
        uint64_t pk[2][2];
        pk[0][0] = a_hat[(int64_t)j * N + z0];
        pk[0][1] = a_hat[(int64_t)j * N + z1];
        pk[1][0] = cq[(int64_t)j * N + z0] + R[(int64_t)j * N + z0];
        pk[1][1] = cq[(int64_t)j * N + z1] + R[(int64_t)j * N + z1];
        if (step == interp - 1) {
#pragma unroll
            for (int r = 0; r < 2; r++)
#pragma unroll
                for (int h = 0; h < 2; h++) s[r][h] = pk[r][h] % QQ;
            continue;
        }
        // gadget_invert (gadget.rs:35-61): row j + k*2 holds digit k of input row j
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int z = h ? z1 : z0;
#pragma unroll
            for (int r = 0; r < 2; r++)
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    const uint32_t d = (uint32_t)((s[r][h] >> (k * GADGET_BITS)) & mask);
                    const int p = r + 2 * k;
                    G[(p * 2 + 0) * N + z] = d;
                    G[(p * 2 + 1) * N + z] = d;
                }
        }
        __syncthreads();
        ntt_forward_smem<12>(G, fw, fwp, [](int p) { return p & 1; });
        // pointwise 2x6 . 6x1 product; results overwrite polys 0..3 at the same slot
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int z = h ? z1 : z0;
#pragma unroll
            for (int l = 0; l < 2; l++) {
                uint64_t sg = 0, acc = 0;
#pragma unroll
                for (int p = 0; p < 6; p++) {
                    const uint32_t gv = G[(p * 2 + l) * N + z];
                    sg += gv;
                    acc += (uint64_t)body[(p * 2 + l) * N + z] * gv;
                }
                const uint32_t p0 = modq((uint64_t)row0[l * N + z] * modq(sg, l), l);
                const uint32_t p1 = modq(acc, l);
                G[(0 * 2 + l) * N + z] = p0;
                G[(1 * 2 + l) * N + z] = p1;
            }
        }
        __syncthreads();
        ntt_inverse_smem<4>(G, iw, iwp, [](int p) { return p & 1; });
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int z = h ? z1 : z0;
#pragma unroll
            for (int r = 0; r < 2; r++) {
                uint64_t v = crt2(G[(r * 2 + 0) * N + z], G[(r * 2 + 1) * N + z], c_q0inv, c_br[1]);
                v += pk[r][h];                      // < q + 2q
                v = v >= QQ ? v - QQ : v;
                v = v >= QQ ? v - QQ : v;
                s[r][h] = v;
            }
        }
        __syncthreads();
    }
    // switch_and_keep: stage s in smem as u64 then emit 7-byte (2 x 28 bit) and
    // 5-byte (2 x 20 bit) little-endian groups
    uint64_t* S64 = reinterpret_cast<uint64_t*>(G);
    S64[z0] = s[0][0]; S64[z1] = s[0][1];
    S64[N + z0] = s[1][0]; S64[N + z1] = s[1][1];
    __syncthreads();
    uint8_t* out = resp + (int64_t)q * resp_query_stride + (int64_t)wp * RESULT_BYTES;
    {
        const int t = threadIdx.x;  // fields 2t, 2t+1 of row 0 -> bytes [7t, 7t+7)
        const uint64_t v = rescale_dev(S64[2 * t], QP2) | (rescale_dev(S64[2 * t + 1], QP2) << 28);
#pragma unroll
        for (int b = 0; b < 7; b++) out[7 * t + b] = (uint8_t)(v >> (8 * b));
        const uint64_t w = rescale_dev(S64[N + 2 * t], QP1) | (rescale_dev(S64[N + 2 * t + 1], QP1) << 20);
#pragma unroll
        for (int b = 0; b < 5; b++) out[7 * N / 2 + 5 * t + b] = (uint8_t)(w >> (8 * b));
    }
}

// serialize_keyword_response framing: [u32 nq] { [u32 len] bytes }* [u32 nstash] { [u32 len] entry }*
__global__ void k_response_frame(uint8_t* __restrict__ resp_all, int nq, int64_t per_query_bytes,
                                 const uint8_t* __restrict__ stash, int64_t stash_count,
                                 int64_t stash_entry, int64_t pstride) {
    uint8_t* resp = resp_all + (int64_t)blockIdx.y * pstride;  // one payload per grid row
    auto put = [](uint8_t* p, uint32_t v) {
        p[0] = (uint8_t)v; p[1] = (uint8_t)(v >> 8); p[2] = (uint8_t)(v >> 16); p[3] = (uint8_t)(v >> 24);
    };
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t tail = 4 + (int64_t)nq * (4 + per_query_bytes);
    if (tid == 0) {
        put(resp, (uint32_t)nq);
        for (int q = 0; q < nq; q++) put(resp + 4 + q * (4 + per_query_bytes), (uint32_t)per_query_bytes);
        put(resp + tail, (uint32_t)stash_count);
    }
    const int64_t rec = 4 + stash_entry;
    for (int64_t i = tid; i < stash_count * rec; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = i / rec, o = i % rec;
        uint8_t* dst = resp + tail + 4 + e * rec;
        if (o < 4) dst[o] = (uint8_t)((uint32_t)stash_entry >> (8 * o));
        else dst[o] = stash[e * stash_entry + (o - 4)];
    }
}

// ---------------------------------------------------------------------------
// Standalone Galois expansion of a key body (the reference's
// gpu_rotation_expand_keys, rotation_kernel.cu:21-59), for the compatibility
// entry points and the automorphism microbenchmark.  Table-free.
// ---------------------------------------------------------------------------
__global__ void k_rotations(const uint64_t* __restrict__ y_body, uint64_t* __restrict__ y_all,
                            uint64_t* __restrict__ y_bar_all, int num_rotations) {
    const int i = blockIdx.x, k = blockIdx.y;
    uint32_t g = 1;
    for (int e = 0; e < i; e++) g = (g * 5) & (2 * N - 1);
    for (int z = threadIdx.x; z < N; z += blockDim.x) {
        const int64_t o = ((int64_t)i * T_EXP + k) * N + z;
        y_all[o] = y_body[k * N + auto_src(g, z)];
        y_bar_all[o] = y_body[k * N + auto_src(2 * N - g, z)];
    }
}

// packing from materialised y_all / y_bar_all (compat path of gpu_packing_online_compute)
__global__ void __launch_bounds__(256) k_pack_materialized(
    const uint64_t* __restrict__ bt, const uint64_t* __restrict__ btb, const uint64_t* __restrict__ bth,
    const uint64_t* __restrict__ y_all, const uint64_t* __restrict__ y_bar_all,
    const uint64_t* __restrict__ z_body, int num_outputs, int n_rot, uint64_t* __restrict__ out) {
    const int j = blockIdx.x;
    const int z = blockIdx.y * blockDim.x + threadIdx.x;
    if (j >= num_outputs || z >= N) return;
    const int n_inner = n_rot * T_EXP;
    const uint64_t* T = bt + (int64_t)j * n_inner * N;
    const uint64_t* Tb = btb + (int64_t)j * n_inner * N;
    uint64_t lo = 0, hi = 0;
    for (int r0 = 0; r0 < n_inner; r0 += 96) {
        const int r1 = r0 + 96 < n_inner ? r0 + 96 : n_inner;
        for (int r = r0; r < r1; r++) {
            const uint64_t y = y_all[(int64_t)r * N + z], t = T[(int64_t)r * N + z];
            const uint64_t yb = y_bar_all[(int64_t)r * N + z], tb = Tb[(int64_t)r * N + z];
            lo += (uint64_t)(uint32_t)y * (uint32_t)t + (uint64_t)(uint32_t)yb * (uint32_t)tb;
            hi += (y >> 32) * (t >> 32) + (yb >> 32) * (tb >> 32);
        }
        lo = modq(lo, 0);
        hi = modq(hi, 1);
    }
    for (int k = 0; k < T_EXP; k++) {
        const uint64_t zv = z_body[k * N + z], tv = bth[((int64_t)j * T_EXP + k) * N + z];
        lo += (uint64_t)(uint32_t)zv * (uint32_t)tv;
        hi += (zv >> 32) * (tv >> 32);
    }
    out[(int64_t)j * 2 * N + z] = modq(lo, 0);
    out[(int64_t)j * 2 * N + N + z] = modq(hi, 1);
}

// standalone negacyclic NTT / INTT over a batch of limb-major polynomial pairs
// ([poly][limb][N] u64 canonical), one CTA per pair (config: kernel microbench)
__global__ void __launch_bounds__(512) k_ntt_batch(uint64_t* __restrict__ data, int forward,
                                                   const uint32_t* __restrict__ w, const uint32_t* __restrict__ wp) {
    __shared__ uint32_t sm[2 * N];
    uint64_t* d = data + (int64_t)blockIdx.x * 2 * N;
    for (int i = threadIdx.x; i < 2 * N; i += blockDim.x) sm[i] = (uint32_t)d[i];
    __syncthreads();
    if (forward) ntt_forward_smem<2>(sm, w, wp, [](int p) { return p; });
    else ntt_inverse_smem<2>(sm, w, wp, [](int p) { return p; });
    for (int i = threadIdx.x; i < 2 * N; i += blockDim.x) d[i] = sm[i];
}

// ---------------------------------------------------------------------------
// seeded synthetic data (identical definition to the oracle's ipr_synth)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t synth(uint64_t seed, uint64_t stream, uint64_t idx) {
    uint64_t x = seed ^ (stream * 0x9E3779B97F4A7C15ull) ^ (idx * 0xD1B54A32D192ED03ull);
    x ^= x >> 30; x *= 0xBF58476D1CE4E5B9ull;
    x ^= x >> 27; x *= 0x94D049BB133111EBull;
    x ^= x >> 31;
    x += 0x9E3779B97F4A7C15ull;
    x ^= x >> 29; x *= 0xBF58476D1CE4E5B9ull;
    x ^= x >> 32;
    return x;
}

// element i of the output is element idx0 + i of the whole synthetic array (a fold-group
// shard of a larger synthetic server is generated alone)
__global__ void k_synth_db(uint16_t* db, int64_t n, uint64_t seed, uint64_t idx0) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        db[i] = (uint16_t)(synth(seed, 1, idx0 + (uint64_t)i) % PT);
}

__global__ void k_synth_condensed(uint64_t* out, int64_t n, uint64_t seed, uint64_t stream, uint64_t idx0) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t x = synth(seed, stream, idx0 + (uint64_t)i);
        out[i] = ((x & 0xffffffffull) % Q0) | (((x >> 32) % Q1) << 32);
    }
}

__global__ void k_synth_modq(uint64_t* out, int64_t n, uint64_t seed, uint64_t stream, uint64_t idx0) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = synth(seed, stream, idx0 + (uint64_t)i) % QQ;
}

// ---------------------------------------------------------------------------
// host launch wrappers
// ---------------------------------------------------------------------------
// per-device kernel attributes (dynamic shared memory above 48 KB); call once
// with the target device current
cudaError_t init_device_kernels() {
    cudaError_t e = cudaFuncSetAttribute(k_pack, cudaFuncAttributeMaxDynamicSharedMemorySize, T_EXP * N * 8);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_gemv_staged_f64<GSF_STAGES>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             gsf_smem(GF_MAX_ROWS));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_gemv_staged<GS_STAGES>, cudaFuncAttributeMaxDynamicSharedMemorySize, GS_SMEM);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_gemv_tma_f64, cudaFuncAttributeMaxDynamicSharedMemorySize, gt_smem());
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_fold_switch, cudaFuncAttributeMaxDynamicSharedMemorySize, 12 * N * 4);
}

namespace {
// the byte ranges one parse launch reads and writes (the bounds-checked build checks them
// against the allocations; the release build compiles the checks away)
cudaError_t parse_extents(const uint8_t* qb, int npay, int64_t pstride, int nq, int db_rows, const uint64_t* y,
                          const uint64_t* z, const uint32_t* a_il, const uint32_t* gsw, const uint8_t* qbytes,
                          int qbase) {
    const uint64_t fpp = 2ull * T_EXP * N + (uint64_t)nq * ((uint64_t)db_rows + 2ull * T_EXP * N);
    const uint64_t keys = (uint64_t)npay * T_EXP * N * 8;
    cudaError_t e;
    if ((e = check_extent(qb, (uint64_t)(npay - 1) * pstride + 1 + 7 * fpp, "parse: payloads")) != cudaSuccess ||
        (e = check_extent(y, keys, "parse: y bodies")) != cudaSuccess ||
        (e = check_extent(z, keys, "parse: z bodies")) != cudaSuccess ||
        (e = check_extent(gsw, (uint64_t)npay * nq * 12 * N * 4, "parse: RGSW bodies")) != cudaSuccess)
        return e;
    if (a_il && (e = check_extent(a_il, (uint64_t)(nq + 1) / 2 * db_rows * 4 * 4, "parse: GEMV operand")) != cudaSuccess)
        return e;
    if (qbytes &&
        (e = check_extent(qbytes, ((uint64_t)qbase + (uint64_t)npay * nq) * 7 * db_rows, "parse: query byte rows")) !=
            cudaSuccess)
        return e;
    return cudaSuccess;
}
}  // namespace

cudaError_t launch_parse_query(const uint8_t* qb, int nq, int db_rows, uint64_t* y, uint64_t* z,
                               uint32_t* a_il, uint32_t* gsw, uint8_t* qbytes, int qbase, cudaStream_t st) {
    cudaError_t e = parse_extents(qb, 1, 0, nq, db_rows, y, z, a_il, gsw, qbytes, qbase);
    if (e != cudaSuccess) return e;
    k_parse_query<<<2 * 148, 256, 0, st>>>(qb, nq, db_rows, y, z, a_il, gsw, qbytes, qbase, 1, 0);
    return cudaGetLastError();
}

cudaError_t launch_parse_batch(const uint8_t* qb, int npay, int64_t pstride, int nq, int db_rows, uint64_t* y,
                               uint64_t* z, uint32_t* gsw, uint8_t* qbytes, cudaStream_t st) {
    cudaError_t e = parse_extents(qb, npay, pstride, nq, db_rows, y, z, nullptr, gsw, qbytes, 0);
    if (e != cudaSuccess) return e;
    k_parse_query<<<8 * 148, 256, 0, st>>>(qb, nq, db_rows, y, z, nullptr, gsw, qbytes, 0, npay, pstride);
    return cudaGetLastError();
}

cudaError_t launch_gemv(const uint16_t* db, int db_rows, int64_t db_cols, int nq, const uint32_t* a_il,
                        uint64_t* c, int sm_count, cudaStream_t st, int form, int* err_flag) {
    const int blocks = sm_count * 4;
    cudaError_t e;
    if ((e = check_extent(db, (uint64_t)db_rows * db_cols * 2, "GEMV: DB")) != cudaSuccess ||
        (e = check_extent(a_il, (uint64_t)db_rows * nq * 8, "GEMV: query residues")) != cudaSuccess ||
        (e = check_extent(c, (uint64_t)nq * db_cols * 8, "GEMV: outputs")) != cudaSuccess)
        return e;
    if (nq == 2 && form == 6 && (!err_flag || (db_rows % (GT_WARPS * GT_ROWS)) || db_rows > (1 << 18)))
        form = db_rows <= 16384 ? 5 : 0;  // the forms whose sums stay exact at these rows
    if (nq == 2 && form == 6) {
        CUtensorMap tm;
        if ((e = make_u16_col_map(&tm, db, db_rows, db_cols, GT_ROWS, GT_COLS)) != cudaSuccess) return e;
        const int64_t ntiles = (db_cols + GT_COLS - 1) / GT_COLS;
        const int grid = ntiles < sm_count ? (int)ntiles : sm_count;
        k_gemv_tma_f64<<<grid, GT_WARPS * 32, gt_smem(), st>>>(tm, db_rows, db_cols, a_il, c, err_flag);
    } else if (nq == 2 && form == 0) k_gemv<2, 8><<<blocks, 256, 0, st>>>(db, db_rows, db_cols, a_il, c);
    else if (nq == 2 && form == 1) k_gemv<2, 4, 2><<<sm_count * 2, 256, 0, st>>>(db, db_rows, db_cols, a_il, c);
    else if (nq == 2 && form == 2) k_gemv<2, 2, 3><<<sm_count * 3, 256, 0, st>>>(db, db_rows, db_cols, a_il, c);
    else if (nq == 2 && form == 3)
        k_gemv_staged<GS_STAGES><<<sm_count, GS_WARPS * 32, GS_SMEM, st>>>(db, db_rows, db_cols, a_il, c);
    else if (nq == 2 && (form == 4 || form == 5) && db_rows > 16384)  // the FP64 sums would pass 2^53
        return cudaErrorInvalidValue;
    else if (nq == 2 && form == 4) k_gemv<2, 8, 1, 1><<<blocks, 256, 0, st>>>(db, db_rows, db_cols, a_il, c);
    else if (nq == 2 && form == 5 && db_rows <= GF_MAX_ROWS)
        k_gemv_staged_f64<GSF_STAGES><<<sm_count, GS_WARPS * 32, gsf_smem(db_rows), st>>>(db, db_rows, db_cols, a_il,
                                                                                           c);
    else if (nq == 2 && form == 5) k_gemv<2, 8, 1, 1><<<blocks, 256, 0, st>>>(db, db_rows, db_cols, a_il, c);
    else if (nq == 1) k_gemv<1, 16><<<blocks, 256, 0, st>>>(db, db_rows, db_cols, a_il, c);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
}

cudaError_t launch_pack(const uint64_t* bt, const uint64_t* btb, const uint64_t* bth, const uint64_t* y,
                        const uint64_t* z, uint32_t* S, int num_outputs, cudaStream_t st) {
    const int smem = T_EXP * N * 8;
    dim3 grid(N / PACK_ZB, num_outputs);
    k_pack<<<grid, PACK_THREADS, smem, st>>>(bt, btb, bth, y, z, S);
    return cudaGetLastError();
}

cudaError_t launch_intt_crt(const uint32_t* S, const uint32_t* iw, const uint32_t* iwp, uint64_t* R,
                            int num_outputs, cudaStream_t st, const uint64_t* z_bodies, const uint64_t* bth,
                            int instances) {
    k_intt_crt<<<(num_outputs + INTT_P - 1) / INTT_P, 512, 0, st>>>(S, iw, iwp, R, num_outputs, z_bodies, bth,
                                                                    instances);
    return cudaGetLastError();
}

cudaError_t launch_fold_switch(const uint32_t* row0, const uint32_t* gsw, const uint64_t* a_hat,
                               const uint64_t* R, const uint64_t* cvec, const uint32_t* fw,
                               const uint32_t* fwp, const uint32_t* iw, const uint32_t* iwp, int interp,
                               int c_groups, int nq, int64_t db_cols, uint8_t* resp,
                               int64_t resp_query_stride, cudaStream_t st) {
    const int smem = 12 * N * 4;
    dim3 grid(c_groups, nq);
    k_fold_switch<<<grid, FOLD_THREADS, smem, st>>>(row0, gsw, a_hat, R, cvec, fw, fwp, iw, iwp, interp,
                                                    c_groups, db_cols, resp, resp_query_stride);
    return cudaGetLastError();
}

cudaError_t launch_response_frame(uint8_t* resp, int nq, int64_t per_query, const uint8_t* stash,
                                  int64_t stash_count, int64_t stash_entry, cudaStream_t st, int npay,
                                  int64_t pstride) {
    const uint64_t frame = 4 + (uint64_t)nq * (4 + per_query) + 4 + (uint64_t)stash_count * (4 + stash_entry);
    cudaError_t e;
    if ((e = check_extent(resp, (uint64_t)(npay - 1) * pstride + frame, "frame: responses")) != cudaSuccess ||
        (e = check_extent(stash, (uint64_t)stash_count * stash_entry, "frame: stash")) != cudaSuccess)
        return e;
    k_response_frame<<<dim3(8, npay), 256, 0, st>>>(resp, nq, per_query, stash, stash_count, stash_entry, pstride);
    return cudaGetLastError();
}

cudaError_t launch_rotations(const uint64_t* y_body, uint64_t* y_all, uint64_t* y_bar_all, int num_rotations,
                             cudaStream_t st) {
    dim3 grid(num_rotations, T_EXP);
    k_rotations<<<grid, 256, 0, st>>>(y_body, y_all, y_bar_all, num_rotations);
    return cudaGetLastError();
}

cudaError_t launch_pack_materialized(const uint64_t* bt, const uint64_t* btb, const uint64_t* bth,
                                     const uint64_t* y_all, const uint64_t* y_bar_all, const uint64_t* z,
                                     int num_outputs, int n_rot, uint64_t* out, cudaStream_t st) {
    dim3 grid(num_outputs, N / 256);
    k_pack_materialized<<<grid, 256, 0, st>>>(bt, btb, bth, y_all, y_bar_all, z, num_outputs, n_rot, out);
    return cudaGetLastError();
}

cudaError_t launch_ntt_batch(uint64_t* data, int npairs, int forward, const uint32_t* w, const uint32_t* wp,
                             cudaStream_t st) {
    k_ntt_batch<<<npairs, 512, 0, st>>>(data, forward, w, wp);
    return cudaGetLastError();
}

cudaError_t launch_synth_db(uint16_t* db, int64_t n, uint64_t seed, cudaStream_t st, uint64_t idx0) {
    k_synth_db<<<148 * 8, 256, 0, st>>>(db, n, seed, idx0);
    return cudaGetLastError();
}
cudaError_t launch_synth_condensed(uint64_t* out, int64_t n, uint64_t seed, uint64_t stream, cudaStream_t st,
                                   uint64_t idx0) {
    k_synth_condensed<<<148 * 8, 256, 0, st>>>(out, n, seed, stream, idx0);
    return cudaGetLastError();
}
cudaError_t launch_synth_modq(uint64_t* out, int64_t n, uint64_t seed, uint64_t stream, cudaStream_t st,
                              uint64_t idx0) {
    k_synth_modq<<<148 * 8, 256, 0, st>>>(out, n, seed, stream, idx0);
    return cudaGetLastError();
}

}  // namespace ipr
