// encode.cu — setup-time database layout and encode on the GPU.
//
// k_raw_db:    KeywordCuckooTable::to_raw_db (rkdud007/inspire-rs
//              src/pir/keyword/cuckoo.rs:314-353): bucket entries (row-major bytes) ->
//              the column-major u16 raw DB, big-endian u16 per byte pair, zero for empty
//              buckets.
// k_encode<I>: gpu_encode_db (native/cuda/encode_kernel.cu:18-228, 264-386): per DB row
//              and fold group, the I = interp polynomials of columns wp*I*N + j*N + k are
//              interpolated by a radix-2 Cooley-Tukey pass over Z_65535[X]/(X^N + 1) with
//              monomial twiddles, then scaled by I^-1 mod 65535.
//
// B200 design.  Every twiddle X^e of the pass has e a multiple of S = 2N/I, so a shift
// moves whole chunks of S coefficients and keeps the offset o = k mod S: the pass
// splits into S independent sub-problems of I polynomials x I/2 chunks.  One CTA takes
// 32 DB rows x one (fold group, offset): it reads its 32 x I x I/2 values once (16-byte
// accesses of 8 rows, 64 bytes per column), runs all log2(I) levels in shared memory
// (in place: each step reads its inputs into registers before a barrier, 8 rows
// per thread and step), scales, and writes them back once — one HBM
// round trip for the whole encode where the reference makes one per level plus a
// gather and a scatter.
#include <cuda_runtime.h>

#include <cstdint>

#include "ipr_b200.h"
#include "ipr_device.cuh"

namespace ipr {
void set_last_error(const char* msg);

namespace {

constexpr int E_ROWS = 32;  // DB rows per CTA (four 16-byte groups per column)
constexpr uint32_t PMOD = 65535;

__device__ __forceinline__ uint32_t fold65535(uint32_t x) {
    uint32_t r = (x & 0xFFFFu) + (x >> 16);
    r = (r & 0xFFFFu) + (r >> 16);
    return r >= PMOD ? r - PMOD : r;
}

// raw[(item * ise + j) * db_rows + row] for bucket row * per + item; one CTA per
// (32 rows, item): the 32 entries are staged in shared memory and written column-wise
__global__ void __launch_bounds__(256) k_raw_db(const uint8_t* __restrict__ entries,
                                                const uint8_t* __restrict__ occupied, int64_t num_buckets,
                                                int entry_size, int64_t db_rows, int64_t per,
                                                uint16_t* __restrict__ raw) {
    extern __shared__ uint8_t ent[];  // [32][stride]: an odd word count per row spreads the column reads
    const int stride = (entry_size + 3) / 4 * 4 + 4;
    const int64_t item = blockIdx.y;
    const int64_t row0 = (int64_t)blockIdx.x * 32;
    for (int i = threadIdx.x; i < 32 * entry_size; i += blockDim.x) {
        const int r = i / entry_size, byte = i % entry_size;
        const int64_t row = row0 + r, b = row * per + item;
        ent[r * stride + byte] = (row < db_rows && b < num_buckets && occupied[b]) ? entries[b * entry_size + byte] : 0;
    }
    __syncthreads();
    const int ise = entry_size / 2;
    for (int i = threadIdx.x; i < 32 * ise; i += blockDim.x) {
        const int r = i & 31, j = i >> 5;
        const int64_t row = row0 + r;
        if (row >= db_rows) continue;
        const uint16_t v = (uint16_t)(((uint16_t)ent[r * stride + 2 * j] << 8) | ent[r * stride + 2 * j + 1]);
        raw[(item * ise + j) * db_rows + row] = v;
    }
}

// interp = 1: the pass is empty, the scale is 1: values reduced mod 65535
__global__ void k_encode_scale1(const uint16_t* __restrict__ in, uint16_t* __restrict__ out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (uint16_t)fold65535(in[i]);
}

// a + b mod 65535 on both 16-bit halves (ones'-complement sum: the carry out of a half is
// added back into it; operands and result in [0, 65535] with 65535 = 0).  One 64-bit add
// gives the high half's carry c1 and the carry c0 out of the low half (bit 16 of
// s ^ a ^ b); c0 moves from the high half back into the low one, c1 re-enters the high
// half, and neither re-addition can carry again.
__device__ __forceinline__ uint32_t oadd2(uint32_t a, uint32_t b) {
    const uint64_t s64 = (uint64_t)a + b;
    const uint32_t s = (uint32_t)s64;
    const uint32_t c1 = (uint32_t)(s64 >> 32);
    const uint32_t c0 = ((s ^ a ^ b) >> 16) & 1u;
    return s + c0 * 0xFFFF0001u + (c1 << 16);
}

// x * 2^K mod 65535 on both halves, canonical (65535 -> 0): multiplying by 2^K modulo
// 2^16 - 1 rotates the 16 bits left by K; afterwards a half that is all ones (a zero
// in ones'-complement form) is cleared
template <int K>
__device__ __forceinline__ uint32_t rotl_canon2(uint32_t w) {
    constexpr uint32_t HI = ((0xFFFFu << K) & 0xFFFFu) * 0x10001u, LO = ((1u << K) - 1) * 0x10001u;
    w = ((w << K) & HI) | ((w >> (16 - K)) & LO);
    const uint32_t nw = ~w;
    const uint32_t nz = ((nw & 0x7FFF7FFFu) + 0x7FFF7FFFu) | nw;  // bit 15 of a half: that half of nw != 0
    const uint32_t ones = ~nz & 0x80008000u;
    return w & ~((ones >> 15) * 0xFFFFu);
}

constexpr int E_THREADS = 256;

template <int I>
__global__ void __launch_bounds__(E_THREADS) k_encode(const uint16_t* __restrict__ in, uint16_t* __restrict__ out,
                                                      int64_t db_rows) {
    constexpr int H = I / 2;        // chunks of S coefficients in [0, N)
    constexpr int S = 2 * N / I;    // coefficient stride between chunks
    constexpr int RG = E_ROWS / 8;  // 8-row groups per column
    constexpr int GROUPS = I * H * RG;
    constexpr int BFLY = (I / 2) * H * RG;  // butterflies (of 8 rows) per level
    constexpr int BPT = (BFLY + E_THREADS - 1) / E_THREADS;
    constexpr int LOGI = I == 2 ? 1 : I == 4 ? 2 : I == 8 ? 3 : I == 16 ? 4 : 5;
    __shared__ __align__(16) uint16_t buf[I][H][E_ROWS];  // [poly][chunk][row], 32 KB at interp 32
    // row tiles vary fastest: the CTAs resident together read whole 4 KB columns between them
    const int64_t row0 = (int64_t)blockIdx.x * E_ROWS;
    const int o = blockIdx.y;         // offset within a chunk, < S
    const int64_t wp = blockIdx.z;    // fold group
    const int64_t col0 = wp * I * N + o;

    // gather in bit-reversed polynomial order, 16 bytes (8 rows) per access; the loads of
    // a thread are all issued before the first store
    {
        constexpr int LPT = (GROUPS + E_THREADS - 1) / E_THREADS;
        uint4 v[LPT];
#pragma unroll
        for (int u = 0; u < LPT; u++) {
            const int i = threadIdx.x + u * E_THREADS;
            if (GROUPS % E_THREADS == 0 || i < GROUPS) {
                const int rg = i % RG, q = i / RG;
                const int j = q / H, kc = q % H;
                v[u] = __ldg(reinterpret_cast<const uint4*>(in + (col0 + (int64_t)j * N + (int64_t)kc * S) * db_rows +
                                                            row0 + rg * 8));
            }
        }
#pragma unroll
        for (int u = 0; u < LPT; u++) {
            const int i = threadIdx.x + u * E_THREADS;
            if (GROUPS % E_THREADS == 0 || i < GROUPS) {
                const int rg = i % RG, q = i / RG;
                const int j = q / H, kc = q % H;
                const int jr = (int)(__brev((unsigned)j) >> (32 - LOGI));
                *reinterpret_cast<uint4*>(&buf[jr][kc][rg * 8]) = v[u];
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int lv = 0; lv < LOGI; lv++) {
        const int gs = 2 << lv, half = 1 << lv;
        // each butterfly reads its two inputs into registers; after a barrier all outputs
        // overwrite them in place
        uint4 ra[BPT], rb[BPT];
#pragma unroll
        for (int u = 0; u < BPT; u++) {
            const int i = threadIdx.x + u * E_THREADS;
            if (BFLY % E_THREADS == 0 || i < BFLY) {
                const int rg = i % RG, rest = i / RG;
                const int kc = rest % H, pr = rest / H;
                const int g = pr / half, t = pr % half;
                const int ev = g * gs + t, od = ev + half;
                const int e = (2 * N - 2 * N * t / gs) % (2 * N);  // twiddle X^e, e a multiple of S
                const int src = (kc + I - e / S) % I;                // chunk of coefficient k - e (mod 2N)
                // two values per 32-bit word in ones'-complement form (65535 stands for 0):
                // -x is ~x and a sum folds its carry back in, so the butterfly runs on packed halves
                const uint4 ov = *reinterpret_cast<const uint4*>(&buf[od][src < H ? src : src - H][rg * 8]);
                const uint4 evv = *reinterpret_cast<const uint4*>(&buf[ev][kc][rg * 8]);
                const bool neg = src >= H;  // X^N = -1
                const uint4 tw = neg ? make_uint4(~ov.x, ~ov.y, ~ov.z, ~ov.w) : ov;
                ra[u] = make_uint4(oadd2(evv.x, tw.x), oadd2(evv.y, tw.y), oadd2(evv.z, tw.z), oadd2(evv.w, tw.w));
                rb[u] = make_uint4(oadd2(evv.x, ~tw.x), oadd2(evv.y, ~tw.y), oadd2(evv.z, ~tw.z), oadd2(evv.w, ~tw.w));
            }
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < BPT; u++) {
            const int i = threadIdx.x + u * E_THREADS;
            if (BFLY % E_THREADS == 0 || i < BFLY) {
                const int rg = i % RG, rest = i / RG;
                const int kc = rest % H, pr = rest / H;
                const int ev = pr / half * gs + pr % half;
                *reinterpret_cast<uint4*>(&buf[ev][kc][rg * 8]) = ra[u];
                *reinterpret_cast<uint4*>(&buf[ev + half][kc][rg * 8]) = rb[u];
            }
        }
        __syncthreads();
    }
    // scale by I^-1 = 2^(16 - log2 I) mod 65535 and store in natural polynomial order
#pragma unroll 4
    for (int i = threadIdx.x; i < GROUPS; i += E_THREADS) {
        const int rg = i % RG, q = i / RG;
        const int j = q / H, kc = q % H;
        uint4 w = *reinterpret_cast<const uint4*>(&buf[j][kc][rg * 8]);
        w = make_uint4(rotl_canon2<16 - LOGI>(w.x), rotl_canon2<16 - LOGI>(w.y), rotl_canon2<16 - LOGI>(w.z),
                       rotl_canon2<16 - LOGI>(w.w));
        *reinterpret_cast<uint4*>(out + (col0 + (int64_t)j * N + (int64_t)kc * S) * db_rows + row0 + rg * 8) = w;
    }
}

int cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return IPR_OK;
    set_last_error(cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? IPR_E_OOM : IPR_E_CUDA;
}

}  // namespace

// interp^-1 mod 65535 for interp a power of two (2^16 = 1 mod 65535)
uint32_t encode_num_inv(uint64_t interp) {
    uint32_t inv = 1;
    unsigned logi = 0;
    while ((1ull << logi) < interp) logi++;
    for (unsigned b = 0; b < (16 - logi) % 16; b++) inv = (inv * 2) % PMOD;
    return inv;
}

int encode_db_device(const uint16_t* d_raw, uint16_t* d_out, uint64_t db_rows, uint64_t db_cols, uint64_t interp,
                     cudaStream_t st) {
    if (!d_raw || !d_out || !interp || (interp & (interp - 1)) || interp > 32 || db_rows % E_ROWS ||
        db_cols % (interp * N) || (reinterpret_cast<uintptr_t>(d_raw) | reinterpret_cast<uintptr_t>(d_out)) % 16) {
        set_last_error("encode: interp must be a power of two <= 32, db_rows a multiple of 32, db_cols of "
                       "interp*2048, buffers 16-byte aligned");
        return IPR_E_ARGS;
    }
    if (d_raw == d_out) {
        set_last_error("encode: input and output must differ");
        return IPR_E_ARGS;
    }
    const uint64_t c = db_cols / (interp * N);
    if (c > 65535 || 2 * N / interp > 65535) {
        set_last_error("encode: shape too large for one launch");
        return IPR_E_ARGS;
    }
    if (interp == 1) {
        k_encode_scale1<<<148 * 8, 256, 0, st>>>(d_raw, d_out, (int64_t)(db_rows * db_cols));
    } else {
        const dim3 grid((unsigned)(db_rows / E_ROWS), (unsigned)(2 * N / interp), (unsigned)c);
        switch (interp) {
            case 2: k_encode<2><<<grid, E_THREADS, 0, st>>>(d_raw, d_out, (int64_t)db_rows); break;
            case 4: k_encode<4><<<grid, E_THREADS, 0, st>>>(d_raw, d_out, (int64_t)db_rows); break;
            case 8: k_encode<8><<<grid, E_THREADS, 0, st>>>(d_raw, d_out, (int64_t)db_rows); break;
            case 16: k_encode<16><<<grid, E_THREADS, 0, st>>>(d_raw, d_out, (int64_t)db_rows); break;
            default: k_encode<32><<<grid, E_THREADS, 0, st>>>(d_raw, d_out, (int64_t)db_rows); break;
        }
    }
    return cuda_status(cudaGetLastError());
}

int raw_db_device(const uint8_t* d_entries, const uint8_t* d_occupied, uint64_t num_buckets, uint64_t entry_size,
                  uint64_t db_rows, uint64_t db_cols, uint64_t per, uint16_t* d_raw, cudaStream_t st) {
    if (!d_entries || !d_occupied || !d_raw || entry_size < 2 || entry_size % 2 || entry_size > 6144 || !per ||
        per * (entry_size / 2) > db_cols || per > 65535) {
        set_last_error("cuckoo_to_raw_db: bad shape (entry size even and <= 6144, per * entry_size/2 <= db_cols)");
        return IPR_E_ARGS;
    }
    int st0 = cuda_status(cudaMemsetAsync(d_raw, 0, db_rows * db_cols * sizeof(uint16_t), st));
    if (st0) return st0;
    const int smem = 32 * ((int)(entry_size + 3) / 4 * 4 + 4);
    st0 = cuda_status(cudaFuncSetAttribute(k_raw_db, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    if (st0) return st0;
    const dim3 grid((unsigned)((db_rows + 31) / 32), (unsigned)per);
    k_raw_db<<<grid, 256, smem, st>>>(d_entries, d_occupied, (int64_t)num_buckets, (int)entry_size, (int64_t)db_rows,
                                      (int64_t)per, d_raw);
    return cuda_status(cudaGetLastError());
}

}  // namespace ipr

extern "C" {

int ipr_encode_db(int device, const uint16_t* d_raw, uint16_t* d_encoded, uint64_t db_rows, uint64_t db_cols,
                  uint64_t interp, void* stream) {
    int st = ipr::cuda_status(cudaSetDevice(device));
    if (st) return st;
    return ipr::encode_db_device(d_raw, d_encoded, db_rows, db_cols, interp, static_cast<cudaStream_t>(stream));
}

int ipr_cuckoo_to_raw_db(int device, const uint8_t* d_entries, const uint8_t* d_occupied, uint64_t num_buckets,
                         uint64_t entry_size, uint64_t db_rows, uint64_t db_cols, uint64_t per, uint16_t* d_raw,
                         void* stream) {
    int st = ipr::cuda_status(cudaSetDevice(device));
    if (st) return st;
    return ipr::raw_db_device(d_entries, d_occupied, num_buckets, entry_size, db_rows, db_cols, per, d_raw,
                              static_cast<cudaStream_t>(stream));
}

}  // extern "C"
