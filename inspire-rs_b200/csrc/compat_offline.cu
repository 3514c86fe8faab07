// compat_offline.cu — the reference's offline-precomputation FFI, same symbol names,
// arguments and results (rkdud007/inspire-rs src/pir/gpu/hint.rs, prep_pack.rs,
// packing.rs, collapse.rs; native/cuda/hint_kernel.cu, prep_pack_kernel.cu,
// packing_kernel.cu, collapse_kernel.cu), so the Rust crate's GPU setup path
// (engine.rs:749-940) runs on this library unchanged.  Like the reference, the state
// lives in process-wide statics, calls return void and failures print to stderr (and
// set ipr_last_error()).
//
// The arithmetic is this library's: register NTTs for the hint and prep_pack columns,
// the packing sums as one NTT over j per slot followed by a slot gather when
// gpu_packing_setup receives the canonical tables (monomial NTTs, the gen_pows index
// tables, N^-1) — every caller in the reference passes those — and a direct sum over the
// given tables otherwise; the collapse is the offline path's chain kernel fed with the
// given W rows.  Outputs are canonical, so they equal the reference kernels' bit for bit.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "host_math.hpp"
#include "ipr_b200.h"
#include "ipr_b200_compat.h"
#include "ipr_device.cuh"
#include "ntt_regs.cuh"

namespace ipr {
void set_last_error(const char* msg);
cudaError_t offline_collapse_arrays(const uint64_t* r_all, const uint64_t* r_bar_all, int64_t cols,
                                    const uint32_t* wrows, const uint32_t* vmask, const uint32_t* tab, uint32_t* F,
                                    uint32_t* r0, uint64_t* xb, uint64_t* bt, uint64_t* btb, uint64_t* bth,
                                    uint64_t* a_hat, cudaStream_t st);
cudaError_t narrow_u64(const uint64_t* in, int64_t n, uint32_t* out, cudaStream_t st);
cudaError_t offline_jntt(const uint32_t* act, int64_t inst, const uint32_t* fw, const uint32_t* fwp, uint32_t* E,
                         cudaStream_t st);

namespace {

using nttr::eA;
using nttr::eD;
using nttr::EPT;
constexpr int CC = 2 * N;    // coefficients of a 2-limb polynomial
constexpr int HALF = N / 2;  // num_to_pack_half
constexpr int XC = 4;        // columns per CTA in the column transforms

bool report(cudaError_t e, const char* where) {
    if (e == cudaSuccess) return false;
    char buf[256];
    snprintf(buf, sizeof(buf), "%s: %s", where, cudaGetErrorString(e));
    set_last_error(buf);
    fprintf(stderr, "[ipr_b200] %s\n", buf);
    return true;
}
void report_msg(const char* msg) {
    set_last_error(msg);
    fprintf(stderr, "[ipr_b200] %s\n", msg);
}
template <typename T>
void dfree(T*& p) {
    if (p) cudaFree(p);
    p = nullptr;
}

// the reference's table layout [limb][fwd, fwd', inv, inv'][N] (u64) -> fw, fwp, iw, iwp [limb][N] (u32)
__global__ void k_tab32(const uint64_t* __restrict__ t64, uint32_t* __restrict__ t32) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < 2 * 4 * N; e += gridDim.x * blockDim.x) {
        const int l = e / (4 * N), kind = (e / N) % 4, i = e % N;
        t32[(kind * 2 + l) * N + i] = (uint32_t)t64[e];
    }
}

// hint column c = raw(sum_row NTT(DB chunk) * query[row]) (hint_multiply_kernel,
// hint_kernel.cu:23-260 / multiply_with_db_ring), stored transposed [z][db_cols] as the
// reference stores it: XC columns per CTA, a limb per 256 threads
__global__ void __launch_bounds__(512, 1)
    k_hint_raw(const uint16_t* __restrict__ db, int64_t db_rows, int64_t ncols, const uint32_t* __restrict__ query,
               const uint32_t* __restrict__ tab, uint64_t* __restrict__ out) {
    extern __shared__ uint32_t csm[];  // [2 groups][XC][N]
    const int g = threadIdx.x >> 8, t = threadIdx.x & 255;
    const uint32_t q = g ? Q1 : Q0;
    const uint64_t br = g ? BR1 : BR0;
    uint32_t* xbuf = csm + g * XC * N;
    const uint32_t *fw = tab + g * N, *fwp = tab + 2 * N + g * N, *iw = tab + 4 * N + g * N,
                   *iwp = tab + 6 * N + g * N;
    const int64_t c0 = (int64_t)blockIdx.x * XC;
    const int polys = (int)(db_rows / N);
    uint32_t acc[XC][EPT];
#pragma unroll
    for (int p = 0; p < XC; p++)
#pragma unroll
        for (int m = 0; m < EPT; m++) acc[p][m] = 0;
    for (int row = 0; row < polys; row++) {
        uint32_t v[XC][EPT];
#pragma unroll
        for (int p = 0; p < XC; p++) {
            const bool live = c0 + p < ncols;
            const uint16_t* col = db + (live ? c0 + p : 0) * db_rows + (int64_t)row * N;
#pragma unroll
            for (int m = 0; m < EPT; m++) v[p][m] = live ? (uint32_t)__ldg(col + eA(t, m)) : 0u;
        }
        nttr::forward<XC>(v, t, xbuf, 1 + g, fw, fwp, q);
        const uint32_t* qr = query + ((int64_t)row * 2 + g) * N;
#pragma unroll
        for (int p = 0; p < XC; p++)
#pragma unroll
            for (int m = 0; m < EPT; m++) acc[p][m] = mod64((uint64_t)v[p][m] * __ldg(qr + eD(t, m)) + acc[p][m], q, br);
    }
    nttr::inverse<XC>(acc, t, xbuf, 1 + g, iw, iwp, q);  // layout A, canonical
    __syncthreads();
#pragma unroll
    for (int p = 0; p < XC; p++)
#pragma unroll
        for (int m = 0; m < EPT; m++) xbuf[p * N + eA(t, m)] = acc[p][m];
    __syncthreads();
    // transposed, as the reference leaves it for prep_pack: out[z][column]
    for (int e = threadIdx.x; e < XC * N; e += 512) {
        const int z = e / XC, p = e % XC;
        if (c0 + p < ncols) out[(int64_t)z * ncols + c0 + p] = crt2(csm[p * N + z], csm[XC * N + p * N + z], Q0INV, BR1);
    }
}

// prepacked column c = NTT(negacyclic_perm(hint column c)) (prep_pack_kernel.cu:22-117 /
// prep_pack_lwes): coefficient 0 stays, k >= 1 takes q - h[N - k]; modulo q_l that is -h[N - k]
__global__ void __launch_bounds__(512, 1)
    k_prep_pack64(const uint64_t* __restrict__ hint, int64_t ncols, const uint32_t* __restrict__ tab,
                  uint64_t* __restrict__ out) {
    extern __shared__ uint32_t psm[];
    const int g = threadIdx.x >> 8, t = threadIdx.x & 255;
    const uint32_t q = g ? Q1 : Q0;
    const uint64_t br = g ? BR1 : BR0;
    const int64_t c0 = (int64_t)blockIdx.x * XC;
    uint32_t v[XC][EPT];
#pragma unroll
    for (int p = 0; p < XC; p++) {
        const bool live = c0 + p < ncols;
        const uint64_t* h = hint + (live ? c0 + p : 0);  // hint[z][column] (transposed)
#pragma unroll
        for (int m = 0; m < EPT; m++) {
            const int k = eA(t, m);
            const uint32_t x = live ? mod64(__ldg(h + (int64_t)(k ? N - k : 0) * ncols), q, br) : 0u;
            v[p][m] = (k == 0 || x == 0) ? x : q - x;
        }
    }
    nttr::forward<XC>(v, t, psm + g * XC * N, 1 + g, tab + g * N, tab + 2 * N + g * N, q);
#pragma unroll
    for (int p = 0; p < XC; p++) {
        if (c0 + p >= ncols) break;
        uint64_t* dst = out + (c0 + p) * CC + g * N;
#pragma unroll
        for (int k = 0; k < EPT; k++) dst[eD(t, k)] = v[p][k];
    }
}

// direct packing sums over the given tables (packing_mul_acc_kernel + scalar_mul_kernel,
// packing_kernel.cu:20-110): r[i][k] = N^-1-scaled sum_j mono[idx[i][j]][k] * a[j][k], four
// rows i per thread so each a[j][k] load feeds four products of each sum
__global__ void __launch_bounds__(256)
    k_pack_direct(const uint64_t* __restrict__ mono, const uint64_t* __restrict__ a_ct, const int* __restrict__ idx,
                  const int* __restrict__ idx_bar, const uint64_t* __restrict__ mod_inv, int nph, int nz, int cc,
                  int poly_len, uint64_t q0, uint64_t q1, int64_t a_stride, int64_t out_stride,
                  uint64_t* __restrict__ r_out, uint64_t* __restrict__ rb_out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int i0 = blockIdx.y * 4;
    const int64_t b = blockIdx.z;
    if (k >= cc) return;
    const uint64_t q = (k / poly_len) ? q1 : q0;
    const uint64_t br = (uint64_t)(~0ull / q);  // floor((2^64 - 1) / q) = floor(2^64 / q) for q not a power of 2
    const uint64_t* a = a_ct + b * a_stride;
    uint64_t acc[4], accb[4];
#pragma unroll
    for (int ii = 0; ii < 4; ii++) acc[ii] = accb[ii] = 0;
    for (int j = 0; j < nz; j++) {
        const uint64_t av = (uint32_t)__ldg(a + (int64_t)j * cc + k);
#pragma unroll
        for (int ii = 0; ii < 4; ii++) {
            if (i0 + ii >= nph) break;
            const int mi = __ldg(idx + (int64_t)(i0 + ii) * nz + j), mb = __ldg(idx_bar + (int64_t)(i0 + ii) * nz + j);
            acc[ii] += (uint64_t)(uint32_t)__ldg(mono + (int64_t)mi * cc + k) * av;
            accb[ii] += (uint64_t)(uint32_t)__ldg(mono + (int64_t)mb * cc + k) * av;
        }
        if ((j & 63) == 63)  // 64 products < 2^64 before each reduction
#pragma unroll
            for (int ii = 0; ii < 4; ii++) {
                acc[ii] = mod64(acc[ii], (uint32_t)q, br);
                accb[ii] = mod64(accb[ii], (uint32_t)q, br);
            }
    }
    const uint64_t inv = __ldg(mod_inv + k) % q;
#pragma unroll
    for (int ii = 0; ii < 4; ii++) {
        if (i0 + ii >= nph) break;
        r_out[b * out_stride + (int64_t)(i0 + ii) * cc + k] = mod64(mod64(acc[ii], (uint32_t)q, br) * inv, (uint32_t)q, br);
        rb_out[b * out_stride + (int64_t)(i0 + ii) * cc + k] =
            mod64(mod64(accb[ii], (uint32_t)q, br) * inv, (uint32_t)q, br);
    }
}

// act[l][j][s] (u32) from prepacked a_ct[j][l*N + s] (u64) of one column group
__global__ void k_act_from_u64(const uint64_t* __restrict__ a_ct, uint32_t* __restrict__ act) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)N * CC;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = e / CC, ls = e % CC;
        act[(ls / N) * (int64_t)N * N + j * N + (ls % N)] = (uint32_t)a_ct[e];
    }
}

// the packing sums before the automorphisms from E = N^-1 NTT_j: r_i[s] = E[s][tau_{g'_i}(s)],
// r_bar_i[s] = E[s][tau_{-g'_i}(s)], g'_i = 5^((N - i) mod N); 8 rows s per CTA (one limb)
__global__ void __launch_bounds__(256) k_pre_gather(const uint32_t* __restrict__ E, uint64_t* __restrict__ r_out,
                                                    uint64_t* __restrict__ rb_out) {
    extern __shared__ __align__(16) uint32_t rows[];  // [8][N]
    const int s0 = blockIdx.x * 8, l = blockIdx.y;
    for (int e = threadIdx.x; e < 8 * N; e += 256) rows[e] = E[((int64_t)l * N + s0) * N + e];
    __syncthreads();
    for (int e = threadIdx.x; e < HALF * 8; e += 256) {
        const int i = e >> 3, ss = e & 7;
        uint32_t gp = 1, bb = 5;
        for (uint32_t x = (uint32_t)((N - i) % N); x; x >>= 1, bb = (bb * bb) & (2 * N - 1))
            if (x & 1) gp = (gp * bb) & (2 * N - 1);
        const uint32_t s = (uint32_t)(s0 + ss);
        r_out[(int64_t)i * CC + l * N + s] = rows[ss * N + auto_src(gp, s)];
        rb_out[(int64_t)i * CC + l * N + s] = rows[ss * N + auto_src(2 * N - gp, s)];
    }
}

// r_all[col][i] = automorph(r_flat[i], gen_pows[i]), r_bar_all[col][i] with 2N - gen_pows[i]
// through the given tables (automorphism_kernel, collapse_kernel.cu:129-175)
__global__ void k_automorph_cols(uint64_t* __restrict__ r_all, uint64_t* __restrict__ r_bar_all,
                                 const uint64_t* __restrict__ r_flat, const uint64_t* __restrict__ rb_flat,
                                 const uint32_t* __restrict__ tables, const uint32_t* __restrict__ gen_pows, int nph,
                                 int poly_len, int crt, int64_t col_stride) {
    const int i = blockIdx.x;
    const int cc = crt * poly_len;
    const uint32_t gp = gen_pows[i];
    const uint32_t* tr = tables + (int64_t)((gp - 1) / 2) * poly_len;
    const uint32_t* tb = tables + (int64_t)((2 * poly_len - gp - 1) / 2) * poly_len;
    for (int e = threadIdx.x; e < cc; e += blockDim.x) {
        const int c = e / poly_len, z = e % poly_len;
        r_all[col_stride + (int64_t)i * cc + e] = r_flat[(int64_t)i * cc + c * poly_len + tr[z]];
        r_bar_all[col_stride + (int64_t)i * cc + e] = rb_flat[(int64_t)i * cc + c * poly_len + tb[z]];
    }
}

// in place: each polynomial of `data` permuted by the table of gen_pows[i] (or 2N - gen_pows[i])
__global__ void k_automorph_inplace(uint64_t* __restrict__ data, const uint32_t* __restrict__ tables,
                                    const uint32_t* __restrict__ gen_pows, int nph, int poly_len, int crt, int is_rbar) {
    extern __shared__ uint64_t abuf[];
    const int64_t blk = blockIdx.x;
    const int i = (int)(blk % nph);
    const int cc = crt * poly_len;
    const uint32_t gp = gen_pows[i];
    const uint32_t* tb = tables + (int64_t)(is_rbar ? (2 * poly_len - gp - 1) / 2 : (gp - 1) / 2) * poly_len;
    uint64_t* d = data + blk * cc;
    for (int e = threadIdx.x; e < cc; e += blockDim.x) abuf[e] = d[e];
    __syncthreads();
    for (int e = threadIdx.x; e < cc; e += blockDim.x) d[e] = abuf[(e / poly_len) * poly_len + tb[e % poly_len]];
}

// ----------------------------- state -----------------------------------------
struct HintState {
    uint64_t* tab64 = nullptr;  // as uploaded (returned by gpu_hint_get_ntt_tables)
    uint32_t* tab32 = nullptr;
    uint32_t* query = nullptr;
    int polys = 0;
    uint64_t* out = nullptr;
    int cols = 0;
} g_hint;

struct PrepState {
    uint64_t* out = nullptr;
    int cols = 0;
    uint32_t* tab32 = nullptr;
} g_prep;

struct PackState {
    bool ready = false, canonical = false;
    int nph = 0, nz = 0, poly_len = 0, crt = 0;
    uint64_t q0 = 0, q1 = 0;
    uint64_t *mono = nullptr, *mod_inv = nullptr, *a_ct = nullptr, *r_out = nullptr, *rb_out = nullptr;
    int *idx = nullptr, *idx_bar = nullptr;
    uint32_t *tab32 = nullptr, *act = nullptr, *E = nullptr;
} g_pack;

struct CollapseSet {  // one set of outputs (primary, or the "_new" set of the fold variants)
    uint64_t *bt = nullptr, *btb = nullptr, *bth = nullptr, *a_hat = nullptr;
};
struct CollapseState {
    uint64_t *r_all = nullptr, *r_bar_all = nullptr;
    int cols = 0, nph = 0, cc = 0;
    uint32_t *wrows = nullptr, *vmask = nullptr, *tab32 = nullptr;
    CollapseSet cur, fresh;
    int out_cols = 0, fresh_cols = 0;
} g_col;

bool upload_tab32(const uint64_t* h_or_d_tab64, bool device, uint32_t*& tab32) {
    if (!tab32 && report(cudaMalloc(&tab32, 8 * N * sizeof(uint32_t)), "table allocation")) return false;
    uint64_t* tmp = nullptr;
    const uint64_t* src = h_or_d_tab64;
    if (!device) {
        if (report(cudaMalloc(&tmp, 8 * N * sizeof(uint64_t)), "table allocation")) return false;
        if (report(cudaMemcpy(tmp, h_or_d_tab64, 8 * N * sizeof(uint64_t), cudaMemcpyHostToDevice), "table upload")) {
            cudaFree(tmp);
            return false;
        }
        src = tmp;
    }
    k_tab32<<<16, 256>>>(src, tab32);
    const bool ok = !report(cudaDeviceSynchronize(), "table conversion");
    if (tmp) cudaFree(tmp);
    return ok;
}

// the canonical packing tables of PackParams::new / the reference's setup (packing.rs:1635-1670,
// 2544-2580): mono[e] = NTT(x^e), mono[N + e] = -NTT(x^e); idx[i][j] the slot of x^(j g'_i mod 2N)
// (g'_i = 5^((N - i) mod N)), idx_bar the slot of x^(-j g'_i mod 2N); mod_inv = N^-1 in every slot
bool tables_canonical(const uint64_t* mono, const int* idx, const int* idx_bar, const uint64_t* mod_inv, int nph,
                      int nz, int poly_len, int crt, uint64_t q0, uint64_t q1) {
    if (poly_len != N || crt != 2 || nph != HALF || nz != N || q0 != Q0 || q1 != Q1) return false;
    const uint64_t q[2] = {q0, q1};
    auto mulm = [](uint64_t a, uint64_t b, uint64_t m) { return (uint64_t)((unsigned __int128)a * b % m); };
    auto powm = [&](uint64_t b, uint64_t e, uint64_t m) {
        uint64_t r = 1;
        for (; e; e >>= 1, b = mulm(b, b, m))
            if (e & 1) r = mulm(r, b, m);
        return r;
    };
    HostParams hp;
    host_params_init(hp);
    for (int l = 0; l < 2; l++) {
        // slot s evaluates at psi^(2 brev(s) + 1); psi = the table's psi^1 (bit-reversed index 1 of fw
        // holds psi^(N/2)... so take it from x^1's NTT: mono[1][l][s] = psi_s)
        const uint64_t inv_n = powm(N, q[l] - 2, q[l]);
        for (int s = 0; s < N; s++) {
            if (mod_inv[l * N + s] != inv_n) return false;
            const uint64_t psi_s = mono[(size_t)1 * CC + l * N + s];
            uint64_t pw = 1;
            for (int e = 0; e < N; e++) {
                if (mono[(size_t)e * CC + l * N + s] != pw) return false;
                const uint64_t neg = pw ? q[l] - pw : 0;
                if (mono[((size_t)N + e) * CC + l * N + s] != neg) return false;
                pw = mulm(pw, psi_s, q[l]);
            }
            if (mulm(pw, 1, q[l]) != q[l] - 1) return false;  // psi_s^N = -1
        }
    }
    // x^1's values must be the NTT slots of this library (exponent 2 brev(s) + 1 of psi)
    {
        std::vector<uint64_t> x1(2 * N, 0);
        x1[1] = 1;
        x1[N + 1] = 1;
        std::vector<uint64_t> t(x1);
        // forward_ntt of x^1 with the library's tables
        for (int l = 0; l < 2; l++) {
            const uint64_t m = q[l];
            uint64_t* op = t.data() + l * N;
            for (int mm = 0; mm < 11; mm++) {
                const int cnt = 1 << mm, tt = N >> (mm + 1);
                for (int i = 0; i < cnt; i++) {
                    const uint64_t w = hp.fw[l * N + cnt + i];
                    for (int j = 0; j < tt; j++) {
                        const uint64_t x = op[2 * tt * i + j], y = mulm(op[2 * tt * i + j + tt], w, m);
                        op[2 * tt * i + j] = (x + y) % m;
                        op[2 * tt * i + j + tt] = (x + m - y) % m;
                    }
                }
            }
        }
        for (int e = 0; e < 2 * N; e++)
            if (mono[CC + e] != t[e]) return false;
    }
    for (int i = 0; i < nph; i++) {
        const uint64_t g = powm(5, (uint64_t)((N - i) % N), 2 * N);
        for (int j = 0; j < nz; j++) {
            const uint64_t ix = ((uint64_t)j * g) % (2 * N);
            const uint64_t ixb = (2 * N - ix) % (2 * N);
            const int want = ix < (uint64_t)N ? (int)ix : (int)(N + ix % N);
            const int wantb = ixb < (uint64_t)N ? (int)ixb : (int)(N + ixb % N);
            if (idx[(size_t)i * nz + j] != want || idx_bar[(size_t)i * nz + j] != wantb) return false;
        }
    }
    return true;
}

// the packing sums of one column group into g_pack.r_out / rb_out (pre-automorphism)
bool pack_sums(const uint64_t* d_a_ct) {
    PackState& P = g_pack;
    if (P.canonical) {
        k_act_from_u64<<<148 * 4, 256>>>(d_a_ct, P.act);
        if (report(offline_jntt(P.act, 1, P.tab32, P.tab32 + 2 * N, P.E, nullptr), "packing transform")) return false;
        if (report(cudaFuncSetAttribute(k_pre_gather, cudaFuncAttributeMaxDynamicSharedMemorySize, 8 * N * 4),
                   "packing gather"))
            return false;
        k_pre_gather<<<dim3(N / 8, 2), 256, 8 * N * 4>>>(P.E, P.r_out, P.rb_out);
    } else {
        k_pack_direct<<<dim3((P.crt * P.poly_len + 255) / 256, (P.nph + 3) / 4, 1), 256>>>(
            P.mono, d_a_ct, P.idx, P.idx_bar, P.mod_inv, P.nph, P.nz, P.crt * P.poly_len, P.poly_len, P.q0, P.q1, 0,
            0, P.r_out, P.rb_out);
    }
    return !report(cudaDeviceSynchronize(), "packing sums");
}

void free_collapse_set(CollapseSet& c) {
    dfree(c.bt);
    dfree(c.btb);
    dfree(c.bth);
    dfree(c.a_hat);
}

bool collapse_weights(const uint64_t* h_w_all, const uint64_t* h_w_bar_all, const uint64_t* h_v_mask,
                      const uint64_t* h_ntt_tables, int nph, int t_exp, int cc) {
    CollapseState& C = g_col;
    if (nph != HALF || t_exp != 3 || cc != CC) {
        report_msg("gpu_collapse_setup: this library supports poly_len 2048, crt_count 2, t_exp 3");
        return false;
    }
    const size_t wn = (size_t)(nph - 1) * t_exp * cc;
    if (!C.wrows && report(cudaMalloc(&C.wrows, 2 * wn * sizeof(uint32_t)), "weights allocation")) return false;
    if (!C.vmask && report(cudaMalloc(&C.vmask, (size_t)t_exp * cc * sizeof(uint32_t)), "weights allocation"))
        return false;
    uint64_t* tmp = nullptr;
    if (report(cudaMalloc(&tmp, wn * sizeof(uint64_t)), "weights staging")) return false;
    bool ok = true;
    const uint64_t* srcs[3] = {h_w_all, h_w_bar_all, h_v_mask};
    uint32_t* dsts[3] = {C.wrows, C.wrows + wn, C.vmask};
    const size_t ns[3] = {wn, wn, (size_t)t_exp * cc};
    for (int k = 0; k < 3 && ok; k++)
        ok = !report(cudaMemcpy(tmp, srcs[k], ns[k] * sizeof(uint64_t), cudaMemcpyHostToDevice), "weights upload") &&
             !report(narrow_u64(tmp, (int64_t)ns[k], dsts[k], nullptr), "weights narrowing") &&
             !report(cudaDeviceSynchronize(), "weights narrowing");
    cudaFree(tmp);
    return ok && upload_tab32(h_ntt_tables, false, C.tab32);
}

bool alloc_collapse_set(CollapseSet& c, int cols) {
    free_collapse_set(c);
    return !report(cudaMalloc(&c.bt, (size_t)cols * NINNER * N * 8), "bold_t allocation") &&
           !report(cudaMalloc(&c.btb, (size_t)cols * NINNER * N * 8), "bold_t_bar allocation") &&
           !report(cudaMalloc(&c.bth, (size_t)cols * 3 * N * 8), "bold_t_hat allocation") &&
           !report(cudaMalloc(&c.a_hat, (size_t)cols * N * 8), "a_hat allocation");
}

void run_collapse(CollapseSet& out, int num_cols, int nph, int t_exp, int bits_per) {
    CollapseState& C = g_col;
    if (!C.r_all || !C.wrows || !C.tab32 || !out.bt) {
        report_msg("gpu_collapse_run: data not set up");
        return;
    }
    if (bits_per != GADGET_BITS || t_exp != 3 || nph != HALF || num_cols > C.cols) {
        report_msg("gpu_collapse_run: unsupported shape (bits_per 19, t_exp 3, nphalf 1024)");
        return;
    }
    // the chains of at most 64 columns at a time share one F buffer
    const int chunk = num_cols < 64 ? num_cols : 64;
    uint32_t *F = nullptr, *r0 = nullptr;
    uint64_t* xb = nullptr;
    if (report(cudaMalloc(&F, (size_t)chunk * 2 * HALF * CC * 4), "collapse scratch") ||
        report(cudaMalloc(&r0, (size_t)chunk * CC * 4), "collapse scratch") ||
        report(cudaMalloc(&xb, (size_t)chunk * N * 8), "collapse scratch")) {
        dfree(F);
        dfree(r0);
        dfree(xb);
        return;
    }
    for (int c0 = 0; c0 < num_cols; c0 += chunk) {
        const int n = num_cols - c0 < chunk ? num_cols - c0 : chunk;
        const size_t ro = (size_t)c0 * HALF * CC;
        if (report(offline_collapse_arrays(C.r_all + ro, C.r_bar_all + ro, n, C.wrows, C.vmask, C.tab32, F, r0, xb,
                                           out.bt + (size_t)c0 * NINNER * N, out.btb + (size_t)c0 * NINNER * N,
                                           out.bth + (size_t)c0 * 3 * N, out.a_hat + (size_t)c0 * N, nullptr),
                   "collapse"))
            break;
    }
    report(cudaDeviceSynchronize(), "collapse");
    dfree(F);
    dfree(r0);
    dfree(xb);
}

}  // namespace
}  // namespace ipr

using namespace ipr;

extern "C" {

// ------------------------------- hint.rs --------------------------------------
void gpu_hint_upload_tables(const uint64_t* h_ntt_tables, int poly_len) {
    if (poly_len != N) return report_msg("gpu_hint_upload_tables: poly_len must be 2048");
    if (!g_hint.tab64 && report(cudaMalloc(&g_hint.tab64, 8 * N * sizeof(uint64_t)), "hint tables")) return;
    if (report(cudaMemcpy(g_hint.tab64, h_ntt_tables, 8 * N * sizeof(uint64_t), cudaMemcpyHostToDevice), "hint tables"))
        return;
    upload_tab32(g_hint.tab64, true, g_hint.tab32);
}

void gpu_hint_upload_query_ffi(const uint64_t* h_query, int db_rows_poly, int poly_len) {
    if (poly_len != N || db_rows_poly < 1) return report_msg("gpu_hint_upload_query_ffi: bad shape");
    const size_t n = (size_t)db_rows_poly * CC;
    dfree(g_hint.query);
    uint64_t* tmp = nullptr;
    if (report(cudaMalloc(&g_hint.query, n * 4), "hint query") || report(cudaMalloc(&tmp, n * 8), "hint query")) {
        dfree(tmp);
        return;
    }
    if (!report(cudaMemcpy(tmp, h_query, n * 8, cudaMemcpyHostToDevice), "hint query") &&
        !report(narrow_u64(tmp, (int64_t)n, g_hint.query, nullptr), "hint query"))
        report(cudaDeviceSynchronize(), "hint query");
    cudaFree(tmp);
    g_hint.polys = db_rows_poly;
}

void gpu_hint_compute_no_d2h(const uint16_t* d_db, int db_rows, int db_rows_poly, int db_cols, uint32_t mod0,
                             uint32_t mod1, uint64_t barrett_cr1_0, uint64_t barrett_cr1_1, uint64_t mod0_inv_mod1,
                             uint64_t mod1_inv_mod0, uint64_t modulus, uint64_t barrett_cr0_mod,
                             uint64_t barrett_cr1_mod) {
    if (!g_hint.tab32 || !g_hint.query) return report_msg("[GPU Hint] Tables or query not uploaded!");
    if (mod0 != Q0 || mod1 != Q1 || db_rows != db_rows_poly * N || db_rows_poly != g_hint.polys || db_cols < 1)
        return report_msg("gpu_hint_compute: unsupported moduli or shape");
    if (db_cols != g_hint.cols) {
        dfree(g_hint.out);
        if (report(cudaMalloc(&g_hint.out, (size_t)db_cols * N * 8), "hint output")) return;
        g_hint.cols = db_cols;
    }
    const int smem = 2 * XC * N * 4;
    if (report(cudaFuncSetAttribute(k_hint_raw, cudaFuncAttributeMaxDynamicSharedMemorySize, smem), "hint kernel"))
        return;
    k_hint_raw<<<(db_cols + XC - 1) / XC, 512, smem>>>(d_db, db_rows, db_cols, g_hint.query, g_hint.tab32, g_hint.out);
    report(cudaDeviceSynchronize(), "hint kernel");
}

void gpu_hint_compute(const uint16_t* d_db, uint64_t* h_output, int db_rows, int db_rows_poly, int db_cols,
                      uint32_t mod0, uint32_t mod1, uint64_t barrett_cr1_0, uint64_t barrett_cr1_1,
                      uint64_t mod0_inv_mod1, uint64_t mod1_inv_mod0, uint64_t modulus, uint64_t barrett_cr0_mod,
                      uint64_t barrett_cr1_mod) {
    gpu_hint_compute_no_d2h(d_db, db_rows, db_rows_poly, db_cols, mod0, mod1, barrett_cr1_0, barrett_cr1_1,
                            mod0_inv_mod1, mod1_inv_mod0, modulus, barrett_cr0_mod, barrett_cr1_mod);
    if (g_hint.out && g_hint.cols == db_cols)
        report(cudaMemcpy(h_output, g_hint.out, (size_t)db_cols * N * 8, cudaMemcpyDeviceToHost), "hint download");
}

void gpu_hint_compute_from_host(const uint16_t* h_db, uint64_t* h_output, int db_rows, int db_rows_poly,
                                int db_cols, uint32_t mod0, uint32_t mod1, uint64_t barrett_cr1_0,
                                uint64_t barrett_cr1_1, uint64_t mod0_inv_mod1, uint64_t mod1_inv_mod0,
                                uint64_t modulus, uint64_t barrett_cr0_mod, uint64_t barrett_cr1_mod) {
    uint16_t* d_db = nullptr;
    const size_t bytes = (size_t)db_rows * db_cols * sizeof(uint16_t);
    if (report(cudaMalloc(&d_db, bytes), "hint DB upload")) return;
    if (!report(cudaMemcpy(d_db, h_db, bytes, cudaMemcpyHostToDevice), "hint DB upload"))
        gpu_hint_compute(d_db, h_output, db_rows, db_rows_poly, db_cols, mod0, mod1, barrett_cr1_0, barrett_cr1_1,
                         mod0_inv_mod1, mod1_inv_mod0, modulus, barrett_cr0_mod, barrett_cr1_mod);
    cudaFree(d_db);
}

void gpu_hint_free_query_only(void) { dfree(g_hint.query); }
void gpu_hint_free_output_and_tables(void) {
    dfree(g_hint.out);
    g_hint.cols = 0;
    dfree(g_hint.tab64);
    dfree(g_hint.tab32);
}
void gpu_hint_free(void) {
    gpu_hint_free_query_only();
    gpu_hint_free_output_and_tables();
}
const uint64_t* gpu_hint_get_device_output(void) { return g_hint.out; }
const uint64_t* gpu_hint_get_ntt_tables(void) { return g_hint.tab64; }
int gpu_hint_get_db_cols(void) { return g_hint.cols; }

// ----------------------------- prep_pack.rs -----------------------------------
void gpu_prep_pack_compute(const uint64_t* d_hint_output, const uint64_t* d_ntt_tables, int db_cols, uint32_t mod0,
                           uint32_t mod1, uint64_t modulus) {
    if (mod0 != Q0 || mod1 != Q1 || db_cols < 1) return report_msg("gpu_prep_pack_compute: unsupported moduli or shape");
    if (db_cols != g_prep.cols) {
        dfree(g_prep.out);
        if (report(cudaMalloc(&g_prep.out, (size_t)db_cols * CC * 8), "[GPU prep_pack] cudaMalloc")) return;
        g_prep.cols = db_cols;
    }
    if (!upload_tab32(d_ntt_tables, true, g_prep.tab32)) return;
    const int smem = 2 * XC * N * 4;
    if (report(cudaFuncSetAttribute(k_prep_pack64, cudaFuncAttributeMaxDynamicSharedMemorySize, smem), "prep_pack"))
        return;
    k_prep_pack64<<<(db_cols + XC - 1) / XC, 512, smem>>>(d_hint_output, db_cols, g_prep.tab32, g_prep.out);
    report(cudaDeviceSynchronize(), "[GPU prep_pack] kernel error");
}
const uint64_t* gpu_prep_pack_get_output(void) { return g_prep.out; }
void gpu_prep_pack_free(void) {
    dfree(g_prep.out);
    g_prep.cols = 0;
    dfree(g_prep.tab32);
}

// ------------------------------ packing.rs ------------------------------------
void gpu_packing_teardown(void) {
    PackState& P = g_pack;
    dfree(P.mono);
    dfree(P.mod_inv);
    dfree(P.a_ct);
    dfree(P.r_out);
    dfree(P.rb_out);
    dfree(P.idx);
    dfree(P.idx_bar);
    dfree(P.tab32);
    dfree(P.act);
    dfree(P.E);
    P.ready = P.canonical = false;
    P.nph = P.nz = 0;
}

void gpu_packing_setup(const uint64_t* h_mono_table, const int* h_idx, const int* h_idx_bar, const uint64_t* h_mod_inv,
                       int num_to_pack_half, int non_zeros, int poly_len, int crt_count, uint64_t mod0, uint64_t mod1,
                       uint64_t barrett_cr0, uint64_t barrett_cr1) {
    gpu_packing_teardown();
    PackState& P = g_pack;
    if (crt_count != 2 || num_to_pack_half < 1 || non_zeros < 1 || poly_len < 1 || mod0 >= (1ull << 32) ||
        mod1 >= (1ull << 32))
        return report_msg("gpu_packing_setup: unsupported shape (crt_count 2, moduli < 2^32)");
    P.nph = num_to_pack_half, P.nz = non_zeros, P.poly_len = poly_len, P.crt = crt_count, P.q0 = mod0, P.q1 = mod1;
    const size_t cc = (size_t)crt_count * poly_len;
    const size_t mono = 2 * (size_t)poly_len * cc, idxn = (size_t)num_to_pack_half * non_zeros;
    P.canonical = tables_canonical(h_mono_table, h_idx, h_idx_bar, h_mod_inv, num_to_pack_half, non_zeros, poly_len,
                                   crt_count, mod0, mod1);
    bool ok = !report(cudaMalloc(&P.a_ct, (size_t)non_zeros * cc * 8), "packing buffers") &&
              !report(cudaMalloc(&P.r_out, (size_t)num_to_pack_half * cc * 8), "packing buffers") &&
              !report(cudaMalloc(&P.rb_out, (size_t)num_to_pack_half * cc * 8), "packing buffers");
    if (ok && P.canonical) {
        HostParams hp;
        host_params_init(hp);
        std::vector<uint32_t> tab(8 * N);
        std::memcpy(tab.data(), hp.fw.data(), 2 * N * 4);
        std::memcpy(tab.data() + 2 * N, hp.fwp.data(), 2 * N * 4);
        std::memcpy(tab.data() + 4 * N, hp.iw.data(), 2 * N * 4);
        std::memcpy(tab.data() + 6 * N, hp.iwp.data(), 2 * N * 4);
        ok = !report(cudaMalloc(&P.tab32, tab.size() * 4), "packing buffers") &&
             !report(cudaMemcpy(P.tab32, tab.data(), tab.size() * 4, cudaMemcpyHostToDevice), "packing tables") &&
             !report(cudaMalloc(&P.act, 2ull * N * N * 4), "packing buffers") &&
             !report(cudaMalloc(&P.E, 2ull * N * N * 4), "packing buffers");
    } else if (ok) {
        for (size_t e = 0; e < idxn && ok; e++)  // the direct sums index the monomial table with these
            if (h_idx[e] < 0 || h_idx[e] >= 2 * poly_len || h_idx_bar[e] < 0 || h_idx_bar[e] >= 2 * poly_len) {
                report_msg("gpu_packing_setup: index table entry outside the monomial table");
                ok = false;
            }
        ok = ok && !report(cudaMalloc(&P.mono, mono * 8), "packing buffers") &&
             !report(cudaMalloc(&P.mod_inv, cc * 8), "packing buffers") &&
             !report(cudaMalloc(&P.idx, idxn * 4), "packing buffers") &&
             !report(cudaMalloc(&P.idx_bar, idxn * 4), "packing buffers") &&
             !report(cudaMemcpy(P.mono, h_mono_table, mono * 8, cudaMemcpyHostToDevice), "packing upload") &&
             !report(cudaMemcpy(P.mod_inv, h_mod_inv, cc * 8, cudaMemcpyHostToDevice), "packing upload") &&
             !report(cudaMemcpy(P.idx, h_idx, idxn * 4, cudaMemcpyHostToDevice), "packing upload") &&
             !report(cudaMemcpy(P.idx_bar, h_idx_bar, idxn * 4, cudaMemcpyHostToDevice), "packing upload");
    }
    P.ready = ok;
}

void gpu_packing_precomp_fast_device_no_d2h(const uint64_t* d_a_ct_device) {
    if (!g_pack.ready) return report_msg("gpu_packing_precomp: packing not set up");
    pack_sums(d_a_ct_device);
}

void gpu_packing_precomp_fast_device(const uint64_t* d_a_ct_device, uint64_t* h_r_out, uint64_t* h_r_bar_out) {
    if (!g_pack.ready) return report_msg("gpu_packing_precomp: packing not set up");
    if (!pack_sums(d_a_ct_device)) return;
    const size_t out = (size_t)g_pack.nph * g_pack.crt * g_pack.poly_len * 8;
    if (!report(cudaMemcpy(h_r_out, g_pack.r_out, out, cudaMemcpyDeviceToHost), "packing download"))
        report(cudaMemcpy(h_r_bar_out, g_pack.rb_out, out, cudaMemcpyDeviceToHost), "packing download");
}

void gpu_packing_precomp_fast(const uint64_t* h_a_ct, uint64_t* h_r_out, uint64_t* h_r_bar_out) {
    if (!g_pack.ready) return report_msg("gpu_packing_precomp: packing not set up");
    const size_t act = (size_t)g_pack.nz * g_pack.crt * g_pack.poly_len * 8;
    if (report(cudaMemcpy(g_pack.a_ct, h_a_ct, act, cudaMemcpyHostToDevice), "packing upload")) return;
    gpu_packing_precomp_fast_device(g_pack.a_ct, h_r_out, h_r_bar_out);
}

void gpu_packing_precomp_batched(const uint64_t* h_mono_table, const uint64_t* h_a_ct_batch, const int* h_idx,
                                 const int* h_idx_bar, const uint64_t* h_mod_inv, uint64_t* h_r_out,
                                 uint64_t* h_r_bar_out, int batch_count, int num_to_pack_half, int non_zeros,
                                 int poly_len, int crt_count, uint64_t mod0, uint64_t mod1, uint64_t barrett_cr0,
                                 uint64_t barrett_cr1) {
    gpu_packing_setup(h_mono_table, h_idx, h_idx_bar, h_mod_inv, num_to_pack_half, non_zeros, poly_len, crt_count,
                      mod0, mod1, barrett_cr0, barrett_cr1);
    const size_t act = (size_t)non_zeros * crt_count * poly_len, out = (size_t)num_to_pack_half * crt_count * poly_len;
    for (int b = 0; b < batch_count && g_pack.ready; b++)
        gpu_packing_precomp_fast(h_a_ct_batch + b * act, h_r_out + b * out, h_r_bar_out + b * out);
    gpu_packing_teardown();
}

void gpu_packing_precomp(const uint64_t* h_mono_table, const uint64_t* h_a_ct, const int* h_idx, const int* h_idx_bar,
                         const uint64_t* h_mod_inv, uint64_t* h_r_out, uint64_t* h_r_bar_out, int num_to_pack_half,
                         int non_zeros, int poly_len, int crt_count, uint64_t mod0, uint64_t mod1,
                         uint64_t barrett_cr0, uint64_t barrett_cr1) {
    gpu_packing_precomp_batched(h_mono_table, h_a_ct, h_idx, h_idx_bar, h_mod_inv, h_r_out, h_r_bar_out, 1,
                                num_to_pack_half, non_zeros, poly_len, crt_count, mod0, mod1, barrett_cr0,
                                barrett_cr1);
}

// packing sums (pre-automorphism) of num_cols column groups straight into d_r_all / d_r_bar_all
// ([col][nphalf][coeff_count]) with the tables of gpu_packing_setup (packing_kernel.cu:782-806)
void gpu_packing_batched_fused(uint64_t* d_r_all, uint64_t* d_r_bar_all, const uint64_t* d_prepacked, int num_cols) {
    if (!g_pack.ready) return report_msg("[GPU packing batched fused] Shared data not set up!");
    const size_t cc = (size_t)g_pack.crt * g_pack.poly_len, act = (size_t)g_pack.nz * cc, out = (size_t)g_pack.nph * cc;
    for (int c = 0; c < num_cols; c++) {
        if (!pack_sums(d_prepacked + c * act)) return;
        if (report(cudaMemcpy(d_r_all + c * out, g_pack.r_out, out * 8, cudaMemcpyDeviceToDevice), "packing copy") ||
            report(cudaMemcpy(d_r_bar_all + c * out, g_pack.rb_out, out * 8, cudaMemcpyDeviceToDevice), "packing copy"))
            return;
    }
}

uint64_t* gpu_packing_get_s_r_out(void) { return g_pack.r_out; }
uint64_t* gpu_packing_get_s_r_bar_out(void) { return g_pack.rb_out; }
int gpu_packing_get_coeff_count(void) { return g_pack.crt * g_pack.poly_len; }
int gpu_packing_get_nphalf(void) { return g_pack.nph; }

// ------------------------------ collapse.rs -----------------------------------
void gpu_collapse_alloc_r(int num_cols, int nphalf, int coeff_count) {
    CollapseState& C = g_col;
    dfree(C.r_all);
    dfree(C.r_bar_all);
    const size_t bytes = (size_t)num_cols * nphalf * coeff_count * sizeof(uint64_t);
    if (report(cudaMalloc(&C.r_all, bytes), "r_all allocation") ||
        report(cudaMalloc(&C.r_bar_all, bytes), "r_all allocation") || report(cudaMemset(C.r_all, 0, bytes), "r_all") ||
        report(cudaMemset(C.r_bar_all, 0, bytes), "r_all")) {
        dfree(C.r_all);
        dfree(C.r_bar_all);
        return;
    }
    C.cols = num_cols, C.nph = nphalf, C.cc = coeff_count;
}
uint64_t* gpu_collapse_get_r_all_col(int col, int nphalf, int coeff_count) {
    return g_col.r_all ? g_col.r_all + (size_t)col * nphalf * coeff_count : nullptr;
}
uint64_t* gpu_collapse_get_r_bar_all_col(int col, int nphalf, int coeff_count) {
    return g_col.r_bar_all ? g_col.r_bar_all + (size_t)col * nphalf * coeff_count : nullptr;
}
uint64_t* gpu_collapse_get_r_all(void) { return g_col.r_all; }
uint64_t* gpu_collapse_get_r_bar_all(void) { return g_col.r_bar_all; }

void gpu_collapse_automorph_column(const uint64_t* d_r_flat, const uint64_t* d_r_bar_flat, int col, int nphalf,
                                   int coeff_count, int poly_len, int crt_count, const uint32_t* d_tables,
                                   const uint32_t* d_gen_pows, int num_tables) {
    if (!g_col.r_all || col >= g_col.cols) return report_msg("gpu_collapse_automorph_column: r_all not allocated");
    k_automorph_cols<<<nphalf, 256>>>(g_col.r_all, g_col.r_bar_all, d_r_flat, d_r_bar_flat, d_tables, d_gen_pows,
                                      nphalf, poly_len, crt_count, (int64_t)col * nphalf * coeff_count);
    report(cudaGetLastError(), "collapse automorphism");  // like the reference, not synchronised
}

void gpu_collapse_batched_automorphism(const uint32_t* d_tables, const uint32_t* d_gen_pows, int num_cols, int nphalf,
                                       int poly_len, int crt_count) {
    if (!g_col.r_all || !g_col.r_bar_all) return report_msg("[GPU Collapse] r_all not allocated for automorphism!");
    const int cc = crt_count * poly_len;
    const size_t smem = (size_t)cc * sizeof(uint64_t);
    if (report(cudaFuncSetAttribute(k_automorph_inplace, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
               "collapse automorphism"))
        return;
    k_automorph_inplace<<<num_cols * nphalf, 256, smem>>>(g_col.r_all, d_tables, d_gen_pows, nphalf, poly_len,
                                                          crt_count, 0);
    k_automorph_inplace<<<num_cols * nphalf, 256, smem>>>(g_col.r_bar_all, d_tables, d_gen_pows, nphalf, poly_len,
                                                          crt_count, 1);
    report(cudaDeviceSynchronize(), "collapse automorphism");
}

void gpu_collapse_setup(const uint64_t* h_w_all, const uint64_t* h_w_bar_all, const uint64_t* h_v_mask,
                        const uint64_t* h_ntt_tables, int num_cols, int nphalf, int t_exp, int coeff_count) {
    if (!collapse_weights(h_w_all, h_w_bar_all, h_v_mask, h_ntt_tables, nphalf, t_exp, coeff_count)) return;
    if (alloc_collapse_set(g_col.cur, num_cols)) g_col.out_cols = num_cols;
}

void gpu_collapse_run(int num_cols, int nphalf, int t_exp, int bits_per, uint32_t mod0, uint32_t mod1,
                      uint64_t barrett_cr1_0, uint64_t barrett_cr1_1, uint64_t mod0_inv_mod1, uint64_t mod1_inv_mod0,
                      uint64_t crt_modulus, uint64_t barrett_cr0_mod, uint64_t barrett_cr1_mod) {
    if (mod0 != Q0 || mod1 != Q1) return report_msg("gpu_collapse_run: unsupported moduli");
    if (num_cols > g_col.out_cols) return report_msg("[GPU Collapse] Data not set up!");
    run_collapse(g_col.cur, num_cols, nphalf, t_exp, bits_per);
}

void gpu_collapse_download_a_hat(uint64_t* h_a_hat, int num_cols) {
    if (g_col.cur.a_hat)
        report(cudaMemcpy(h_a_hat, g_col.cur.a_hat, (size_t)num_cols * N * 8, cudaMemcpyDeviceToHost), "a_hat download");
}
uint64_t* gpu_collapse_get_bold_t(void) { return g_col.cur.bt; }
uint64_t* gpu_collapse_get_bold_t_bar(void) { return g_col.cur.btb; }
uint64_t* gpu_collapse_get_bold_t_hat(void) { return g_col.cur.bth; }

void gpu_collapse_setup_fold(const uint64_t* h_w_all, const uint64_t* h_w_bar_all, const uint64_t* h_v_mask,
                             const uint64_t* h_ntt_tables, int num_cols, int nphalf, int t_exp, int coeff_count) {
    if (!collapse_weights(h_w_all, h_w_bar_all, h_v_mask, h_ntt_tables, nphalf, t_exp, coeff_count)) return;
    if (alloc_collapse_set(g_col.fresh, num_cols)) g_col.fresh_cols = num_cols;
}
void gpu_collapse_run_fold(int num_cols, int nphalf, int t_exp, int bits_per, uint32_t mod0, uint32_t mod1,
                           uint64_t barrett_cr1_0, uint64_t barrett_cr1_1, uint64_t mod0_inv_mod1,
                           uint64_t mod1_inv_mod0, uint64_t crt_modulus, uint64_t barrett_cr0_mod,
                           uint64_t barrett_cr1_mod) {
    if (mod0 != Q0 || mod1 != Q1) return report_msg("gpu_collapse_run_fold: unsupported moduli");
    if (num_cols > g_col.fresh_cols) return report_msg("[GPU Collapse] Fold data not set up!");
    run_collapse(g_col.fresh, num_cols, nphalf, t_exp, bits_per);
}
void gpu_collapse_download_a_hat_new(uint64_t* h_a_hat, int num_cols) {
    if (g_col.fresh.a_hat)
        report(cudaMemcpy(h_a_hat, g_col.fresh.a_hat, (size_t)num_cols * N * 8, cudaMemcpyDeviceToHost),
               "a_hat download");
}
uint64_t* gpu_collapse_get_bold_t_new(void) { return g_col.fresh.bt; }
uint64_t* gpu_collapse_get_bold_t_bar_new(void) { return g_col.fresh.btb; }
uint64_t* gpu_collapse_get_bold_t_hat_new(void) { return g_col.fresh.bth; }
void gpu_collapse_swap_bold_t(void) {
    CollapseSet t = g_col.cur;
    g_col.cur = g_col.fresh;
    g_col.fresh = t;
    const int c = g_col.out_cols;
    g_col.out_cols = g_col.fresh_cols;
    g_col.fresh_cols = c;
}

void gpu_collapse_free_working(void) {
    CollapseState& C = g_col;
    dfree(C.r_all);
    dfree(C.r_bar_all);
    dfree(C.wrows);
    dfree(C.vmask);
    dfree(C.tab32);
    C.cols = 0;
}
void gpu_collapse_free_all(void) {
    gpu_collapse_free_working();
    free_collapse_set(g_col.cur);
    free_collapse_set(g_col.fresh);
    g_col.out_cols = g_col.fresh_cols = 0;
}

}  // extern "C"
