// compat.cu — reference-named respond-path entry points (include/ipr_b200_compat.h)
// implemented on this library's kernels.  Semantics follow
// native/cuda/{gemv,rotation,packing_online}_kernel.cu of rkdud007/inspire-rs:
// process-wide state, one query stream, void returns with errors reported on
// stderr (and kept for ipr_last_error()).
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>
#include <string>

#include "host_math.hpp"
#include "ipr_b200.h"
#include "ipr_b200_compat.h"
#include "ipr_device.cuh"
#include "kernels.cuh"

namespace ipr {
uint32_t encode_num_inv(uint64_t interp);
int encode_db_device(const uint16_t* d_raw, uint16_t* d_out, uint64_t db_rows, uint64_t db_cols, uint64_t interp,
                     cudaStream_t st);
}  // namespace ipr

namespace {

std::mutex g_mu;
cudaStream_t g_stream = nullptr;
int g_const_device = -1;
thread_local std::string g_compat_err;

uint32_t *d_tables = nullptr, *d_gen_pows = nullptr;
int g_num_tables = 0, g_num_rot = 0;
uint64_t* d_y_body = nullptr;
uint64_t *d_bold_t = nullptr, *d_bold_t_bar = nullptr, *d_bold_t_hat = nullptr, *d_output = nullptr;
uint64_t *d_y_all = nullptr, *d_y_bar_all = nullptr, *d_z_body = nullptr;
bool g_adopted = false;
int g_n_inner = 0, g_poly_len = 0;
uint16_t* g_encoded_db = nullptr;      // gpu_encode_db_from_host's result, kept on the device
uint16_t* g_encoded_db_new = nullptr;  // gpu_encode_db_from_host_fold's result until the swap

bool report(const char* tag, cudaError_t e, int line) {
    if (e == cudaSuccess) return false;
    char buf[256];
    snprintf(buf, sizeof(buf), "[%s] CUDA error at compat.cu:%d: %s", tag, line, cudaGetErrorString(e));
    fprintf(stderr, "%s\n", buf);
    g_compat_err = buf;
    return true;
}
#define CHK(tag, call) \
    if (report(tag, (call), __LINE__)) return

bool bad_shape(const char* tag, int t_exp_left, int poly_len) {
    if (t_exp_left == ipr::T_EXP && poly_len == ipr::N) return false;
    fprintf(stderr, "[%s] unsupported shape t_exp_left=%d poly_len=%d (kernels are built for 3, 2048)\n", tag,
            t_exp_left, poly_len);
    return true;
}

cudaError_t ensure_stream_and_constants() {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (!g_stream) {
        int lo, hi;
        cudaDeviceGetStreamPriorityRange(&lo, &hi);
        e = cudaStreamCreateWithPriority(&g_stream, cudaStreamNonBlocking, hi);
        if (e != cudaSuccess) return e;
    }
    if (g_const_device != dev) {
        ipr::HostParams hp;
        ipr::host_params_init(hp);
        e = ipr::set_constants(hp.barrett, hp.q0_inv_mod_q1);
        if (e != cudaSuccess) return e;
        e = ipr::init_device_kernels();
        if (e != cudaSuccess) return e;
        g_const_device = dev;
    }
    return cudaSuccess;
}

// y_all[i][k][z] = y[k][tables[(g_i-1)/2][z]], y_bar_all from tables[(2N-g_i-1)/2]
__global__ void k_rotations_tables(const uint64_t* __restrict__ y_body, const uint32_t* __restrict__ tables,
                                   const uint32_t* __restrict__ gen_pows, uint64_t* __restrict__ y_all,
                                   uint64_t* __restrict__ y_bar_all, int num_rotations, int t_exp_left) {
    const int i = blockIdx.x, k = blockIdx.y;
    const uint32_t t = gen_pows[i];
    const uint32_t* t1 = tables + (size_t)((t - 1) / 2) * ipr::N;
    const uint32_t* t2 = tables + (size_t)((2 * ipr::N - t - 1) / 2) * ipr::N;
    for (int z = threadIdx.x; z < ipr::N; z += blockDim.x) {
        const size_t o = ((size_t)i * t_exp_left + k) * ipr::N + z;
        y_all[o] = y_body[(size_t)k * ipr::N + t1[z]];
        y_bar_all[o] = y_body[(size_t)k * ipr::N + t2[z]];
    }
}

}  // namespace

extern "C" {

void gpu_init_memory_pool(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, 0) == cudaSuccess) {
        uint64_t threshold = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
    }
    CHK("GPU", ensure_stream_and_constants());
}

void gpu_encode_db(uint16_t* d_db_in, uint16_t* d_db_out, int db_rows, int db_cols, int interp_degree, int gamma,
                   int c, uint32_t modulus, uint32_t num_inv) {
    if (gamma != ipr::N || modulus != 65535u || interp_degree < 1 || db_rows < 1 || db_cols < 1 ||
        (int64_t)interp_degree * gamma * c != db_cols || num_inv != ipr::encode_num_inv((uint64_t)interp_degree)) {
        fprintf(stderr, "[GPU Encode] unsupported arguments (gamma %d, modulus %u, interp %d, c %d)\n", gamma,
                modulus, interp_degree, c);
        return;
    }
    int st = ipr::encode_db_device(d_db_in, d_db_out, (uint64_t)db_rows, (uint64_t)db_cols, (uint64_t)interp_degree,
                                   cudaStreamPerThread);
    if (st) fprintf(stderr, "[GPU Encode] %s\n", ipr_last_error());
    cudaStreamSynchronize(cudaStreamPerThread);
}

void gpu_encode_db_from_host(const uint16_t* h_db_in, uint16_t* h_db_out, int db_rows, int db_cols,
                             int interp_degree, int gamma, int c, uint32_t modulus, uint32_t num_inv) {
    (void)h_db_out;  // the encoded DB stays on the device (gpu_encode_get_device_db)
    std::lock_guard<std::mutex> lk(g_mu);
    const size_t bytes = (size_t)db_rows * (size_t)db_cols * sizeof(uint16_t);
    uint16_t *d_in = nullptr, *d_out = nullptr;
    if (report("GPU Encode", cudaMalloc(&d_in, bytes), __LINE__) ||
        report("GPU Encode", cudaMalloc(&d_out, bytes), __LINE__) ||
        report("GPU Encode", cudaMemcpy(d_in, h_db_in, bytes, cudaMemcpyHostToDevice), __LINE__)) {
        if (d_in) cudaFree(d_in);
        if (d_out) cudaFree(d_out);
        return;
    }
    gpu_encode_db(d_in, d_out, db_rows, db_cols, interp_degree, gamma, c, modulus, num_inv);
    cudaFree(d_in);
    if (g_encoded_db) cudaFree(g_encoded_db);
    g_encoded_db = d_out;
}

const uint16_t* gpu_encode_get_device_db(void) { return g_encoded_db; }

void gpu_encode_free_device_db(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_encoded_db) cudaFree(g_encoded_db);
    g_encoded_db = nullptr;
}

// encode_kernel.cu:452-516: encode a new DB into the secondary slot while the primary keeps
// serving; the upload goes in 256 MB pieces on the per-thread stream so that query copies
// on other streams interleave with it
void gpu_encode_db_from_host_fold(const uint16_t* h_db_in, int db_rows, int db_cols, int interp_degree, int gamma,
                                  int c, uint32_t modulus, uint32_t num_inv) {
    std::lock_guard<std::mutex> lk(g_mu);
    const size_t bytes = (size_t)db_rows * (size_t)db_cols * sizeof(uint16_t);
    uint16_t *d_in = nullptr, *d_out = nullptr;
    if (report("GPU Encode Fold", cudaMalloc(&d_in, bytes), __LINE__) ||
        report("GPU Encode Fold", cudaMalloc(&d_out, bytes), __LINE__)) {
        if (d_in) cudaFree(d_in);
        if (d_out) cudaFree(d_out);
        return;
    }
    const size_t chunk = 256ull << 20;
    for (size_t off = 0; off < bytes; off += chunk) {
        const size_t n = off + chunk <= bytes ? chunk : bytes - off;
        if (report("GPU Encode Fold",
                   cudaMemcpyAsync(reinterpret_cast<uint8_t*>(d_in) + off, reinterpret_cast<const uint8_t*>(h_db_in) + off,
                                   n, cudaMemcpyHostToDevice, cudaStreamPerThread),
                   __LINE__)) {
            cudaStreamSynchronize(cudaStreamPerThread);
            cudaFree(d_in);
            cudaFree(d_out);
            return;
        }
    }
    cudaStreamSynchronize(cudaStreamPerThread);
    gpu_encode_db(d_in, d_out, db_rows, db_cols, interp_degree, gamma, c, modulus, num_inv);
    cudaFree(d_in);
    if (g_encoded_db_new && g_encoded_db_new != d_out) cudaFree(g_encoded_db_new);
    g_encoded_db_new = d_out;
}

const uint16_t* gpu_encode_get_device_db_fold(void) { return g_encoded_db_new; }

// free the primary encoded DB and promote the secondary one
void gpu_encode_swap_primary(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_encoded_db && g_encoded_db != g_encoded_db_new) cudaFree(g_encoded_db);
    g_encoded_db = g_encoded_db_new;
    g_encoded_db_new = nullptr;
}

void gpu_trim_memory_pool(void) {
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, 0) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
}

uint64_t gpu_available_memory_bytes(void) {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return 0;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, 0) == cudaSuccess) {
        size_t reserved = 0, used = 0;
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used);
        if (reserved > used) free_b += reserved - used;
    }
    return (uint64_t)free_b;
}

void gpu_gemv_upload_db(const uint16_t* h_db, uint16_t** d_db_out, size_t db_size_bytes) {
    *d_db_out = nullptr;
    void* p = nullptr;
    CHK("GPU GEMV", cudaMalloc(&p, db_size_bytes));
    if (report("GPU GEMV", cudaMemcpy(p, h_db, db_size_bytes, cudaMemcpyHostToDevice), __LINE__)) {
        cudaFree(p);
        return;
    }
    *d_db_out = static_cast<uint16_t*>(p);
}

void gpu_gemv_set_device_db(uint16_t** d_db_out, const uint16_t* d_db_in, size_t) {
    *d_db_out = const_cast<uint16_t*>(d_db_in);
}

void gpu_gemv_free_db(uint16_t* d_db) {
    if (d_db) cudaFree(d_db);
}

void gpu_gemv_query(uint64_t* h_c, const uint64_t* h_a, const uint16_t* d_db, int db_rows, int b_cols, uint64_t mod0,
                    uint64_t mod1, uint64_t, uint64_t, uint64_t, uint64_t, uint64_t modulus, uint64_t, uint64_t) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (mod0 != ipr::Q0 || mod1 != ipr::Q1 || modulus != ipr::QQ || db_rows < 256 || (db_rows & 255) ||
        b_cols <= 0 || (b_cols & 15)) {
        fprintf(stderr, "[GPU GEMV] unsupported arguments (moduli or db_rows=%d b_cols=%d)\n", db_rows, b_cols);
        return;
    }
    CHK("GPU GEMV", ensure_stream_and_constants());
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    uint64_t *d_a = nullptr, *d_c = nullptr;
    CHK("GPU GEMV", cudaMallocAsync((void**)&d_a, (size_t)db_rows * 8, g_stream));
    CHK("GPU GEMV", cudaMallocAsync((void**)&d_c, (size_t)b_cols * 8, g_stream));
    // a condensed u64 (lo32 = mod q0, hi32 = mod q1) is already the single-query operand layout
    CHK("GPU GEMV", cudaMemcpyAsync(d_a, h_a, (size_t)db_rows * 8, cudaMemcpyHostToDevice, g_stream));
    CHK("GPU GEMV", ipr::launch_gemv(d_db, db_rows, b_cols, 1, reinterpret_cast<const uint32_t*>(d_a), d_c, sms,
                                     g_stream));
    CHK("GPU GEMV", cudaMemcpyAsync(h_c, d_c, (size_t)b_cols * 8, cudaMemcpyDeviceToHost, g_stream));
    CHK("GPU GEMV", cudaStreamSynchronize(g_stream));
    cudaFreeAsync(d_a, g_stream);
    cudaFreeAsync(d_c, g_stream);
}

void gpu_rotation_upload_tables(const uint32_t* h_tables, const uint32_t* h_gen_pows, int num_tables,
                                int num_rotations, int poly_len) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (poly_len != ipr::N) {
        fprintf(stderr, "[GPU Rotation] unsupported poly_len %d\n", poly_len);
        return;
    }
    if (d_tables) cudaFree(d_tables);
    if (d_gen_pows) cudaFree(d_gen_pows);
    d_tables = d_gen_pows = nullptr;
    CHK("GPU Rotation", cudaMalloc(&d_tables, (size_t)num_tables * poly_len * 4));
    CHK("GPU Rotation", cudaMalloc(&d_gen_pows, (size_t)num_rotations * 4));
    CHK("GPU Rotation", cudaMemcpy(d_tables, h_tables, (size_t)num_tables * poly_len * 4, cudaMemcpyHostToDevice));
    CHK("GPU Rotation", cudaMemcpy(d_gen_pows, h_gen_pows, (size_t)num_rotations * 4, cudaMemcpyHostToDevice));
    g_num_tables = num_tables;
    g_num_rot = num_rotations;
}

void gpu_rotation_expand_keys(uint64_t* d_y_all_out, uint64_t* d_y_bar_all_out, const uint64_t* h_y_body,
                              int num_rotations, int t_exp_left, int poly_len) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (bad_shape("GPU Rotation", t_exp_left, poly_len)) return;
    if (!d_tables || num_rotations > g_num_rot || g_num_tables < ipr::N) {
        fprintf(stderr, "[GPU Rotation] tables not uploaded\n");
        return;
    }
    CHK("GPU Rotation", ensure_stream_and_constants());
    if (!d_y_body) CHK("GPU Rotation", cudaMalloc(&d_y_body, (size_t)t_exp_left * poly_len * 8));
    CHK("GPU Rotation", cudaMemcpyAsync(d_y_body, h_y_body, (size_t)t_exp_left * poly_len * 8,
                                        cudaMemcpyHostToDevice, g_stream));
    dim3 grid(num_rotations, t_exp_left);
    k_rotations_tables<<<grid, 256, 0, g_stream>>>(d_y_body, d_tables, d_gen_pows, d_y_all_out, d_y_bar_all_out,
                                                    num_rotations, t_exp_left);
    CHK("GPU Rotation", cudaGetLastError());
    CHK("GPU Rotation", cudaStreamSynchronize(g_stream));
}

void gpu_rotation_free(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (d_tables) cudaFree(d_tables);
    if (d_gen_pows) cudaFree(d_gen_pows);
    if (d_y_body) cudaFree(d_y_body);
    d_tables = d_gen_pows = nullptr;
    d_y_body = nullptr;
}

void gpu_packing_online_ensure_key_buffers(int n_inner, int t_exp_left, int poly_len) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (d_y_all && n_inner == g_n_inner && poly_len == g_poly_len) return;
    if (d_y_all) cudaFree(d_y_all);
    if (d_y_bar_all) cudaFree(d_y_bar_all);
    if (d_z_body) cudaFree(d_z_body);
    d_y_all = d_y_bar_all = d_z_body = nullptr;
    CHK("GPU Packing Online", cudaMalloc(&d_y_all, (size_t)n_inner * poly_len * 8));
    CHK("GPU Packing Online", cudaMalloc(&d_y_bar_all, (size_t)n_inner * poly_len * 8));
    CHK("GPU Packing Online", cudaMalloc(&d_z_body, (size_t)t_exp_left * poly_len * 8));
    g_n_inner = n_inner;
    g_poly_len = poly_len;
}

uint64_t* gpu_packing_online_get_d_y_all(void) { return d_y_all; }
uint64_t* gpu_packing_online_get_d_y_bar_all(void) { return d_y_bar_all; }

void gpu_packing_online_upload_z_body(const uint64_t* h_z_body, int t_exp_left, int poly_len) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!d_z_body) {
        fprintf(stderr, "[GPU Packing Online] key buffers not allocated\n");
        return;
    }
    CHK("GPU Packing Online", ensure_stream_and_constants());
    CHK("GPU Packing Online", cudaMemcpyAsync(d_z_body, h_z_body, (size_t)t_exp_left * poly_len * 8,
                                              cudaMemcpyHostToDevice, g_stream));
}

void gpu_packing_online_upload_precomp(const uint64_t* h_bold_t, const uint64_t* h_bold_t_bar,
                                       const uint64_t* h_bold_t_hat, int num_outputs, int n_inner, int t_exp_left,
                                       int poly_len) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_adopted) {
        if (d_bold_t) cudaFree(d_bold_t);
        if (d_bold_t_bar) cudaFree(d_bold_t_bar);
        if (d_bold_t_hat) cudaFree(d_bold_t_hat);
    }
    if (d_output) cudaFree(d_output);
    d_bold_t = d_bold_t_bar = d_bold_t_hat = d_output = nullptr;
    g_adopted = false;
    const size_t bt = (size_t)num_outputs * n_inner * poly_len * 8;
    const size_t bh = (size_t)num_outputs * t_exp_left * poly_len * 8;
    CHK("GPU Packing Online", cudaMalloc(&d_bold_t, bt));
    CHK("GPU Packing Online", cudaMalloc(&d_bold_t_bar, bt));
    CHK("GPU Packing Online", cudaMalloc(&d_bold_t_hat, bh));
    CHK("GPU Packing Online", cudaMalloc(&d_output, (size_t)num_outputs * 2 * poly_len * 8));
    CHK("GPU Packing Online", cudaMemcpy(d_bold_t, h_bold_t, bt, cudaMemcpyHostToDevice));
    CHK("GPU Packing Online", cudaMemcpy(d_bold_t_bar, h_bold_t_bar, bt, cudaMemcpyHostToDevice));
    CHK("GPU Packing Online", cudaMemcpy(d_bold_t_hat, h_bold_t_hat, bh, cudaMemcpyHostToDevice));
}

void gpu_packing_online_upload_keys(const uint64_t* h_y_all, const uint64_t* h_y_bar_all, const uint64_t* h_z_body,
                                    int n_inner, int t_exp_left, int poly_len) {
    gpu_packing_online_ensure_key_buffers(n_inner, t_exp_left, poly_len);
    std::lock_guard<std::mutex> lk(g_mu);
    if (!d_y_all) return;
    CHK("GPU Packing Online", ensure_stream_and_constants());
    const size_t ys = (size_t)n_inner * poly_len * 8, zs = (size_t)t_exp_left * poly_len * 8;
    CHK("GPU Packing Online", cudaMemcpyAsync(d_y_all, h_y_all, ys, cudaMemcpyHostToDevice, g_stream));
    CHK("GPU Packing Online", cudaMemcpyAsync(d_y_bar_all, h_y_bar_all, ys, cudaMemcpyHostToDevice, g_stream));
    CHK("GPU Packing Online", cudaMemcpyAsync(d_z_body, h_z_body, zs, cudaMemcpyHostToDevice, g_stream));
}

void gpu_packing_online_compute(uint64_t* h_output, int num_outputs, int nphalf_minus_1, int t_exp_left,
                                int poly_len, int, uint64_t mod0, uint64_t mod1, uint64_t, uint64_t) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!d_bold_t || !d_y_all) {
        fprintf(stderr, "[GPU Packing Online] Data not uploaded!\n");
        return;
    }
    if (bad_shape("GPU Packing Online", t_exp_left, poly_len)) return;
    if (mod0 != ipr::Q0 || mod1 != ipr::Q1) {
        fprintf(stderr, "[GPU Packing Online] unsupported moduli\n");
        return;
    }
    CHK("GPU Packing Online", ensure_stream_and_constants());
    CHK("GPU Packing Online", ipr::launch_pack_materialized(d_bold_t, d_bold_t_bar, d_bold_t_hat, d_y_all,
                                                            d_y_bar_all, d_z_body, num_outputs, nphalf_minus_1,
                                                            d_output, g_stream));
    CHK("GPU Packing Online", cudaMemcpyAsync(h_output, d_output, (size_t)num_outputs * 2 * poly_len * 8,
                                              cudaMemcpyDeviceToHost, g_stream));
    CHK("GPU Packing Online", cudaStreamSynchronize(g_stream));
}

void gpu_packing_online_adopt_precomp(uint64_t* bt, uint64_t* btb, uint64_t* bth, int num_outputs, int n_inner,
                                      int, int poly_len) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_adopted) {
        if (d_bold_t) cudaFree(d_bold_t);
        if (d_bold_t_bar) cudaFree(d_bold_t_bar);
        if (d_bold_t_hat) cudaFree(d_bold_t_hat);
    }
    d_bold_t = bt;
    d_bold_t_bar = btb;
    d_bold_t_hat = bth;
    g_adopted = true;
    g_n_inner = n_inner;
    if (d_output) cudaFree(d_output);
    d_output = nullptr;
    CHK("GPU Packing Online", cudaMalloc(&d_output, (size_t)num_outputs * 2 * poly_len * 8));
}

void gpu_packing_online_swap_precomp(uint64_t* bt, uint64_t* btb, uint64_t* bth, int num_outputs, int n_inner,
                                     int, int poly_len) {
    std::lock_guard<std::mutex> lk(g_mu);
    d_bold_t = bt;
    d_bold_t_bar = btb;
    d_bold_t_hat = bth;
    g_adopted = true;
    g_n_inner = n_inner;
    if (d_output) cudaFree(d_output);
    d_output = nullptr;
    CHK("GPU Packing Online", cudaMalloc(&d_output, (size_t)num_outputs * 2 * poly_len * 8));
}

void gpu_packing_online_free(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_adopted) {
        if (d_bold_t) cudaFree(d_bold_t);
        if (d_bold_t_bar) cudaFree(d_bold_t_bar);
        if (d_bold_t_hat) cudaFree(d_bold_t_hat);
    }
    d_bold_t = d_bold_t_bar = d_bold_t_hat = nullptr;
    g_adopted = false;
    for (uint64_t** p : {&d_y_all, &d_y_bar_all, &d_z_body, &d_output})
        if (*p) {
            cudaFree(*p);
            *p = nullptr;
        }
}

}  // extern "C"
