// state.cu — the server state file: the setup outputs a server was built from, written
// once and loaded on restart, so that a restart skips the DB encode and the offline
// precomputation (the reference has no such file: its setup reruns both on every start,
// src/pir/server/keyword.rs:366-457).
//
// Layout (little-endian, every section 4096-byte aligned):
//   [0, 4096)  header: magic "IPRSTATE", version, the plan, the public parameters, the
//              stash shape, one {offset, bytes, checksum} entry per section, and a
//              checksum of the header itself
//   sections   encoded DB [db_cols][db_rows] u16, a_hat [instances][2048] u64,
//              bold_t and bold_t_bar [instances][3069][2048] u64 condensed,
//              bold_t_hat [instances][3][2048] u64 condensed, stash bytes
// i.e. exactly the arrays of ipr_server_data.  Section checksums are
//   sum over 64-bit words w_i of mix64(w_i + i * 0x9E3779B97F4A7C15)   (mod 2^64)
// with mix64 the splitmix64 finaliser (a sum of position-keyed hashes: order-independent
// to compute, so each device section is checked by one reduction kernel on the GPU, yet
// sensitive to any changed, moved or swapped word).  The stash's last word is zero-padded.
//
// Both directions stream through two pinned 64 MB staging buffers: while one chunk
// crosses PCIe asynchronously the host reads or writes the other.
#include <cuda_runtime.h>
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <cstdarg>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ipr_b200.h"
#include "server_internal.hpp"

namespace {

constexpr char kMagic[8] = {'I', 'P', 'R', 'S', 'T', 'A', 'T', 'E'};
constexpr uint32_t kVersion = 1;
constexpr uint64_t kHeaderBytes = 4096;
constexpr uint64_t kChunk = 64ull << 20;
constexpr int kN = 2048;
constexpr int kNInner = 3069;
enum { SEC_DB, SEC_AHAT, SEC_BT, SEC_BTB, SEC_BTH, SEC_STASH, SEC_COUNT };
const char* const kSectionName[SEC_COUNT] = {"db", "a_hat", "bold_t", "bold_t_bar", "bold_t_hat", "stash"};

struct SectionEntry {
    uint64_t offset, bytes, checksum, reserved;
};
struct FileHeader {
    char magic[8];
    uint32_t version, header_bytes;
    uint64_t plan[10];  // ipr_plan fields in declaration order
    uint64_t key_size, value_size, num_records, stash_count, stash_entry;
    uint8_t cuckoo_seed[16];
    SectionEntry sec[SEC_COUNT];
    uint64_t header_checksum;  // of every byte before this field
};
static_assert(sizeof(FileHeader) <= kHeaderBytes, "header must fit its block");

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    ipr::set_last_error(buf);
    return code;
}

#define CU(call)                                                                                      \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess)                                                                        \
            return fail(e_ == cudaErrorMemoryAllocation ? IPR_E_OOM : IPR_E_CUDA, "%s: %s", #call, \
                        cudaGetErrorString(e_));                                                      \
    } while (0)

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t x) {
    x ^= x >> 30;
    x *= 0xBF58476D1CE4E5B9ull;
    x ^= x >> 27;
    x *= 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
constexpr uint64_t kPosKey = 0x9E3779B97F4A7C15ull;

uint64_t host_checksum(const uint8_t* p, uint64_t bytes) {
    uint64_t acc = 0, i = 0;
    for (; (i + 1) * 8 <= bytes; i++) {
        uint64_t w;
        std::memcpy(&w, p + i * 8, 8);
        acc += mix64(w + i * kPosKey);
    }
    if (i * 8 < bytes) {
        uint64_t w = 0;
        std::memcpy(&w, p + i * 8, bytes - i * 8);
        acc += mix64(w + i * kPosKey);
    }
    return acc;
}

// grid-stride partial sums, one atomic add per block (addition mod 2^64 is commutative,
// so the result does not depend on the schedule)
__global__ void __launch_bounds__(256) k_state_checksum(const uint64_t* __restrict__ p, uint64_t nwords,
                                                        unsigned long long* out) {
    uint64_t acc = 0;
    for (uint64_t i = blockIdx.x * 256ull + threadIdx.x; i < nwords; i += (uint64_t)gridDim.x * 256)
        acc += mix64(__ldg(p + i) + i * kPosKey);
#pragma unroll
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
    __shared__ uint64_t part[8];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint64_t s = 0;
        for (int w = 0; w < 8; w++) s += part[w];
        atomicAdd(out, (unsigned long long)s);
    }
}

int device_checksum(ipr_server* s, const void* d, uint64_t bytes, uint64_t* out) {
    unsigned long long* d_sum = nullptr;
    CU(cudaMallocAsync(&d_sum, sizeof(*d_sum), s->stream));
    cudaError_t e = cudaMemsetAsync(d_sum, 0, sizeof(*d_sum), s->stream);
    if (e == cudaSuccess) {
        k_state_checksum<<<s->sm_count * 8, 256, 0, s->stream>>>(static_cast<const uint64_t*>(d), bytes / 8, d_sum);
        e = cudaGetLastError();
    }
    unsigned long long h = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d_sum, sizeof(h), cudaMemcpyDeviceToHost, s->stream);
    cudaFreeAsync(d_sum, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    CU(e);
    *out = h;
    return IPR_OK;
}

// two pinned staging buffers and their events; released on every exit path
struct Staging {
    void* buf[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    int init() {
        for (int b = 0; b < 2; b++) {
            CU(cudaMallocHost(&buf[b], kChunk));
            CU(cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming));
        }
        return IPR_OK;
    }
    ~Staging() {
        for (int b = 0; b < 2; b++) {
            if (ev[b]) cudaEventSynchronize(ev[b]), cudaEventDestroy(ev[b]);
            if (buf[b]) cudaFreeHost(buf[b]);
        }
    }
};

struct Fd {
    int fd = -1;
    ~Fd() {
        if (fd >= 0) close(fd);
    }
};

int write_all(int fd, const void* p, uint64_t n, uint64_t off, const char* path) {
    const uint8_t* c = static_cast<const uint8_t*>(p);
    while (n) {
        const ssize_t w = pwrite(fd, c, n, (off_t)off);
        if (w <= 0) return fail(IPR_E_IO, "state file %s: write failed at offset %llu (%s)", path,
                                (unsigned long long)off, strerror(errno));
        c += w, n -= (uint64_t)w, off += (uint64_t)w;
    }
    return IPR_OK;
}

int read_all(int fd, void* p, uint64_t n, uint64_t off, const char* path) {
    uint8_t* c = static_cast<uint8_t*>(p);
    while (n) {
        const ssize_t r = pread(fd, c, n, (off_t)off);
        if (r < 0) return fail(IPR_E_IO, "state file %s: read failed at offset %llu (%s)", path,
                               (unsigned long long)off, strerror(errno));
        if (r == 0) return fail(IPR_E_FORMAT, "state file %s: truncated at offset %llu", path, (unsigned long long)off);
        c += r, n -= (uint64_t)r, off += (uint64_t)r;
    }
    return IPR_OK;
}

// device -> file: chunk k is copied into buffer k % 2 while chunk k - 1 is written
int save_section(ipr_server* s, Staging& sg, int fd, const void* d, uint64_t bytes, uint64_t off, const char* path) {
    const uint64_t chunks = (bytes + kChunk - 1) / kChunk;
    for (uint64_t k = 0; k <= chunks; k++) {
        if (k < chunks) {
            const int b = (int)(k & 1);
            const uint64_t n = std::min(kChunk, bytes - k * kChunk);
            CU(cudaEventSynchronize(sg.ev[b]));  // the buffer's previous chunk has been written (host side)
            CU(cudaMemcpyAsync(sg.buf[b], static_cast<const uint8_t*>(d) + k * kChunk, n, cudaMemcpyDeviceToHost,
                               s->stream));
            CU(cudaEventRecord(sg.ev[b], s->stream));
        }
        if (k > 0) {
            const uint64_t j = k - 1;
            const int b = (int)(j & 1);
            const uint64_t n = std::min(kChunk, bytes - j * kChunk);
            CU(cudaEventSynchronize(sg.ev[b]));
            int st = write_all(fd, sg.buf[b], n, off + j * kChunk, path);
            if (st) return st;
        }
    }
    return IPR_OK;
}

// file -> device: the host reads chunk k into buffer k % 2 while chunk k - 1 crosses PCIe
int load_section(ipr_server* s, Staging& sg, int fd, void* d, uint64_t bytes, uint64_t off, const char* path) {
    for (uint64_t k = 0; k * kChunk < bytes; k++) {
        const int b = (int)(k & 1);
        const uint64_t n = std::min(kChunk, bytes - k * kChunk);
        CU(cudaEventSynchronize(sg.ev[b]));  // the copy out of this buffer has finished
        int st = read_all(fd, sg.buf[b], n, off + k * kChunk, path);
        if (st) return st;
        CU(cudaMemcpyAsync(static_cast<uint8_t*>(d) + k * kChunk, sg.buf[b], n, cudaMemcpyHostToDevice, s->stream));
        CU(cudaEventRecord(sg.ev[b], s->stream));
    }
    return IPR_OK;
}

void section_shapes(const ipr::Plan& p, uint64_t stash_bytes, uint64_t (&bytes)[SEC_COUNT]) {
    const uint64_t no = p.instances;
    bytes[SEC_DB] = p.db_rows * p.db_cols * 2;
    bytes[SEC_AHAT] = no * kN * 8;
    bytes[SEC_BT] = bytes[SEC_BTB] = no * (uint64_t)kNInner * kN * 8;
    bytes[SEC_BTH] = no * 3ull * kN * 8;
    bytes[SEC_STASH] = stash_bytes;
}

uint64_t align_up(uint64_t x) { return (x + kHeaderBytes - 1) / kHeaderBytes * kHeaderBytes; }

}  // namespace

extern "C" {

int ipr_server_save(ipr_server* s, const char* path) {
    if (!s || !path) return fail(IPR_E_ARGS, "null argument");
    std::lock_guard<std::mutex> lock(s->mu);
    CU(cudaSetDevice(s->device));
    CU(cudaStreamSynchronize(s->stream));
    const ipr::Plan& p = s->plan;
    FileHeader h;
    std::memset(&h, 0, sizeof(h));
    std::memcpy(h.magic, kMagic, 8);
    h.version = kVersion;
    h.header_bytes = (uint32_t)kHeaderBytes;
    const uint64_t pf[10] = {p.num_items, p.entry_size, p.item_size_bits, p.dim0, p.db_rows,
                             p.db_cols,   p.instances,  p.interp,         p.c,    p.peak_bytes};
    std::memcpy(h.plan, pf, sizeof(pf));
    h.key_size = s->key_size;
    h.value_size = s->value_size;
    h.num_records = s->num_records;
    h.stash_count = s->stash_count;
    h.stash_entry = s->stash_entry;
    std::memcpy(h.cuckoo_seed, s->cuckoo_seed, 16);
    uint64_t bytes[SEC_COUNT];
    section_shapes(p, s->stash_count * s->stash_entry, bytes);
    const void* dev[SEC_COUNT] = {s->d_db, s->d_ahat, s->d_bt, s->d_btb, s->d_bth, s->d_stash};
    std::vector<uint8_t> stash(bytes[SEC_STASH]);
    if (!stash.empty()) CU(cudaMemcpy(stash.data(), s->d_stash, stash.size(), cudaMemcpyDeviceToHost));
    uint64_t off = kHeaderBytes;
    for (int k = 0; k < SEC_COUNT; k++) {
        h.sec[k].offset = off;
        h.sec[k].bytes = bytes[k];
        int st = k == SEC_STASH ? (h.sec[k].checksum = host_checksum(stash.data(), stash.size()), IPR_OK)
                                : device_checksum(s, dev[k], bytes[k], &h.sec[k].checksum);
        if (st) return st;
        off = align_up(off + bytes[k]);
    }
    h.header_checksum = host_checksum(reinterpret_cast<const uint8_t*>(&h), offsetof(FileHeader, header_checksum));

    Fd f;
    f.fd = open(path, O_WRONLY | O_CREAT | O_TRUNC, 0644);
    if (f.fd < 0) return fail(IPR_E_IO, "state file %s: cannot create (%s)", path, strerror(errno));
    std::vector<uint8_t> block(kHeaderBytes, 0);
    std::memcpy(block.data(), &h, sizeof(h));
    int st = write_all(f.fd, block.data(), kHeaderBytes, 0, path);
    if (st) return st;
    Staging sg;
    if ((st = sg.init())) return st;
    for (int k = 0; k < SEC_STASH; k++)
        if ((st = save_section(s, sg, f.fd, dev[k], bytes[k], h.sec[k].offset, path))) return st;
    if (!stash.empty() && (st = write_all(f.fd, stash.data(), stash.size(), h.sec[SEC_STASH].offset, path))) return st;
    // the file ends on a section boundary, so its size alone tells a truncated copy apart
    if (ftruncate(f.fd, (off_t)off) != 0) return fail(IPR_E_IO, "state file %s: %s", path, strerror(errno));
    if (fsync(f.fd) != 0) return fail(IPR_E_IO, "state file %s: fsync failed (%s)", path, strerror(errno));
    return IPR_OK;
}

int ipr_state_file_plan(const char* path, ipr_plan* out) {
    if (!path || !out) return fail(IPR_E_ARGS, "null argument");
    Fd f;
    f.fd = open(path, O_RDONLY);
    if (f.fd < 0) return fail(IPR_E_IO, "state file %s: cannot open (%s)", path, strerror(errno));
    std::vector<uint8_t> block(kHeaderBytes);
    int st = read_all(f.fd, block.data(), kHeaderBytes, 0, path);
    if (st) return st;
    FileHeader h;
    std::memcpy(&h, block.data(), sizeof(h));
    if (std::memcmp(h.magic, kMagic, 8) != 0) return fail(IPR_E_FORMAT, "state file %s: bad magic", path);
    if (h.version != kVersion || h.header_bytes != kHeaderBytes)
        return fail(IPR_E_FORMAT, "state file %s: version %u not supported (this build reads %u)", path, h.version,
                    kVersion);
    if (h.header_checksum != host_checksum(block.data(), offsetof(FileHeader, header_checksum)))
        return fail(IPR_E_FORMAT, "state file %s: header checksum mismatch", path);
    uint64_t* o = &out->num_items;
    for (int i = 0; i < 10; i++) o[i] = h.plan[i];
    return IPR_OK;
}

int ipr_server_load(int device, const char* path, ipr_server** out) {
    if (!path || !out) return fail(IPR_E_ARGS, "null argument");
    *out = nullptr;
    ipr_plan plan;
    int st = ipr_state_file_plan(path, &plan);
    if (st) return st;
    if (!plan.instances || plan.instances > (1u << 20) || plan.db_rows > (1u << 24) ||
        plan.db_cols != plan.instances * kN)
        return fail(IPR_E_FORMAT, "state file %s: implausible plan in the header", path);
    Fd f;
    f.fd = open(path, O_RDONLY);
    if (f.fd < 0) return fail(IPR_E_IO, "state file %s: cannot open (%s)", path, strerror(errno));
    FileHeader h;
    if ((st = read_all(f.fd, &h, sizeof(h), 0, path))) return st;
    struct stat sb;
    if (fstat(f.fd, &sb) != 0) return fail(IPR_E_IO, "state file %s: %s", path, strerror(errno));
    // the section table must match the plan's shapes and lie inside the file, in order
    ipr::Plan pp{};
    pp.db_rows = plan.db_rows, pp.db_cols = plan.db_cols, pp.instances = plan.instances;
    if (h.stash_count && !h.stash_entry) return fail(IPR_E_FORMAT, "state file %s: bad stash shape", path);
    if (h.stash_entry && h.stash_count > (1ull << 40) / h.stash_entry)
        return fail(IPR_E_FORMAT, "state file %s: bad stash shape", path);
    uint64_t bytes[SEC_COUNT];
    section_shapes(pp, h.stash_count * h.stash_entry, bytes);
    uint64_t off = kHeaderBytes;
    for (int k = 0; k < SEC_COUNT; k++) {
        if (h.sec[k].offset != off || h.sec[k].bytes != bytes[k])
            return fail(IPR_E_FORMAT, "state file %s: section %s does not match the plan", path, kSectionName[k]);
        off = align_up(off + bytes[k]);
    }
    if ((uint64_t)sb.st_size != off)
        return fail(IPR_E_FORMAT, "state file %s: %llu bytes, the header describes %llu", path,
                    (unsigned long long)sb.st_size, (unsigned long long)off);
    std::vector<uint8_t> stash(bytes[SEC_STASH]);
    if (!stash.empty() && (st = read_all(f.fd, stash.data(), stash.size(), h.sec[SEC_STASH].offset, path))) return st;
    if (host_checksum(stash.data(), stash.size()) != h.sec[SEC_STASH].checksum)
        return fail(IPR_E_FORMAT, "state file %s: section stash checksum mismatch", path);

    auto* s = new ipr_server();
    auto bail = [&](int code) {
        ipr_server_destroy(s);
        return code;
    };
    if ((st = ipr::server_init(s, device, &plan))) return bail(st);
    void* dev[SEC_STASH] = {s->d_db, s->d_ahat, s->d_bt, s->d_btb, s->d_bth};
    {
        Staging sg;
        if ((st = sg.init())) return bail(st);
        for (int k = 0; k < SEC_STASH; k++)
            if ((st = load_section(s, sg, f.fd, dev[k], bytes[k], h.sec[k].offset, path))) return bail(st);
    }
    for (int k = 0; k < SEC_STASH; k++) {
        uint64_t sum = 0;
        if ((st = device_checksum(s, dev[k], bytes[k], &sum))) return bail(st);
        if (sum != h.sec[k].checksum)
            return bail(fail(IPR_E_FORMAT, "state file %s: section %s checksum mismatch", path, kSectionName[k]));
    }
    ipr_server_data d;
    std::memset(&d, 0, sizeof(d));
    d.stash = stash.empty() ? nullptr : stash.data();
    d.stash_count = h.stash_count;
    d.stash_entry_bytes = h.stash_entry;
    d.key_size = h.key_size;
    d.value_size = h.value_size;
    d.num_records = h.num_records;
    std::memcpy(d.cuckoo_seed, h.cuckoo_seed, 16);
    if ((st = ipr::server_finish(s, false, &d))) return bail(st);
    *out = s;
    return IPR_OK;
}

}  // extern "C"
