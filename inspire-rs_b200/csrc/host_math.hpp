// host_math.hpp — host-side parameter derivation for the respond() path:
// moduli constants, NTT twiddle tables, the RGSW mask row, and the keyword
// server shape plan.  Restates (rkdud007/inspire-rs):
//   Params::init                    src/core/params.rs:225-301
//   build_ntt_tables                src/core/ntt.rs:74-108
//   get_minimal_primitive_root      src/core/number_theory.rs:41-55
//   ChaCha20Rng + random_rng        rand_chacha 0.10 / src/core/poly.rs:211-231
//   params_rgswpir_given_input_size_and_dim0  src/protocol/wire.rs:386-477
//   KeywordServerSetupPlan::from_shape        src/pir/server/keyword.rs:145-233
#pragma once
#include <cstdint>
#include <vector>

namespace ipr {

struct HostParams {
    uint64_t q[2];
    uint64_t modulus;
    uint64_t barrett[2];      // floor(2^64 / q_l)
    uint32_t q0_inv_mod_q1;
    // [limb][N] u32 twiddle tables: forward psi powers (bit-reversed order) and
    // their Shoup companions; inverse powers pre-halved and companions
    std::vector<uint32_t> fw, fwp, iw, iwp;
    std::vector<uint32_t> row0;  // [2][N] NTT(-a), a from ChaCha20Rng([7;32])
    // for inverse transforms that leave out N^-1 (the fold folds it into its operands):
    // plain inverse twiddles (2 x the pre-halved ones) with Shoup companions, row 0 times
    // N^-1, and N^-1 mod q_l with its companion as {w0, wp0, w1, wp1}
    std::vector<uint32_t> iwu, iwup, row0s;
    uint32_t ninv[4];
    // the one-chain fold's Montgomery operands (R = 2^32): row 0 x N^-1 x R and N^-1 x R
    // (with its Shoup companion) per limb, so that a Montgomery reduction of a product with
    // them leaves the product with N^-1
    std::vector<uint32_t> row0m;
    uint32_t ninvr[4];
    // the forward and plain inverse twiddles interleaved with their companions: [limb][N][2]
    std::vector<uint32_t> fwi, iwi;
};

void host_params_init(HostParams& p);

// ChaCha20Rng keystream (rand_chacha 0.10 layout): 64-bit block counter in words 12-13,
// 64-bit stream id in words 14-15, u64 = two consecutive words, low first
struct ChaCha {
    uint32_t key[8];
    uint64_t counter = 0;
    uint64_t stream = 0;
    uint32_t buf[16];
    int idx = 16;
    static uint32_t rotl(uint32_t x, int n);
    void block();
    uint64_t next_u64();
};
ChaCha chacha_from_seed(const uint8_t seed[32], uint64_t stream = 0);

// ntt_forward (src/core/ntt.rs:111-160) of a [2][N] array of limb residues, in place,
// reference evaluation order
void forward_ntt_u64(const HostParams& p, uint64_t* a);

// Inputs of the offline precomputation derived from fixed seeds: the hint query of
// generate_pseudorandom_query(SEED_0) ([polys][2][N] NTT) and the W / V masks of
// OfflinePackingKeys::init_full ([3][2][N] NTT each).
void offline_host_inputs(const HostParams& p, unsigned polys, std::vector<uint32_t>& query,
                         std::vector<uint32_t>& w_mask, std::vector<uint32_t>& v_mask);

// Only the two reduction constants the kernels keep in constant memory
// (floor(2^64 / q_l) and q0^-1 mod q1); computes them without touching the heap.
void host_moduli_constants(uint64_t barrett[2], uint32_t* q0_inv_mod_q1);

struct Plan {
    uint64_t num_items, entry_size, item_size_bits, dim0;
    uint64_t db_rows, db_cols, instances, interp, c;
    uint64_t peak_bytes;
};
// returns 0 or a negative IPR_E_* status
int plan_from_shape(uint64_t record_count, uint64_t key_size, uint64_t value_size, uint64_t buckets,
                    uint64_t dim0, Plan& out);

uint64_t query_bytes(uint64_t db_rows, unsigned nq);

}  // namespace ipr
