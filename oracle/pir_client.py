"""A seeded keyword-PIR client for end-to-end tests.  TEST INFRASTRUCTURE ONLY.

It restates the client side of inspire-rs, so that a test can encrypt a real
query, send its bytes through a server (the device library or the oracle),
and decrypt the response back to the database values:

* secret key: `gen_ternary_mat` (src/pir/client/base.rs:126-139), 256
  coefficients +1 and 256 coefficients -1 in shuffled positions;
* first-dimension query: `generate_query_impl` / `generate_query_b_values`
  (client/online.rs:216-287, 340-357) with the public `a` polynomials drawn
  from ChaCha20Rng(get_seed(SEED_0)), and `pack_query` (online.rs:26-52);
* RGSW bodies: `build_query_for_index` (client/keyword.rs:137-191), the `a`
  polynomials drawn from ChaCha20Rng(RGSW_SEEDS[i]) (protocol/wire.rs:88);
* packing keys: `PackingKeys::init_full` (src/pir/packing.rs:1895-1943) and
  `generate_ksk_body` (packing.rs:3272-3293) under the offline W/V masks;
* wire encoding: `serialize_keyword_query` (protocol/wire.rs:542-615);
* decryption: `recover_how_many` (pir/modulus_switch.rs:102-130), then
  `decrypt_ct_reg_measured` (client/online.rs:118-135) and `extract`
  (client/keyword.rs:232-283).

What is not restated bit for bit: the reference seeds its noise and secret
key generators from `rand::random()` and samples the discrete Gaussian with
its own sampler (discrete_gaussian.rs); here both come from a seeded NumPy
generator with the same width (s = 16.042421, sigma = s / sqrt(2 pi) = 6.4).
The server's answer does not depend on which noise the client drew, and
decryption only needs the noise small, so a response that decrypts to the
database values shows the whole respond() path computes what the scheme
needs, independently of the oracle's restatement of each step.

The reference keyword client never calls `generate_secret_keys`, so its
secret key is the zero polynomial (`Client::init`, base.rs:370-389, leaves it
zero and `setup_from_public_params`, keyword.rs:60-115, keeps it); a zero key
would hide wrong key-switching keys, so this client draws a real one.
"""
from __future__ import annotations

import numpy as np

import oracle as _o

N = _o.N
Q0, Q1, Q = _o.Q0, _o.Q1, _o.Q
P = 65535                      # pt_modulus, params_rgswpir_given_input_size_and_dim0 (wire.rs:419-424)
SCALE_K = Q // P               # params.modulus / params.pt_modulus (online.rs:229)
BITS_PER = 19                  # get_bits_per(params, 3) (gadget.rs:3-9): floor(56 / 3) + 1
T = 3                          # t_gsw = t_exp_left = 3
SIGMA = 6.4
HAMMING = 256
Q1_PRIME, Q2_PRIME = 1 << 20, 268369921      # get_q_prime_1 / get_q_prime_2
Q1_BITS, Q2_BITS = 20, 28
PUBLIC_SEED_0 = bytes(32)                    # STATIC_PUBLIC_SEED with byte 0 = SEED_0 = 0 (scheme.rs:38-39)
RGSW_SEED = bytes([7] * 32)                  # every entry of RGSW_SEEDS (wire.rs:88-113)
LIMB_Q = np.array([Q0, Q1], dtype=np.uint64).reshape(2, 1)


# --- arithmetic on NTT-domain polynomials: [2][N] limb-major residues ------
def ntt_mul(a, b):
    return (a.reshape(2, N) * b.reshape(2, N)) % LIMB_Q


def ntt_add(*xs):
    acc = np.zeros((2, N), dtype=np.uint64)
    for x in xs:
        acc = (acc + x.reshape(2, N)) % LIMB_Q
    return acc


def ntt_neg(a):
    return (LIMB_Q - a.reshape(2, N)) % LIMB_Q


def ntt_const(c: int):
    """NTT of the constant polynomial c: c in every evaluation slot"""
    return np.repeat(np.array([[c % Q0], [c % Q1]], dtype=np.uint64), N, axis=1)


def to_ntt(raw):
    return _o.to_ntt(np.ascontiguousarray(raw, dtype=np.uint64)).reshape(2, N)


def from_ntt(x):
    return _o.from_ntt(np.ascontiguousarray(x, dtype=np.uint64).reshape(-1))


def condense(x):
    """condense_matrix (packing.rs:867-884): lo32 = mod q0 residue, hi32 = mod q1 residue"""
    x = x.reshape(2, N)
    return x[0] | (x[1] << np.uint64(32))


_MASKS = None


def _masks():
    """w_mask, v_mask (OfflinePackingKeys::init_full, packing.rs:1837-1870), computed once"""
    global _MASKS
    if _MASKS is None:
        w_mask, v_mask, _, _ = _o.offline_keys()
        _MASKS = (w_mask, v_mask)
    return _MASKS


class TestClient:
    """Keyword-PIR client for a server plan: db_rows, interp (interpolation
    degree), c (fold groups), per (buckets per DB row), item_elems (u16
    elements per entry)."""

    def __init__(self, db_rows: int, interp: int, c: int, per: int, item_elems: int, seed: int):
        self.db_rows, self.interp, self.c, self.per, self.item_elems = db_rows, interp, c, per, item_elems
        self.rng = np.random.default_rng(seed)
        s = np.zeros(N, dtype=np.int64)
        s[:HAMMING], s[HAMMING:2 * HAMMING] = 1, -1
        self.rng.shuffle(s)
        self.s_raw = (s % Q).astype(np.uint64)
        self.s_ntt = to_ntt(self.s_raw)

    # --- sampling ---------------------------------------------------------
    def noise_raw(self):
        e = np.rint(self.rng.normal(0.0, SIGMA, N)).astype(np.int64)
        return (e % Q).astype(np.uint64)

    def body(self, a_raw, msg_ntt):
        """row 1 of encrypt_matrix_reg (base.rs:426-436, 502-511): NTT(e) + s * a + msg"""
        return ntt_add(to_ntt(self.noise_raw()), ntt_mul(self.s_ntt, to_ntt(a_raw)), msg_ntt)

    # --- packing keys -----------------------------------------------------
    def ksk_body(self, generator: int, mask):
        """generate_ksk_body (packing.rs:3272-3293): -s * mask + e + tau_g(s) * g, 3 columns"""
        tau_s = to_ntt(_o.automorph_poly(self.s_raw, generator))
        out = np.zeros((T, 2, N), dtype=np.uint64)
        for k in range(T):
            out[k] = ntt_add(ntt_mul(self.s_ntt, ntt_neg(mask[k])), to_ntt(self.noise_raw()),
                             ntt_mul(tau_s, ntt_const(1 << (BITS_PER * k))))
        return out

    def packing_keys(self):
        """PackingKeys::init_full: (y_body, z_body) NTT [3][2][N], generators 5 and 2N - 1"""
        w_mask, v_mask = _masks()
        return self.ksk_body(_o.gen_pow(1), w_mask), self.ksk_body(2 * N - 1, v_mask)

    # --- one sub-query ------------------------------------------------------
    def target(self, bucket: int):
        """(target_row, target_col, target_sub_col) of build_query_for_index (keyword.rs:138-141)"""
        row = bucket // self.per
        col = (bucket % self.per) * self.item_elems
        sub = (col % (self.interp * N)) // N
        return row, col, sub

    def query_row(self, target_row: int):
        """packed_query_row: b values of the db_rows / N scaled-Regev samples, condensed"""
        polys = self.db_rows // N
        a_all = _o.random_raw(PUBLIC_SEED_0, polys * N).reshape(polys, N)
        out = np.zeros(self.db_rows, dtype=np.uint64)
        for i in range(polys):
            msg = np.zeros(N, dtype=np.uint64)
            if i == target_row // N:
                msg[target_row % N] = SCALE_K
            b_raw = from_ntt(self.body(a_all[i], to_ntt(msg)))
            out[i * N:(i + 1) * N] = (b_raw % np.uint64(Q0)) | ((b_raw % np.uint64(Q1)) << np.uint64(32))
        return out

    def rgsw_body(self, sub: int):
        """ct_gsw_body [6][2][N] NTT: column 2j+1 encrypts sigma_j = +-2^(19 j) X^(e mod N),
        column 2j encrypts s * sigma_j (keyword.rs:148-181)"""
        a = _o.random_raw(RGSW_SEED, N)          # every RGSW_SEEDS entry restarts the same stream
        e = (2 * N * sub // self.interp) % (2 * N)
        out = np.zeros((2 * T, 2, N), dtype=np.uint64)
        for j in range(T):
            sig = np.zeros(N, dtype=np.uint64)
            v = 1 << (BITS_PER * j)
            sig[e % N] = v if e < N else Q - v
            sig_ntt = to_ntt(sig)
            out[2 * j + 1] = self.body(a, sig_ntt)
            out[2 * j] = self.body(a, ntt_mul(self.s_ntt, sig_ntt))
        return out

    # --- the payload ----------------------------------------------------------
    def query(self, buckets):
        """query bytes for the given buckets (one sub-query each), plus the fields"""
        y, z = self.packing_keys()
        subs = [(self.query_row(self.target(b)[0]), self.rgsw_body(self.target(b)[2])) for b in buckets]
        fields = {"y_body": [condense(y[k]) for k in range(T)], "z_body": [condense(z[k]) for k in range(T)],
                  "queries": subs}
        return serialize_query(fields), fields

    # --- decryption -------------------------------------------------------------
    def decrypt_result(self, chunk: bytes):
        """one 12,288-byte result -> its N plaintext values mod 65535"""
        bits = np.unpackbits(np.frombuffer(chunk, dtype=np.uint8), bitorder="little")
        w0 = bits[:Q2_BITS * N].reshape(N, Q2_BITS).astype(np.uint64)
        w1 = bits[Q2_BITS * N:(Q2_BITS + Q1_BITS) * N].reshape(N, Q1_BITS).astype(np.uint64)
        v0 = (w0 << np.arange(Q2_BITS, dtype=np.uint64)).sum(axis=1, dtype=np.uint64)
        v1 = (w1 << np.arange(Q1_BITS, dtype=np.uint64)).sum(axis=1, dtype=np.uint64)
        row0 = _o.rescale_many(v0, Q2_PRIME, Q)
        row1 = _o.rescale_many(v1, Q1_PRIME, Q)
        dec = from_ntt(ntt_add(ntt_mul(self.s_ntt, to_ntt(row0)), to_ntt(row1)))
        return _o.rescale_many(dec, Q, P)

    def decrypt(self, response: bytes):
        """the response bytes -> per sub-query, the c results' plaintexts [c][N], and the stash"""
        off = 0

        def u32():
            nonlocal off
            v = int.from_bytes(response[off:off + 4], "little")
            off += 4
            return v
        results = []
        for _ in range(u32()):
            n = u32()
            body = response[off:off + n]
            off += n
            step = n // self.c
            results.append(np.stack([self.decrypt_result(body[w * step:(w + 1) * step]) for w in range(self.c)]))
        stash = []
        for _ in range(u32()):
            n = u32()
            stash.append(bytes(response[off:off + n]))
            off += n
        return results, stash

    def extract(self, bucket: int, plaintext) -> bytes:
        """the entry bytes of `bucket` from its sub-query's plaintexts (keyword.rs:246-257);
        None when the entry crosses a polynomial boundary and is not in the returned one"""
        _, col, _ = self.target(bucket)
        poly, coeff = col // N, col % N
        off = (poly // self.interp) * N + coeff
        flat = np.asarray(plaintext, dtype=np.uint64).reshape(-1)
        if coeff + self.item_elems > N:
            return None
        vals = flat[off:off + self.item_elems].astype(np.uint16)
        return vals.astype(">u2").tobytes()


def serialize_query(fields) -> bytes:
    """serialize_keyword_query (wire.rs:542-615): a count byte, then 56-bit fields
    (crt0 | crt1 << 28) LSB first: y/z keys interleaved per (column, slot), then per
    sub-query its packed row and its 6 RGSW bodies"""
    m28 = np.uint64((1 << 28) - 1)
    parts = []
    for k in range(T):
        yz = np.empty(2 * N, dtype=np.uint64)
        yz[0::2], yz[1::2] = fields["y_body"][k], fields["z_body"][k]
        parts.append((yz & m28) | ((yz >> np.uint64(32)) << np.uint64(28)))
    for row, gsw in fields["queries"]:
        parts.append((row & m28) | ((row >> np.uint64(32)) << np.uint64(28)))
        g = np.asarray(gsw, dtype=np.uint64).reshape(2 * T, 2, N)
        parts.append((g[:, 0, :] | (g[:, 1, :] << np.uint64(28))).reshape(-1))
    words = np.concatenate(parts).astype("<u8")
    return bytes([len(fields["queries"])]) + words.view(np.uint8).reshape(-1, 8)[:, :7].tobytes()


class SeededClient(TestClient):
    """The device client's deterministic randomness (ipr_client_*), restated for parity:
    the ternary key is placed by a Fisher-Yates shuffle of [+1 x 256, -1 x 256, 0 ...] whose
    step i (from N-1 down to 1) swaps with j = (u * (i + 1)) >> 64, u the next u64 of
    ChaCha20(seed, stream 1); the noise of a query with nonce n is, for its global coefficient
    index g, a centered binomial sample with eta = 82 from ChaCha20 block g of stream 2 + n
    (popcount of words 0, 1 and the low 18 bits of word 2 minus that of words 3, 4, 5).  The
    noise polynomials follow the order in which TestClient.query draws them."""

    def __init__(self, db_rows: int, interp: int, c: int, per: int, item_elems: int, seed: bytes):
        super().__init__(db_rows, interp, c, per, item_elems, seed=0)
        self.seed = bytes(seed)
        words = _o.chacha_blocks(self.seed, 1, 0, N // 8).astype(np.uint64).reshape(-1)
        u64 = [int(words[2 * k]) | (int(words[2 * k + 1]) << 32) for k in range(N)]
        s = [1] * HAMMING + [-1] * HAMMING + [0] * (N - 2 * HAMMING)
        for step, i in enumerate(range(N - 1, 0, -1)):
            j = (u64[step] * (i + 1)) >> 64
            s[i], s[j] = s[j], s[i]
        self.s = np.array(s, dtype=np.int8)
        self.s_raw = (self.s.astype(np.int64) % Q).astype(np.uint64)
        self.s_ntt = to_ntt(self.s_raw)
        self._noise, self._next = None, 0

    def noise_raw(self):
        e = self._noise[self._next]
        self._next += 1
        return (e % Q).astype(np.uint64)

    def query(self, buckets, nonce: int = 0):
        npolys = 6 + len(buckets) * (self.db_rows // N + 6)
        w = _o.chacha_blocks(self.seed, 2 + nonce, 0, npolys * N)
        m = np.uint32((1 << 18) - 1)
        pos = np.bitwise_count(w[:, 0]) + np.bitwise_count(w[:, 1]) + np.bitwise_count(w[:, 2] & m)
        neg = np.bitwise_count(w[:, 3]) + np.bitwise_count(w[:, 4]) + np.bitwise_count(w[:, 5] & m)
        self._noise = (pos.astype(np.int64) - neg.astype(np.int64)).reshape(npolys, N)
        self._next = 0
        out = super().query(buckets)
        assert self._next == npolys
        return out


# --- cuckoo positions (src/pir/keyword/cuckoo.rs:105-131) -------------------------------------
_M64 = (1 << 64) - 1


def siphash24(k0: int, k1: int, msg: bytes) -> int:
    """SipHash-2-4 (Aumasson and Bernstein, 2012) of msg under the 64-bit keys k0, k1"""
    def rotl(x, b):
        return ((x << b) | (x >> (64 - b))) & _M64
    v = [k0 ^ 0x736f6d6570736575, k1 ^ 0x646f72616e646f6d, k0 ^ 0x6c7967656e657261, k1 ^ 0x7465646279746573]

    def rnd():
        v[0] = (v[0] + v[1]) & _M64; v[1] = rotl(v[1], 13) ^ v[0]; v[0] = rotl(v[0], 32)
        v[2] = (v[2] + v[3]) & _M64; v[3] = rotl(v[3], 16) ^ v[2]
        v[0] = (v[0] + v[3]) & _M64; v[3] = rotl(v[3], 21) ^ v[0]
        v[2] = (v[2] + v[1]) & _M64; v[1] = rotl(v[1], 17) ^ v[2]; v[2] = rotl(v[2], 32)
    full = len(msg) // 8 * 8
    blocks = [int.from_bytes(msg[i:i + 8], "little") for i in range(0, full, 8)]
    blocks.append(int.from_bytes(msg[full:], "little") | ((len(msg) & 0xFF) << 56))
    for m in blocks:
        v[3] ^= m
        rnd()
        rnd()
        v[0] ^= m
    v[2] ^= 0xFF
    for _ in range(4):
        rnd()
    return v[0] ^ v[1] ^ v[2] ^ v[3]


def cuckoo_positions(seed: bytes, num_buckets: int, num_hashes: int, key: bytes):
    """CuckooHash::all_positions: SipHash-2-4 with keys (seed[..8] ^ i, seed[8..] ^ (i << 32)) mod
    num_buckets; the all-zero seed is the identity layout (cuckoo.rs:105-121)"""
    if bytes(seed) == bytes(16):
        idx = int.from_bytes(key[-8:].ljust(8, b"\0") if len(key) < 8 else key[-8:], "big")
        half = num_buckets // 2
        return [idx % half if i == 0 else half + idx % half for i in range(num_hashes)]
    s0, s1 = int.from_bytes(seed[:8], "little"), int.from_bytes(seed[8:16], "little")
    return [siphash24(s0 ^ i, s1 ^ (i << 32), bytes(key)) % num_buckets for i in range(num_hashes)]


# --- the e2e test's target selection (tests/e2e_mlkem.rs:17-19) -------------------------------
def chacha_u32_stream(seed_u64: int):
    """next_u32 of ChaCha20Rng::seed_from_u64(seed) (rand_core's PCG32 key expansion, then the
    keystream words in order); a restatement of the crates' published algorithms"""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import oracle as orc
    key = orc.seed_from_u64(seed_u64)
    ctr = 0
    while True:
        for w in orc.chacha_blocks(key, 0, ctr, 1)[0]:
            yield int(w)
        ctr += 1


def random_range_u32(words, n: int) -> int:
    """a uniform index in [0, n) from u32 words by the widening multiply with one
    bias-correcting step (the single-sample integer method of rand 0.9 / 0.10 for ranges
    that fit u32); which record the e2e test picks does not change what it checks"""
    hi, lo = divmod(next(words) * n, 1 << 32)
    if lo > (-n) % (1 << 32):
        hi2 = (next(words) * n) >> 32
        hi += (lo + hi2) >> 32
    return hi
