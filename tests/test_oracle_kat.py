"""Pins the CPU oracle to the reference's own known-answer tests.

Each test restates a #[test] of rkdud007/inspire-rs (file:line given) against
the oracle (oracle/ipr_oracle.c).  Runs on CPU.
"""
import numpy as np
import pytest


def test_build_ntt_tables_kat(orc):
    # src/core/ntt.rs:797-815
    t = orc.ntt_tables()
    assert t.shape == (2, 4, 2048)
    assert int(t[0, 2, 0]) == 134184961
    assert int(t[0, 2, 1]) == 96647580
    x = 0
    for v in t.reshape(-1):
        x ^= int(v)
    assert x == 519370102


def test_ntt_forward_delta(orc):
    # src/core/ntt.rs:818-826: forward NTT of 100*delta is all 100
    v = np.zeros(4096, dtype=np.uint64)
    v[0] = 100
    v[2048] = 100
    out = orc.ntt_forward(v)
    assert int(out[50]) == 100 and int(out[2048 + 50]) == 100
    assert np.all(out == 100)


def test_ntt_inverse_constant(orc):
    # src/core/ntt.rs:828-840: inverse NTT of all-100 is 100*delta
    out = orc.ntt_inverse(np.full(4096, 100, dtype=np.uint64))
    assert int(out[0]) == 100 and int(out[2048]) == 100
    assert int(out[50]) == 0 and int(out[2048 + 50]) == 0


def test_ntt_roundtrip(orc):
    # src/core/ntt.rs:843-907 (round trip of random residues, seeded here)
    rng = np.random.default_rng(11)
    for _ in range(20):
        v = np.concatenate([rng.integers(0, orc.Q0, 2048), rng.integers(0, orc.Q1, 2048)]).astype(np.uint64)
        assert np.array_equal(orc.ntt_inverse(orc.ntt_forward(v)), v)


def test_get_barrett_crs_kat(orc):
    # src/core/arith.rs:483-497
    assert orc.get_barrett_crs(268369921) == (16144578669088582089, 68736257792)
    assert orc.get_barrett_crs(249561089) == (10966983149909726427, 73916747789)
    assert orc.get_barrett_crs(66974689739603969) == (7906011006380390721, 275)


def test_div2_uint_mod_kat(orc):
    # src/core/arith.rs:463-466
    assert orc.div2_uint_mod(3, 7) == 5


def test_barrett_u128_kat(orc):
    # src/core/arith.rs:499-515
    m = 66974689739603969

    def ex(v):
        return orc.barrett_reduction_u128_raw(m, 7906011006380390721, 275, v & (2**64 - 1), v >> 64)
    assert ex(m) == 0
    assert ex(m + 1) == 1
    assert ex(m * 7 + 5) == 5
    rng = np.random.default_rng(3)
    for _ in range(200):
        v = int(rng.integers(0, 2**63)) * 2**20 + int(rng.integers(0, 2**20))
        assert ex(v) == v % m


def test_barrett_u64_kat(orc):
    # src/core/arith.rs:517-528
    m, cr1 = 66974689739603969, 275
    rng = np.random.default_rng(5)
    for _ in range(200):
        v = int(rng.integers(0, 2**63)) * 2 + 1
        assert orc.barrett_raw_u64(v, cr1, m) == v % m


def test_crt_compose(orc):
    rng = np.random.default_rng(9)
    for _ in range(200):
        v = int(rng.integers(0, orc.Q))
        assert orc.crt_compose(v % orc.Q0, v % orc.Q1) == v


def test_gadget_invert_kat(orc):
    # src/core/gadget.rs:79-96: 2x1 -> 2*log_q rows, 1 bit per digit, row j + k*2
    mat = np.zeros((2, 2048), dtype=np.uint64)
    mat[0, 37] = 3
    mat[1, 37] = 6
    log_q = int(orc.params().modulus_log2)
    assert log_q == 56
    r = orc.gadget_invert_general(mat, log_q)
    assert r.shape == (2 * log_q, 2048)
    assert r[0, 37] == 1 and r[2, 37] == 1 and r[4, 37] == 0
    assert r[1, 37] == 0 and r[3, 37] == 1 and r[5, 37] == 1 and r[7, 37] == 0


def test_gadget_invert_three_digits(orc):
    # the respond() fold's gadget: 3 digits of 19 bits (gadget.rs:3-9), recomposes exactly
    rng = np.random.default_rng(1)
    rows = rng.integers(0, orc.Q, size=(2, 2048), dtype=np.uint64)
    g = orc.gadget_invert_2(rows)
    assert np.array_equal(g, orc.gadget_invert_general(rows, 3))
    for j in range(2):
        rec = g[j] + (g[j + 2] << np.uint64(19)) + (g[j + 4] << np.uint64(38))
        assert np.array_equal(rec, rows[j])
    assert int(g.max()) < 2**19


def test_full_multiply_kat(orc):
    # src/core/poly.rs:1027-1039: (100 x) * (7 x) = 700 x^2 through NTT
    a = np.zeros(2048, dtype=np.uint64)
    b = np.zeros(2048, dtype=np.uint64)
    a[1], b[1] = 100, 7
    an, bn = orc.to_ntt(a), orc.to_ntt(b)
    prod = np.concatenate([(an[:2048] * bn[:2048]) % np.uint64(orc.Q0), (an[2048:] * bn[2048:]) % np.uint64(orc.Q1)])
    c = orc.from_ntt(prod)
    assert int(c[2]) == 700
    assert int(c.sum()) == 700


@pytest.mark.parametrize("t", [3, 9, 17, 33, 65, 129, 257, 513, 1025, 2049])
def test_automorph_tables_kat(orc, t):
    # src/pir/packing.rs:3943-3985: NTT-domain automorphism through the table
    # equals the coefficient automorphism (poly.rs:531-543)
    rng = np.random.default_rng(t)
    poly = rng.integers(0, orc.Q, 2048, dtype=np.uint64)
    tab = orc.automorph_table(t)
    pn = orc.to_ntt(poly)
    rot = np.concatenate([pn[:2048][tab], pn[2048:][tab]])
    assert np.array_equal(orc.from_ntt(rot), orc.automorph_poly(poly, t))


def test_automorph_closed_form_matches_bruteforce(orc):
    # generate_automorph_tables_brute_force (packing.rs:1423-1468) vs the closed form,
    # over every generator power the rotations use plus a spread of odd t
    ts = sorted({int(orc.gen_pow(i)) for i in range(0, 1023, 37)} |
                {4096 - int(orc.gen_pow(i)) for i in range(0, 1023, 53)} | {1, 3, 4095, 2047, 2049})
    for t in ts:
        bf = orc.automorph_table_bruteforce(t, seed=t)
        assert bf is not None
        assert np.array_equal(bf, orc.automorph_table(t)), t


def test_gen_pows(orc):
    # PackParams::new (packing.rs:1639-1652): generator 5 for num_to_pack = poly_len
    assert [int(orc.gen_pow(i)) for i in range(5)] == [1, 5, 25, 125, 625]
    assert int(orc.gen_pow(1023)) == pow(5, 1023, 4096)


def test_read_write_arbitrary_bits_kat(orc):
    # src/core/util.rs:410-428
    ln, nb = 4096, 9
    data = np.zeros(ln, dtype=np.uint8)
    n = ln * 8 // nb - 64
    for i in range(n):
        orc.write_bits(data, (i * 7 + 13) % (1 << nb), i * nb, nb)
    for i in range(n):
        assert orc.read_bits(data, i * nb, nb) == (i * 7 + 13) % (1 << nb)


def test_chacha20_rfc8439_vector(orc):
    # RFC 8439 section 2.3.2 block function test vector (rand_chacha's core)
    key = bytes(range(32))
    nonce = bytes.fromhex("000000090000004a00000000")
    out = orc.chacha20_rfc8439_block(key, 1, nonce)
    assert out[:16].hex() == "10f1e7e4d13b5915500fdd1fa32071c4"


def test_rescale_properties(orc):
    # rescale (arith.rs:436-452): centred rounding q -> q'
    q, q2 = orc.Q, 268369921
    assert orc.rescale(0, q, q2) == 0
    assert orc.rescale(q - 1, q, q2) == 0           # -1 rounds to 0
    assert orc.rescale(q // 2 - 1, q, q2) == round((q // 2 - 1) * q2 / q) % q2
    rng = np.random.default_rng(2)
    for _ in range(300):
        v = int(rng.integers(0, q))
        c = v - q if v >= q // 2 else v
        s = 1 if c >= 0 else -1
        want = int((abs(c) * q2 + q // 2) // q) * s % q2
        assert orc.rescale(v, q, q2) == want


def test_plan_matches_reference_estimates(orc):
    # perf.md:46-69 figures the reference's estimate formula reproduces (keyword.rs:105-141)
    p = orc.plan_from_shape(5_000_000, 32, 1184, 8_388_608, 65_536)
    assert p["peak_bytes"] == 32_205_963_264
    assert (p["db_rows"], p["db_cols"], p["instances"]) == (65536, 131072, 64)
    assert orc.plan_from_shape(5_000_000, 32, 1184)["peak_bytes"] == 669_207_494_656


def test_plan_configs(orc):
    c0 = orc.plan_from_shape(10_000, 32, 1184)
    assert (c0["num_items"], c0["db_rows"], c0["db_cols"], c0["instances"], c0["interp"], c0["c"]) == \
        (32768, 2048, 16384, 8, 8, 1)
    c1 = orc.plan_from_shape(1_000_000, 32, 1184, 2_097_152, 2048)
    assert (c1["db_rows"], c1["db_cols"], c1["instances"], c1["interp"], c1["c"]) == (2048, 720896, 352, 32, 11)
    # buckets < records is rejected (keyword.rs:171-180)
    assert orc.plan_from_shape(1_000_000, 32, 1184, 262_144, 2048) is None
    # entry size not a multiple of 16 bits, zero records
    assert orc.plan_from_shape(100, 3, 0) is None
    assert orc.plan_from_shape(0, 32, 1184) is None


def test_query_size(orc):
    # 2 queries at dim0 = 2048: 286,721 bytes
    assert orc.query_bytes(2048, 2) == 286721
