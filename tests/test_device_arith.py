"""Exactness of the integer arithmetic the first-dimension GEMM relies on, restated in Python
over the full input ranges the kernels accept (CPU only):

* the parse's CRT composition (`crt2m`, csrc/ipr_device.cuh) of a query value's two residues
  into X < q0 q1 < 2^56 with X = residue_l mod q_l, for residues that need not be reduced;
* the epilogue's recombination of the 7 x 2 byte-plane sums into W0 + 2^32 W1 and its
  single Montgomery reduction per limb (`mod96m`), at the largest sums 32,768 DB rows give.

The GPU parity tests compare the kernels' bytes with the oracle; these pin the bounds the
kernels' comments state, including the extremes no seeded case reaches."""
import random

Q0, Q1 = 268369921, 249561089
M32 = (1 << 32) - 1


def _neg_inv32(q):
    x = q
    for _ in range(5):
        x = (x * (2 - q * x)) & M32
    return (-x) & M32


QNEG = {Q0: _neg_inv32(Q0), Q1: _neg_inv32(Q1)}
R1 = {q: (1 << 32) % q for q in (Q0, Q1)}
R2 = {q: R1[q] * R1[q] % q for q in (Q0, Q1)}
R3 = {q: R2[q] * R1[q] % q for q in (Q0, Q1)}
Q0INV = pow(Q0, -1, Q1)
Q0INV_R = (Q0INV << 32) % Q1


def _redc(x, q):
    assert 0 <= x < 1 << 64
    m = ((x & M32) * QNEG[q]) & M32
    s = x + m * q
    assert s < 1 << 64, "the Montgomery sum must not wrap"
    return s >> 32


def _umin(a, b):  # min of two u32 values, as the kernels' min(t, t - k q)
    return min(a & M32, b & M32)


def _crt2m(x, y):
    xm = x - Q1 if x >= Q1 else x
    d = y - xm if y >= xm else y + Q1 - xm
    kr = _redc(d * Q0INV_R, Q1)
    k = _umin(kr, kr - Q1)
    return x + Q0 * k


def _mod96m(w0, w1, q):
    t = w1 + (w0 >> 32)
    x = (w0 & M32) * R1[q] + (t & M32) * R2[q] + (t >> 32) * R3[q]
    assert x < 1 << 64
    r = _redc(x, q)
    assert r < 4 * q
    r1 = _umin(r, r - 2 * q)
    return _umin(r1, r1 - q)


def test_crt_composition_of_unreduced_residues():
    rng = random.Random(5)
    edges = [0, 1, Q1 - 1, Q1, Q0 - 1, Q0, (1 << 28) - 1]
    cases = [(a, b) for a in edges for b in edges]
    cases += [(rng.randrange(1 << 28), rng.randrange(1 << 28)) for _ in range(20000)]
    for lo, hi in cases:
        x = _crt2m(lo, hi)
        assert x < 1 << 56
        assert x % Q0 == lo % Q0 and x % Q1 == hi % Q1


def test_byte_plane_recombination_at_the_row_limit():
    rng = random.Random(6)
    p_max = 255 * 255 * 32768  # a byte-pair sum over 32,768 DB rows
    s_max = p_max + 256 * p_max  # S_b = P_0b + 256 P_1b
    trials = [[s_max] * 7, [0] * 7, [s_max if b < 4 else 0 for b in range(7)],
              [0 if b < 4 else s_max for b in range(7)]]
    trials += [[rng.randrange(s_max + 1) for _ in range(7)] for _ in range(20000)]
    for s in trials:
        w0 = sum(s[b] << (8 * b) for b in range(4))
        w1 = sum(s[b] << (8 * (b - 4)) for b in range(4, 7))
        assert w0 < 1 << 64 and w1 < 1 << 56
        v = w0 + (w1 << 32)
        assert v == sum(s[b] << (8 * b) for b in range(7))
        for q in (Q0, Q1):
            assert _mod96m(w0, w1, q) == v % q


def test_gemm_sum_of_crt_values_gives_both_limbs():
    """sum_k D[k] X[k] mod q_l equals sum_k D[k] a_l[k] mod q_l: the one 7-byte product sum
    serves both limbs"""
    rng = random.Random(7)
    rows = 64
    d = [rng.randrange(1 << 16) for _ in range(rows)]
    a0 = [rng.randrange(1 << 28) for _ in range(rows)]
    a1 = [rng.randrange(1 << 28) for _ in range(rows)]
    x = [_crt2m(u, v) for u, v in zip(a0, a1)]
    # the byte-plane form the GEMM computes
    planes = [[v & 0xFF for v in d], [v >> 8 for v in d]]
    xb = [[(v >> (8 * b)) & 0xFF for v in x] for b in range(7)]
    total = 0
    for p in range(2):
        for b in range(7):
            total += sum(planes[p][k] * xb[b][k] for k in range(rows)) << (8 * (p + b))
    assert total == sum(dk * xk for dk, xk in zip(d, x))
    assert total % Q0 == sum(dk * ak for dk, ak in zip(d, a0)) % Q0
    assert total % Q1 == sum(dk * ak for dk, ak in zip(d, a1)) % Q1
