"""Kernel-level building blocks (ipr_ntt_batch, ipr_automorph_batch) against the oracle.

The batched limb NTT must equal the oracle's ntt_forward / ntt_inverse
(src/core/ntt.rs:111-160, 731-780) for every polynomial, including a batch
size that leaves a partial tile; the automorphism gather must map NTT(a) to
NTT(a(x^t)) for the oracle's coefficient-domain automorphism (the reference's
packing.rs:3943-3985 equivalence), for t at the edges of the odd range.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 2048
Q = (268369921, 249561089)


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("count", [1, 37, 512])
def test_ntt_batch_matches_oracle(pkg, orc, count):
    rng = np.random.default_rng(count)
    for limb in (0, 1):
        polys = rng.integers(0, Q[limb], (count, N), dtype=np.uint64)
        d = _dev(polys.view(np.int64))
        pkg.ntt_batch(d.data_ptr(), count, limb)
        got = d.cpu().numpy().view(np.uint64)
        for p in sorted({0, count // 2, count - 1}):
            both = np.zeros((2, N), dtype=np.uint64)
            both[limb] = polys[p]
            assert np.array_equal(got[p], orc.ntt_forward(both)[limb])
        pkg.ntt_batch(d.data_ptr(), count, limb, inverse=True)
        assert np.array_equal(d.cpu().numpy().view(np.uint64), polys)  # round trip, every polynomial


def test_intt_batch_matches_oracle(pkg, orc):
    rng = np.random.default_rng(5)
    polys = rng.integers(0, Q[1], (9, N), dtype=np.uint64)
    d = _dev(polys.view(np.int64))
    pkg.ntt_batch(d.data_ptr(), 9, 1, inverse=True)
    got = d.cpu().numpy().view(np.uint64)
    for p in (0, 4, 8):
        both = np.zeros((2, N), dtype=np.uint64)
        both[1] = polys[p]
        assert np.array_equal(got[p], orc.ntt_inverse(both)[1])


def test_automorph_batch_matches_oracle(pkg, orc):
    import torch
    rng = np.random.default_rng(11)
    count = 6
    raw = rng.integers(0, Q[0] * Q[1], (count, N), dtype=np.uint64)
    ntt = np.stack([orc.to_ntt(r) for r in raw])  # [count][2N], limb-major
    ks = np.array([1, 3, 5, 4095, 2049, 25, 4093], dtype=np.uint32)
    d_ks = _dev(ks.view(np.int32))
    for limb in (0, 1):
        d_in = _dev(np.ascontiguousarray(ntt[:, limb * N:(limb + 1) * N]).view(np.int64))
        d_out = torch.zeros((len(ks), count, N), dtype=torch.int64, device="cuda")
        pkg.automorph_batch(d_in.data_ptr(), count, d_ks.data_ptr(), len(ks), d_out.data_ptr())
        got = d_out.cpu().numpy().view(np.uint64)
        for j, t in enumerate(ks):
            for p in (0, count - 1):
                want = orc.to_ntt(orc.automorph_poly(raw[p], int(t)))[limb * N:(limb + 1) * N]
                assert np.array_equal(got[j, p], want), (limb, t, p)


def test_micro_argument_errors(pkg):
    import torch
    with pytest.raises(pkg.IprError):
        pkg.ntt_batch(0, 4, 0)  # null buffer
    d = torch.zeros(N, dtype=torch.int64, device="cuda")
    with pytest.raises(pkg.IprError):
        pkg.ntt_batch(d.data_ptr(), 1, 2)  # no limb 2
