"""Output-layer drop-ins (dpf_out_sums / dpf_out_scatter_g) against the
oracle on the out_hash_cuda_bitexact fixture and on ragged shapes."""
import numpy as np
import pytest

import oracle_lib as O
from gpu_helpers import dev

pytestmark = pytest.mark.gpu
P = O.P


def fixture_bitexact():
    """GPU_baseline/test/out_hash_cuda_bitexact.cu:50-59: t=3, B=9, D=1024,
    mt19937_64(12345) leaves (lo then hi) followed by CW[b] = rng() % P."""
    t, B, D = 3, 9, 1024
    r = O.mt64(12345, 2 * B * D + B)
    leaves = np.ascontiguousarray(r[: 2 * B * D].reshape(B * D, 2))
    CW = r[2 * B * D:] % np.uint64(P)
    return t, B, D, leaves, CW


@pytest.mark.parametrize("party", [0, 1])
def test_out_hash_bitexact_fixture(pcg, party):
    t, B, D, leaves, CW = fixture_bitexact()
    N = t * (D // 2)
    d = dev(pcg, leaves)
    sc, st = pcg.dpf_out_sums(d.ptr, B, D)
    g = pcg.dpf_out_scatter_g(d.ptr, B, D, t, party, CW, N)
    wc, wt = O.out_sums(leaves, B, D)
    assert (sc == wc).all() and (st == wt).all()
    assert (g == O.out_scatter_g(leaves, B, D, t, party, CW, N)).all()


@pytest.mark.parametrize("B,t,n,extra", [(16, 4, 8, 0), (7, 4, 6, 0), (9, 3, 10, 64), (1, 1, 12, 0),
                                         (64, 8, 9, 1 << 9)])
def test_convert_ragged_shapes(pcg, B, t, n, extra):
    rng = np.random.default_rng(B * 1000 + n)
    D = 1 << n
    leaves = rng.integers(0, 2**64 - 1, (B * D, 2), dtype=np.uint64)
    CW = rng.integers(0, 2**64 - 1, B, dtype=np.uint64)  # reduced mod p by both sides
    s_max = (B - 1) // t + t - 1
    N = max(t * (D // 2), (s_max + 2) * (D // 2) // 2) + extra
    d = dev(pcg, leaves)
    for party in (0, 1):
        g = pcg.dpf_out_scatter_g(d.ptr, B, D, t, party, CW, N)
        assert (g == O.out_scatter_g(leaves, B, D, t, party, CW, N)).all()
    sc, st = pcg.dpf_out_sums(d.ptr, B, D)
    wc, wt = O.out_sums(leaves, B, D)
    assert (sc == wc).all() and (st == wt).all()


def test_convert_rejects_bad_arguments(pcg):
    d = pcg.DeviceBuffer(16 * 64)
    with pytest.raises(pcg.PcgError, match="project prime"):
        pcg.dpf_out_sums(d.ptr, 2, 32, prime=97)
    with pytest.raises(pcg.PcgError, match="N smaller"):
        pcg.dpf_out_scatter_g(d.ptr, 4, 16, 2, 0, np.zeros(4, np.uint64), 8)
