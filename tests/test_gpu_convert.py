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


@pytest.mark.parametrize("B,t,n", [(9, 3, 10), (16, 4, 8), (7, 4, 6), (64, 8, 9)])
def test_convert_keep_then_scatter_matches_drop_ins(pcg, B, t, n):
    """pcgb_dpf_out_convert_device + pcgb_dpf_out_scatter_g_conv_device (each
    leaf hashed once, its converted word kept) give the drop-ins' sums and g
    bit for bit, and the oracle's."""
    rng = np.random.default_rng(7 * B + n)
    D = 1 << n
    leaves = rng.integers(0, 2**64 - 1, (B * D, 2), dtype=np.uint64, endpoint=True)
    CW = rng.integers(0, P, B, dtype=np.uint64)
    s_max = (B - 1) // t + t - 1
    N = max(t * (D // 2), (s_max + 2) * (D // 2) // 2)
    d = dev(pcg, leaves)
    conv, sums = pcg.DeviceBuffer(8 * B * D), pcg.DeviceBuffer(16 * B)
    pcg.dpf_out_convert_device(d.ptr, B, D, conv.ptr, sums.ptr, sums.ptr + 8 * B)
    pcg.synchronize()
    s = sums.download(np.uint64, 2 * B)
    wc, wt = O.out_sums(leaves, B, D)
    assert (s[:B] == wc).all() and (s[B:] == wt).all()
    words = conv.download(np.uint64, B * D)
    assert ((words >> np.uint64(63)) == (leaves[:, 0] & np.uint64(1))).all()
    d_cw, d_g = pcg.to_device(CW), pcg.DeviceBuffer(8 * N)
    for party in (0, 1):
        pcg.dpf_out_scatter_g_conv_device(conv.ptr, B, D, t, party, d_cw.ptr, d_g.ptr, N)
        pcg.synchronize()
        g = d_g.download(np.uint64, N)
        assert (g == pcg.dpf_out_scatter_g(d.ptr, B, D, t, party, CW, N)).all()
        assert (g == O.out_scatter_g(leaves, B, D, t, party, CW, N)).all()


def test_output_layer_beaver_on_device(pcg):
    """Both parties' opens and closes on the device (the exchange done here
    in-process): the CW shares add to A*B with A = sumT0 - sumT1 and
    B = sumC1 - sumC0 + beta (pcg_ole_impl.h:222-290), for sums and shares
    anywhere in [0, 2^64)."""
    rng = np.random.default_rng(99)
    B = 1000
    u64 = lambda: rng.integers(0, 2**64 - 1, B, dtype=np.uint64, endpoint=True)
    sumC, sumT, beta = [u64(), u64()], [u64(), u64()], [u64(), u64()]
    r, s = u64() % np.uint64(P), u64() % np.uint64(P)
    rs_v = [int(a) * int(b) % P for a, b in zip(r, s)]
    sh = lambda v: (lambda x0: [x0, np.array([(int(a) - int(b)) % P for a, b in zip(v, x0)],
                                              np.uint64)])(u64() % np.uint64(P))
    r_sh, s_sh, rs_sh = sh(r), sh(s), sh(rs_v)
    dv = lambda a: pcg.to_device(np.ascontiguousarray(a, np.uint64))
    keep = []
    de = []
    for p in (0, 1):
        bufs = [dv(x) for x in (sumC[p], sumT[p], beta[p], r_sh[p], s_sh[p], rs_sh[p])]
        d_de = pcg.DeviceBuffer(16 * B)
        pcg.out_beaver_open_device(B, p, *[b.ptr for b in bufs[:5]], d_de.ptr)
        keep.append(bufs)
        de.append(d_de)
    cw = []
    for p in (0, 1):
        bufs, d_cw = keep[p], pcg.DeviceBuffer(8 * B)
        pcg.out_beaver_close_device(B, p, de[p].ptr, de[1 - p].ptr, bufs[3].ptr, bufs[4].ptr,
                                    bufs[5].ptr, d_cw.ptr)
        cw.append(d_cw)
    d_sum = pcg.DeviceBuffer(8 * B)
    pcg.add_mod_p_device(d_sum.ptr, cw[0].ptr, cw[1].ptr, B)
    pcg.synchronize()
    got = d_sum.download(np.uint64, B)
    for k in range(B):
        A = (int(sumT[0][k]) - int(sumT[1][k])) % P
        Bv = (int(sumC[1][k]) - int(sumC[0][k]) + int(beta[0][k]) + int(beta[1][k])) % P
        assert int(got[k]) == A * Bv % P, k


def test_one_hash_output_layer_rejects_bad_arguments(pcg):
    d = pcg.DeviceBuffer(16 * 64)
    s = pcg.DeviceBuffer(64)
    with pytest.raises(pcg.PcgError, match="null pointer"):
        pcg.dpf_out_convert_device(d.ptr, 2, 32, None, s.ptr, s.ptr + 16)
    with pytest.raises(pcg.PcgError, match="power of two"):
        pcg.dpf_out_convert_device(d.ptr, 2, 24, d.ptr, s.ptr, s.ptr + 16)
    with pytest.raises(pcg.PcgError, match="N smaller"):
        pcg.dpf_out_scatter_g_conv_device(d.ptr, 4, 16, 2, 0, s.ptr, d.ptr, 8)
    with pytest.raises(pcg.PcgError, match="party"):
        pcg.out_beaver_open_device(4, 2, s.ptr, s.ptr, s.ptr, s.ptr, s.ptr, d.ptr)
    with pytest.raises(pcg.PcgError, match="null pointer"):
        pcg.out_beaver_close_device(4, 0, s.ptr, None, s.ptr, s.ptr, s.ptr, d.ptr)
