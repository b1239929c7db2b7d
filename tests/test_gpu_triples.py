"""Beaver-triple extraction and the on-device OLE / triple relation checks
(CPU_baseline/pcg_ole_2pc/triple.h:45-110, test/pcg_ole_2pc.cpp:199-214)."""
import numpy as np
import pytest

import oracle_lib as O
from gpu_helpers import dev

pytestmark = pytest.mark.gpu
P = O.P


@pytest.mark.parametrize("N", [2, 16, 1 << 10, 1 << 12])
@pytest.mark.parametrize("party", [0, 1])
def test_triples_match_oracle(pcg, N, party):
    """Arbitrary 64-bit inputs: the slot shares equal the oracle's triple.h
    restatement (whose NTT is pinned to the reference's ntt.h)."""
    rng = np.random.default_rng(N + party)
    x1, z1, x2, z2 = (rng.integers(0, 2**64 - 1, N, dtype=np.uint64) for _ in range(4))
    d = [dev(pcg, v) for v in (x1, z1, x2, z2)]
    out = [pcg.DeviceBuffer(8 * N) for _ in range(3)]
    pcg.triples_device(N, party, *[b.ptr for b in d], *[b.ptr for b in out])
    got = [b.download(np.uint64, N) for b in out]
    want = O.triples(N, party, x1, z1, x2, z2)
    for g, w in zip(got, want):
        assert (g == w).all()


def _expand_both(pcg, N, c, t, seed, w=1):
    s = O.shape(N, c, t)
    e = pcg.Expander(N, c, t, w, pcg.PRG_CHACHA8, public_a=O.public_a(s, 7))
    K, L = e.K, e.levels
    r0, r1 = pcg.DeviceBuffer(16 * K), pcg.DeviceBuffer(16 * K)
    cws, cwo = pcg.DeviceBuffer(16 * K * L * e.nk), pcg.DeviceBuffer(8 * K)
    e.deal_keys_device(seed, r0.ptr, r1.ptr, cws.ptr, cwo.ptr)
    outs = []
    for party, roots in ((0, r0), (1, r1)):
        pos, val = pcg.noise(N, c, t, seed, party)
        dp, dv = pcg.to_device(pos), pcg.to_device(val)
        x, z = pcg.DeviceBuffer(8 * N), pcg.DeviceBuffer(8 * N)
        e.expand_device(party, roots.ptr, cws.ptr, cwo.ptr, dp.ptr, dv.ptr, x.ptr, z.ptr)
        outs.append((x, z))
    pcg.synchronize()
    e.close()
    return outs


def test_relations_on_real_expansions(pcg):
    """Two OLEs from the fused expansion: the OLE relation holds on the
    device (0 bad slots), the extracted triples hold for every slot, and a
    planted error (on the host copy) is counted exactly."""
    N = 1 << 14
    ole1 = _expand_both(pcg, N, 2, 8, 101)
    ole2 = _expand_both(pcg, N, 2, 8, 202)
    bad = pcg.DeviceBuffer(8)
    for (x0, z0), (x1, z1) in (ole1, ole2):
        pcg.verify_ole_device(N, x0.ptr, z0.ptr, x1.ptr, z1.ptr, bad.ptr)
        assert int(bad.download(np.uint64, 1)[0]) == 0
    shares = []
    for party in (0, 1):
        (x1, z1), (x2, z2) = ole1[party], ole2[party]
        out = [pcg.DeviceBuffer(8 * N) for _ in range(3)]
        pcg.triples_device(N, party, x1.ptr, z1.ptr, x2.ptr, z2.ptr, *[b.ptr for b in out])
        shares.append(out)
    flat = [b.ptr for b in shares[0]] + [b.ptr for b in shares[1]]
    pcg.verify_triples_device(N, *flat, bad.ptr)
    assert int(bad.download(np.uint64, 1)[0]) == 0
    # Host cross-check of a few slots, then a planted error in one share.
    a0, b0, c0 = (b.download(np.uint64, N) for b in shares[0])
    a1, b1, c1 = (b.download(np.uint64, N) for b in shares[1])
    for k in (0, 1, N // 2, N - 1):
        lhs = (int(a0[k]) + int(a1[k])) % P * ((int(b0[k]) + int(b1[k])) % P) % P
        assert lhs == (int(c0[k]) + int(c1[k])) % P
    c0[[3, 77]] = (c0[[3, 77]] + np.uint64(1)) % np.uint64(P)
    d_c0 = dev(pcg, c0)
    pcg.verify_triples_device(N, shares[0][0].ptr, shares[0][1].ptr, d_c0.ptr,
                              *[b.ptr for b in shares[1]], bad.ptr)
    assert int(bad.download(np.uint64, 1)[0]) == 2
    (x0, z0), (x1, z1) = ole1
    z_bad = z0.download(np.uint64, N)
    z_bad[5] = (z_bad[5] + np.uint64(1)) % np.uint64(P)
    d_z = dev(pcg, z_bad)
    pcg.verify_ole_device(N, x0.ptr, d_z.ptr, x1.ptr, z1.ptr, bad.ptr)
    assert int(bad.download(np.uint64, 1)[0]) > 0


def test_triples_rejects_bad_args(pcg):
    b = pcg.DeviceBuffer(64)
    with pytest.raises(pcg.PcgError):
        pcg.triples_device(6, 0, *([b.ptr] * 7))
    with pytest.raises(pcg.PcgError):
        pcg.triples_device(8, 2, *([b.ptr] * 7))


@pytest.mark.parametrize("w", [1, 2, 3])
def test_triples_at_the_reference_test_shape(pcg, w):
    """The reference's triple test shape (CPU_baseline/test/triple.cpp:
    N = 128, t = 4, w in {1, 2, 3}): two OLEs from the fused expansion, their
    triples, and c0 + c1 = (a0 + a1)(b0 + b1) in every slot, checked on the
    device and on the host."""
    N = 128
    oles = [_expand_both(pcg, N, 2, 4, seed, w) for seed in (11, 22)]
    bad = pcg.DeviceBuffer(8)
    for (x0, z0), (x1, z1) in oles:
        pcg.verify_ole_device(N, x0.ptr, z0.ptr, x1.ptr, z1.ptr, bad.ptr)
        assert int(bad.download(np.uint64, 1)[0]) == 0
    shares = []
    for party in (0, 1):
        (x1, z1), (x2, z2) = oles[0][party], oles[1][party]
        out = [pcg.DeviceBuffer(8 * N) for _ in range(3)]
        pcg.triples_device(N, party, x1.ptr, z1.ptr, x2.ptr, z2.ptr, *[b.ptr for b in out])
        shares.append([b.download(np.uint64, N) for b in out])
        want = O.triples(N, party, x1.download(np.uint64, N), z1.download(np.uint64, N),
                         x2.download(np.uint64, N), z2.download(np.uint64, N))
        for g, ww in zip(shares[-1], want):
            assert (g == ww).all()
    (a0, b0, c0), (a1, b1, c1) = shares
    for k in range(N):
        lhs = (int(a0[k]) + int(a1[k])) % P * ((int(b0[k]) + int(b1[k])) % P) % P
        assert lhs == (int(c0[k]) + int(c1[k])) % P, k
