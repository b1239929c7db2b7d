"""Fused expansion (keyed DPF -> convert -> gather -> NTT products) against
the oracle's restatement of gen_and_expand's algebra, plus the OLE relation
at the full N=2^20, c=4, t=16 shape."""
import numpy as np
import pytest

import oracle_lib as O
from gpu_helpers import dev

pytestmark = pytest.mark.gpu
P = O.P
MASTER = np.array([0x2B, 0x7E, 0x15, 0x16, 0x28, 0xAE, 0xD2, 0xA6, 0xAB, 0xF7, 0x15, 0x88, 0x09,
                   0xCF, 0x4F, 0x3C], np.uint8)  # pcg_ole_impl.h:89-90


def material(s, seed, a_seed, prg):
    rks = O.aes_tree_round_keys(MASTER, s.nk) if prg == O.PRG_AES else None
    r0, r1, cws, cwo = O.deal_keys(s, seed, rks)
    a = O.public_a(s, a_seed)
    n0 = O.noise(s, seed, 0)
    n1 = O.noise(s, seed, 1)
    return rks, (r0, r1), cws, cwo, a, (n0, n1)


SHAPES = [(4096, 2, 4, 1, O.PRG_CHACHA8),   # the CPU-runnable configuration
          (1024, 3, 8, 1, O.PRG_CHACHA8),
          (2048, 4, 8, 1, O.PRG_AES),
          (4096, 2, 8, 2, O.PRG_CHACHA8),  # n = 10, w = 2
          (8192, 1, 64, 1, O.PRG_CHACHA8),
          (16384, 2, 32, 2, O.PRG_AES)]


@pytest.mark.parametrize("N,c,t,w,prg", SHAPES)
def test_expand_matches_oracle(pcg, N, c, t, w, prg):
    s = O.shape(N, c, t, w, prg)
    rks, roots, cws, cwo, a, noise = material(s, 1000 + N + c, 7, prg)
    e = pcg.Expander(N, c, t, w, prg, public_a=a if c > 1 else None,
                     master_key=MASTER if prg == O.PRG_AES else None)
    xs, zs = [], []
    for party in (0, 1):
        x, z = e.expand_host(party, roots[party], cws, cwo, *noise[party])
        wx, wz = O.expand(s, party, roots[party], cws, cwo, *noise[party], a, rks)
        assert (x == wx).all(), ("x", party)
        assert (z == wz).all(), ("z", party)
        xs.append(x), zs.append(z)
    prod = O.poly_mul(xs[0], xs[1], N)
    zz = (zs[0].astype(object) + zs[1].astype(object)) % P
    assert all(int(p) == int(q) for p, q in zip(prod, zz))
    e.close()


@pytest.mark.parametrize("N,c,t,w,prg", SHAPES[:3])
def test_g_prime_matches_oracle(pcg, N, c, t, w, prg):
    s = O.shape(N, c, t, w, prg)
    rks, roots, cws, cwo, a, noise = material(s, 77, 7, prg)
    e = pcg.Expander(N, c, t, w, prg, public_a=a if c > 1 else None,
                     master_key=MASTER if prg == O.PRG_AES else None)
    d_cws, d_cwo = dev(pcg, cws), dev(pcg, cwo)
    for party in (0, 1):
        _, _, g = O.expand(s, party, roots[party], cws, cwo, *noise[party], a, rks, want_g=True)
        g = g.reshape(c, c, N)
        d_r = dev(pcg, roots[party])
        d_g = pcg.DeviceBuffer(8 * N * e.Q)
        e.expand_g_device(party, d_r.ptr, d_cws.ptr, d_cwo.ptr, d_g.ptr)
        got = d_g.download(np.uint64, N * e.Q).reshape(e.Q, N)
        q = 0
        for i in range(c):
            for j in range(i, c):
                want = g[i, j] if i == j else (g[i, j].astype(object) + g[j, i]) % P
                assert (got[q] == np.asarray(want, dtype=np.uint64)).all(), (party, i, j)
                q += 1
    e.close()


@pytest.mark.parametrize("N,c,t,w,prg", [(4096, 2, 4, 1, O.PRG_CHACHA8), (1 << 14, 4, 16, 1, O.PRG_AES),
                                         (1 << 15, 4, 16, 2, O.PRG_CHACHA8)])
def test_gpu_dealer_matches_oracle(pcg, N, c, t, w, prg):
    s = O.shape(N, c, t, w, prg)
    rks = O.aes_tree_round_keys(MASTER, s.nk) if prg == O.PRG_AES else None
    r0, r1, cws, cwo = O.deal_keys(s, 4242, rks)
    a = O.public_a(s, 1)
    e = pcg.Expander(N, c, t, w, prg, public_a=a, master_key=MASTER if prg == O.PRG_AES else None)
    bufs = [pcg.DeviceBuffer(x.nbytes) for x in (r0, r1, cws, cwo)]
    e.deal_keys_device(4242, *[b.ptr for b in bufs])
    for b, want in zip(bufs, (r0, r1, cws, cwo)):
        assert (b.download(np.uint64, want.size).reshape(want.shape) == want).all()
    e.close()


def test_ole_relation_full_shape(pcg):
    """N = 2^20, c = 4, t = 16 (256 keys of domain 2^17 per block, 4096 keys):
    z0 + z1 == x0 * x1, with the product on the (oracle-checked) GPU NTT."""
    N, c, t = 1 << 20, 4, 16
    a = pcg.public_a(N, c, 12)
    e = pcg.Expander(N, c, t, 1, pcg.PRG_CHACHA8, public_a=a)
    K, L = e.K, e.levels
    d_r0, d_r1 = pcg.DeviceBuffer(16 * K), pcg.DeviceBuffer(16 * K)
    d_cws, d_cwo = pcg.DeviceBuffer(16 * K * L * e.nk), pcg.DeviceBuffer(8 * K)
    e.deal_keys_device(31337, d_r0.ptr, d_r1.ptr, d_cws.ptr, d_cwo.ptr)
    xs, zs = [], []
    for party, d_r in ((0, d_r0), (1, d_r1)):
        pos, val = pcg.noise(N, c, t, 31337, party)
        d_pos, d_val = dev(pcg, pos), dev(pcg, val)
        d_x, d_z = pcg.DeviceBuffer(8 * N), pcg.DeviceBuffer(8 * N)
        e.expand_device(party, d_r.ptr, d_cws.ptr, d_cwo.ptr, d_pos.ptr, d_val.ptr, d_x.ptr,
                        d_z.ptr)
        xs.append(d_x.download(np.uint64, N))
        zs.append(d_z.download(np.uint64, N))
    prod, _ = pcg.poly_mul_u64_gpuntt(xs[0], xs[1], 1, N)
    zsum = zs[0] + zs[1]
    zsum = np.where(zsum >= np.uint64(P), zsum - np.uint64(P), zsum)
    assert (prod == zsum).all()
    # x = sum a_i e_i has exactly the dealt noise in a_0's slot.
    assert np.count_nonzero(xs[0]) > N // 2
    e.close()


def test_full_shape_against_independent_paths(pcg):
    """N = 2^20, c = 4, t = 16: x against the oracle's products of the same
    public a and noise; z against sum_q (a_i a_j) * g'_q computed with the
    poly-mul drop-in on the fused kernel's g' (an independent NTT path); and
    two separately built expanders agree (resident plans are deterministic)."""
    N, c, t, seed = 1 << 20, 4, 16, 4242
    a = pcg.public_a(N, c, 21)
    e1 = pcg.Expander(N, c, t, 1, pcg.PRG_CHACHA8, public_a=a)
    K, L = e1.K, e1.levels
    d_r0, d_r1 = pcg.DeviceBuffer(16 * K), pcg.DeviceBuffer(16 * K)
    d_cws, d_cwo = pcg.DeviceBuffer(16 * K * L * e1.nk), pcg.DeviceBuffer(8 * K)
    e1.deal_keys_device(seed, d_r0.ptr, d_r1.ptr, d_cws.ptr, d_cwo.ptr)
    pos, val = pcg.noise(N, c, t, seed, 0)
    d_pos, d_val = dev(pcg, pos), dev(pcg, val)
    outs = []
    for e in (e1, pcg.Expander(N, c, t, 1, pcg.PRG_CHACHA8, public_a=a)):
        d_x, d_z = pcg.DeviceBuffer(8 * N), pcg.DeviceBuffer(8 * N)
        e.expand_device(0, d_r0.ptr, d_cws.ptr, d_cwo.ptr, d_pos.ptr, d_val.ptr, d_x.ptr, d_z.ptr)
        outs.append((d_x.download(np.uint64, N), d_z.download(np.uint64, N)))
    x, z = outs[0]
    assert (outs[1][0] == x).all() and (outs[1][1] == z).all()
    # x = e_0 + sum_{i>=1} a_i * e_i, on the CPU.
    want = np.zeros(N, dtype=object)
    for i in range(c):
        ei = np.zeros(N, np.uint64)
        ei[pos[i * t:(i + 1) * t].astype(np.int64)] = val[i * t:(i + 1) * t]
        if i == 0:
            prod = ei
        else:
            prod = O.poly_mul(a[(i - 1) * N:i * N], ei, N)
        want = (want + prod.astype(object)) % P
    assert (x == np.asarray(want, dtype=np.uint64)).all()
    # z through g' and the drop-in products.
    d_g = pcg.DeviceBuffer(8 * N * e1.Q)
    e1.expand_g_device(0, d_r0.ptr, d_cws.ptr, d_cwo.ptr, d_g.ptr)
    g = d_g.download(np.uint64, N * e1.Q).reshape(e1.Q, N)
    av = [np.eye(1, N, 0, dtype=np.uint64)[0]] + [a[(i - 1) * N:i * N] for i in range(1, c)]
    zz = np.zeros(N, dtype=object)
    q = 0
    for i in range(c):
        for j in range(i, c):
            aa, _ = pcg.poly_mul_u64_gpuntt(av[i], av[j], 1, N)
            p, _ = pcg.poly_mul_u64_gpuntt(aa, g[q], 1, N)
            zz = (zz + p.astype(object)) % P
            q += 1
    assert (z == np.asarray(zz, dtype=np.uint64)).all()


@pytest.mark.parametrize("N,c,t", [(1 << 12, 2, 4), (1 << 12, 3, 4), (1 << 11, 1, 2)])
def test_public_a0_expander_matches_oracle(pcg, N, c, t):
    """pcgb_expander_create_public_a0: all c public polynomials given (a_0
    too).  x and z equal the oracle's step 4 on the oracle's own block
    outputs, for both parties, and satisfy the OLE relation."""
    s = O.shape(N, c, t)
    rng = np.random.default_rng(N + c)
    a_all = rng.integers(0, P, c * N, dtype=np.uint64)
    r0, r1, cws, cwo = O.deal_keys(s, 404)
    e = pcg.Expander(N, c, t, 1, pcg.PRG_CHACHA8, public_a=a_all, a0_public=True)
    xs, zs = [], []
    for p in (0, 1):
        pos, val = O.noise(s, 404, p)
        _, _, g = O.expand(s, p, (r0, r1)[p], cws, cwo, pos, val,
                           O.public_a(s, 1) if c > 1 else np.zeros(0, np.uint64), want_g=True)
        wx, wz = O.step4(N, c, t, pos, val, a_all, g)
        x, z = e.expand_host(p, (r0, r1)[p], cws, cwo, pos, val)
        assert (x == wx).all() and (z == wz).all(), p
        xs.append(x)
        zs.append(z)
    prod = O.poly_mul(xs[0], xs[1], N)
    zz = (zs[0].astype(object) + zs[1].astype(object)) % P
    assert all(int(u) == int(v) for u, v in zip(prod, zz))
    e.close()


def test_public_a0_expander_ole_relation_full_shape(pcg):
    """The same mode at N = 2^20, c = 4, t = 16, checked on the device."""
    N, c, t = 1 << 20, 4, 16
    a_all = np.random.default_rng(9).integers(0, P, c * N, dtype=np.uint64)
    e = pcg.Expander(N, c, t, 1, pcg.PRG_CHACHA8, public_a=a_all, a0_public=True)
    K, L = e.K, e.levels
    d_r0, d_r1 = pcg.DeviceBuffer(16 * K), pcg.DeviceBuffer(16 * K)
    d_cws, d_cwo = pcg.DeviceBuffer(16 * K * L * e.nk), pcg.DeviceBuffer(8 * K)
    e.deal_keys_device(777, d_r0.ptr, d_r1.ptr, d_cws.ptr, d_cwo.ptr)
    outs = []
    for party, d_r in ((0, d_r0), (1, d_r1)):
        pos, val = pcg.noise(N, c, t, 777, party)
        d_pos, d_val = dev(pcg, pos), dev(pcg, val)
        d_x, d_z = pcg.DeviceBuffer(8 * N), pcg.DeviceBuffer(8 * N)
        e.expand_device(party, d_r.ptr, d_cws.ptr, d_cwo.ptr, d_pos.ptr, d_val.ptr, d_x.ptr,
                        d_z.ptr)
        outs += [d_x, d_z]
    bad = pcg.DeviceBuffer(8)
    pcg.verify_ole_device(N, *[b.ptr for b in outs], bad.ptr)
    pcg.synchronize()
    assert int(bad.download(np.uint64, 1)[0]) == 0
    e.close()
