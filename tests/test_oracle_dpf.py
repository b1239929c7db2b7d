"""Oracle self-consistency: keyed dealer == interactive two-party protocol,
point-function property, output-layer correctness, OLE relation (no GPU)."""
import numpy as np
import pytest

import oracle_lib as O

P = O.P


@pytest.mark.parametrize("prg", [O.PRG_CHACHA8, O.PRG_AES])
@pytest.mark.parametrize("n,w", [(6, 1), (8, 2), (9, 3), (8, 4)])
def test_keyed_equals_interactive(prg, n, w):
    rng = np.random.default_rng(100 * n + w + prg)
    B, nk, L = 5, (1 << w) - 1, n // w
    rks = O.aes_tree_round_keys(np.arange(16, dtype=np.uint8), nk) if prg == O.PRG_AES else None
    roots0 = rng.integers(0, 2**63, (B, 2), dtype=np.uint64)
    deltas = rng.integers(0, 2**63, (B, 2), dtype=np.uint64)
    deltas[:, 0] |= np.uint64(1)
    roots1 = roots0 ^ deltas
    alphas = rng.integers(0, 1 << n, B)
    betas = rng.integers(1, P, B, dtype=np.uint64)
    dlt0 = rng.integers(0, 2**63, (B * L * nk, 2), dtype=np.uint64)
    dlt1 = np.zeros_like(dlt0)
    cws = np.zeros_like(dlt0)
    for b in range(B):
        s = slice(b * L * nk, (b + 1) * L * nk)
        c, _, d1 = O.dpf_deal(n, w, roots0[b], deltas[b], int(alphas[b]), int(betas[b]), prg, rks,
                              np.ascontiguousarray(dlt0[s]))
        cws[s], dlt1[s] = c, d1
    l0, l1, rec = O.dpf_full_eval_2p(B, n, w, roots0, roots1, dlt0, dlt1, prg, rks)
    assert (rec == cws).all()
    assert (O.dpf_keyed_full_eval(B, n, w, roots0, cws, prg, rks) == l0).all()
    assert (O.dpf_keyed_full_eval(B, n, w, roots1, cws, prg, rks) == l1).all()
    D = 1 << n
    x = (l0 ^ l1).reshape(B, D, 2)
    for b in range(B):
        assert list(np.nonzero(x[b].any(axis=1))[0]) == [alphas[b]]
        assert (x[b, alphas[b]] == deltas[b]).all()


def test_output_layer_sums_to_beta():
    rng = np.random.default_rng(5)
    n, D = 7, 128
    for trial in range(8):
        r0 = rng.integers(0, 2**63, 2, dtype=np.uint64)
        dl = rng.integers(0, 2**63, 2, dtype=np.uint64)
        dl[0] |= np.uint64(1)
        alpha, beta = int(rng.integers(0, D)), int(rng.integers(1, P))
        cws, cwo, _ = O.dpf_deal(n, 1, r0, dl, alpha, beta)
        l0 = O.dpf_keyed_full_eval(1, n, 1, r0.reshape(1, 2), cws)
        l1 = O.dpf_keyed_full_eval(1, n, 1, (r0 ^ dl).reshape(1, 2), cws)
        cw = np.array([cwo], np.uint64)
        g0 = O.out_scatter_g(l0, 1, D, 1, 0, cw, D // 2)
        g1 = O.out_scatter_g(l1, 1, D, 1, 1, cw, D // 2)
        s = [(int(a) + int(b)) % P for a, b in zip(g0, g1)]
        exp = [0] * (D // 2)
        exp[alpha % (D // 2)] = beta if alpha < D // 2 else (P - beta) % P
        assert s == exp


def test_dpf_eval_matches_full_eval():
    rng = np.random.default_rng(9)
    n, w = 8, 2
    r0 = rng.integers(0, 2**63, 2, dtype=np.uint64)
    dl = rng.integers(0, 2**63, 2, dtype=np.uint64)
    dl[0] |= np.uint64(1)
    cws, _, _ = O.dpf_deal(n, w, r0, dl, 77, 5)
    leaves = O.dpf_keyed_full_eval(1, n, w, r0.reshape(1, 2), cws)
    for j in [0, 1, 77, 200, 255]:
        e = O.lib().orc_dpf_eval(O.Blk(int(r0[0]), int(r0[1])), cws, n, w, None, O.PRG_CHACHA8, j)
        assert (e.lo, e.hi) == (int(leaves[j, 0]), int(leaves[j, 1]))


@pytest.mark.parametrize("N,c,t", [(4096, 2, 4), (1024, 3, 8), (512, 1, 4)])
def test_ole_relation(N, c, t):
    """z0 + z1 = x0 * x1 in Z_p[X]/(X^N+1) (CPU_baseline/test/pcg_ole_2pc.cpp:199-214)."""
    s = O.shape(N, c, t)
    r0, r1, cws, cwo = O.deal_keys(s, 2024 + N)
    a = O.public_a(s, 99)
    p0, v0 = O.noise(s, 2024 + N, 0)
    p1, v1 = O.noise(s, 2024 + N, 1)
    x0, z0 = O.expand(s, 0, r0, cws, cwo, p0, v0, a)
    x1, z1 = O.expand(s, 1, r1, cws, cwo, p1, v1, a)
    prod = O.poly_mul(x0, x1, N)
    zz = (z0.astype(object) + z1.astype(object)) % P
    assert all(int(p) == int(q) for p, q in zip(prod, zz))


def test_step4_with_a_public_a0_keeps_the_ole_relation():
    """orc_step4 with a_0 = 1 is orc_expand's own step 4; with a_0 drawn
    uniformly as well, the two parties' outputs still satisfy
    z0 + z1 = x0 * x1 (x_p = sum a_i e_i^p, so the relation holds for any a)."""
    N, c, t = 1 << 10, 2, 4
    s = O.shape(N, c, t)
    a = O.public_a(s, 7)
    r0, r1, cws, cwo = O.deal_keys(s, 55)
    noise = [O.noise(s, 55, p) for p in (0, 1)]
    outs = [O.expand(s, p, (r0, r1)[p], cws, cwo, *noise[p], a, want_g=True) for p in (0, 1)]
    one = np.zeros(N, np.uint64)
    one[0] = 1
    for p in (0, 1):
        x, z = O.step4(N, c, t, *noise[p], np.concatenate([one, a]), outs[p][2])
        assert (x == outs[p][0]).all() and (z == outs[p][1]).all()
    a0 = np.random.default_rng(3).integers(0, O.P, N, dtype=np.uint64)
    (x0, z0), (x1, z1) = [O.step4(N, c, t, *noise[p], np.concatenate([a0, a]), outs[p][2])
                          for p in (0, 1)]
    prod = O.poly_mul(x0, x1, N)
    zz = (z0.astype(object) + z1.astype(object)) % O.P
    assert all(int(u) == int(v) for u, v in zip(prod, zz))
