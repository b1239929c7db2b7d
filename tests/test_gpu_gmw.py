"""Boolean preprocessing by two-party GMW on the GPU (pcgb_gmw_*): two
processes, one per party, exchanging AND-gate openings through
torch.distributed (gloo).

* position add: the XOR of the two alpha shares is off0 + off1 (the
  Kogge-Stone adder's sum with carry-out, bool_circuit/adder.h:22-63);
* DltSft: the XOR of the two shares is [digit_i(alpha) == k] * Delta with
  lsb(Delta) forced to 1 -- checked against the oracle's dealer (which
  restates dpf.cpp's Gen) and a numpy statement of the circuit;
* one exchange per AND depth;
* the full interactive expansion, with its DltSft shares and roots from
  GMW, equals the fused keyed expansion built from the same alpha and Delta,
  bit for bit, and satisfies the OLE relation.
AND triples, beta shares and F_p Beaver triples come from a dealer standing
in for the OT layer."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu
P = O.P


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run_two(target, *args):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=target, args=(p, port, q) + args) for p in (0, 1)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=600) for _ in range(2))
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    return out


def _init(party, port):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=party, world_size=2,
                            timeout=datetime.timedelta(seconds=120))
    return dist


# ---- circuits alone ----------------------------------------------------------
ADD_CASES = [(1, 1), (33, 5), (100, 15), (4096, 16), (70, 40)]          # (B, off_bits)
DLT_CASES = [(1, 4, 1), (37, 6, 2), (64, 8, 4), (100, 17, 1), (33, 9, 3)]  # (B, n, w)


def _circuit_material(seed):
    import pcg_b200 as L
    from pcg_b200 import twoparty as T
    rng = np.random.default_rng(seed)
    adds, dlts = [], []
    for B, m in ADD_CASES:
        off = rng.integers(0, 1 << m, (2, B), dtype=np.uint64)
        tri = T.bool_triples_dealer(L.gmw_position_add_gates(m), B, rng)
        adds.append((B, m, off, tri))
    for B, n, w in DLT_CASES:
        alpha = rng.integers(0, 1 << n, B, dtype=np.uint64)
        a0 = rng.integers(0, 1 << n, B, dtype=np.uint64)
        delta = rng.integers(0, 2**64 - 1, (2, B, 2), dtype=np.uint64, endpoint=True)
        tri = T.bool_triples_dealer(L.gmw_dltsft_gates(n, w), B, rng)
        dlts.append((B, n, w, alpha, np.stack([a0, a0 ^ alpha]), delta, tri))
    return adds, dlts


def _circuit_party(party, port, q, seed):
    dist = _init(party, port)
    try:
        import pcg_b200 as L
        from pcg_b200 import twoparty as T
        adds, dlts = _circuit_material(seed)
        chan = T.Channel(party)
        res = {"add": [], "dlt": []}
        for B, m, off, tri in adds:
            before = chan.messages
            a = L.gmw_position_add(party, off[party], m, tri[party], chan.exchange)
            res["add"].append((a, chan.messages - before))
        for B, n, w, _, ash, delta, tri in dlts:
            before = chan.messages
            d, s = L.gmw_dltsft(party, ash[party], delta[party], n, w, tri[party], chan.exchange)
            res["dlt"].append((d, s, chan.messages - before))
        q.put((party, res))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _and_depth_adder(m):
    """AND depth of the Kogge-Stone adder (adder.h:22-63) with every gate
    evaluated as soon as its inputs are: at most 1 + ceil(log2 m), less where
    a prefix step reads an already final generate bit (m = 5: 3)."""
    G, P = [1] * m, [0] * m
    d = 1
    while d < m:
        G = G[:d] + [max(G[i], max(P[i], G[i - d]) + 1) for i in range(d, m)]
        P = P[:d] + [max(P[i], P[i - d]) + 1 for i in range(d, m)]
        d *= 2
    return max(G + P)


def test_gmw_circuits_reconstruct(pcg):
    seed = 2024
    out = _run_two(_circuit_party, seed)
    adds, dlts = _circuit_material(seed)
    for (B, m, off, _), r0, r1 in zip(adds, out[0]["add"], out[1]["add"]):
        assert ((r0[0] ^ r1[0]) == off[0] + off[1]).all(), (B, m)
        assert r0[1] == r1[1] == _and_depth_adder(m), (m, r0[1])
    for (B, n, w, alpha, _, delta, _), r0, r1 in zip(dlts, out[0]["dlt"], out[1]["dlt"]):
        levels, nk = n // w, (1 << w) - 1
        d0, d1 = r0[0], r1[0]
        assert (d0[:, 0] & np.uint64(1)).all() and not (d1[:, 0] & np.uint64(1)).any()
        one = np.uint64(1)
        for p, d in ((0, d0), (1, d1)):   # every other bit as given
            assert ((d[:, 0] | one) == (delta[p][:, 0] | one)).all() and (d[:, 1] == delta[p][:, 1]).all()
        Delta = d0 ^ d1
        got = (r0[1] ^ r1[1]).reshape(B, levels, nk, 2)
        for b in range(B):
            digit = [(int(alpha[b]) >> (n - w * (i + 1))) & ((1 << w) - 1) for i in range(levels)]
            want = np.zeros((levels, nk, 2), np.uint64)
            for i in range(levels):
                if digit[i] < nk:
                    want[i, digit[i]] = Delta[b]
            assert (got[b] == want).all(), (n, w, b)
            if b < 3:   # the oracle's dealer: dlt1 = dlt0 ^ [digit == k] * Delta
                _, _, dl = O.dpf_deal(n, w, (1, 2), Delta[b], int(alpha[b]), 1, O.PRG_CHACHA8,
                                      None, np.zeros((levels * nk, 2), np.uint64))
                assert (dl.reshape(levels, nk, 2) == got[b]).all(), (n, w, b)
        assert r0[2] == r1[2] == (1 + (w - 1).bit_length()), (n, w, r0[2])


# ---- the whole interactive expansion from GMW preprocessing -----------------
def _pipeline_material(N, c, t, seed):
    import pcg_b200 as L
    from pcg_b200 import twoparty as T
    rng = np.random.default_rng(seed)
    B = c * c * t * t
    g_add, g_dlt = T.preprocess_gates(N, c, t)
    noise = [L.noise(N, c, t, seed, p) for p in (0, 1)]
    beta = np.zeros((2, c * c, t * t), np.uint64)
    bt = np.zeros((3, 2, c * c, t * t), np.uint64)
    for blk in range(c * c):
        ii, jj = divmod(blk, c)
        for idx in range(t * t):
            kk, ll = divmod(idx, t)
            b = int(noise[0][1][ii * t + kk]) * int(noise[1][1][jj * t + ll]) % P
            b0 = int(rng.integers(0, P))
            beta[:, blk, idx] = (b0, (b - b0) % P)
            r, s = int(rng.integers(0, P)), int(rng.integers(0, P))
            for k, v in enumerate((r, s, r * s % P)):
                sh = int(rng.integers(0, P))
                bt[k, :, blk, idx] = (sh, (v - sh) % P)
    return dict(noise=noise, beta=beta, bt=bt,
                delta=rng.integers(0, 2**64 - 1, (2, B, 2), dtype=np.uint64, endpoint=True),
                tri_add=T.bool_triples_dealer(g_add, B, rng),
                tri_dlt=T.bool_triples_dealer(g_dlt, B, rng),
                a=O.public_a(O.shape(N, c, t), 7))


def _pipeline_party(party, port, q, N, c, t, seed):
    dist = _init(party, port)
    try:
        import pcg_b200 as L
        from pcg_b200 import twoparty as T
        mat = _pipeline_material(N, c, t, seed)
        pos, val = mat["noise"][party]
        chan = T.Channel(party)
        roots, dlt, delta, alpha = T.preprocess(party, chan, N, c, t, pos, mat["delta"][party],
                                                mat["tri_add"][party], mat["tri_dlt"][party])
        pre_msgs = chan.messages
        e = L.Expander(N, c, t, 1, L.PRG_CHACHA8, public_a=mat["a"])
        m = T.PartyMaterial(roots=roots, dltsft=dlt, beta=mat["beta"][party],
                            r=mat["bt"][0][party], s=mat["bt"][1][party], rs=mat["bt"][2][party],
                            pos=pos, val=val)
        d_x, d_z = T.gen_and_expand(party, chan, e, m)
        L.synchronize()
        q.put((party, dict(x=d_x.download(np.uint64, N), z=d_z.download(np.uint64, N),
                           roots=roots, delta=delta, alpha=alpha, pre=pre_msgs,
                           msgs=chan.messages)))
        e.close()
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("N,c,t", [(1 << 12, 2, 4), (1 << 13, 2, 8)])
def test_expansion_from_gmw_preprocessing_matches_fused(pcg, N, c, t):
    from pcg_b200 import twoparty as T
    seed = 6100 + N
    out = _run_two(_pipeline_party, N, c, t, seed)
    mat = _pipeline_material(N, c, t, seed)
    s = O.shape(N, c, t)
    n, B = s.n, t * t
    off_bits = n - 1
    pre = _and_depth_adder(off_bits) + 1
    assert out[0]["pre"] == out[1]["pre"] == pre
    assert out[0]["msgs"] == pre + n + 2
    off = [T.instance_offsets(p, N, c, t, mat["noise"][p][0]) for p in (0, 1)]
    alpha = out[0]["alpha"] ^ out[1]["alpha"]
    assert (alpha == off[0] + off[1]).all()
    Delta = out[0]["delta"] ^ out[1]["delta"]
    assert ((out[0]["roots"] ^ out[1]["roots"]).reshape(-1, 2) == Delta).all()
    # Keyed view of the same DPFs: root0 and Delta from GMW, alpha = off0 + off1.
    K = c * c * B
    cws = np.zeros((K * n, 2), np.uint64)
    cwo = np.zeros(K, np.uint64)
    beta = (mat["beta"][0].astype(object) + mat["beta"][1].astype(object)) % P
    r0 = out[0]["roots"].reshape(K, 2)
    for key in range(K):
        cw, co, _ = O.dpf_deal(n, 1, r0[key], Delta[key], int(alpha[key]),
                               int(beta.reshape(-1)[key]), O.PRG_CHACHA8)
        cws[key * n:(key + 1) * n], cwo[key] = cw, co
    pcg_e = pcg.Expander(N, c, t, 1, pcg.PRG_CHACHA8, public_a=mat["a"])
    for party in (0, 1):
        roots = out[party]["roots"].reshape(K, 2)
        x, z = pcg_e.expand_host(party, roots, cws, cwo, *mat["noise"][party])
        assert (out[party]["x"] == x).all(), party
        assert (out[party]["z"] == z).all(), party
    pcg_e.close()
    prod = O.poly_mul(out[0]["x"], out[1]["x"], N)
    zz = (out[0]["z"].astype(object) + out[1]["z"].astype(object)) % P
    assert all(int(a) == int(b) for a, b in zip(prod, zz))


def test_gmw_rejects_bad_arguments(pcg):
    """Argument errors come back as PCGB_EINVAL before any exchange."""
    from pcg_b200 import twoparty as T
    rng = np.random.default_rng(5)
    B = 40
    tri = T.bool_triples_dealer(pcg.gmw_position_add_gates(8), B, rng)[0]
    off = np.arange(B, dtype=np.uint64)
    never = lambda my: (_ for _ in ()).throw(AssertionError("no exchange expected"))
    with pytest.raises(pcg.PcgError, match="party") as e:
        pcg.gmw_position_add(2, off, 8, tri, never)
    assert e.value.code == -1
    with pytest.raises(pcg.PcgError, match="off_bits"):
        pcg.gmw_position_add(0, off, 64, ((), (), ()), never)
    with pytest.raises(pcg.PcgError, match="exchange callback is required"):
        pcg.gmw_position_add(0, off, 8, tri, None)
    with pytest.raises(ValueError, match="triples"):
        pcg.gmw_position_add(0, off, 8, [v[:-1] for v in tri], never)
    delta = np.zeros((B, 2), np.uint64)
    for n, w in ((7, 2), (18, 9)):
        with pytest.raises(pcg.PcgError, match=r"w \| n"):
            pcg.gmw_dltsft(0, off, delta, n, w, ((), (), ()), never)
    # Calls with B = 0 are no-ops.
    assert pcg.gmw_position_add(0, np.zeros(0, np.uint64), 8, ((), (), ()), never).size == 0
