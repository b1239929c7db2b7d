"""GPU DPF parity through the C ABI: keyed eval and the interactive drop-in
(pcg_cuda::dpf_gpu_batch_full_eval) against the oracle and the reference's
dpf_real_bench golden checksums."""
import numpy as np
import pytest

import oracle_lib as O
from gpu_helpers import dealt_keys, dev, real_bench_checksum, real_bench_inputs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prg", [O.PRG_CHACHA8, O.PRG_AES])
@pytest.mark.parametrize("n,w", [(6, 1), (11, 1), (8, 2), (9, 3), (8, 4)])
def test_keyed_full_eval_matches_oracle(pcg, prg, n, w):
    nk = (1 << w) - 1
    rks = O.aes_tree_round_keys(np.arange(16, dtype=np.uint8), nk) if prg == O.PRG_AES else None
    K = 6
    k = dealt_keys(n, w, K, 11 * n + w, prg, rks)
    want = O.dpf_keyed_full_eval(K, n, w, k["roots0"], k["cws"], prg, rks)
    d_r, d_c = dev(pcg, k["roots0"]), dev(pcg, k["cws"])
    d_l = pcg.DeviceBuffer(want.nbytes)
    pcg.dpf_keyed_full_eval_device(K, n, w, prg, d_r.ptr, d_c.ptr, d_l.ptr, round_keys=rks)
    got = d_l.download(np.uint64, want.size).reshape(-1, 2)
    assert (got == want).all()


# ChaCha8 w = 1 top-walk stages take the compile-time-depth walk of their
# depth, 1 .. 8 levels; a deeper last stage is split in two.  Six keys give
# stages of n levels for n <= 5; 2^14 keys give a 5-level stage and then the
# last stage (2^19 or more subtrees) of n - 5 levels: 6, 7, 8, and 9 split
# into 1 + 8.
@pytest.mark.parametrize("K,n", [(6, 2), (6, 3), (6, 4), (1 << 14, 11), (1 << 14, 12),
                                 (1 << 14, 13), (1 << 14, 14)])
def test_keyed_eval_every_walk_depth(pcg, K, n):
    rng = np.random.default_rng(900 + n)
    roots = rng.integers(0, 2**64 - 1, (K, 2), dtype=np.uint64)
    cws = rng.integers(0, 2**64 - 1, (K, n, 2), dtype=np.uint64)
    D = 1 << n
    d_r, d_c = dev(pcg, roots), dev(pcg, cws.reshape(-1, 2))
    d_l = pcg.DeviceBuffer(16 * K * D)
    pcg.dpf_keyed_full_eval_device(K, n, 1, O.PRG_CHACHA8, d_r.ptr, d_c.ptr, d_l.ptr)
    pick = np.unique(np.concatenate([[0, K - 1], rng.integers(0, K, 30)]))
    want = O.dpf_keyed_full_eval(len(pick), n, 1, roots[pick], cws[pick].reshape(-1, 2))
    got = np.empty((len(pick), D, 2), np.uint64)
    for i, k in enumerate(pick):
        rc = pcg.lib.pcgb_memcpy_d2h(got[i].ctypes.data, d_l.ptr + 16 * D * int(k), 16 * D, None)
        assert rc == 0
    assert (got.reshape(-1, 2) == want).all()


@pytest.mark.parametrize("prg", [O.PRG_CHACHA8, O.PRG_AES])
@pytest.mark.parametrize("n,w", [(1, 1), (10, 1), (10, 2), (9, 3), (12, 4)])
def test_interactive_stub_exchange_matches_oracle(pcg, prg, n, w):
    rng = np.random.default_rng(n * 7 + w)
    B, nk = 7, (1 << w) - 1
    rks = O.aes_tree_round_keys(rng.integers(0, 256, 16, dtype=np.uint8), nk) \
        if prg == O.PRG_AES else None
    roots = rng.integers(0, 2**64 - 1, (B, 2), dtype=np.uint64)
    dlt = rng.integers(0, 2**64 - 1, (B * (n // w) * nk, 2), dtype=np.uint64)
    want = O.dpf_batch_full_eval(B, n, w, roots, dlt, prg, rks)
    got = pcg.dpf_gpu_batch_full_eval(B, n, w, roots, dlt, round_keys=rks, prg=prg)
    assert (got == want).all()


@pytest.mark.parametrize("prg", [O.PRG_CHACHA8, O.PRG_AES])
@pytest.mark.parametrize("n,w", [(10, 1), (10, 2), (8, 4), (14, 1), (14, 2)])
def test_interactive_two_party_matches_keyed(pcg, prg, n, w):
    """Real DltSft shares; the peer's share is my ^ CW (what the other party
    sends), so the drop-in must reproduce the dealer's keyed leaves.  n = 14
    reaches levels of 4096+ parents, where the AES levels hash with the
    replicated table and several parents per thread."""
    nk, L = (1 << w) - 1, n // w
    rks = O.aes_tree_round_keys(np.arange(16, dtype=np.uint8), nk) if prg == O.PRG_AES else None
    B = 5
    k = dealt_keys(n, w, B, 99 + n, prg, rks, with_dlt=True)
    cw = k["cws"].reshape(B, L, nk, 2)
    for party, roots, dlt in ((0, k["roots0"], k["dlt0"]), (1, k["roots1"], k["dlt1"])):
        level = [0]

        def exchange(my):
            peer = my.reshape(B, nk, 2) ^ cw[:, level[0]]
            level[0] += 1
            return peer.reshape(-1, 2)

        got = pcg.dpf_gpu_batch_full_eval(B, n, w, roots, dlt, round_keys=rks, party=party,
                                          exchange=exchange, prg=prg)
        assert level[0] == L
        want = O.dpf_keyed_full_eval(B, n, w, roots, k["cws"], prg, rks)
        assert (got == want).all()


def test_interactive_errors(pcg):
    roots = np.zeros((2, 2), np.uint64)
    with pytest.raises(pcg.PcgError, match="w must divide n"):
        pcg.dpf_gpu_batch_full_eval(2, 5, 2, roots, np.zeros((20, 2), np.uint64),
                                    prg=pcg.PRG_CHACHA8)
    with pytest.raises(pcg.PcgError, match=r"w must be in \[1,4\]"):
        pcg.dpf_gpu_batch_full_eval(2, 10, 5, roots, np.zeros((20, 2), np.uint64),
                                    prg=pcg.PRG_CHACHA8)
    with pytest.raises(pcg.PcgError, match="AES PRG requires round_keys"):
        pcg.dpf_gpu_batch_full_eval(2, 4, 1, roots, np.zeros((8, 2), np.uint64), prg=pcg.PRG_AES)
    with pytest.raises(pcg.PcgError, match="exchange callback"):
        pcg.dpf_gpu_batch_full_eval(2, 4, 1, roots, np.zeros((8, 2), np.uint64),
                                    exchange=lambda my: 1 / 0, prg=pcg.PRG_CHACHA8)
    assert pcg.dpf_gpu_batch_full_eval_device(0, 4, 1, roots, roots) is None


# GPU_baseline/results_l40s/plateau.txt: dpf_real_bench checksums (w=1, chacha8).
GOLDEN = [(18, 64, 8, 0x16E395FEBFD6D23F), (18, 256, 16, 0x27CB4298E84744ED),
          (20, 64, 8, 0x104646E15A59C497), (20, 256, 16, 0x204A14F81D54AA7E),
          (24, 16, 4, 0x02A9707398F918D0)]


@pytest.mark.parametrize("n,B,t,want", GOLDEN)
def test_dpf_real_bench_golden_checksums(pcg, n, B, t, want):
    roots, dlt, CW = real_bench_inputs(n, B)
    d_leaves = pcg.dpf_gpu_batch_full_eval_device(B, n, 1, roots, dlt, prg=pcg.PRG_CHACHA8)
    D = 1 << n
    sc, st = pcg.dpf_out_sums(d_leaves, B, D)
    g = pcg.dpf_out_scatter_g(d_leaves, B, D, t, 0, CW, t * (D // 2))
    assert real_bench_checksum(sc, st, g) == want


@pytest.mark.parametrize("prg", [O.PRG_CHACHA8, O.PRG_AES])
@pytest.mark.parametrize("n,w,B", [(1, 1, 3), (10, 1, 5), (10, 2, 5), (9, 3, 4), (8, 4, 6),
                                   (12, 1, 300), (13, 1, 4), (14, 2, 3), (16, 4, 2)])
def test_interactive_fused_convert_matches_two_calls(pcg, prg, n, w, B):
    """pcgb_dpf_batch_full_eval_convert_device (last level fused with the
    sums pass, no leaves stored) gives the converted words and sums of
    dpf_gpu_batch_full_eval_device + pcgb_dpf_out_convert_device, and the
    oracle's sums, with a real per-level exchange.  (13,1), (14,2) and (16,4)
    have 4096 last-level parents, where the AES expand levels walk 8 parents
    per thread and the fused last level must still take one each."""
    nk, L = (1 << w) - 1, n // w
    rks = O.aes_tree_round_keys(np.arange(16, dtype=np.uint8), nk) if prg == O.PRG_AES else None
    rng = np.random.default_rng(31 * n + w + B)
    roots = rng.integers(0, 2**64 - 1, (B, 2), dtype=np.uint64, endpoint=True)
    dlt = rng.integers(0, 2**64 - 1, (B * L * nk, 2), dtype=np.uint64, endpoint=True)
    mask = rng.integers(0, 2**64 - 1, (B * nk, 2), dtype=np.uint64, endpoint=True)
    exchange = lambda my: my ^ mask            # a deterministic stand-in for the peer
    D = 1 << n
    d_leaves = pcg.dpf_gpu_batch_full_eval_device(B, n, w, roots, dlt, round_keys=rks,
                                                  exchange=exchange, prg=prg)
    conv0, sums0 = pcg.DeviceBuffer(8 * B * D), pcg.DeviceBuffer(16 * B)
    pcg.dpf_out_convert_device(d_leaves, B, D, conv0.ptr, sums0.ptr, sums0.ptr + 8 * B)
    pcg.synchronize()
    leaves = np.zeros((B * D, 2), np.uint64)
    pcg.lib.pcgb_memcpy_d2h(leaves.ctypes.data, d_leaves, leaves.nbytes, None)
    conv1, sums1 = pcg.DeviceBuffer(8 * B * D), pcg.DeviceBuffer(16 * B)
    pcg.lib.pcgb_memset(conv1.ptr, 0xA5, conv1.nbytes, None)   # every word must be written
    pcg.dpf_gpu_batch_full_eval_convert_device(B, n, w, roots, dlt, conv1.ptr, sums1.ptr,
                                               sums1.ptr + 8 * B, round_keys=rks,
                                               exchange=exchange, prg=prg)
    assert (conv1.download(np.uint64, B * D) == conv0.download(np.uint64, B * D)).all()
    s0, s1 = sums0.download(np.uint64, 2 * B), sums1.download(np.uint64, 2 * B)
    assert (s0 == s1).all()
    wc, wt = O.out_sums(leaves, B, D)
    assert (s1[:B] == wc).all() and (s1[B:] == wt).all()


@pytest.mark.parametrize("prg", [O.PRG_CHACHA8, O.PRG_AES])
def test_interactive_fused_convert_device_exchange(pcg, prg):
    """pcgb_dpf_batch_full_eval_convert_device_dx: the per-level shares go to
    a device-side callback (here a one-GPU loopback, peer = my ^ mask
    computed by torch on the device) and the outputs equal the host-exchange
    call's with the same peer values, one callback per level."""
    torch = pytest.importorskip("torch")
    from pcg_b200.twoparty import device_words
    B, n, w = 64, 12, 1
    nk, L = (1 << w) - 1, n // w
    rks = O.aes_tree_round_keys(np.arange(16, dtype=np.uint8), nk) if prg == O.PRG_AES else None
    rng = np.random.default_rng(77)
    roots = rng.integers(0, 2**64 - 1, (B, 2), dtype=np.uint64, endpoint=True)
    dlt = rng.integers(0, 2**64 - 1, (B * L * nk, 2), dtype=np.uint64, endpoint=True)
    mask = rng.integers(0, 2**64 - 1, (B * nk, 2), dtype=np.uint64, endpoint=True)
    d_mask = torch.from_numpy(mask.view(np.int64).reshape(-1).copy()).cuda()
    calls = []

    def dex(d_my, d_peer, count):
        my, peer = device_words(d_my, 2 * count), device_words(d_peer, 2 * count)
        peer.copy_(my ^ d_mask)
        torch.cuda.synchronize()
        calls.append(count)

    D = 1 << n
    outs = []
    for use_dev in (False, True):
        conv, sums = pcg.DeviceBuffer(8 * B * D), pcg.DeviceBuffer(16 * B)
        if use_dev:
            pcg.dpf_gpu_batch_full_eval_convert_device_dx(B, n, w, roots, dlt, conv.ptr, sums.ptr,
                                                          sums.ptr + 8 * B, dex, round_keys=rks,
                                                          prg=prg)
        else:
            pcg.dpf_gpu_batch_full_eval_convert_device(B, n, w, roots, dlt, conv.ptr, sums.ptr,
                                                       sums.ptr + 8 * B, round_keys=rks,
                                                       exchange=lambda my: my ^ mask, prg=prg)
        outs.append((conv.download(np.uint64, B * D), sums.download(np.uint64, 2 * B)))
    assert calls == [B * nk] * L
    assert (outs[0][0] == outs[1][0]).all() and (outs[0][1] == outs[1][1]).all()


MULTI_CASES = [
    (O.PRG_CHACHA8, 1, [(64, 10), (7, 12), (300, 8), (1, 16), (0, 9), (2048, 12)]),
    (O.PRG_CHACHA8, 2, [(100, 10), (16, 12), (1, 4)]),
    (O.PRG_AES, 1, [(64, 10), (9, 12), (0, 6), (33, 7)]),
    # A final stage of 2^19+ threads: the PRMT-addressed AES walk.
    (O.PRG_AES, 1, [(4096, 10), (2048, 12), (3, 8)]),
]


@pytest.mark.parametrize("prg,w,groups", MULTI_CASES)
def test_keyed_multi_domain_batch(pcg, prg, w, groups):
    """pcgb_dpf_keyed_full_eval_multi: key groups of different domains in one
    batch give each group's single-call leaves (and the oracle's for the
    smallest group), in as many launches as the deepest group's stage plan
    (ChaCha8, w = 1: one per stage and walk depth, so at least that many and
    fewer than one call per group)."""
    nk = (1 << w) - 1
    rks = O.aes_tree_round_keys(np.arange(16, dtype=np.uint8), nk) if prg == O.PRG_AES else None
    rng = np.random.default_rng(len(groups) * 10 + w)
    bufs, want, stages = [], [], []
    for K, n in groups:
        roots = rng.integers(0, 2**64 - 1, (max(K, 1), 2), dtype=np.uint64, endpoint=True)
        cws = rng.integers(0, 2**64 - 1, (max(K, 1) * (n // w) * nk, 2), dtype=np.uint64,
                           endpoint=True)
        d_r, d_c = pcg.to_device(roots), pcg.to_device(cws)
        d_one = pcg.DeviceBuffer(16 * max(K, 1) << n)
        before = pcg.launch_count()
        pcg.dpf_keyed_full_eval_device(K, n, w, prg, d_r.ptr, d_c.ptr, d_one.ptr, round_keys=rks)
        pcg.synchronize()
        stages.append(pcg.launch_count() - before)
        want.append(d_one.download(np.uint64, 2 * (K << n)))
        if 0 < K <= 9 and n <= 12:   # pinned to the oracle too
            o = O.dpf_keyed_full_eval(K, n, w, roots[:K], cws[:K * (n // w) * nk], prg, rks)
            assert (want[-1] == o.reshape(-1)).all()
        d_out = pcg.DeviceBuffer(16 * max(K, 1) << n)
        pcg.lib.pcgb_memset(d_out.ptr, 0x5A, d_out.nbytes, None)
        bufs.append((K, n, d_r, d_c, d_out))
    before = pcg.launch_count()
    pcg.dpf_keyed_full_eval_multi_device([(K, n, r.ptr, c.ptr, o.ptr) for K, n, r, c, o in bufs],
                                         w, prg, round_keys=rks)
    pcg.synchronize()
    launches = pcg.launch_count() - before
    if prg == O.PRG_CHACHA8 and w == 1:
        assert max(stages) <= launches < sum(stages)
    else:
        assert launches == max(stages)
    for (K, n, _, _, d_out), wv in zip(bufs, want):
        assert (d_out.download(np.uint64, 2 * (K << n)) == wv).all(), (K, n)


def test_keyed_multi_rejects_bad_groups(pcg):
    d = pcg.DeviceBuffer(16 * 64)
    with pytest.raises(pcg.PcgError, match="bad"):
        pcg.dpf_keyed_full_eval_multi_device([(4, 7, d.ptr, d.ptr, d.ptr)], 2, pcg.PRG_CHACHA8)
    with pytest.raises(pcg.PcgError, match="negative"):
        pcg.dpf_keyed_full_eval_multi_device([(-1, 6, d.ptr, d.ptr, d.ptr)], 1, pcg.PRG_CHACHA8)
    with pytest.raises(pcg.PcgError, match="round keys"):
        pcg.dpf_keyed_full_eval_multi_device([(4, 6, d.ptr, d.ptr, d.ptr)], 1, pcg.PRG_AES)


@pytest.mark.parametrize("prg", [O.PRG_CHACHA8, O.PRG_AES])
@pytest.mark.parametrize("n,w,K", [(10, 1, 9), (14, 1, 5), (14, 2, 4), (16, 4, 3)])
def test_point_function_property(pcg, prg, n, w, K):
    """The reference's half_tree_dpf test (CPU_baseline/test/half_tree_dpf.cpp:80-94):
    the two parties' leaves XOR to Delta at alpha and to zero everywhere else,
    for the keyed evaluation and for the interactive drop-in with real DltSft
    shares (levels of 4096+ parents take the PRMT-addressed AES kernel)."""
    nk, L = (1 << w) - 1, n // w
    rks = O.aes_tree_round_keys(np.arange(16, dtype=np.uint8), nk) if prg == O.PRG_AES else None
    k = dealt_keys(n, w, K, 500 + n + w, prg, rks, with_dlt=True)
    D = 1 << n
    want = np.zeros((K, D, 2), np.uint64)
    want[np.arange(K), k["alphas"]] = k["deltas"]
    d_c = dev(pcg, k["cws"])
    keyed = []
    for roots in (k["roots0"], k["roots1"]):
        d_r, d_l = dev(pcg, roots), pcg.DeviceBuffer(16 * K * D)
        pcg.dpf_keyed_full_eval_device(K, n, w, prg, d_r.ptr, d_c.ptr, d_l.ptr, round_keys=rks)
        keyed.append(d_l.download(np.uint64, 2 * K * D).reshape(K, D, 2))
    assert (keyed[0] ^ keyed[1] == want).all()
    cw = k["cws"].reshape(K, L, nk, 2)
    inter = []
    for party, roots, dlt in ((0, k["roots0"], k["dlt0"]), (1, k["roots1"], k["dlt1"])):
        level = [0]

        def exchange(my):
            peer = my.reshape(K, nk, 2) ^ cw[:, level[0]]
            level[0] += 1
            return peer.reshape(-1, 2)

        inter.append(pcg.dpf_gpu_batch_full_eval(K, n, w, roots, dlt, round_keys=rks, party=party,
                                                 exchange=exchange, prg=prg).reshape(K, D, 2))
    assert (inter[0] ^ inter[1] == want).all()
