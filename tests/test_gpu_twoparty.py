"""The interactive two-party expansion (pcg_b200.twoparty): two processes,
one per party, exchanging each level's correction-word shares and the two
Beaver opens through torch.distributed (gloo), each running the drop-in
DPF and convert entry points on the GPU.  Their outputs must equal the fused
keyed expansion's on the same material, bit for bit, and satisfy the OLE
relation.  The preprocessing (DltSft shares, beta shares, Beaver triples)
comes from a dealer written with the oracle, standing in for the OT layer."""
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


def dealer(N, c, t, seed):
    """Material for both parties (interactive) and the keyed view of it."""
    import pcg_b200 as L
    s = O.shape(N, c, t)
    n, B, bin_ = s.n, t * t, N // t
    rng = np.random.default_rng(seed)
    noise = [L.noise(N, c, t, seed, p) for p in (0, 1)]
    roots = np.zeros((2, c * c, B, 2), np.uint64)
    dlt = np.zeros((2, c * c, B * n, 2), np.uint64)
    cws = np.zeros((c * c * B * n, 2), np.uint64)
    cwo = np.zeros(c * c * B, np.uint64)
    beta = np.zeros((2, c * c, B), np.uint64)
    r_, s_, rs_ = (np.zeros((2, c * c, B), np.uint64) for _ in range(3))
    for blk in range(c * c):
        ii, jj = divmod(blk, c)
        for idx in range(B):
            kk, ll = divmod(idx, t)
            p0, v0 = int(noise[0][0][ii * t + kk]), int(noise[0][1][ii * t + kk])
            p1, v1 = int(noise[1][0][jj * t + ll]), int(noise[1][1][jj * t + ll])
            alpha = (p0 - kk * bin_) + (p1 - ll * bin_)
            b = v0 * v1 % P
            root0 = rng.integers(0, 2**64 - 1, 2, dtype=np.uint64)
            delta = rng.integers(0, 2**64 - 1, 2, dtype=np.uint64)
            delta[0] |= np.uint64(1)
            d0 = rng.integers(0, 2**64 - 1, (n, 2), dtype=np.uint64)
            cw, co, d1 = O.dpf_deal(n, 1, root0, delta, alpha, b, O.PRG_CHACHA8, None, d0)
            key = blk * B + idx
            cws[key * n:(key + 1) * n], cwo[key] = cw, co
            roots[0, blk, idx], roots[1, blk, idx] = root0, root0 ^ delta
            dlt[0, blk, idx * n:(idx + 1) * n], dlt[1, blk, idx * n:(idx + 1) * n] = d0, d1
            b0 = int(rng.integers(0, P))
            beta[0, blk, idx], beta[1, blk, idx] = b0, (b - b0) % P
            r, s2 = int(rng.integers(0, P)), int(rng.integers(0, P))
            for arr, v in ((r_, r), (s_, s2), (rs_, r * s2 % P)):
                sh = int(rng.integers(0, P))
                arr[0, blk, idx], arr[1, blk, idx] = sh, (v - sh) % P
    return dict(noise=noise, roots=roots, dlt=dlt, cws=cws, cwo=cwo, beta=beta, r=r_, s=s_,
                rs=rs_, a=O.public_a(s, 7))


def _party(party, port, N, c, t, mat, q, batched, device_channel=False):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=party, world_size=2,
                            timeout=datetime.timedelta(seconds=120))
    try:
        import pcg_b200 as L
        from pcg_b200 import twoparty
        e = L.Expander(N, c, t, 1, L.PRG_CHACHA8, public_a=mat["a"])
        m = twoparty.PartyMaterial(
            roots=mat["roots"][party], dltsft=mat["dlt"][party], beta=mat["beta"][party],
            r=mat["r"][party], s=mat["s"][party], rs=mat["rs"][party],
            pos=mat["noise"][party][0], val=mat["noise"][party][1])
        # DeviceChannel: messages stay in device memory up to the transport
        # (gloo here, staged through the host; NCCL moves them device to
        # device when each party has its own GPU).
        chan = twoparty.DeviceChannel(party) if device_channel else twoparty.Channel(party)
        d_x, d_z = twoparty.gen_and_expand(party, chan, e, m, batched=batched)
        L.synchronize()
        q.put((party, d_x.download(np.uint64, N), d_z.download(np.uint64, N), chan.messages))
        e.close()
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("N,c,t,batched,device_channel",
                         [(1 << 12, 2, 4, False, False), (1 << 12, 2, 4, True, False),
                          (1 << 13, 2, 8, True, False), (1 << 13, 2, 8, True, True),
                          (1 << 12, 2, 4, False, True)])
def test_two_processes_match_the_fused_expansion(pcg, N, c, t, batched, device_channel):
    mat = dealer(N, c, t, 5150 + N)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_party, args=(p, port, N, c, t, mat, q, batched, device_channel))
             for p in (0, 1)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(2):
        party, x, z, msgs = q.get(timeout=300)
        out[party] = (x, z, msgs)
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    levels = O.shape(N, c, t).n
    # Per-level CW exchanges and two Beaver opens, per block or for all blocks.
    assert out[0][2] == (levels + 2) * (1 if batched else c * c)
    e = pcg.Expander(N, c, t, 1, pcg.PRG_CHACHA8, public_a=mat["a"])
    K = e.K
    for party in (0, 1):
        roots = mat["roots"][party].reshape(K, 2)
        x, z = e.expand_host(party, roots, mat["cws"], mat["cwo"], *mat["noise"][party])
        assert (out[party][0] == x).all(), party
        assert (out[party][1] == z).all(), party
    e.close()
    prod = O.poly_mul(out[0][0], out[1][0], N)
    zz = (out[0][1].astype(object) + out[1][1].astype(object)) % P
    assert all(int(a) == int(b) for a, b in zip(prod, zz))
