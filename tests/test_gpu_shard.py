"""Intra-expansion sharding (pcgb_expander_create_shard): the pair blocks of
one expansion split over `world` shards.  The shards' partial z must sum
(mod p) to the unsharded z bit for bit, every shard's x must be the full x,
and the pairs must be partitioned.  The multi-process form sums the partial
z's with a torch.distributed all-reduce (gloo, host tensors) between two
processes that share the GPU, followed by the mod-p fix-up."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu
P = O.P


def _expand(pcg, e, N, c, t, seed, party=0):
    K, L = e.K, e.levels
    r0, r1 = pcg.DeviceBuffer(16 * K), pcg.DeviceBuffer(16 * K)
    cws, cwo = pcg.DeviceBuffer(16 * K * L * e.nk), pcg.DeviceBuffer(8 * K)
    e.deal_keys_device(seed, r0.ptr, r1.ptr, cws.ptr, cwo.ptr)
    pos, val = pcg.noise(N, c, t, seed, party)
    dp, dv = pcg.to_device(pos), pcg.to_device(val)
    x, z = pcg.DeviceBuffer(8 * N), pcg.DeviceBuffer(8 * N)
    e.expand_device(party, (r1 if party else r0).ptr, cws.ptr, cwo.ptr, dp.ptr, dv.ptr, x.ptr,
                    z.ptr)
    pcg.synchronize()
    return x.download(np.uint64, N), z.download(np.uint64, N)


@pytest.mark.parametrize("N,c,t", [(1 << 12, 2, 4), (1 << 14, 4, 8)])
@pytest.mark.parametrize("world", [2, 3, 4])
def test_shards_sum_to_the_expansion(pcg, N, c, t, world):
    s = O.shape(N, c, t)
    a = O.public_a(s, 7)
    full = pcg.Expander(N, c, t, 1, pcg.PRG_CHACHA8, public_a=a)
    x_full, z_full = _expand(pcg, full, N, c, t, 31, party=1)
    assert full.world == 1 and full.Q == full.Q_total == c * (c + 1) // 2
    zsum = np.zeros(N, dtype=object)
    pairs = 0
    for rank in range(world):
        e = pcg.Expander(N, c, t, 1, pcg.PRG_CHACHA8, public_a=a, rank=rank, world=world)
        assert (e.rank, e.world, e.Q_total) == (rank, world, full.Q)
        pairs += e.Q
        x, z = _expand(pcg, e, N, c, t, 31, party=1)
        assert (x == x_full).all()
        zsum += z.astype(object)
        e.close()
    assert pairs == full.Q
    zsum = np.array([int(v) % P for v in zsum], np.uint64)
    assert (zsum == z_full).all()
    full.close()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _shard_rank(rank, port, N, c, t, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=2,
                            timeout=datetime.timedelta(seconds=120))
    try:
        import pcg_b200 as L
        s = O.shape(N, c, t)
        e = L.Expander(N, c, t, 1, L.PRG_CHACHA8, public_a=O.public_a(s, 7), rank=rank, world=2)
        x, z = _expand(L, e, N, c, t, 77)
        zt = torch.from_numpy(z.view(np.int64).copy())
        dist.all_reduce(zt)                       # uint64 sum, exact for 2 shards
        d = L.to_device(zt.numpy().view(np.uint64))
        L.reduce_mod_p(d.ptr, d.ptr, N)
        q.put((rank, x, d.download(np.uint64, N)))
        e.close()
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_process_shards_all_reduce(pcg):
    N, c, t = 1 << 14, 4, 8
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_rank, args=(r, port, N, c, t, q)) for r in (0, 1)]
    for p in procs:
        p.start()
    got = dict((r, (x, z)) for r, x, z in (q.get(timeout=300) for _ in range(2)))
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    s = O.shape(N, c, t)
    full = pcg.Expander(N, c, t, 1, pcg.PRG_CHACHA8, public_a=O.public_a(s, 7))
    x_full, z_full = _expand(pcg, full, N, c, t, 77)
    for r in (0, 1):
        assert (got[r][0] == x_full).all() and (got[r][1] == z_full).all()
    full.close()
