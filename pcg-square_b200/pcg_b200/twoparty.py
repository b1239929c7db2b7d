"""Interactive two-party PCG-OLE expansion over the drop-in entry points.

The online part of the reference's device path, PCG_OLE::gen_and_expand
(CPU_baseline/pcg_ole_2pc/pcg_ole_impl.h:213-312, then step 4 at :453-484),
run by each party in its own process:

  for every block (i, j):
    leaves = dpf_gpu_batch_full_eval_device(...)   one CW exchange per level
    sumC, sumT = dpf_out_sums(leaves)
    <A> = (-1)^party sumT, <B> = (-1)^(1-party) sumC + <beta>
    open d = A - r, e = B - s                      Beaver triple (r, s, rs)
    <CW> = d<s> + e<r> + <rs> (+ d e for party 0); open CW
    g_ij = dpf_out_scatter_g(leaves, ..., CW)
  x, z = step 4 over the g_ij (pcgb_expand_from_g_device)

By default all c*c blocks run as one batch (see gen_and_expand), which
leaves levels + 2 message exchanges per expansion instead of c*c*(levels+2).

The preprocessing the reference draws from OT and boolean circuits
(DltSft shares, Delta shares, beta shares, Beaver triples; pcg_ole_impl.h:
100-200) is an input here (`PartyMaterial`); the OT layer itself is outside
this library.  Messages travel over a `Channel`: party 0 sends first and
party 1 receives first, as the reference's NetIO exchange does.  With
torch.distributed the two parties may share one GPU: they exchange through
the host between kernels and no kernel waits on the other party.
"""
from dataclasses import dataclass

import numpy as np

from . import (DeviceBuffer, P, PRG_CHACHA8, dpf_gpu_batch_full_eval_device, dpf_out_sums,
               dpf_out_scatter_g_device, synchronize, to_device)


@dataclass
class PartyMaterial:
    """One party's preprocessing for an expansion of shape (N, c, t), w = 1.

    roots:  [c*c, t*t, 2] uint64   DPF root seeds of the t*t keys of each block
    dltsft: [c*c, t*t*levels, 2]   DltSft shares, layout [key][level][k]
    beta:   [c*c, t*t] uint64      additive shares of beta = pay0 * pay1 mod p
    r, s, rs: [c*c, t*t] uint64    additive shares of Beaver triples (rs = r*s)
    pos, val: [c*t] uint64         this party's regular noise
    """
    roots: np.ndarray
    dltsft: np.ndarray
    beta: np.ndarray
    r: np.ndarray
    s: np.ndarray
    rs: np.ndarray
    pos: np.ndarray
    val: np.ndarray


class Channel:
    """Ordered two-party exchange of uint64 arrays over torch.distributed
    point-to-point messages (any backend that supports send/recv)."""

    def __init__(self, party, peer_rank=None):
        import torch
        import torch.distributed as dist
        self.torch, self.dist = torch, dist
        self.party = party
        self.peer = (1 - dist.get_rank()) if peer_rank is None else peer_rank
        self.messages = 0
        self.bytes = 0

    def exchange(self, mine):
        """Send this party's array, return the peer's array of the same shape."""
        mine = np.ascontiguousarray(mine, np.uint64)
        t_my = self.torch.from_numpy(mine.view(np.int64).copy())
        t_peer = self.torch.empty_like(t_my)
        if self.party == 0:
            self.dist.send(t_my, self.peer)
            self.dist.recv(t_peer, self.peer)
        else:
            self.dist.recv(t_peer, self.peer)
            self.dist.send(t_my, self.peer)
        self.messages += 1
        self.bytes += mine.nbytes
        return t_peer.numpy().view(np.uint64).reshape(mine.shape)


def _beaver_cw(party, chan, sumC, sumT, beta, r, s, rs):
    """Output-layer correction words of a batch of instances: <A> =
    (-1)^party sumT, <B> = (-1)^(1-party) sumC + <beta>, CW = A*B by one
    Beaver triple per instance (two opens; pcg_ole_impl.h:222-290)."""
    A = [(P - int(v) % P) % P if party == 1 else int(v) % P for v in sumT]
    Bsh = [((P - int(v)) % P if party == 0 else int(v)) for v in sumC]
    Bsh = [(b + int(x)) % P for b, x in zip(Bsh, beta)]
    n = len(A)
    de_my = np.array([(a - int(x)) % P for a, x in zip(A, r)] +
                     [(b - int(x)) % P for b, x in zip(Bsh, s)], np.uint64)
    de_peer = chan.exchange(de_my)
    cw_my = np.empty(n, np.uint64)
    for k in range(n):
        d = (int(de_my[k]) + int(de_peer[k])) % P
        e = (int(de_my[n + k]) + int(de_peer[n + k])) % P
        v = (d * int(s[k]) + e * int(r[k]) + int(rs[k])) % P
        if party == 0:
            v = (v + d * e) % P
        cw_my[k] = v
    cw_peer = chan.exchange(cw_my)
    return np.array([(int(a) + int(b)) % P for a, b in zip(cw_my, cw_peer)], np.uint64)


def gen_and_expand(party, chan, expander, material, prg=PRG_CHACHA8, batched=True):
    """One party's online expansion; returns device buffers (x, z) of N words.

    `expander` is this party's pcg_b200.Expander for (N, c, t), w = 1 (its
    resident a_i images serve step 4).  batched=True evaluates the c*c
    blocks' t*t keys as one batch of c*c*t*t instances -- levels + 2 message
    exchanges in all -- where the reference runs block by block
    (c*c*(levels + 2) exchanges; batched=False does the same).  Both parties
    must use the same mode.  The output layers stay on the device."""
    e = expander
    N, c, t = e.N, e.c, e.t
    B, n = t * t, e.levels
    D = 1 << n
    m = material
    d_g = DeviceBuffer(8 * c * c * N)
    groups = [list(range(c * c))] if batched else [[blk] for blk in range(c * c)]
    for blocks in groups:
        nb = len(blocks)
        roots = np.ascontiguousarray(np.concatenate([m.roots[b] for b in blocks]))
        dlt = np.ascontiguousarray(np.concatenate([m.dltsft[b] for b in blocks]))
        d_leaves = dpf_gpu_batch_full_eval_device(nb * B, n, 1, roots, dlt, party=party,
                                                  exchange=chan.exchange, prg=prg)
        sumC, sumT = dpf_out_sums(d_leaves, nb * B, D)
        cat = lambda a: np.concatenate([a[b] for b in blocks])
        CW = _beaver_cw(party, chan, sumC, sumT, cat(m.beta), cat(m.r), cat(m.s), cat(m.rs))
        d_cw = to_device(CW)
        for k, blk in enumerate(blocks):
            dpf_out_scatter_g_device(d_leaves + 16 * k * B * D, B, D, t, party,
                                     d_cw.ptr + 8 * k * B, d_g.ptr + 8 * blk * N, N)
        synchronize()   # d_leaves is valid until the next DPF call
    d_pos, d_val = to_device(m.pos), to_device(m.val)
    d_x, d_z = DeviceBuffer(8 * N), DeviceBuffer(8 * N)
    e.expand_from_g_device(d_g.ptr, d_pos.ptr, d_val.ptr, d_x.ptr, d_z.ptr)
    return d_x, d_z
