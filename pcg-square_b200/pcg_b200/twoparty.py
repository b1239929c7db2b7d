"""Interactive two-party PCG-OLE expansion over the drop-in entry points.

The online part of the reference's device path, PCG_OLE::gen_and_expand
(CPU_baseline/pcg_ole_2pc/pcg_ole_impl.h:213-312, then step 4 at :453-484),
run by each party in its own process:

  for every block (i, j):
    leaves = dpf_gpu_batch_full_eval_device(...)   one CW exchange per level
    sumC, sumT = dpf_out_sums(leaves)              (one call, pcgb_dpf_batch_full_
                                                    eval_convert_device: the last
                                                    level keeps C | tau<<63 per
                                                    leaf, no leaves stored)
    <A> = (-1)^party sumT, <B> = (-1)^(1-party) sumC + <beta>
    open d = A - r, e = B - s                      Beaver triple (r, s, rs), on
    <CW> = d<s> + e<r> + <rs> (+ d e for party 0);  the device; open CW
    g_ij = dpf_out_scatter_g(leaves, ..., CW)      (from the kept words)
  x, z = step 4 over the g_ij (pcgb_expand_from_g_device)

By default all c*c blocks run as one batch (see gen_and_expand), which
leaves levels + 2 message exchanges per expansion instead of c*c*(levels+2).

The boolean part of the reference's preprocessing (pcg_ole_impl.h:118-199:
Kogge-Stone position add, then the DltSft circuit) runs on the GPU by
two-party GMW (`preprocess`, over pcgb_gmw_*), given AND triples.  What the
reference draws from OT -- the AND triples, beta shares (Gilboa) and the F_p
Beaver triples -- is an input (`PartyMaterial`, `bool_triples_dealer`); the
OT layer itself is outside this library.  Messages travel over a
`Channel`: party 0 sends first and party 1 receives first, as the
reference's NetIO exchange does.  With
torch.distributed the two parties may share one GPU: they exchange through
the host between kernels and no kernel waits on the other party.
"""
from dataclasses import dataclass

import numpy as np

from . import (DeviceBuffer, PRG_CHACHA8, add_mod_p_device,
               dpf_gpu_batch_full_eval_convert_device,
               dpf_gpu_batch_full_eval_convert_device_dx, dpf_out_scatter_g_conv_device, gmw_dltsft,
               gmw_position_add, out_beaver_close_device, out_beaver_open_device, synchronize,
               to_device)

# The public block W both parties add to their Delta share to form the DPF
# root (HalfTreeDPF::setup_params, dpf.cpp:289-296, draws it from a PRG with
# a fixed seed): any constant known to both parties serves.  Hex digits of pi.
PUBLIC_W = np.array([0x243F6A8885A308D3, 0x13198A2E03707344], np.uint64)


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


# Device scratch reused across calls in this process (the converted leaf
# words alone are 8 bytes per leaf: 4.3 GB at N = 2^20, c = 4, t = 16).
_scratch = {}


def release_scratch():
    """Free the device scratch gen_and_expand keeps between calls."""
    for b in _scratch.values():
        b.free()
    _scratch.clear()


def _scratch_buf(name, nbytes):
    b = _scratch.get(name)
    if b is None or b.nbytes < nbytes:
        if b is not None:
            b.free()
        b = _scratch[name] = DeviceBuffer(nbytes)
    return b


def device_words(ptr, nwords):
    """A torch int64 view (no copy) of nwords device words at ptr."""
    import torch

    class _Cai:
        __cuda_array_interface__ = {"shape": (nwords,), "typestr": "<i8", "data": (ptr, False),
                                    "version": 3}
    return torch.as_tensor(_Cai(), device="cuda")


class DeviceChannel(Channel):
    """Exchange that keeps the messages in device memory: gen_and_expand
    hands it the per-level CW shares and the Beaver openings as device
    pointers (pcgb_dpf_batch_full_eval_convert_device_dx), so they never
    visit the host.  Over NCCL (one GPU per party) the words go device to
    device.  Backends without device send/recv (gloo) stage each message
    through host memory (`stage`, default: on unless the backend is NCCL);
    that is how two processes sharing one GPU run this same code path.
    `exchange` (host arrays in and out) serves the callers that work on
    host arrays, the GMW circuits of `preprocess`."""

    def __init__(self, party, peer_rank=None, stage=None):
        super().__init__(party, peer_rank)
        self.stage = (self.dist.get_backend() != "nccl") if stage is None else stage

    def exchange_device(self, d_my, d_peer, nwords):
        my, peer = device_words(d_my, nwords), device_words(d_peer, nwords)
        if self.stage:
            self.torch.cuda.current_stream().synchronize()
            t_my, t_peer = my.cpu(), self.torch.empty(nwords, dtype=self.torch.int64)
        else:
            t_my, t_peer = my, peer
        if self.party == 0:
            self.dist.send(t_my, self.peer)
            self.dist.recv(t_peer, self.peer)
        else:
            self.dist.recv(t_peer, self.peer)
            self.dist.send(t_my, self.peer)
        if self.stage:
            peer.copy_(t_peer)
        self.torch.cuda.current_stream().synchronize()
        self.messages += 1
        self.bytes += 8 * nwords

    def exchange(self, mine):
        mine = np.ascontiguousarray(mine, np.uint64)
        t_my = self.torch.from_numpy(mine.view(np.int64).copy()).cuda()
        t_peer = self.torch.empty_like(t_my)
        self.exchange_device(t_my.data_ptr(), t_peer.data_ptr(), t_my.numel())
        return t_peer.cpu().numpy().view(np.uint64).reshape(mine.shape)


def _beaver_cw_device(party, chan, nB, d_sumC, d_sumT, beta, r, s, rs, d_cw):
    """Output-layer correction words of nB instances into d_cw (a
    DeviceBuffer of nB words): <A> =
    (-1)^party sumT, <B> = (-1)^(1-party) sumC + <beta>, CW = A*B by one
    Beaver triple per instance (two opens; pcg_ole_impl.h:222-290).  The
    arithmetic runs on the device; only the 2nB + nB words of the two
    openings cross to the host for the exchange."""
    w = 8 * nB
    d_in = _scratch_buf("beaver_in", 4 * w)          # beta | r | s | rs
    for k, a in enumerate((beta, r, s, rs)):
        d_in.upload_at(np.ascontiguousarray(a, np.uint64), k * w)
    d_beta, d_r, d_s, d_rs = (d_in.ptr + k * w for k in range(4))
    d_de = _scratch_buf("beaver_de", 4 * w)          # mine (2nB) | peer (2nB)
    out_beaver_open_device(nB, party, d_sumC, d_sumT, d_beta, d_r, d_s, d_de.ptr)
    d_peer = _scratch_buf("beaver_cw_peer", w)
    if hasattr(chan, "exchange_device"):       # openings stay on the device
        synchronize()
        chan.exchange_device(d_de.ptr, d_de.ptr + 2 * w, 2 * nB)
        out_beaver_close_device(nB, party, d_de.ptr, d_de.ptr + 2 * w, d_r, d_s, d_rs, d_cw.ptr)
        synchronize()
        chan.exchange_device(d_cw.ptr, d_peer.ptr, nB)
    else:
        peer = chan.exchange(d_de.download(np.uint64, 2 * nB))
        d_de.upload_at(peer, 2 * w)
        out_beaver_close_device(nB, party, d_de.ptr, d_de.ptr + 2 * w, d_r, d_s, d_rs, d_cw.ptr)
        d_peer.upload(chan.exchange(d_cw.download(np.uint64, nB)))
    add_mod_p_device(d_cw.ptr, d_cw.ptr, d_peer.ptr, nB)


def gen_and_expand(party, chan, expander, material, prg=PRG_CHACHA8, batched=True):
    """One party's online expansion; returns device buffers (x, z) of N words.

    `expander` is this party's pcg_b200.Expander for (N, c, t), w = 1 (its
    resident a_i images serve step 4).  batched=True evaluates the c*c
    blocks' t*t keys as one batch of c*c*t*t instances -- levels + 2 message
    exchanges in all -- where the reference runs block by block
    (c*c*(levels + 2) exchanges; batched=False does the same).  Both parties
    must use the same mode.  Everything but the messages stays on the
    device: the sums pass keeps each leaf's converted word, so the scatter
    after the Beaver opens hashes no leaf a second time."""
    e = expander
    N, c, t = e.N, e.c, e.t
    B, n = t * t, e.levels
    D = 1 << n
    m = material
    d_g = DeviceBuffer(8 * c * c * N)
    groups = [list(range(c * c))] if batched else [[blk] for blk in range(c * c)]
    for blocks in groups:
        nb = len(blocks)
        nB = nb * B
        roots = np.ascontiguousarray(np.concatenate([m.roots[b] for b in blocks]))
        dlt = np.ascontiguousarray(np.concatenate([m.dltsft[b] for b in blocks]))
        d_conv = _scratch_buf("conv", 8 * nB * D)
        d_sums = _scratch_buf("sums", 2 * 8 * nB)     # sumC | sumT
        d_sumC, d_sumT = d_sums.ptr, d_sums.ptr + 8 * nB
        d_cw = _scratch_buf("cw", 8 * nB)
        # DPF levels with their CW exchanges, the last level fused with the
        # sums pass (leaves hashed as they are made, never stored).
        if hasattr(chan, "exchange_device"):
            dpf_gpu_batch_full_eval_convert_device_dx(
                nB, n, 1, roots, dlt, d_conv.ptr, d_sumC, d_sumT,
                lambda d_my, d_peer, count: chan.exchange_device(d_my, d_peer, 2 * count),
                party=party, prg=prg)
        else:
            dpf_gpu_batch_full_eval_convert_device(nB, n, 1, roots, dlt, d_conv.ptr, d_sumC,
                                                   d_sumT, party=party, exchange=chan.exchange,
                                                   prg=prg)
        cat = lambda a: np.concatenate([a[b] for b in blocks])
        _beaver_cw_device(party, chan, nB, d_sumC, d_sumT, cat(m.beta), cat(m.r), cat(m.s),
                          cat(m.rs), d_cw)
        for k, blk in enumerate(blocks):
            dpf_out_scatter_g_conv_device(d_conv.ptr + 8 * k * B * D, B, D, t, party,
                                          d_cw.ptr + 8 * k * B, d_g.ptr + 8 * blk * N, N)
        synchronize()
    d_pos, d_val = to_device(m.pos), to_device(m.val)
    d_x, d_z = DeviceBuffer(8 * N), DeviceBuffer(8 * N)
    e.expand_from_g_device(d_g.ptr, d_pos.ptr, d_val.ptr, d_x.ptr, d_z.ptr)
    return d_x, d_z


def bool_triples_dealer(rows, B, rng):
    """Both parties' shares of `rows` bit-sliced AND triples for B instances,
    ((a0, b0, c0), (a1, b1, c1)) with (a0^a1) & (b0^b1) == c0^c1 -- a trusted
    dealer standing in for the reference's OT-based TripleGen in tests and
    benchmarks (whoever runs it sees both shares)."""
    W = (B + 31) // 32
    a0, a1, b0, b1, c0 = (rng.integers(0, 1 << 32, rows * W, dtype=np.uint32) for _ in range(5))
    return (a0, b0, c0), (a1, b1, ((a0 ^ a1) & (b0 ^ b1)) ^ c0)


def instance_offsets(party, N, c, t, pos):
    """This party's private adder input for every instance of the c*c blocks
    (block (i, j) = i*c + j, instance k*t + l): the in-bin offset of its noise
    position i*t + k (party 0) or j*t + l (party 1) (pcg_ole_impl.h:132-139)."""
    bin_ = N // t
    pos = np.asarray(pos, np.uint64)
    blk = np.arange(c * c)[:, None]
    idx = np.arange(t * t)[None, :]
    sel = (blk // c) * t + idx // t if party == 0 else (blk % c) * t + idx % t
    return (pos[sel] % np.uint64(bin_)).reshape(-1)


def preprocess_gates(N, c, t):
    """AND-triple rows the two circuits of `preprocess` consume:
    (position adder, DltSft), each for c*c*t*t instances."""
    from . import gmw_dltsft_gates, gmw_position_add_gates
    bin_ = N // t
    off_bits = max(1, bin_.bit_length() - 1)
    return gmw_position_add_gates(off_bits), gmw_dltsft_gates(off_bits + 1, 1)


def preprocess(party, chan, N, c, t, pos, delta_share, adder_triples, dltsft_triples):
    """Boolean preprocessing of one expansion, all c*c blocks in one circuit
    each (the reference runs both circuits per block, pcg_ole_impl.h:118-199):

      alpha = off0 + off1   Kogge-Stone adder, log2(bin) + 1 bits
      DltSft = [digit_i(alpha) == 0] * Delta   (w = 1)
      root = Delta share ^ PUBLIC_W

    delta_share: [c*c*t*t, 2] this party's random Delta shares.  Returns
    (roots, dltsft) in PartyMaterial's layout plus the forced Delta shares and
    the alpha shares.  Costs 1 + ceil(log2(off_bits)) + 1 exchanges."""
    bin_ = N // t
    off_bits = max(1, bin_.bit_length() - 1)
    n = off_bits + 1
    off = instance_offsets(party, N, c, t, pos)
    alpha = gmw_position_add(party, off, off_bits, adder_triples, chan.exchange)
    delta, dlt = gmw_dltsft(party, alpha, delta_share, n, 1, dltsft_triples, chan.exchange)
    roots = delta ^ PUBLIC_W[None, :]
    return (roots.reshape(c * c, t * t, 2), dlt.reshape(c * c, t * t * n, 2), delta, alpha)
