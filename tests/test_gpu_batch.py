"""Expansions of different (N, c, t) as one batch (pcgb_expand_batch_device):
one launch per stage for the whole batch, each request's x and z bit-exact
against its own pcgb_expand_device call, and one request against the oracle."""
import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu

SHAPES = [(1 << 14, 2, 8), (1 << 16, 4, 16), (1 << 14, 4, 32), (1 << 18, 2, 8),
          (1 << 16, 2, 32), (1 << 20, 4, 16), (1 << 14, 2, 8)]


def _request(pcg, e, seed, party):
    K, L, nk = e.K, e.levels, e.nk
    d_r0, d_r1 = pcg.DeviceBuffer(16 * K), pcg.DeviceBuffer(16 * K)
    d_cws, d_cwo = pcg.DeviceBuffer(16 * K * L * nk), pcg.DeviceBuffer(8 * K)
    e.deal_keys_device(seed, d_r0.ptr, d_r1.ptr, d_cws.ptr, d_cwo.ptr)
    pos, val = pcg.noise(e.N, e.c, e.t, seed, party)
    d_pos, d_val = pcg.to_device(pos), pcg.to_device(val)
    d_x, d_z = pcg.DeviceBuffer(8 * e.N), pcg.DeviceBuffer(8 * e.N)
    roots = d_r1 if party else d_r0
    keep = (d_r0, d_r1, d_cws, d_cwo, d_pos, d_val, d_x, d_z)
    return (e, party, roots.ptr, d_cws.ptr, d_cwo.ptr, d_pos.ptr, d_val.ptr, d_x.ptr,
            d_z.ptr), keep


@pytest.fixture(scope="module")
def expanders(pcg):
    es = []
    for N, c, t in SHAPES:
        e = pcg.Expander(N, c, t, 1, pcg.PRG_CHACHA8, public_a=pcg.public_a(N, c, 7))
        e.set_leaf_shape(64, 8)
        es.append(e)
    yield es
    for e in es:
        e.close()


def test_batch_equals_single_expansions(pcg, expanders):
    reqs, keep = [], []
    for i, e in enumerate(expanders):
        r, k = _request(pcg, e, 100 + i, i % 2)
        reqs.append(r)
        keep.append(k)
    # One request at a time.
    want = []
    before = pcg.launch_count()
    for (e, party, *ptrs), k in zip(reqs, keep):
        e.expand_device(party, *ptrs)
        pcg.synchronize()
        want.append((k[6].download(np.uint64, e.N), k[7].download(np.uint64, e.N)))
    single_launches = pcg.launch_count() - before
    for k in keep:   # poison the outputs: the batch must write every word
        pcg.lib.pcgb_memset(k[6].ptr, 0xA5, k[6].nbytes, None)
        pcg.lib.pcgb_memset(k[7].ptr, 0xA5, k[7].nbytes, None)
    before = pcg.launch_count()
    pcg.expand_batch_device(reqs)
    pcg.synchronize()
    batch_launches = pcg.launch_count() - before
    for (e, *_), k, (wx, wz) in zip(reqs, keep, want):
        assert (k[6].download(np.uint64, e.N) == wx).all(), (e.N, e.c, e.t)
        assert (k[7].download(np.uint64, e.N) == wz).all(), (e.N, e.c, e.t)
    # Top walk (one launch per stage and walk depth), leaf, x, three NTT
    # passes, against eight launches per request one at a time.
    assert batch_launches <= single_launches // 2


def test_batch_request_matches_oracle(pcg, expanders):
    """The first request of a batch (N = 2^14, c = 2, t = 8) against the
    oracle's expansion on the same keys and noise, both parties."""
    e = expanders[0]
    s = O.shape(e.N, e.c, e.t)
    r0, r1, cws, cwo = O.deal_keys(s, 4242)
    a = O.public_a(s, 7)
    for party, roots in ((0, r0), (1, r1)):
        pos, val = O.noise(s, 4242, party)
        d = [pcg.to_device(np.ascontiguousarray(v)) for v in (roots, cws, cwo, pos, val)]
        d_x, d_z = pcg.DeviceBuffer(8 * e.N), pcg.DeviceBuffer(8 * e.N)
        other, keep = _request(pcg, expanders[1], 7, 0)
        pcg.expand_batch_device([(e, party, *[b.ptr for b in d], d_x.ptr, d_z.ptr), other])
        pcg.synchronize()
        wx, wz = O.expand(s, party, roots, cws, cwo, pos, val, a)
        assert (d_x.download(np.uint64, e.N) == wx).all()
        assert (d_z.download(np.uint64, e.N) == wz).all()


def test_batch_rejects_mismatched_requests(pcg, expanders):
    e0 = expanders[0]
    r0, k0 = _request(pcg, e0, 1, 0)
    odd = pcg.Expander(1 << 14, 2, 8, 1, pcg.PRG_CHACHA8, public_a=pcg.public_a(1 << 14, 2, 7))
    odd.set_leaf_shape(64, 4)
    r1, k1 = _request(pcg, odd, 2, 0)
    with pytest.raises(pcg.PcgError, match="same w and leaf shape"):
        pcg.expand_batch_device([r0, r1])
    small = pcg.Expander(1 << 12, 2, 4, 1, pcg.PRG_CHACHA8, public_a=pcg.public_a(1 << 12, 2, 7))
    small.set_leaf_shape(64, 8)
    r2, k2 = _request(pcg, small, 3, 0)
    with pytest.raises(pcg.PcgError, match="2\\^14 .. 2\\^20"):
        pcg.expand_batch_device([r0, r2])
    odd.close()
    small.close()
