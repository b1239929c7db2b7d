"""CUDA-graph replay of the expansion and the leaf-kernel autotuner: both
must leave every output bit-identical to direct launches (and to the
oracle), and graph replays must still be counted as kernel launches."""
import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu


def _material(pcg, N, c, t, seed):
    s = O.shape(N, c, t)
    a = O.public_a(s, 7)
    e = pcg.Expander(N, c, t, 1, pcg.PRG_CHACHA8, public_a=a)
    K, L = e.K, e.levels
    d = {k: pcg.DeviceBuffer(n) for k, n in
         (("r0", 16 * K), ("r1", 16 * K), ("cws", 16 * K * L * e.nk), ("cwo", 8 * K))}
    e.deal_keys_device(seed, d["r0"].ptr, d["r1"].ptr, d["cws"].ptr, d["cwo"].ptr)
    pos, val = pcg.noise(N, c, t, seed, 0)
    d["pos"], d["val"] = pcg.to_device(pos), pcg.to_device(val)
    return s, a, e, d, (pos, val)


def _expand(pcg, e, d, x, z):
    e.expand_device(0, d["r0"].ptr, d["cws"].ptr, d["cwo"].ptr, d["pos"].ptr, d["val"].ptr,
                    x.ptr, z.ptr)
    pcg.synchronize()
    N = e.N
    return x.download(np.uint64, N), z.download(np.uint64, N)


@pytest.mark.parametrize("N,c,t", [(1 << 12, 2, 4), (1 << 16, 4, 16)])
def test_graph_replay_is_bit_exact_and_counted(pcg, N, c, t):
    s, a, e, d, noise = _material(pcg, N, c, t, 4242)
    x0, z0 = pcg.DeviceBuffer(8 * N), pcg.DeviceBuffer(8 * N)
    want = _expand(pcg, e, d, x0, z0)
    if N == 1 << 12:   # small enough for the oracle: pins the direct path too
        r0 = d["r0"].download(np.uint64, 2 * e.K).reshape(e.K, 2)
        cws = d["cws"].download(np.uint64, 2 * e.K * e.levels).reshape(-1, 2)
        cwo = d["cwo"].download(np.uint64, e.K)
        wx, wz = O.expand(s, 0, r0, cws, cwo, *noise, a, None)
        assert (want[0] == wx).all() and (want[1] == wz).all()
    e.set_graph(True)
    x1, z1 = pcg.DeviceBuffer(8 * N), pcg.DeviceBuffer(8 * N)
    per_call = []
    for _ in range(4):       # direct (warm), capture, replay, replay
        before = pcg.launch_count()
        got = _expand(pcg, e, d, x1, z1)
        per_call.append(pcg.launch_count() - before)
        assert (got[0] == want[0]).all() and (got[1] == want[1]).all()
    assert per_call[0] == per_call[1] == per_call[2] == per_call[3] > 0, per_call
    # New output buffers: re-capture and update the executable graph.
    x2, z2 = pcg.DeviceBuffer(8 * N), pcg.DeviceBuffer(8 * N)
    for _ in range(2):
        got = _expand(pcg, e, d, x2, z2)
        assert (got[0] == want[0]).all() and (got[1] == want[1]).all()
    e.set_graph(False)
    got = _expand(pcg, e, d, x1, z1)
    assert (got[0] == want[0]).all() and (got[1] == want[1]).all()
    e.close()


@pytest.mark.parametrize("N,c,t", [(1 << 14, 2, 8), (1 << 16, 2, 8), (1 << 18, 4, 16)])
def test_autotune_keeps_outputs(pcg, N, c, t):
    _, _, e, d, _ = _material(pcg, N, c, t, 99)
    x, z = pcg.DeviceBuffer(8 * N), pcg.DeviceBuffer(8 * N)
    want = _expand(pcg, e, d, x, z)
    tpb = e.autotune()
    assert tpb in (32, 64, 128, 256)
    assert e.autotune() == tpb          # cached per shape
    got = _expand(pcg, e, d, x, z)
    assert (got[0] == want[0]).all() and (got[1] == want[1]).all()
    e.close()


def test_async_host_expansions_match_sync(pcg):
    """pcgb_expand_host_async over alternating parties and buffer sets equals
    pcgb_expand_host, call for call."""
    N, c, t = 1 << 14, 2, 8
    s = O.shape(N, c, t)
    a = O.public_a(s, 7)
    e = pcg.Expander(N, c, t, 1, pcg.PRG_CHACHA8, public_a=a)
    r0, r1, cws, cwo = O.deal_keys(s, 1234)
    noise = [O.noise(s, 1234, p) for p in (0, 1)]
    want = [e.expand_host(p, (r0, r1)[p], cws, cwo, *noise[p]) for p in (0, 1)]
    bufs = []
    for k in range(6):
        p = k % 2
        ins = [np.ascontiguousarray(v, np.uint64) for v in ((r0, r1)[p], cws, cwo, *noise[p])]
        outs = [np.zeros(N, np.uint64), np.zeros(N, np.uint64)]
        bufs.append((p, ins, outs))
        rc = pcg.lib.pcgb_expand_host_async(e.h, p, *[v.ctypes.data for v in ins + outs])
        assert rc == 0, pcg.lib.pcgb_last_error()
    assert pcg.lib.pcgb_expander_wait(e.h) == 0
    for p, _, (x, z) in bufs:
        assert (x == want[p][0]).all() and (z == want[p][1]).all()
    e.close()


def test_pinned_leaf_shape_keeps_outputs(pcg):
    """pcgb_expander_set_leaf_shape: every candidate shape gives the same x, z;
    shapes outside the candidates are refused; a captured graph is dropped
    and re-captured with the new shape."""
    N, c, t = 1 << 14, 2, 8
    _, _, e, d, _ = _material(pcg, N, c, t, 321)
    x, z = pcg.DeviceBuffer(8 * N), pcg.DeviceBuffer(8 * N)
    want = _expand(pcg, e, d, x, z)
    e.set_graph(True)
    for tpb, lpt in ((128, 16), (64, 8), (32, 4), (256, 4)):
        e.set_leaf_shape(tpb, lpt)
        assert e.leaf_shape() == (tpb, lpt)
        for _ in range(2):
            got = _expand(pcg, e, d, x, z)
            assert (got[0] == want[0]).all() and (got[1] == want[1]).all(), (tpb, lpt)
    for tpb, lpt in ((96, 16), (128, 2), (128, 32), (256, 16)):
        with pytest.raises(pcg.PcgError):
            e.set_leaf_shape(tpb, lpt)
    assert e.leaf_shape() == (256, 4)
    e.close()
