"""Serving loop: continuous batching of mixed-shape expansion requests.

Each result must be the same alone and in the mix (digests of x and z are
exact integer fingerprints), and equal to a direct expansion of the same
request through the expander API."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
A_SEED = 7


def direct_digests(pcg, N, c, t, seed, party):
    a = pcg.public_a(N, c, A_SEED)
    e = pcg.Expander(N, c, t, 1, pcg.PRG_CHACHA8, public_a=a)
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
    out = pcg.digest_device(x.ptr, N), pcg.digest_device(z.ptr, N)
    e.close()
    return out


def test_served_request_equals_direct_expansion(pcg):
    srv = pcg.Server(n_streams=2, a_seed=A_SEED)
    for (N, c, t, seed, party) in [(1 << 14, 2, 8, 11, 0), (1 << 12, 4, 16, 12, 1)]:
        res = srv.wait(srv.submit(N, c, t, seed, party), timeout_ms=60000)
        assert res.status == 0
        assert (res.digest_x, res.digest_z) == direct_digests(pcg, N, c, t, seed, party)
    srv.close()


def mixed_trace(n, seed, rate):
    rng = np.random.default_rng(seed)
    shapes = [(1 << lg, c, t) for lg in (12, 14, 16, 18) for c in (2, 4) for t in (8, 16, 32)
              if (1 << lg) // t >= 4]
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n))
    out = []
    for i in range(n):
        N, c, t = shapes[rng.integers(len(shapes))]
        out.append((N, c, t, int(rng.integers(2)), int(rng.integers(1, 2**62)), float(arrivals[i])))
    return out


def test_results_are_the_same_alone_and_in_the_mix(pcg):
    trace = mixed_trace(48, 5, rate=400.0)
    mix = pcg.Server(n_streams=4, a_seed=A_SEED)
    got = mix.run_trace(trace, timeout_s=300)
    # Overlap actually happened: some request started before an earlier one finished.
    overlap = any(got[i].start_s < got[j].done_s for j in range(len(got))
                  for i in range(j + 1, len(got)))
    mix.close()
    alone = pcg.Server(n_streams=1, max_in_flight=1, a_seed=A_SEED)
    ref = [alone.wait(alone.submit(N, c, t, seed, party)) for (N, c, t, party, seed, _) in trace]
    alone.close()
    for a, b in zip(got, ref):
        assert a.status == 0 and b.status == 0
        assert (a.digest_x, a.digest_z) == (b.digest_x, b.digest_z)
    assert overlap


def test_small_memory_budget_still_serves_everything(pcg):
    srv = pcg.Server(n_streams=4, mem_budget=1, a_seed=A_SEED)  # admits one at a time
    tickets = [srv.submit(1 << 12, 2, 8, s, s & 1) for s in range(6)]
    res = [srv.wait(tk, timeout_ms=60000) for tk in tickets]
    assert all(r.status == 0 for r in res)
    # With the budget exceeded by any second request, runs never overlap.
    for a, b in zip(res, res[1:]):
        assert b.start_s >= a.done_s - 1e-6
    srv.close()


def test_failures_are_reported_on_the_host(pcg):
    srv = pcg.Server(n_streams=1, max_in_flight=1, a_seed=A_SEED)
    with pytest.raises(pcg.PcgError) as e:
        srv.submit(1000, 2, 8, 1)            # N not a power of two
    assert e.value.code == -1
    with pytest.raises(pcg.PcgError):
        srv.wait(123456789, timeout_ms=10)   # unknown ticket
    srv.prepare(1 << 20, 4, 16)
    tks = [srv.submit(1 << 20, 4, 16, s) for s in range(3)]
    with pytest.raises(pcg.PcgError) as e:
        srv.wait(tks[-1], timeout_ms=0)      # queued behind two full expansions
    assert e.value.code == -6
    assert srv.wait(tks[0], timeout_ms=60000).status == 0
    srv.close(timeout_ms=60000)               # cancels or drains the rest


def test_large_requests_run_one_at_a_time_and_small_ones_pass(pcg):
    """Two large requests (c^2 N > 2^20) never overlap; a small one submitted
    after both starts while the first large one is still running."""
    srv = pcg.Server(n_streams=4, a_seed=A_SEED)
    big, small = (1 << 18, 4, 16), (1 << 12, 2, 8)
    srv.prepare(*big)
    srv.prepare(*small)
    t_big = [srv.submit(*big, s) for s in (1, 2)]
    t_small = srv.submit(*small, 3)
    rb = [srv.wait(t, timeout_ms=60000) for t in t_big]
    rs = srv.wait(t_small, timeout_ms=60000)
    assert all(r.status == 0 for r in rb + [rs])
    assert rb[1].start_s >= rb[0].done_s - 1e-6
    assert rs.start_s < rb[0].done_s
    srv.close()


def test_queued_small_requests_run_as_batches(pcg):
    """Small requests of mixed shapes (N in 2^14 .. 2^18) queued together run
    as batches: the same digests as one at a time, in far fewer launches."""
    shapes = [(1 << 14, 2, 8), (1 << 16, 4, 16), (1 << 14, 4, 32), (1 << 18, 2, 8),
              (1 << 16, 2, 32), (1 << 14, 2, 16)]
    trace = [(*shapes[i % len(shapes)], i & 1, 700 + i, 0.0) for i in range(24)]
    runs = {}
    for name, kw in (("batched", dict(n_streams=1, max_in_flight=32)),
                     ("alone", dict(n_streams=1, max_in_flight=1))):
        srv = pcg.Server(a_seed=A_SEED, **kw)
        for shp in shapes:
            srv.prepare(*shp)
        srv.run_trace(trace[:6])          # warm: plans, pool
        before = pcg.launch_count()
        res = srv.run_trace(trace, timeout_s=300)
        runs[name] = ([(r.digest_x, r.digest_z) for r in res], pcg.launch_count() - before)
        assert all(r.status == 0 for r in res)
        srv.close()
    assert runs["batched"][0] == runs["alone"][0]
    assert runs["batched"][1] * 2 < runs["alone"][1]
