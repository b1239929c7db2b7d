"""The allocation-free sums entry point (pcgb_dpf_out_sums_noalloc) against
the allocating one (pcgb_dpf_out_sums), through the C ABI.

Some callers cannot allocate device memory — a framework's allocator owns
it, a fixed budget caps it, or a hot loop cannot afford cudaMalloc's
implicit synchronisation — so this variant keeps its scratch in a static
device array and writes into caller-provided device outputs.  The test runs
it twice in a row on different shapes (the second call must not see the
first call's leftovers in the shared array) and checks each result word for
word (these are exact integer sums) against the existing entry point.  It
is collected last so a failure here comes after every other test has run.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
P = 4611686018326724609


def _sums_noalloc(pcg, d_leaves, B, D):
    out_c, out_t = pcg.DeviceBuffer(8 * B), pcg.DeviceBuffer(8 * B)
    rc = pcg.lib.pcgb_dpf_out_sums_noalloc(d_leaves, B, D, P, out_c.ptr, out_t.ptr, None)
    assert rc == 0, pcg.lib.pcgb_last_error().decode()
    assert pcg.lib.pcgb_stream_synchronize(None) == 0
    return out_c.download(np.uint64, B), out_t.download(np.uint64, B)


def _sums_existing(pcg, d_leaves, B, D):
    sc, st = np.zeros(B, np.uint64), np.zeros(B, np.uint64)
    rc = pcg.lib.pcgb_dpf_out_sums(d_leaves, B, D, P, sc, st)
    assert rc == 0, pcg.lib.pcgb_last_error().decode()
    return sc, st


def test_noalloc_sums_match_existing_entry_point(pcg):
    rng = np.random.default_rng(2024)
    # Two calls in a row: a larger shape first, then a smaller, ragged one.
    for B, n in ((300, 12), (37, 9)):
        D = 1 << n
        leaves = rng.integers(0, 2**64 - 1, (B * D, 2), dtype=np.uint64)
        d = pcg.to_device(leaves)
        got_c, got_t = _sums_noalloc(pcg, d.ptr, B, D)
        want_c, want_t = _sums_existing(pcg, d.ptr, B, D)
        assert (got_c == want_c).all() and (got_t == want_t).all(), (B, n)


def test_noalloc_sums_with_fewer_partials_than_the_allocating_path(pcg):
    """B = 4096 instances of 2^16 leaves: the allocating path uses 32 partials
    per instance, more than the static array holds for this B (16 each), so
    the allocation-free call runs fewer CTAs with more leaves per thread.
    The 4 GiB of leaves come from the keyed evaluator on the device.  Then a
    small call again, which must not see the large call's partials."""
    rng = np.random.default_rng(77)
    for B, n in ((4096, 16), (5, 10)):
        D = 1 << n
        roots = rng.integers(0, 2**64 - 1, (B, 2), dtype=np.uint64, endpoint=True)
        cws = rng.integers(0, 2**64 - 1, (B * n, 2), dtype=np.uint64, endpoint=True)
        d_r, d_c = pcg.to_device(roots), pcg.to_device(cws)
        d_leaves = pcg.DeviceBuffer(16 * B * D)
        pcg.dpf_keyed_full_eval_device(B, n, 1, pcg.PRG_CHACHA8, d_r.ptr, d_c.ptr, d_leaves.ptr)
        pcg.synchronize()
        got_c, got_t = _sums_noalloc(pcg, d_leaves.ptr, B, D)
        want_c, want_t = _sums_existing(pcg, d_leaves.ptr, B, D)
        assert (got_c == want_c).all() and (got_t == want_t).all(), (B, n)
        d_leaves.free()


def test_noalloc_rejects_sizes_beyond_the_static_scratch(pcg):
    d = pcg.DeviceBuffer(16 * 64)
    out = pcg.DeviceBuffer(8)
    rc = pcg.lib.pcgb_dpf_out_sums_noalloc(d.ptr, 70000, 2, P, out.ptr, out.ptr, None)
    assert rc == -1
    assert "65535" in pcg.lib.pcgb_last_error().decode()
