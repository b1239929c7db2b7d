"""Bit-exactness against the reference's own GPU kernels
(GPU_baseline/common/*.cu compiled unmodified into oracle/_ref)."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O
from gpu_helpers import dealt_keys, dev, ref_exchange_fn

pytestmark = pytest.mark.gpu
P = O.P


@pytest.fixture(scope="module")
def ref():
    R = O.ref_gpu()
    if R is None:
        pytest.skip("oracle/_ref/libref_gpu.so not built")
    return R


CASES = [(prg, n, w, 16) for prg in (O.PRG_CHACHA8, O.PRG_AES) for n, w in
         ((12, 1), (12, 2), (12, 4))]
# Levels of 4096+ parents: the AES level kernel stages the per-lane
# replicated T-table and walks 8 parents per thread (grid-stride).
CASES += [(O.PRG_AES, 14, 1, 5), (O.PRG_AES, 14, 2, 3), (O.PRG_AES, 16, 4, 2),
          (O.PRG_AES, 16, 1, 3)]


@pytest.mark.parametrize("prg,n,w,B", CASES)
def test_interactive_leaves_match_reference_kernels(pcg, ref, prg, n, w, B):
    rng = np.random.default_rng(n + 10 * w + prg)
    nk = (1 << w) - 1
    rks = O.aes_tree_round_keys(rng.integers(0, 256, 16, dtype=np.uint8), nk) \
        if prg == O.PRG_AES else None
    roots = rng.integers(0, 2**64 - 1, (B, 2), dtype=np.uint64)
    dlt = rng.integers(0, 2**64 - 1, (B * (n // w) * nk, 2), dtype=np.uint64)
    want = np.zeros((B << n, 2), np.uint64)
    rc = ref.ref_dpf_batch_full_eval(B, n, w, roots.ctypes.data, dlt.ctypes.data,
                                     None if rks is None else rks.ctypes.data, 0, None, None,
                                     want.ctypes.data, 1 if prg == O.PRG_CHACHA8 else 0)
    assert rc == 0, ref.ref_last_error()
    got = pcg.dpf_gpu_batch_full_eval(B, n, w, roots, dlt, round_keys=rks, prg=prg)
    assert (got == want).all()


def test_convert_matches_reference_kernels(pcg, ref):
    rng = np.random.default_rng(4)
    t, n = 4, 11
    B, D = t * t, 1 << n
    leaves = rng.integers(0, 2**64 - 1, (B * D, 2), dtype=np.uint64)
    CW = rng.integers(0, P, B, dtype=np.uint64)
    N = t * (D // 2)
    d = dev(pcg, leaves)
    sc, st = pcg.dpf_out_sums(d.ptr, B, D)
    rc_, rt_ = np.zeros(B, np.uint64), np.zeros(B, np.uint64)
    assert ref.ref_dpf_out_sums(d.ptr, B, D, P, rc_, rt_) == 0
    assert (sc == rc_).all() and (st == rt_).all()
    for party in (0, 1):
        g = pcg.dpf_out_scatter_g(d.ptr, B, D, t, party, CW, N)
        rg = np.zeros(N, np.uint64)
        assert ref.ref_dpf_out_scatter_g(d.ptr, B, D, t, party, P, CW, rg, N) == 0
        assert (g == rg).all()


def test_poly_mul_v1_matches_reference_kernels(pcg, ref):
    for N in (128, 4096, 32768):
        r = O.mt64(N, 4 * N)
        a, b = r[: 2 * N] % np.uint64(P), r[2 * N:] % np.uint64(P)
        want = np.zeros(2 * N, np.uint64)
        ms = C.c_double()
        assert ref.ref_poly_mul_u64(want, a, b, 2, N, P, C.byref(ms)) == 0
        got, _ = pcg.poly_mul_u64(a, b, 2, N)
        assert (got == want).all()


def test_keyed_g_matches_reference_pipeline(pcg, ref):
    """One expansion block through the reference's interactive kernels driven
    by an exchange that supplies peer = my ^ CW (keyed evaluation), then its
    dpf_out_scatter_g, versus the fused kernel's g' for a diagonal pair."""
    N, c, t = 1 << 14, 2, 8
    s = O.shape(N, c, t)
    r0, r1, cws, cwo = O.deal_keys(s, 555)
    a = O.public_a(s, 3)
    e = pcg.Expander(N, c, t, 1, pcg.PRG_CHACHA8, public_a=a)
    B, n, L = t * t, s.n, s.levels
    D = 1 << n
    d_cws, d_cwo = dev(pcg, cws), dev(pcg, cwo)
    for party, roots in ((0, r0), (1, r1)):
        d_g = pcg.DeviceBuffer(8 * N * e.Q)
        e.expand_g_device(party, dev(pcg, roots).ptr, d_cws.ptr, d_cwo.ptr, d_g.ptr)
        got = d_g.download(np.uint64, N * e.Q).reshape(e.Q, N)
        blk = 0  # block (0, 0) -> pair q = 0
        cw = cws[blk * B * L:(blk + 1) * B * L].reshape(B, L, 2)
        level = [0]

        def ex(my, peer, count, user):
            m = np.ctypeslib.as_array(C.cast(my, C.POINTER(C.c_uint64)), shape=(count, 2))
            p = np.ctypeslib.as_array(C.cast(peer, C.POINTER(C.c_uint64)), shape=(count, 2))
            p[:] = m ^ cw[:, level[0]]
            level[0] += 1

        cb = ref_exchange_fn()(ex)
        dl = C.c_void_p()
        rts = np.ascontiguousarray(roots[blk * B:(blk + 1) * B])
        dz = np.zeros((B * L, 2), np.uint64)
        assert ref.ref_dpf_batch_full_eval_device(B, n, 1, rts.ctypes.data, dz.ctypes.data, None,
                                                  party, C.cast(cb, C.c_void_p), None, 1,
                                                  C.byref(dl)) == 0
        # The reference sizes its CW buffer in dpf_out_sums
        # (leaf_convert_cuda.cu:350), so the pipeline calls it first.
        sc, st = np.zeros(B, np.uint64), np.zeros(B, np.uint64)
        assert ref.ref_dpf_out_sums(dl.value, B, D, P, sc, st) == 0
        g = np.zeros(N, np.uint64)
        cwb = np.ascontiguousarray(cwo[blk * B:(blk + 1) * B])
        assert ref.ref_dpf_out_scatter_g(dl.value, B, D, t, party, P, cwb, g, N) == 0, \
            ref.ref_last_error()
        assert (got[0] == g).all()
    e.close()
