"""Batched DPF full-domain evaluation plus leaf convert at its full stated
shape: 4096 half-tree DPF keys x 2^16 leaves (w = 1), ChaCha8 and AES tree
PRGs, bit for bit against the reference's own GPU kernels
(GPU_baseline/common/dpf_gpu.cu:339-535 and leaf_convert_cuda.cu:245-308,
compiled unmodified into oracle/_ref/libref_gpu.so).

Keys are random roots and per-level correction words.  The reference entry
point is interactive: after each level it hands over its CW shares and takes
the peer's; the exchange here returns peer = my ^ CW, which makes the
interactive evaluation equal to the keyed one.  Checked:
  * every leaf (4 GiB) of the library's keyed evaluation and of its
    interactive drop-in against the reference's leaves, compared on the
    device;
  * every instance's sums (C mod p and T) of dpf_out_sums;
  * the whole scattered g of dpf_out_scatter_g at t = 64 (B = t^2, N = 2^21);
  * the fused last-level convert's sums against the reference's sums.
"""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O
from gpu_helpers import ref_exchange_fn

pytestmark = pytest.mark.gpu
P = O.P
B, n, w, t = 4096, 16, 1, 64
D, L, nk = 1 << n, n // w, (1 << w) - 1
N = t * D // 2


@pytest.fixture(scope="module")
def ref():
    R = O.ref_gpu()
    if R is None:
        pytest.skip("oracle/_ref/libref_gpu.so not built")
    return R


@pytest.mark.parametrize("prg", [O.PRG_CHACHA8, O.PRG_AES])
def test_config3_full_shape_matches_reference_kernels(pcg, ref, prg):
    torch = pytest.importorskip("torch")
    from pcg_b200.twoparty import device_words
    rng = np.random.default_rng(3 + prg)
    rks = O.aes_tree_round_keys(rng.integers(0, 256, 16, dtype=np.uint8), nk) \
        if prg == O.PRG_AES else None
    roots = rng.integers(0, 2**64 - 1, (B, 2), dtype=np.uint64, endpoint=True)
    cws = rng.integers(0, 2**64 - 1, (B * L * nk, 2), dtype=np.uint64, endpoint=True)
    cw_out = rng.integers(0, P, B, dtype=np.uint64)
    cw = cws.reshape(B, L, nk, 2)
    zeros = np.zeros((B * L * nk, 2), np.uint64)
    words = 2 * B * D

    # Reference: interactive kernels, then its sums and scatter.
    level = [0]

    def ex(my, peer, count, user):
        m = np.ctypeslib.as_array(C.cast(my, C.POINTER(C.c_uint64)), shape=(count, 2))
        p = np.ctypeslib.as_array(C.cast(peer, C.POINTER(C.c_uint64)), shape=(count, 2))
        p[:] = m ^ cw[:, level[0]].reshape(-1, 2)
        level[0] += 1

    cb = ref_exchange_fn()(ex)
    dl = C.c_void_p()
    assert ref.ref_dpf_batch_full_eval_device(
        B, n, w, roots.ctypes.data, zeros.ctypes.data,
        None if rks is None else rks.ctypes.data, 0, C.cast(cb, C.c_void_p), None,
        1 if prg == O.PRG_CHACHA8 else 0, C.byref(dl)) == 0, ref.ref_last_error()
    assert level[0] == L
    rsc, rst = np.zeros(B, np.uint64), np.zeros(B, np.uint64)
    assert ref.ref_dpf_out_sums(dl.value, B, D, P, rsc, rst) == 0, ref.ref_last_error()
    rg = np.zeros(N, np.uint64)
    assert ref.ref_dpf_out_scatter_g(dl.value, B, D, t, 0, P, cw_out, rg, N) == 0, \
        ref.ref_last_error()
    ref.ref_sync()
    ref_leaves = device_words(dl.value, words)

    # Keyed evaluation (no exchange): every leaf, then the convert drop-ins.
    d_r, d_c = pcg.to_device(roots), pcg.to_device(cws)
    d_keyed = pcg.DeviceBuffer(8 * words)
    pcg.dpf_keyed_full_eval_device(B, n, w, prg, d_r.ptr, d_c.ptr, d_keyed.ptr, round_keys=rks)
    pcg.synchronize()
    assert torch.equal(device_words(d_keyed.ptr, words), ref_leaves)
    sc, st = pcg.dpf_out_sums(d_keyed.ptr, B, D)
    assert (sc == rsc).all() and (st == rst).all()
    g = pcg.dpf_out_scatter_g(d_keyed.ptr, B, D, t, 0, cw_out, N)
    assert (g == rg).all()
    d_keyed.free()

    # Interactive drop-in with the same exchange.
    lv = [0]

    def exchange(my):
        peer = my.reshape(B, nk, 2) ^ cw[:, lv[0]]
        lv[0] += 1
        return peer.reshape(-1, 2)

    d_drop = pcg.dpf_gpu_batch_full_eval_device(B, n, w, roots, zeros, round_keys=rks,
                                                exchange=exchange, prg=prg)
    pcg.synchronize()
    assert lv[0] == L
    assert torch.equal(device_words(d_drop, words), ref_leaves)
    sc2, st2 = pcg.dpf_out_sums(d_drop, B, D)
    assert (sc2 == rsc).all() and (st2 == rst).all()

    # Last level fused with the sums pass (no leaves stored).
    lv[0] = 0
    conv, sums = pcg.DeviceBuffer(8 * B * D), pcg.DeviceBuffer(16 * B)
    pcg.dpf_gpu_batch_full_eval_convert_device(B, n, w, roots, zeros, conv.ptr, sums.ptr,
                                               sums.ptr + 8 * B, round_keys=rks,
                                               exchange=exchange, prg=prg)
    s = sums.download(np.uint64, 2 * B)
    assert (s[:B] == rsc).all() and (s[B:] == rst).all()
