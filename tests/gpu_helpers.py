"""Shared helpers for the GPU parity tests."""
import ctypes as C

import numpy as np

import oracle_lib as O

P = O.P


def dev(L, arr):
    return L.to_device(np.ascontiguousarray(arr))


def dealt_keys(n, w, K, seed, prg=O.PRG_CHACHA8, rks=None, with_dlt=False):
    """K random keyed instances dealt by the oracle: roots0/1, cws, cw_out, (dlt0, dlt1)."""
    rng = np.random.default_rng(seed)
    nk, L = (1 << w) - 1, n // w
    roots0 = rng.integers(0, 2**64 - 1, (K, 2), dtype=np.uint64)
    deltas = rng.integers(0, 2**64 - 1, (K, 2), dtype=np.uint64)
    deltas[:, 0] |= np.uint64(1)
    alphas = rng.integers(0, 1 << n, K)
    betas = rng.integers(1, P, K, dtype=np.uint64)
    dlt0 = rng.integers(0, 2**64 - 1, (K * L * nk, 2), dtype=np.uint64)
    cws = np.zeros((K * L * nk, 2), np.uint64)
    dlt1 = np.zeros_like(dlt0)
    cwo = np.zeros(K, np.uint64)
    for k in range(K):
        s = slice(k * L * nk, (k + 1) * L * nk)
        c, co, d1 = O.dpf_deal(n, w, roots0[k], deltas[k], int(alphas[k]), int(betas[k]), prg, rks,
                               np.ascontiguousarray(dlt0[s]))
        cws[s], dlt1[s], cwo[k] = c, d1, co
    out = dict(roots0=roots0, roots1=roots0 ^ deltas, cws=cws, cw_out=cwo, alphas=alphas,
               betas=betas, deltas=deltas)
    if with_dlt:
        out.update(dlt0=dlt0, dlt1=dlt1)
    return out


def real_bench_inputs(n, B):
    """dpf_real_bench synthetic inputs (GPU_baseline/dpf_real_bench.cu:256-263, :285-286)."""
    roots = np.zeros((B, 2), np.uint64)
    b = np.arange(B, dtype=np.uint64)
    with np.errstate(over="ignore"):
        roots[:, 0] = np.uint64(0x9E3779B97F4A7C15) * (b + np.uint64(1))
        roots[:, 1] = b + np.uint64(1)
        i = np.arange(B * n, dtype=np.uint64)
        dlt = np.stack([np.uint64(0x1234567) * (i + np.uint64(1)), i], axis=1)
    CW = np.array([(0xABCDEF * (k + 1)) % P for k in range(B)], np.uint64)
    return roots, np.ascontiguousarray(dlt), CW


def real_bench_checksum(sumC, sumT, g):
    c = 0
    for x, y in zip(sumC.tolist(), sumT.tolist()):
        c ^= x ^ y
    return c ^ int(np.bitwise_xor.reduce(g[::97]))


def ref_exchange_fn():
    return C.CFUNCTYPE(None, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p)
