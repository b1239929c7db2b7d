"""Pins the CPU oracle to the reference's own known answers (no GPU)."""
import time

import numpy as np
import pytest

import oracle_lib as O

P = O.P


def test_aes_fips197_kat():
    # GPU_baseline/test/aes_gpu.cpp:57-60
    key = np.arange(16, dtype=np.uint8)
    pt = np.array([0x00, 0x11, 0x22, 0x33, 0x44, 0x55, 0x66, 0x77,
                   0x88, 0x99, 0xaa, 0xbb, 0xcc, 0xdd, 0xee, 0xff], np.uint8)
    ct = O.aes_encrypt(O.aes_expand_key(key), pt)
    assert bytes(ct).hex() == "69c4e0d86a7b0430d8cdb78070b4c55a"


def test_mt19937_64_known_value():
    # The C++ standard pins the 10000th output of default-seeded mt19937_64.
    assert int(O.mt64(5489, 10000)[-1]) == 9981545732273789042


def test_chacha8_matches_reference_header():
    R = O.ref_cpu()
    if R is None:
        pytest.skip("oracle/_ref not built (reference tree absent)")
    rng = np.random.default_rng(1)
    for _ in range(64):
        k8 = rng.integers(0, 2**32, 8, dtype=np.uint32)
        nonce = int(rng.integers(0, 2**63))
        ctr = int(rng.integers(0, 2**40))
        ks = np.zeros(64, np.uint8)
        R.ref_chacha8_keystream(np.ascontiguousarray(k8.view(np.uint8)), nonce, ctr, ks, 1)
        assert (ks.view(np.uint32) == O.chacha8_block(k8, ctr, nonce)).all()


@pytest.mark.parametrize("N", [2, 4, 16, 256, 4096])
def test_ntt_matches_reference_header(N):
    R = O.ref_cpu()
    if R is None:
        pytest.skip("oracle/_ref not built (reference tree absent)")
    rng = np.random.default_rng(N)
    a = rng.integers(0, 2**64 - 1, 3 * N, dtype=np.uint64)
    b = rng.integers(0, 2**64 - 1, 3 * N, dtype=np.uint64)
    got = O.poly_mul(a, b, N)
    want = np.zeros_like(got)
    R.ref_ntt_poly_mul(want, a, b, 3, N)
    assert (got == want).all()


@pytest.mark.parametrize("N", [8, 64, 256])
def test_ntt_matches_schoolbook(N):
    rng = np.random.default_rng(7 + N)
    a = rng.integers(0, P, N, dtype=np.uint64)
    b = rng.integers(0, P, N, dtype=np.uint64)
    assert (O.poly_mul(a, b, N) == O.poly_mul_schoolbook(a, b, N)).all()


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
    """dpf_real_bench.cu:310-312."""
    c = 0
    for x, y in zip(sumC.tolist(), sumT.tolist()):
        c ^= x ^ y
    return c ^ int(np.bitwise_xor.reduce(g[::97]))


@pytest.mark.slow
def test_dpf_convert_golden_checksum():
    # GPU_baseline/results_l40s/plateau.txt:1 — n=18 B=64 t=8 w=1 chacha8.
    n, B, t = 18, 64, 8
    roots, dlt, CW = real_bench_inputs(n, B)
    leaves = O.dpf_batch_full_eval(B, n, 1, roots, dlt)
    D = 1 << n
    sc, st = O.out_sums(leaves, B, D)
    g = O.out_scatter_g(leaves, B, D, t, 0, CW, t * (D // 2))
    assert real_bench_checksum(sc, st, g) == 0x16E395FEBFD6D23F


def fourstep_inputs(N, batch):
    """ntt_batch_bench.cu:45-49."""
    j = np.arange(N * batch, dtype=np.uint64)
    with np.errstate(over="ignore"):
        a = (np.uint64(0x9E3779B97F4A7C15) * (j + np.uint64(1))) % np.uint64(P)
        b = (np.uint64(0xC2B2AE3D27D4EB4F) * (j + np.uint64(7))) % np.uint64(P)
    return a, b


def naive_inputs(N, batch):
    """naive_ntt_bench.cu:200-203: mt19937_64(11), a then b."""
    r = O.mt64(11, 2 * N * batch)
    return r[: N * batch] % np.uint64(P), r[N * batch:] % np.uint64(P)


def fnv64(v):
    h = 1469598103934665603
    for x in v.tolist():
        h = ((h ^ x) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


@pytest.mark.slow
def test_ntt_golden_checksums():
    # results_l40s/ntt_4step.txt:7 and ntt_naive.txt:1 (N=2^20, batch 16).
    N, batch = 1 << 20, 16
    a, b = fourstep_inputs(N, batch)
    c = O.poly_mul(a, b, N)
    assert int(np.bitwise_xor.reduce(c)) == 0x3969340B039F5D5D
    a, b = naive_inputs(N, batch)
    assert fnv64(O.poly_mul(a, b, N)) == 0x8599DD17BF241164


def test_oracle_slot_order_is_the_references():
    R = O.ref_cpu()
    if R is None:
        pytest.skip("oracle/_ref not built")
    a = np.random.default_rng(3).integers(0, 2**64 - 1, 2 * 512, dtype=np.uint64)
    want = a.copy()
    R.ref_ntt_forward(want, 2, 512)
    assert (O.ntt_forward(a, 512) == want).all()


def test_oracle_triples_hold_on_oracle_oles():
    """Two OLEs from the oracle's expansion at the CPU-runnable shape: the
    triple.h restatement yields slot shares with (a0+a1)(b0+b1) = c0+c1."""
    s = O.shape(4096, 2, 4)
    a = O.public_a(s, 7)
    oles = []
    for seed in (11, 12):
        r0, r1, cws, cwo = O.deal_keys(s, seed)
        outs = []
        for party, roots in ((0, r0), (1, r1)):
            outs.append(O.expand(s, party, roots, cws, cwo, *O.noise(s, seed, party), a, None))
        oles.append(outs)
    N, P = 4096, O.P
    sh = [O.triples(N, party, *oles[0][party], *oles[1][party]) for party in (0, 1)]
    for k in range(0, N, 97):
        lhs = (int(sh[0][0][k]) + int(sh[1][0][k])) * (int(sh[0][1][k]) + int(sh[1][1][k])) % P
        assert lhs == (int(sh[0][2][k]) + int(sh[1][2][k])) % P
