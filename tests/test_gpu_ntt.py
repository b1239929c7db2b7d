"""Negacyclic poly-mul drop-ins and the device batch API against the oracle
(CPU_baseline/ntt.h restated), schoolbook products and the reference's NTT
checksums."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O
from gpu_helpers import dev

pytestmark = pytest.mark.gpu
P = O.P


def pattern(N, batch, kind, seed):
    """GPU_baseline/test/poly_mul_cuda.cpp:173-188."""
    if kind == "zero":
        return np.zeros(N * batch, np.uint64)
    if kind == "one":
        return np.ones(N * batch, np.uint64)
    if kind == "impulse":
        v = np.zeros((batch, N), np.uint64)
        for b in range(batch):
            v[b, b % N] = 1
        return v.reshape(-1)
    if kind == "max":
        return np.full(N * batch, P - 1, np.uint64)
    return O.mt64(seed, N * batch) % np.uint64(P)


VARIANTS = {
    "v1": (lambda L: L.poly_mul_u64, [128, 256, 512, 1024, 8192, 16384, 32768]),
    "merge": (lambda L: L.poly_mul_u64_gpuntt, [2, 4, 128, 1024, 32768, 1 << 18, 1 << 20]),
    "4step": (lambda L: L.poly_mul_u64_gpuntt_4step, [4096, 65536, 1 << 18, 1 << 20]),
    "square": (lambda L: L.poly_mul_u64_gpuntt_square, [256, 4096, 1 << 20]),
}


@pytest.mark.parametrize("variant", list(VARIANTS))
def test_poly_mul_patterns(pcg, variant):
    fn, sizes = VARIANTS[variant]
    f = fn(pcg)
    for N in sizes:
        batch = 4 if N <= 1024 else 2
        for lhs, rhs in [("zero", "zero"), ("one", "one"), ("impulse", "one"), ("max", "max"),
                         ("random", "random")]:
            a = pattern(N, batch, lhs, 1234 + N + batch)
            b = pattern(N, batch, rhs, 5678 + 3 * N + batch)
            got, _ = f(a, b, batch, N)
            assert (got == O.poly_mul(a, b, N)).all(), (variant, N, lhs)


def test_poly_mul_alias_out_is_lhs(pcg):
    N, batch = 256, 4
    a = pattern(N, batch, "random", 111)
    b = pattern(N, batch, "random", 222)
    want = O.poly_mul(a, b, N)
    ms = C.c_double()
    rc = pcg.lib.pcgb_poly_mul_u64(pcg.POLYMUL_MERGE, a, a, b, batch, N, P, C.byref(ms))
    assert rc == 0 and (a == want).all()


def test_unreduced_inputs(pcg):
    rng = np.random.default_rng(3)
    N = 2048
    a = rng.integers(P, 2**64 - 1, N, dtype=np.uint64)
    b = rng.integers(0, 2**64 - 1, N, dtype=np.uint64)
    got, _ = pcg.poly_mul_u64_gpuntt(a, b, 1, N)
    assert (got == O.poly_mul(a, b, N)).all()


@pytest.mark.parametrize("lg", [8, 9, 10, 11, 12])
def test_square_verify_schoolbook(pcg, lg):
    """GPU_baseline/square_verify.cu:309-346: vs the schoolbook negacyclic product."""
    N = 1 << lg
    r = O.mt64(12345 + lg, 8 * N)
    for batch, off in ((1, 0), (3, 2 * N)):
        a = r[off: off + batch * N] % np.uint64(P)
        b = r[off + batch * N: off + 2 * batch * N] % np.uint64(P)
        got, _ = pcg.poly_mul_u64_gpuntt_square(a, b, batch, N)
        for k in range(batch):
            s = slice(k * N, (k + 1) * N)
            assert (got[s] == O.poly_mul_schoolbook(a[s], b[s], N)).all()


def test_supported_rules(pcg):
    assert pcg.poly_mul_supported(P, 32768)[0] and not pcg.poly_mul_supported(P, 65536)[0]
    assert not pcg.poly_mul_gpuntt_4step_supported(P, 2048)[0]
    assert pcg.poly_mul_gpuntt_supported(P, 1 << 24)[0]
    assert not pcg.poly_mul_gpuntt_supported(P, 1 << 25)[0]
    assert not pcg.poly_mul_gpuntt_square_supported(P, 128)[0]
    ok, why = pcg.poly_mul_supported(97, 1024)
    assert not ok and "prime" in why
    with pytest.raises(pcg.PcgError):
        pcg.poly_mul_u64(np.zeros(8, np.uint64), np.zeros(8, np.uint64), 0, 8)


def fnv64(v):
    h = 1469598103934665603
    for x in v.tolist():
        h = ((h ^ x) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def test_golden_checksums_2e20_batch16(pcg):
    """results_l40s/ntt_4step.txt:7 (XOR) and ntt_naive.txt:1 (FNV)."""
    N, batch = 1 << 20, 16
    j = np.arange(N * batch, dtype=np.uint64)
    with np.errstate(over="ignore"):
        a = (np.uint64(0x9E3779B97F4A7C15) * (j + np.uint64(1))) % np.uint64(P)
        b = (np.uint64(0xC2B2AE3D27D4EB4F) * (j + np.uint64(7))) % np.uint64(P)
    got, _ = pcg.poly_mul_u64_gpuntt_square(a, b, batch, N)
    assert int(np.bitwise_xor.reduce(got)) == 0x3969340B039F5D5D
    r = O.mt64(11, 2 * N * batch)
    got, _ = pcg.poly_mul_u64_gpuntt(r[: N * batch] % np.uint64(P), r[N * batch:] % np.uint64(P),
                                     batch, N)
    assert fnv64(got) == 0x8599DD17BF241164


@pytest.mark.parametrize("lg", [21, 22, 24])
def test_large_n_against_oracle(pcg, lg):
    N = 1 << lg
    r = O.mt64(lg, 2 * N)
    a, b = r[:N] % np.uint64(P), r[N:] % np.uint64(P)
    got, _ = pcg.poly_mul_u64_gpuntt(a, b, 1, N)
    assert (got == O.poly_mul(a, b, N)).all()


def test_device_batch_api_uneven(pcg):
    rng = np.random.default_rng(5)
    sizes = [1 << 16, 1 << 18, 1 << 20]
    polys = [(rng.integers(0, P, N, dtype=np.uint64), rng.integers(0, P, N, dtype=np.uint64))
             for N in sizes]
    bufs = [(dev(pcg, a), dev(pcg, b), pcg.DeviceBuffer(a.nbytes)) for a, b in polys]
    arr = lambda k: (C.c_void_p * len(sizes))(*[x[k].ptr for x in bufs])
    Ns = (C.c_int * len(sizes))(*sizes)
    rc = pcg.lib.pcgb_poly_mul_device_multi(len(sizes), arr(2), arr(0), arr(1), Ns, None)
    assert rc == 0, pcg.lib.pcgb_last_error()
    for (a, b), (_, _, dc), N in zip(polys, bufs, sizes):
        assert (dc.download(np.uint64, N) == O.poly_mul(a, b, N)).all()


def _multi(pcg, outs, As, Bs, sizes):
    arr = lambda bufs: (C.c_void_p * len(sizes))(*[x.ptr for x in bufs])
    Ns = (C.c_int * len(sizes))(*sizes)
    rc = pcg.lib.pcgb_poly_mul_device_multi(len(sizes), arr(outs), arr(As), arr(Bs), Ns, None)
    assert rc == 0, pcg.lib.pcgb_last_error()
    pcg.synchronize()


def test_mixed_lengths_one_launch_per_pass(pcg):
    """Lengths 2^16..2^20 in any order and multiplicity, unreduced inputs, one
    output aliasing its first operand: five launches for the whole batch and
    every product equal to the single-length path's."""
    rng = np.random.default_rng(17)
    sizes = [1 << 17, 1 << 20, 1 << 16, 1 << 19, 1 << 17, 1 << 18]
    A = [rng.integers(0, 2**64 - 1, N, dtype=np.uint64) for N in sizes]
    B = [rng.integers(0, 2**64 - 1, N, dtype=np.uint64) for N in sizes]
    dA, dB = [dev(pcg, a) for a in A], [dev(pcg, b) for b in B]
    want = []
    for a, b, N in zip(dA, dB, sizes):
        out = pcg.DeviceBuffer(8 * N)
        pcg.poly_mul_device(out.ptr, a.ptr, b.ptr, 1, N)
        pcg.synchronize()
        want.append(out.download(np.uint64, N))
    outs = [pcg.DeviceBuffer(8 * N) for N in sizes]
    outs[3] = dA[3]                                  # c aliases a
    _multi(pcg, outs, dA, dB, sizes)                 # plans warm
    dA[3] = dev(pcg, A[3])
    outs[3] = dA[3]
    before = pcg.launch_count()
    _multi(pcg, outs, dA, dB, sizes)
    assert pcg.launch_count() - before == 5
    for o, w, N in zip(outs, want, sizes):
        assert (o.download(np.uint64, N) == w).all()


def test_multi_outside_mixed_range_falls_back(pcg):
    rng = np.random.default_rng(18)
    sizes = [1 << 12, 1 << 16, 1 << 21]
    polys = [(rng.integers(0, P, N, dtype=np.uint64), rng.integers(0, P, N, dtype=np.uint64))
             for N in sizes]
    dA = [dev(pcg, a) for a, _ in polys]
    dB = [dev(pcg, b) for _, b in polys]
    outs = [pcg.DeviceBuffer(8 * N) for N in sizes]
    _multi(pcg, outs, dA, dB, sizes)
    for (a, b), o, N in zip(polys, outs, sizes):
        assert (o.download(np.uint64, N) == O.poly_mul(a, b, N)).all()
