"""The C-ABI library loads and exports every symbol include/*.h declares
(no device compute here)."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "pcg-square_b200", "lib", "libpcg_b200.so")


def declared_c_symbols():
    text = open(os.path.join(ROOT, "include", "pcg_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pcgb_[a-z0-9_]+)\s*\(", text)))


def test_library_loads_and_exports_c_abi():
    assert os.path.exists(LIB), "library not built"
    lib = ctypes.CDLL(LIB)
    syms = declared_c_symbols()
    assert len(syms) > 30
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_exports_pcg_cuda_compat_symbols():
    out = subprocess.run(["nm", "-DC", LIB], capture_output=True, text=True, check=True).stdout
    for name in ["pcg_cuda::dpf_gpu_batch_full_eval(", "pcg_cuda::dpf_gpu_batch_full_eval_device(",
                 "pcg_cuda::dpf_out_sums(", "pcg_cuda::dpf_out_scatter_g(",
                 "pcg_cuda::poly_mul_u64(", "pcg_cuda::poly_mul_u64_gpuntt(",
                 "pcg_cuda::poly_mul_u64_gpuntt_4step(", "pcg_cuda::poly_mul_u64_gpuntt_square(",
                 "pcg_cuda::poly_mul_supported(", "pcg_cuda::poly_mul_gpuntt_supported(",
                 "pcg_cuda::poly_mul_gpuntt_4step_supported(",
                 "pcg_cuda::poly_mul_gpuntt_square_supported(", "pcg_cuda::is_cuda_available(",
                 "pcg_cuda::device_name[abi:cxx11](", "pcg_cuda::runtime_version[abi:cxx11](",
                 "pcg_cuda::aes128_expand_key_host(", "pcg_cuda::aes128_ecb_encrypt_gpu("]:
        assert name in out, name


@pytest.mark.parametrize("driver", ["test_poly_mul_cuda", "dpf_real_bench", "e2e_full_bench"])
def test_reference_drivers_resolve_every_pcg_cuda_symbol(driver):
    """The reference's own drivers, compiled unchanged (oracle/Makefile
    `drivers`), import only pcg_cuda:: symbols the library defines, and load
    the in-tree library."""
    path = os.path.join(ROOT, "oracle", "_ref", "drivers", driver)
    if not os.path.exists(path):
        pytest.skip("reference drivers not built (needs the reference tree)")
    nm = lambda *a: subprocess.run(["nm", "-D", *a], capture_output=True, text=True,
                                   check=True).stdout
    need = {l.split()[-1] for l in nm("--undefined-only", path).splitlines()
            if "pcg_cuda" in l}
    have = {l.split()[-1] for l in nm("--defined-only", LIB).splitlines()}
    assert need, "driver imports no pcg_cuda symbol"
    assert need <= have, sorted(need - have)
    ldd = subprocess.run(["ldd", path], capture_output=True, text=True, check=True).stdout
    line = next(l for l in ldd.splitlines() if "libpcg_b200.so" in l)
    assert os.path.realpath(line.split("=>")[1].split("(")[0].strip()) == os.path.realpath(LIB)


def test_host_side_calls_without_device():
    import pcg_b200 as L
    if L.is_cuda_available():
        pytest.skip("device present: covered by the gpu tests")
    # Host-only helpers work; device calls fail loudly (no CPU fallback).
    rk = L.aes128_expand_key_host(bytes(range(16)))
    assert rk[:16].tobytes() == bytes(range(16))
    ok, why = L.poly_mul_supported(L.P, 1024)
    assert not ok and "CUDA" in why
    with pytest.raises(L.PcgError) as e:
        L.poly_mul_u64([1] * 8, [1] * 8, 1, 8)
    assert e.value.code == -3


def test_synthetic_material_matches_oracle():
    import numpy as np

    import oracle_lib as O
    import pcg_b200 as L
    s = O.shape(4096, 4, 16)
    for party in (0, 1):
        p_lib, v_lib = L.noise(4096, 4, 16, 77, party)
        p_orc, v_orc = O.noise(s, 77, party)
        assert (p_lib == p_orc).all() and (v_lib == v_orc).all()
    assert (L.public_a(4096, 4, 5) == O.public_a(s, 5)).all()


def test_gmw_gate_counts_follow_the_reference_circuits():
    """AND gates of the two preprocessing circuits: the Kogge-Stone adder
    (bool_circuit/adder.h:22-63: m initial generates, then 2(m - d) per
    prefix step d = 1, 2, 4, ...) and DltSft (dpf.cpp:214-238: per level and
    branch, a w-1 gate AND tree and 128 ANDs with Delta)."""
    import numpy as np

    import pcg_b200 as L
    from pcg_b200 import twoparty as T
    for m in (1, 2, 3, 5, 15, 16, 40, 63):
        want = m + sum(2 * (m - (1 << k)) for k in range(6) if (1 << k) < m)
        assert L.gmw_position_add_gates(m) == want, m
    assert L.gmw_position_add_gates(0) == 0 and L.gmw_position_add_gates(64) == 0
    for n, w in ((16, 1), (17, 1), (8, 4), (6, 2), (9, 3), (8, 8)):
        assert L.gmw_dltsft_gates(n, w) == (n // w) * ((1 << w) - 1) * (w - 1 + 128), (n, w)
    assert L.gmw_dltsft_gates(7, 2) == 0 and L.gmw_dltsft_gates(18, 9) == 0
    assert T.preprocess_gates(1 << 20, 4, 16) == (114, 17 * 128)
    # The dealer's triples hold, and the instance offsets follow the block order.
    (a0, b0, c0), (a1, b1, c1) = T.bool_triples_dealer(7, 100, np.random.default_rng(1))
    assert a0.size == 7 * 4 and (((a0 ^ a1) & (b0 ^ b1)) == (c0 ^ c1)).all()
    N, c, t = 1 << 10, 2, 4
    pos = np.array([k * (N // t) + 3 * k + i for i in range(c) for k in range(t)], np.uint64)
    off0, off1 = T.instance_offsets(0, N, c, t, pos), T.instance_offsets(1, N, c, t, pos)
    for blk in range(c * c):
        ii, jj = divmod(blk, c)
        for idx in range(t * t):
            kk, ll = divmod(idx, t)
            assert off0[blk * t * t + idx] == 3 * kk + ii
            assert off1[blk * t * t + idx] == 3 * ll + jj
