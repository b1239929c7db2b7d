"""The reference's own driver programs, compiled unchanged from their sources
and linked with libpcg_b200.so (oracle/Makefile, target `drivers`), run on the
GPU.  They reach the library through its pcg_cuda:: C++ layer (std::function
exchange, std::string reasons, exceptions), exactly as the reference's
callers would:

  GPU_baseline/test/poly_mul_cuda.cpp   every poly-mul name (v1, gpuntt merge,
                                        gpuntt 4-step) against the reference's
                                        CPU ntt.h, aliasing included; exit 0
  GPU_baseline/dpf_real_bench.cu        the five checksums of
                                        GPU_baseline/results_l40s/plateau.txt
  GPU_baseline/e2e_full_bench.cu        the serial arm (interactive DPF per
                                        block, out_sums, out_scatter_g, two
                                        batched square products); checksum
                                        recomputed from the reference kernels
                                        and the oracle's product

The e2e driver's --batch-blocks arm is not run: it asks for B*c^2 instances
while its root and DltSft vectors hold B (e2e_full_bench.cu:83-84,134-136), a
host over-read in the reference driver itself.
"""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import oracle_lib as O
from gpu_helpers import real_bench_inputs

pytestmark = pytest.mark.gpu
P = O.P
DRV = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                   "drivers")


def run(name, *args, timeout=600):
    path = os.path.join(DRV, name)
    if not os.path.exists(path):
        pytest.skip(f"{name} not built (make -C oracle REF=<reference tree> drivers)")
    r = subprocess.run([path, *map(str, args)], capture_output=True, text=True, timeout=timeout,
                       env={**os.environ, "PCG_RTT_US": "0"})
    return r.returncode, r.stdout + r.stderr


def test_reference_poly_mul_test_passes(pcg):
    rc, out = run("test_poly_mul_cuda")
    assert rc == 0, out[-3000:]
    assert "Mismatch" not in out
    for backend in ("v1", "gpuntt-merge", "gpuntt-4step"):
        assert f"PASS [{backend}] alias output==lhs" in out, out[-2000:]
    # Every size the driver lists for the gpuntt backends, up to 2^20.
    assert "PASS [gpuntt-4step] N=1048576 batch=2 random*random" in out
    assert "PASS [gpuntt-merge] N=1048576 batch=2 random*random" in out


# GPU_baseline/results_l40s/plateau.txt:1,7,13,19,25
PLATEAU = [(18, 64, 8, "16e395febfd6d23f"), (18, 256, 16, "27cb4298e84744ed"),
           (20, 64, 8, "104646e15a59c497"), (20, 256, 16, "204a14f81d54aa7e"),
           (24, 16, 4, "02a9707398f918d0")]


@pytest.mark.parametrize("n,B,t,want", PLATEAU)
def test_reference_dpf_real_bench_checksums(pcg, n, B, t, want):
    rc, out = run("dpf_real_bench", "--n", n, "--B", B, "--t", t, "--iters", 1)
    assert rc == 0, out[-2000:]
    m = re.search(r"checksum=([0-9a-f]{16})", out)
    assert m and m.group(1) == want, out[-2000:]


def _e2e_expected(c, t, logN):
    """The checksum e2e_full_bench.cu:154-196 prints for --iters 1 (serial):
    each of the c^2 identical blocks XORs in a sample of its sums and g, then
    the product of the first polynomial pair adds pc[0] ^ pc[N/2].  The block
    part comes from the reference's own kernels (oracle/_ref/libref_gpu.so),
    the product from the oracle's NTT."""
    N = 1 << logN
    n = logN + 1 - (t.bit_length() - 1)
    B, D = t * t, 1 << n
    gN = t * (D // 2)
    cks = 0
    if (c * c) % 2:
        R = O.ref_gpu()
        if R is None:
            pytest.skip("oracle/_ref/libref_gpu.so not built")
        roots, dlt, CW = real_bench_inputs(n, B)
        dl = C.c_void_p()
        assert R.ref_dpf_batch_full_eval_device(B, n, 1, roots.ctypes.data, dlt.ctypes.data, None,
                                                0, None, None, 1, C.byref(dl)) == 0
        sc, st = np.zeros(B, np.uint64), np.zeros(B, np.uint64)
        assert R.ref_dpf_out_sums(dl.value, B, D, P, sc, st) == 0
        g = np.zeros(gN, np.uint64)
        assert R.ref_dpf_out_scatter_g(dl.value, B, D, t, 0, P, CW, g, gN) == 0
        for b in range(0, B, 97):
            cks ^= int(sc[b]) ^ int(st[b])
        cks ^= int(np.bitwise_xor.reduce(g[::9973]))
    i = np.arange(N, dtype=object)
    pa = np.array([(0x9E37 * k + 1) % P for k in i], dtype=np.uint64)
    pb = np.array([(0xBEEF * k + 7) % P for k in i], dtype=np.uint64)
    pc = O.poly_mul(pa, pb, N)
    return cks ^ int(pc[0]) ^ int(pc[N // 2])


@pytest.mark.parametrize("c", [3, 4])
def test_reference_e2e_full_bench_serial_arm(pcg, c):
    t, logN = 16, 20
    rc, out = run("e2e_full_bench", "--c", c, "--t", t, "--logN", logN, "--iters", 1)
    assert rc == 0, out[-2000:]
    m = re.search(r"RESULT .*checksum=([0-9a-f]{16}) STATUS=OK", out)
    assert m, out[-2000:]
    assert int(m.group(1), 16) == _e2e_expected(c, t, logN), out[-2000:]
    print(out.strip().splitlines()[-1])
