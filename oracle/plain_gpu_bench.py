"""Plain per-stage GPU path: the reference's own GPU kernels (oracle/_ref,
compiled unmodified from GPU_baseline/common) driven one request at a time
the way GPU_baseline/e2e_full_bench.cu's serial arm drives them
(e2e_full_bench.cu:154-180): for each of the c^2 blocks,
dpf_gpu_batch_full_eval_device (B = t^2 instances, n = log2(2N/t)) ->
dpf_out_sums (D2H) -> dpf_out_scatter_g (D2H g); then the step-4 products.

TEST INFRASTRUCTURE: this is a baseline measurement, not product code.
Differences from the reference bench, all stated in the output:
  * the per-level exchange returns peer = my ^ CW (CWs from the keyed
    dealer) instead of a zero stub, so the outputs are the real expansion
    and are checked against the library's fused path (bit-exact);
  * the reference's step-4 backend (GPU-NTT "square") is not in the tree,
    so the 2 batched products of batch c^2 (e2e_full_bench.cu:177-180) run
    through the library's host-API poly-mul (same host-in/host-out
    contract, H2D/D2H inside), which is at least as fast as the reference's
    published B200 figure.

Usage: python oracle/plain_gpu_bench.py [--iters 3] [--N 1048576 --c 4 --t 16]
"""
import argparse
import ctypes as C
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "pcg-square_b200"))

import oracle_lib as O  # noqa: E402


def run(L, N=1 << 20, c=4, t=16, iters=3, seed=1000):
    """Times the plain path (one warm-up iteration, then `iters`) and checks
    its g against the library's fused g'; returns the result dict, or None
    when oracle/_ref/libref_gpu.so is not built."""
    R = O.ref_gpu()
    if R is None:
        return None
    s = O.shape(N, c, t)
    B, n, levels = t * t, s.n, s.levels
    D = 1 << n
    a = L.public_a(N, c, 7)
    e = L.Expander(N, c, t, 1, L.PRG_CHACHA8, public_a=a)
    K = e.K
    d_r0, d_r1 = L.DeviceBuffer(16 * K), L.DeviceBuffer(16 * K)
    d_cws, d_cwo = L.DeviceBuffer(16 * K * levels * e.nk), L.DeviceBuffer(8 * K)
    e.deal_keys_device(seed, d_r0.ptr, d_r1.ptr, d_cws.ptr, d_cwo.ptr)
    roots = d_r0.download(np.uint64, 2 * K).reshape(K, 2)
    cws = d_cws.download(np.uint64, 2 * K * levels).reshape(K, levels, 2)
    cwo = d_cwo.download(np.uint64, K)

    # Library's fused g' for the bit-exactness check of the plain path.
    d_g = L.DeviceBuffer(8 * N * e.Q)
    e.expand_g_device(0, d_r0.ptr, d_cws.ptr, d_cwo.ptr, d_g.ptr)
    fused = d_g.download(np.uint64, N * e.Q).reshape(e.Q, N)

    EX = C.CFUNCTYPE(None, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p)
    pa = np.ascontiguousarray(np.tile(a[:N], c * c).astype(np.uint64))
    pc = np.zeros_like(pa)
    dz = np.zeros((B * levels, 2), np.uint64)
    timings = []
    g_blocks = {}
    for it in range(iters + 1):
        st = {"dpf": 0.0, "sums": 0.0, "scatter": 0.0, "ntt": 0.0}
        w0 = time.perf_counter()
        for blk in range(c * c):
            cw_blk = cws[blk * B:(blk + 1) * B]
            level = [0]

            def ex(my, peer, count, user, cw_blk=cw_blk, level=level):
                m = np.ctypeslib.as_array(C.cast(my, C.POINTER(C.c_uint64)), shape=(count, 2))
                p = np.ctypeslib.as_array(C.cast(peer, C.POINTER(C.c_uint64)), shape=(count, 2))
                p[:] = m ^ cw_blk[:, level[0]]
                level[0] += 1

            cb = EX(ex)
            rts = np.ascontiguousarray(roots[blk * B:(blk + 1) * B])
            dl = C.c_void_p()
            t0 = time.perf_counter()
            rc = R.ref_dpf_batch_full_eval_device(B, n, 1, rts.ctypes.data, dz.ctypes.data, None, 0,
                                                  C.cast(cb, C.c_void_p), None, 1, C.byref(dl))
            assert rc == 0, R.ref_last_error()
            R.ref_sync()
            t1 = time.perf_counter()
            sc, stt = np.zeros(B, np.uint64), np.zeros(B, np.uint64)
            assert R.ref_dpf_out_sums(dl.value, B, D, O.P, sc, stt) == 0
            t2 = time.perf_counter()
            g = np.zeros(N, np.uint64)   # (dpf_out_sums above sized the CW buffer)
            cwb = np.ascontiguousarray(cwo[blk * B:(blk + 1) * B])
            assert R.ref_dpf_out_scatter_g(dl.value, B, D, t, 0, O.P, cwb, g, N) == 0
            t3 = time.perf_counter()
            st["dpf"] += t1 - t0
            st["sums"] += t2 - t1
            st["scatter"] += t3 - t2
            if it == 0:
                g_blocks[blk] = g
        t4 = time.perf_counter()
        for _ in range(2):
            pc, _ = L.poly_mul_u64_gpuntt_square(pa, pa, c * c, N)
        t5 = time.perf_counter()
        st["ntt"] = t5 - t4
        st["wall"] = t5 - w0
        if it > 0:
            timings.append(st)

    # Bit-exactness: merged pairs of the plain path == the fused kernel's g'.
    ok = True
    q = 0
    for i in range(c):
        for j in range(i, c):
            want = g_blocks[i * c + j] if i == j else \
                (g_blocks[i * c + j].astype(object) + g_blocks[j * c + i]) % O.P
            ok &= bool((fused[q] == np.asarray(want, dtype=np.uint64)).all())
            q += 1
    mean = {k: float(np.mean([x[k] for x in timings])) for k in timings[0]}
    e.close()
    return {"path": "plain per-stage GPU (reference kernels, serial arm)", "N": N, "c": c, "t": t,
            "B_per_block": B, "n": n, "iters": iters,
            "ms": {k: 1e3 * v for k, v in mean.items()},
            "corr_per_s": N / mean["wall"], "g_bit_exact_vs_fused": ok,
            "device": L.device_name()}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--N", type=int, default=1 << 20)
    ap.add_argument("--c", type=int, default=4)
    ap.add_argument("--t", type=int, default=16)
    ap.add_argument("--iters", type=int, default=3)
    ap.add_argument("--seed", type=int, default=1000)
    args = ap.parse_args()
    import pcg_b200 as L
    out = run(L, args.N, args.c, args.t, args.iters, args.seed)
    if out is None:
        raise SystemExit("oracle/_ref/libref_gpu.so not built")
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
