"""Batched DPF full-domain evaluation + leaf convert, 4096 keys x 2^16 leaves
(w = 1), ChaCha8 and AES tree PRGs: the library against the reference's own
GPU kernels (oracle/_ref/libref_gpu.so, GPU_baseline/common/{dpf_gpu,
leaf_convert_cuda}.cu compiled unmodified).

TEST INFRASTRUCTURE: a measurement script, not product code.

Keys are random roots and per-level correction words.  The reference's GPU
entry point is interactive (dpf_gpu.h:55-75): after every level it hands the
host the current shares and takes the peer's back.  Here the exchange
returns peer = my ^ CW, which makes the interactive evaluation equal to the
keyed one, so three paths compute the same leaves:

  ref      reference dpf_gpu_batch_full_eval_device + dpf_out_sums +
           dpf_out_scatter_g
  drop_in  the library's dpf_gpu_batch_full_eval_device + dpf_out_sums +
           dpf_out_scatter_g, same exchange callback
  keyed    the library's pcgb_dpf_keyed_full_eval (no exchange) + the same
           convert calls

The scatter uses the t = 64 geometry (B = t^2 = 4096 instances, N = t*D/2 =
2^21), party 0, uniform F_p output CWs.  Bit-exactness: per-instance sums
(C mod p and T), the whole scattered g, and the leaves of the first and last
instance must agree across the three paths.
Times are wall-clock per call with the device synchronised (the interactive
paths include their per-level host round trips, as the reference's do).

Usage: python oracle/dpf_convert_bench.py [--B 4096] [--n 16] [--w 1] [--iters 3]

--mixed instead times a batch of key groups with different domains (ChaCha8,
w = 1): one pcgb_dpf_keyed_full_eval_multi call against one
pcgb_dpf_keyed_full_eval call per group, device time by CUDA events.
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


MIXED_GROUPS = [(256, 17), (512, 16), (1024, 14), (2048, 12), (4096, 10), (64, 8), (8, 6)]


def mixed_main(args):
    import pcg_b200 as L
    rng = np.random.default_rng(args.seed)
    groups = []
    for K, n in MIXED_GROUPS:
        roots = rng.integers(0, 2**64 - 1, (K, 2), dtype=np.uint64)
        cws = rng.integers(0, 2**64 - 1, (K * n, 2), dtype=np.uint64)
        groups.append((K, n, L.to_device(roots), L.to_device(cws), L.DeviceBuffer(16 * K << n)))
    spec = [(K, n, r.ptr, c.ptr, o.ptr) for K, n, r, c, o in groups]

    def timed(fn):
        fn()                                     # warm
        best = None
        for _ in range(args.iters):
            a, b = L.Event(), L.Event()
            a.record()
            fn()
            b.record()
            ms = a.elapsed_ms(b)
            best = ms if best is None else min(best, ms)
        return best

    def each():
        for K, n, r, c, o in spec:
            L.dpf_keyed_full_eval_device(K, n, 1, L.PRG_CHACHA8, r, c, o)

    def batch():
        L.dpf_keyed_full_eval_multi_device(spec, 1, L.PRG_CHACHA8)

    c0 = L.launch_count()
    each()
    per_group_launches = L.launch_count() - c0
    c0 = L.launch_count()
    batch()
    batch_launches = L.launch_count() - c0
    t_each, t_batch = timed(each), timed(batch)
    leaves = sum(K << n for K, n in MIXED_GROUPS)
    print(json.dumps({
        "workload": "keyed DPF full-domain eval, ChaCha8 w=1, groups (K, n) = "
                    + str(MIXED_GROUPS), "leaves": leaves,
        "per_group_calls": {"ms": t_each, "launches": per_group_launches},
        "one_batch": {"ms": t_batch, "launches": batch_launches},
        "speedup": t_each / t_batch, "device": L.device_name()}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--B", type=int, default=4096)
    ap.add_argument("--n", type=int, default=16)
    ap.add_argument("--w", type=int, default=1)
    ap.add_argument("--iters", type=int, default=3)
    ap.add_argument("--seed", type=int, default=33)
    ap.add_argument("--mixed", action="store_true",
                    help="time a batch of key groups of different domains")
    args = ap.parse_args()
    if args.mixed:
        return mixed_main(args)
    import pcg_b200 as L

    R = O.ref_gpu()
    if R is None:
        raise SystemExit("oracle/_ref/libref_gpu.so not built")
    B, n, w = args.B, args.n, args.w
    D, levels, nk = 1 << n, n // w, (1 << w) - 1
    t = int(round(B ** 0.5))
    assert t * t == B and n % w == 0
    N = t * D // 2
    rng = np.random.default_rng(args.seed)
    roots = rng.integers(0, 2**64 - 1, (B, 2), dtype=np.uint64)
    cws = rng.integers(0, 2**64 - 1, (B, levels, nk, 2), dtype=np.uint64)
    CW = rng.integers(0, O.P, B, dtype=np.uint64)
    zero_dlt = np.zeros((B * levels * nk, 2), np.uint64)
    d_roots, d_cws = L.to_device(roots), L.to_device(cws)
    d_keyed = L.DeviceBuffer(16 * B * D)

    EX = C.CFUNCTYPE(None, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p)
    out = {"workload": f"{B} keys x 2^{n} leaves, w={w}, DPF full-domain eval + out_sums + "
                       f"out_scatter_g (t={t}, N=2^{N.bit_length() - 1})",
           "device": L.device_name(), "iters": args.iters}

    for prg_name, prg in (("chacha8", L.PRG_CHACHA8), ("aes", L.PRG_AES)):
        rks = O.aes_tree_round_keys(rng.integers(0, 256, 16, dtype=np.uint8), nk) \
            if prg == L.PRG_AES else None
        level = [0]

        def ex(my, peer, count, user):
            m = np.ctypeslib.as_array(C.cast(my, C.POINTER(C.c_uint64)), shape=(count, 2))
            p = np.ctypeslib.as_array(C.cast(peer, C.POINTER(C.c_uint64)), shape=(count, 2))
            p[:] = m ^ cws[:, level[0]].reshape(-1, 2)
            level[0] += 1

        cb = EX(ex)

        def run_ref():
            level[0] = 0
            d = C.c_void_p()
            rc = R.ref_dpf_batch_full_eval_device(
                B, n, w, roots.ctypes.data, zero_dlt.ctypes.data,
                None if rks is None else rks.ctypes.data, 0, C.cast(cb, C.c_void_p), None,
                1 if prg == L.PRG_CHACHA8 else 0, C.byref(d))
            assert rc == 0, R.ref_last_error()
            R.ref_sync()
            t1 = time.perf_counter()
            sc, st = np.zeros(B, np.uint64), np.zeros(B, np.uint64)
            assert R.ref_dpf_out_sums(d.value, B, D, O.P, sc, st) == 0
            t2 = time.perf_counter()
            g = np.zeros(N, np.uint64)
            assert R.ref_dpf_out_scatter_g(d.value, B, D, t, 0, O.P, CW, g, N) == 0
            return d.value, sc, st, g, t1, t2

        def run_drop_in():
            level[0] = 0
            d = L.dpf_gpu_batch_full_eval_device(
                B, n, w, roots, zero_dlt, round_keys=rks,
                exchange=lambda my: my ^ cws[:, _next(level)].reshape(-1, 2), prg=prg)
            L.synchronize()
            t1 = time.perf_counter()
            sc, st = L.dpf_out_sums(d, B, D)
            t2 = time.perf_counter()
            g = L.dpf_out_scatter_g(d, B, D, t, 0, CW, N)
            return d, sc, st, g, t1, t2

        def run_keyed():
            L.dpf_keyed_full_eval_device(B, n, w, prg, d_roots.ptr, d_cws.ptr, d_keyed.ptr,
                                         round_keys=rks)
            L.synchronize()
            t1 = time.perf_counter()
            sc, st = L.dpf_out_sums(d_keyed.ptr, B, D)
            t2 = time.perf_counter()
            g = L.dpf_out_scatter_g(d_keyed.ptr, B, D, t, 0, CW, N)
            return d_keyed.ptr, sc, st, g, t1, t2

        res = {}
        for name, fn in (("ref", run_ref), ("drop_in", run_drop_in), ("keyed", run_keyed)):
            fn()                                   # warm-up
            ev, cv, sv = [], [], []
            for _ in range(args.iters):
                t0 = time.perf_counter()
                d, sc, st, g, t1, t2 = fn()
                t3 = time.perf_counter()
                ev.append(t1 - t0)
                cv.append(t2 - t1)
                sv.append(t3 - t2)
            first = _download(L, d, 0, D)
            last = _download(L, d, (B - 1) * D, D)
            res[name] = {"eval_ms": 1e3 * float(np.median(ev)),
                         "convert_ms": 1e3 * float(np.median(cv)),
                         "scatter_ms": 1e3 * float(np.median(sv)),
                         "sums": (sc.copy(), st.copy(), g.copy()), "leaves": (first, last)}
        base = res["ref"]
        entry = {}
        for name, r in res.items():
            same = all((a == b).all() for a, b in zip(r["sums"], base["sums"])) and \
                all((a == b).all() for a, b in zip(r["leaves"], base["leaves"]))
            entry[name] = {"eval_ms": r["eval_ms"], "convert_ms": r["convert_ms"],
                           "scatter_ms": r["scatter_ms"],
                           "total_ms": r["eval_ms"] + r["convert_ms"],
                           "leaves_per_s": B * D / ((r["eval_ms"] + r["convert_ms"]) * 1e-3),
                           "bit_exact_vs_ref": bool(same)}
        for name in ("drop_in", "keyed"):
            entry[name]["speedup_vs_ref"] = entry["ref"]["total_ms"] / entry[name]["total_ms"]
        out[prg_name] = entry
    print(json.dumps(out), flush=True)


def _next(level):
    v = level[0]
    level[0] += 1
    return v


def _download(L, d_ptr, first_blk, count):
    h = np.empty((count, 2), np.uint64)
    L.lib.pcgb_memcpy_d2h(h.ctypes.data, d_ptr + 16 * first_blk, h.nbytes, None)
    return h


if __name__ == "__main__":
    main()
