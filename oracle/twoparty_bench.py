"""Wall time of the interactive two-party expansion (pcg_b200.twoparty):
two processes, one per party, on one GPU, exchanging each level's CW shares
and the two Beaver opens through torch.distributed (gloo over 127.0.0.1).

TEST INFRASTRUCTURE: the preprocessing (DltSft shares, beta shares, Beaver
triples) comes from the oracle dealer of tests/test_gpu_twoparty.py,
standing in for the OT layer.  With --gmw the DltSft shares and roots are
instead computed online by the GPU GMW circuits (twoparty.preprocess: the
Kogge-Stone position add and the DltSft circuit) from dealt AND triples and
random Delta shares, and that time is reported separately.  Reports
per-party wall time of gen_and_expand (after one warm-up run), its message
count and bytes sent.

Usage: python oracle/twoparty_bench.py [--N 1048576 --c 4 --t 16] [--iters 2] [--gmw]
"""
import argparse
import json
import multiprocessing as mp
import os
import socket
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (HERE, os.path.join(ROOT, "pcg-square_b200"), os.path.join(ROOT, "tests")):
    sys.path.insert(0, p)


def _party(party, port, N, c, t, mat, iters, q, batched, gmw):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=party, world_size=2,
                            timeout=datetime.timedelta(seconds=600))
    try:
        import pcg_b200 as L
        from pcg_b200 import twoparty
        e = L.Expander(N, c, t, 1, L.PRG_CHACHA8, public_a=mat["a"])
        m = twoparty.PartyMaterial(
            roots=mat["roots"][party], dltsft=mat["dlt"][party], beta=mat["beta"][party],
            r=mat["r"][party], s=mat["s"][party], rs=mat["rs"][party],
            pos=mat["noise"][party][0], val=mat["noise"][party][1])
        times, pre = [], []
        d_x = d_z = None
        for it in range(iters + 1):
            chan = twoparty.Channel(party)
            del d_x, d_z              # the previous outputs, freed before the clock starts
            L.synchronize()
            dist.barrier()
            t0 = time.perf_counter()
            if gmw:
                m.roots, m.dltsft, _, _ = twoparty.preprocess(
                    party, chan, N, c, t, m.pos, mat["delta"][party], mat["tri_add"][party],
                    mat["tri_dlt"][party])
                t_pre = time.perf_counter() - t0
            d_x, d_z = twoparty.gen_and_expand(party, chan, e, m, batched=batched)
            L.synchronize()
            if it:
                times.append(time.perf_counter() - t0)
                if gmw:
                    pre.append(t_pre)
        q.put((party, times, chan.messages, chan.bytes,
               d_x.download(np.uint64, N), d_z.download(np.uint64, N),
               float(np.median(pre)) if pre else None))
        e.close()
        dist.barrier()
    finally:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--N", type=int, default=1 << 20)
    ap.add_argument("--c", type=int, default=4)
    ap.add_argument("--t", type=int, default=16)
    ap.add_argument("--iters", type=int, default=2)
    ap.add_argument("--per-block", action="store_true",
                    help="the reference's block-by-block order (one batch per block)")
    ap.add_argument("--gmw", action="store_true",
                    help="DltSft shares and roots from the GPU GMW circuits, timed")
    args = ap.parse_args()
    from test_gpu_twoparty import dealer
    import oracle_lib as O
    N, c, t = args.N, args.c, args.t
    t0 = time.perf_counter()
    mat = dealer(N, c, t, 777)
    if args.gmw:
        from pcg_b200 import twoparty
        rng = np.random.default_rng(778)
        B = c * c * t * t
        g_add, g_dlt = twoparty.preprocess_gates(N, c, t)
        mat["delta"] = rng.integers(0, 2**64 - 1, (2, B, 2), dtype=np.uint64, endpoint=True)
        mat["tri_add"] = twoparty.bool_triples_dealer(g_add, B, rng)
        mat["tri_dlt"] = twoparty.bool_triples_dealer(g_dlt, B, rng)
    deal_s = time.perf_counter() - t0
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_party, args=(p, port, N, c, t, mat, args.iters, q,
                                              not args.per_block, args.gmw))
             for p in (0, 1)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        party, times, msgs, nbytes, x, z, pre = q.get(timeout=1800)
        res[party] = (float(np.median(times)), msgs, nbytes, x, z, pre, times)
    for p in procs:
        p.join(timeout=300)
    import pcg_b200 as L
    d = [L.to_device(v) for v in (res[0][3], res[0][4], res[1][3], res[1][4])]
    bad = L.DeviceBuffer(8)
    L.verify_ole_device(N, d[0].ptr, d[1].ptr, d[2].ptr, d[3].ptr, bad.ptr)
    ok = int(bad.download(np.uint64, 1)[0]) == 0
    wall = max(res[0][0], res[1][0])
    print(json.dumps({
        "path": "interactive two-party expansion, 2 processes on 1 GPU, gloo exchange",
        "mode": ("per block" if args.per_block else "all blocks batched")
                + (", DltSft by GPU GMW" if args.gmw else ", DltSft dealt"),
        "N": N, "c": c, "t": t, "levels": O.shape(N, c, t).n,
        "ms_per_party": {p: 1e3 * res[p][0] for p in (0, 1)},
        "ms_iterations_party0": [round(1e3 * v, 2) for v in res[0][6]],
        "corr_per_s": N / wall, "messages_per_party": res[0][1],
        "bytes_sent_per_party": res[0][2], "ole_relation": ok,
        "gmw_preprocess_ms_per_party": ({p: 1e3 * res[p][5] for p in (0, 1)}
                                        if args.gmw else None),
        "dealer_s": deal_s, "device": L.device_name()}), flush=True)


if __name__ == "__main__":
    main()
