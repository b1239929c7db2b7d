#!/usr/bin/env python
"""Throughput of the PCG-OLE expansion hot path on B200.

A step is one party's full PCG-OLE expansion at N=2^20, c=4, t=16 (w=1,
ChaCha8 tree PRG): 4096 keyed half-tree DPF instances of domain 2^17
(2^29 leaves) -> output-layer hash/convert -> gather into the folded
g_ij -> NTT products with the resident a_i images -> x, z.  It yields N OLE
correlations for that party, so the metric is N / step time (corr/s).

  value   whole-job corr/s, inputs (keys, noise) already resident in HBM,
          device-timed with CUDA events on the library's stream; L2 flushed
          (256 MiB write) between timed steps.
  e2e     the same through pcgb_expand_host with pinned host buffers: the
          H2D of the step's keys and noise and the D2H of x and z are inside
          the timed region.
  roofline  the dominant kernel (the fused leaf/out-hash/gather kernel) is
          integer-ALU bound (ChaCha8 ARX); achieved = its algorithmic int ops
          per launch / its mean duration, peak = the ARX throughput probe run
          in this process.  roofline_ntt gives the HBM view of the NTT stage.
  cpu_baseline  the oracle's CPU restatement of the same expansion, timed on
          a bounded sample on this host's cores (rank 0, N=1 only).

`--impl reference` times the reference's CPU implementation of the path (the
oracle port; the reference's own CPU DPF needs emp-tool, absent here) on the
host cores and prints its line with "impl": "reference".

Multi-GPU (torchrun): every rank runs its own expansions (independent
replicas, no data-path collective); value = total correlations of all ranks
/ max over ranks of the timed region.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "pcg-square_b200"))

METRIC = "OLE corr/s at N=2^20,c=4,t=16, bit-exact; serve p50/p99 vs plain one-shot"
N, C_, T_, W_ = 1 << 20, 4, 16, 1
A_SEED = 7
L2_BYTES = 126 * 1024 * 1024
# Published figure for this metric and shape (1x L40S, serial arm,
# GPU_baseline/final_l40s/e2e_arms.csv:32): 2^20 / 192.11 ms.
PUBLISHED = 2 ** 20 / 0.19211


def chacha8_live_ops(ctr, nonce, words):
    """ARX ops (32-bit add, xor, rotate) a ChaCha8 block must execute to
    produce keystream `words` when the key is a 128-bit DPF node followed by
    128 zero bits (the tree PRG and output hash of CPU_baseline/tree_prg.h:80-148).

    Ops whose inputs are all constants fold away, x+0 and x^0 are free, and
    only the backward slice of the requested words is counted -- the same
    pruning the compiler applies to the kernel.  The ALU probe counts every
    op of its (fully live) double rounds the same way, so achieved/peak
    compares like with like."""
    M = 0xFFFFFFFF
    deps = []

    def node(*ins):
        deps.append(tuple(x[1] for x in ins if x[0] == "v"))
        return ("v", len(deps) - 1)

    def add(a, b):
        if a[0] == "c" and b[0] == "c":
            return ("c", (a[1] + b[1]) & M)
        if a == ("c", 0):
            return b
        return a if b == ("c", 0) else node(a, b)

    def xor(a, b):
        if a[0] == "c" and b[0] == "c":
            return ("c", a[1] ^ b[1])
        if a == ("c", 0):
            return b
        return a if b == ("c", 0) else node(a, b)

    def rot(a, r):
        return ("c", ((a[1] << r) | (a[1] >> (32 - r))) & M) if a[0] == "c" else node(a)

    key = [node() for _ in range(4)]
    n_in = len(deps)
    x = ([("c", v) for v in (0x61707865, 0x3320646E, 0x79622D32, 0x6B206574)] + key +
         [("c", 0)] * 4 + [("c", ctr), ("c", 0), ("c", nonce[0]), ("c", nonce[1])])
    init = list(x)

    def qr(a, b, c, d):
        x[a] = add(x[a], x[b]); x[d] = rot(xor(x[d], x[a]), 16)
        x[c] = add(x[c], x[d]); x[b] = rot(xor(x[b], x[c]), 12)
        x[a] = add(x[a], x[b]); x[d] = rot(xor(x[d], x[a]), 8)
        x[c] = add(x[c], x[d]); x[b] = rot(xor(x[b], x[c]), 7)

    for _ in range(4):
        for q in ((0, 4, 8, 12), (1, 5, 9, 13), (2, 6, 10, 14), (3, 7, 11, 15),
                  (0, 5, 10, 15), (1, 6, 11, 12), (2, 7, 8, 13), (3, 4, 9, 14)):
            qr(*q)
    stack = [o[1] for o in (add(x[i], init[i]) for i in words) if o[0] == "v"]
    live = set()
    while stack:
        v = stack.pop()
        if v not in live:
            live.add(v)
            stack.extend(deps[v])
    return sum(1 for v in live if v >= n_in)


# Output hash: nonce "out_hash", counter 0, low 64 bits (words 0-1).
OPS_OUT_HASH = chacha8_live_ops(0, (0x68617368, 0x6F75745F), [0, 1])
# Binary tree node (w = 1): H_0 = words 0-3 of block 0, nonce 0.
OPS_TREE_W1 = chacha8_live_ops(0, (0, 0), [0, 1, 2, 3])
# An unpruned block: 8 rounds x 4 quarter rounds x 12 ops + 4 feed-forward adds.
OPS_FULL_BLOCK = 388


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-verify", action="store_true")
    ap.add_argument("--no-polymul", dest="polymul", action="store_false",
                    help="skip the batched 16 x 2^20 poly-mul measurement")
    ap.add_argument("--no-graph", dest="graph", action="store_false",
                    help="time direct launches instead of CUDA-graph replays")
    ap.add_argument("--arx-variants", action="store_true",
                    help="only the ARX probe with quarter-round adds moved to the FMA pipe")
    ap.add_argument("--polymul-only", action="store_true",
                    help="only the batched poly-mul measurement (profiler captures)")
    ap.add_argument("--serve-requests", type=int, default=1000,
                    help="seeded sample of the 10,000-request serving stream (0 = skip)")
    ap.add_argument("--no-plain-gpu", dest="plain_gpu", action="store_false",
                    help="skip the plain per-stage GPU path (the reference's kernels)")
    # Smaller shapes for profiler captures; the bench line is quoted at the defaults.
    ap.add_argument("--leaf-shape", default=None,
                    help="pin the leaf kernel to THREADSxLEAVES (e.g. 128x8) instead of "
                         "autotuning it (profiler captures need one fixed shape)")
    ap.add_argument("--a0-public", action="store_true",
                    help="all c public polynomials a_0 .. a_{c-1} uniform (the reference "
                         "fixes a_0 = 1)")
    ap.add_argument("--N", type=int, default=N)
    ap.add_argument("--c", type=int, default=C_)
    ap.add_argument("--t", type=int, default=T_)
    return ap.parse_args()


# ---- distributed plumbing ---------------------------------------------------
class Dist:
    def __init__(self):
        self.rank = int(os.environ.get("RANK", 0))
        self.world = int(os.environ.get("WORLD_SIZE", 1))
        self.local = int(os.environ.get("LOCAL_RANK", 0))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            backend = "nccl" if torch.cuda.is_available() else "gloo"
            if backend == "nccl":
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
            self.pg = dist
            self.torch = torch
            self.device = torch.device("cuda", self.local) if backend == "nccl" else None

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x):
        if not self.pg:
            return x
        t = self.torch.tensor([float(x)], dtype=self.torch.float64, device=self.device)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.barrier()
            self.pg.destroy_process_group()


# ---- clocks -----------------------------------------------------------------
class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.gpu)],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
                power.append(float(f[3]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "power_w_max": max(power) if power else None,
                "samples": len(sm), "reasons": sorted(reasons)}


# ---- CPU baseline (oracle port, whole units of work) -------------------------
def host_info():
    """Core count and model of this host (for the CPU figures)."""
    model = None
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    try:
        usable = len(os.sched_getaffinity(0))
    except AttributeError:
        usable = os.cpu_count()
    return {"nproc": usable, "cpu_count": os.cpu_count(), "model": model}


class CpuExpansion:
    """One party's expansion on the host (the oracle's CPU restatement of the
    reference algorithm), cut into c^2 steps of equal work: step k runs every
    key of block k mod c^2 (keyed DPF, output hash, convert, scatter into the
    block's g) and its share of the c + 2c^2 step-4 products (2 or 3 of 36
    at c = 4, so that any c^2 consecutive steps run all of them), from one
    task queue on `threads` threads.  c^2 consecutive steps are exactly one
    expansion; nothing is extrapolated."""

    def __init__(self, shape=None):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle_lib as O
        self.O = O
        self.N, self.c, self.t = shape or (N, C_, T_)
        self.s = O.shape(self.N, self.c, self.t)
        r0, _, cws, cwo = O.deal_keys(self.s, 1000)
        self.material = (r0, cws, cwo, O.public_a(self.s, A_SEED))
        self.blocks = self.c * self.c
        self.products = self.c + 2 * self.c * self.c   # pcg_ole_impl.h:460-483

    def products_of_step(self, k):
        return (self.products * (k + 1)) // self.blocks - (self.products * k) // self.blocks

    def step(self, k, threads):
        r0, cws, cwo, a = self.material
        return self.O.bench_block(self.s, 0, r0, cws, cwo, a, k % self.blocks,
                                  self.products_of_step(k), threads)

    def corr_per_step(self):
        return self.N / self.blocks


def cpu_sample(threads, shape=None):
    """One whole expansion on `threads` host threads (c^2 block steps):
    returns (corr/s, seconds, description)."""
    cpu = CpuExpansion(shape)
    sec = [cpu.step(k, threads) for k in range(cpu.blocks)]
    desc = (f"one whole expansion: {cpu.blocks} blocks x {cpu.t * cpu.t} keys "
            f"(DPF+convert+scatter) and {cpu.products} length-2^{cpu.N.bit_length() - 1} "
            f"products on {threads} threads")
    return cpu.N / sum(sec), sum(sec), desc


def run_reference(args, d):
    if d.rank != 0:
        return
    threads = host_info()["nproc"] or 1
    cpu = CpuExpansion()
    for k in range(args.warmup):
        cpu.step(k, threads)
    sec = [cpu.step(k, threads) for k in range(args.steps)]
    value = cpu.corr_per_step() * args.steps / sum(sec)
    desc = (f"each step one of the {cpu.blocks} blocks of one party's expansion: "
            f"{cpu.t * cpu.t} keys (DPF+convert+scatter) and 2-3 of the {cpu.products} "
            f"products, cycling; {cpu.blocks} steps = one expansion; {threads} threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "corr/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * float(np.mean(sec)), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": value / PUBLISHED, "dtype": "u64", "data": "synthetic",
        "config": {"workload": "pcg-ole expansion N=2^20 c=4 t=16 w=1 chacha8 (one party)",
                   "N": N, "c": C_, "t": T_, "host_threads": threads,
                   "step": f"1/{cpu.blocks} of one expansion (one whole block)"},
        "cpu_baseline": {"value": value, "unit": "corr/s", "cores": threads, "kind": "port",
                         "sample": desc, "host": host_info(),
                         "step_ms": [round(1e3 * x, 2) for x in sec]},
        "e2e": {"value": value, "unit": "corr/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---- our arm -----------------------------------------------------------------
def run_ours(args, d):
    import pcg_b200 as L
    N, C_, T_ = args.N, args.c, args.t
    L.set_device(d.local)
    if args.a0_public:          # all c public polynomials uniform, a_0 too
        a = L.public_a(N, C_ + 1, A_SEED)
    else:                       # the reference's a_0 = 1, a_1 .. a_{c-1} uniform
        a = L.public_a(N, C_, A_SEED)
    e = L.Expander(N, C_, T_, W_, L.PRG_CHACHA8, public_a=a, a0_public=args.a0_public)
    K, levels = e.K, e.levels
    seed = 1000 + d.rank
    d_r0, d_r1 = L.DeviceBuffer(16 * K), L.DeviceBuffer(16 * K)
    d_cws, d_cwo = L.DeviceBuffer(16 * K * levels * e.nk), L.DeviceBuffer(8 * K)
    e.deal_keys_device(seed, d_r0.ptr, d_r1.ptr, d_cws.ptr, d_cwo.ptr)
    pos0, val0 = L.noise(N, C_, T_, seed, 0)
    pos1, val1 = L.noise(N, C_, T_, seed, 1)
    d_pos, d_val = L.to_device(pos0), L.to_device(val0)
    d_x, d_z = L.DeviceBuffer(8 * N), L.DeviceBuffer(8 * N)
    flush = L.DeviceBuffer(2 * L2_BYTES)
    args_dev = (d_r0.ptr, d_cws.ptr, d_cwo.ptr, d_pos.ptr, d_val.ptr, d_x.ptr, d_z.ptr)

    if args.leaf_shape:         # leaf-kernel shape pinned, or tuned for this shape (untimed)
        e.set_leaf_shape(*(int(v) for v in args.leaf_shape.lower().split("x")))
    else:
        e.autotune()
    leaf_tpb, leaf_lpt = e.leaf_shape()
    for _ in range(args.warmup):
        e.expand_device(0, *args_dev)
    L.synchronize()
    # The ALU peak: 15 launches of the ARX probe (about 36 ms each), with
    # the SM clock sampled while they run; the roofline divides by the median.
    probe_clk = Clocks(d.local)
    probe_clk.start()
    probe = sorted(L.arx_peak_samples(15, 16384))
    probe_clocks = probe_clk.stop()
    gops_peak = float(np.median(probe))

    # Per-stage device times: a profiled pass of the same steps (direct
    # launches, events between the stages), not part of the timed region.
    e.set_profiling(args.steps)
    for i in range(args.steps):
        L.lib.pcgb_memset(flush.ptr, i & 0xFF, flush.nbytes, None)
        e.expand_device(0, *args_dev)
    stages = e.stage_times()
    e.set_profiling(0)
    if args.graph:
        # Timed region replays the expansion as one CUDA graph per step
        # (first call direct, second captures; both untimed).
        e.set_graph(True)
        for _ in range(2):
            e.expand_device(0, *args_dev)
    L.synchronize()

    evs = [(L.Event(), L.Event()) for _ in range(args.steps)]
    clocks = Clocks(d.local)
    d.barrier()
    L.synchronize()
    clocks.start()
    launches0 = L.launch_count()
    for i in range(args.steps):
        L.lib.pcgb_memset(flush.ptr, i & 0xFF, flush.nbytes, None)  # L2 flush, not timed
        evs[i][0].record()
        e.expand_device(0, *args_dev)
        evs[i][1].record()
    L.synchronize()
    launches = L.launch_count() - launches0
    clk = clocks.stop()
    step_ms = [s.elapsed_ms(t) for s, t in evs]
    e.set_graph(False)
    total_ms = float(np.sum(step_ms))
    total_ms_max = d.max(total_ms)
    d.barrier()
    value = N * args.steps * d.world / (total_ms_max / 1e3)

    # Correctness check (untimed): party 1 on the same keys, then the OLE
    # relation z0 + z1 = x0 * x1 over the whole ring, checked slot by slot on
    # the device (pcgb_verify_ole_device) and, independently, on the host
    # through the library's product of x0 and x1.
    verified = None
    if not args.no_verify:
        d_pos1, d_val1 = L.to_device(pos1), L.to_device(val1)
        d_x1, d_z1 = L.DeviceBuffer(8 * N), L.DeviceBuffer(8 * N)
        e.expand_device(1, d_r1.ptr, d_cws.ptr, d_cwo.ptr, d_pos1.ptr, d_val1.ptr, d_x1.ptr,
                        d_z1.ptr)
        d_bad = L.DeviceBuffer(8)
        L.verify_ole_device(N, d_x.ptr, d_z.ptr, d_x1.ptr, d_z1.ptr, d_bad.ptr)
        bad_slots = int(d_bad.download(np.uint64, 1)[0])
        x0, z0 = d_x.download(np.uint64, N), d_z.download(np.uint64, N)
        x1, z1 = d_x1.download(np.uint64, N), d_z1.download(np.uint64, N)
        prod, _ = L.poly_mul_u64_gpuntt(x0, x1, 1, N)
        zs = z0 + z1
        zs = np.where(zs >= np.uint64(L.P), zs - np.uint64(L.P), zs)
        verified = bool((prod == zs).all()) and bad_slots == 0

    # e2e through the public host API with pinned buffers.
    e2e = None
    if args.e2e_steps > 0:
        try:
            import torch
            pin = lambda n: torch.empty(n, dtype=torch.int64, pin_memory=True)
        except Exception:
            pin = None
        h_r0 = d_r0.download(np.uint64, 2 * K)
        h_cws = d_cws.download(np.uint64, 2 * K * levels)
        h_cwo = d_cwo.download(np.uint64, K)
        keep = []

        def host_set():
            """Inputs and output buffers of one step (pinned when torch can)."""
            arrs = [h_r0, h_cws, h_cwo, pos0, val0, np.zeros(N, np.uint64),
                    np.zeros(N, np.uint64)]
            if pin:
                for i, arr in enumerate(arrs):
                    t = pin(arr.size)
                    v = t.numpy().view(np.uint64)
                    v[:] = arr
                    keep.append(t)
                    arrs[i] = v
            return arrs

        # Two host buffer sets, alternating: each step copies its own inputs
        # in and its own x, z out, while pcgb_expand_host_async overlaps one
        # step's copies with the next step's kernels.
        sets = [host_set(), host_set()]
        ptrs = [[h.ctypes.data for h in hs] for hs in sets]
        h2d = sum(h.nbytes for h in sets[0][:5])
        d2h = sets[0][5].nbytes + sets[0][6].nbytes
        lib = L.lib

        def check(rc):
            if rc:
                raise RuntimeError(lib.pcgb_last_error().decode())

        for k in range(2):                       # warm both slots
            check(lib.pcgb_expand_host_async(e.h, 0, *ptrs[k]))
        check(lib.pcgb_expander_wait(e.h))
        s, t = L.Event(), L.Event()
        d.barrier()                              # all ranks start together
        L.synchronize()
        s.record()
        for i in range(args.e2e_steps):
            check(lib.pcgb_expand_host_async(e.h, 0, *ptrs[i & 1]))
        check(lib.pcgb_expander_wait(e.h))
        t.record()
        e2e_ms = d.max(s.elapsed_ms(t))
        same = bool((sets[0][5] == sets[1][5]).all() and (sets[0][6] == sets[1][6]).all())
        e2e = {"value": N * args.e2e_steps * d.world / (e2e_ms / 1e3), "unit": "corr/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "pinned": bool(pin), "api": "pcgb_expand_host_async (two host buffer sets)",
               "outputs_agree": same}

    # Roofline of the dominant kernel (fused leaf gather), ALU bound.
    leaf_ms = float(np.mean([s[1] for s in stages])) if stages else None
    D = 1 << e.levels
    S = leaf_lpt                # leaves per thread of the leaf kernel
    # Per leaf: one output hash; per internal node below the frontier (S - 1
    # of them per S leaves): one tree block.
    ops = K * D * (OPS_OUT_HASH + OPS_TREE_W1 * (S - 1) / S)
    ops_full = K * D * (2 - 1 / S) * OPS_FULL_BLOCK
    achieved = ops / (leaf_ms * 1e-3) / 1e12 if leaf_ms else None
    peak = gops_peak / 1e3
    # DRAM traffic of one launch: frontier nodes read (one per S leaves) and
    # g' words written, at the per-node and per-word rates of the ncu capture.
    traffic = (LEAF_READ_BYTES_PER_NODE * K * D / S + LEAF_WRITE_BYTES_PER_WORD * e.Q * N)
    roofline = {"bound": "int_alu",
                "kernel": f"leaf_gather_kernel<1,{S.bit_length() - 1},chacha8>",
                "achieved": achieved, "peak": peak, "unit": "Tops/s",
                "frac": achieved / peak if achieved else None,
                "traffic": traffic,
                "traffic_unit": "bytes per launch: frontier reads + g' writes at the rates "
                                "of the ncu capture (profiles/leaf_gather_chacha8_*.txt)",
                "algorithmic_bytes": 16 * K * D / S + 8 * e.Q * N,
                "peak_source": "median of 15 launches of the ARX probe (pcgb_arx_peak_samples) "
                               "in this run; MEASURED_PEAKS.json has no integer-ALU figure",
                "peak_spread": {"min": probe[0] / 1e3, "median": peak, "max": probe[-1] / 1e3,
                                "launches": len(probe), "clocks": probe_clocks},
                "ops_per_launch": ops, "ops_per_block": {"out_hash": OPS_OUT_HASH,
                                                         "tree": OPS_TREE_W1},
                "frac_at_full_blocks": (ops_full / (leaf_ms * 1e-3) / 1e12 / peak
                                        if leaf_ms else None),
                "full_block_ops": OPS_FULL_BLOCK,
                "launch_ms": leaf_ms}
    ntt_ms = float(np.mean([s[3] for s in stages])) if stages else None
    Q = e.Q
    ntt_bytes = 8 * N * (4 * Q + 3)
    roofline_ntt = {"bound": "hbm", "achieved": ntt_bytes / (ntt_ms * 1e-3) / 1e9 if ntt_ms else None,
                    "peak": hbm_peak(), "peak_source": hbm_peak_source()[1], "unit": "GB/s",
                    "bytes_per_step": ntt_bytes,
                    "stage_ms": ntt_ms}
    if roofline_ntt["achieved"]:
        roofline_ntt["frac"] = roofline_ntt["achieved"] / roofline_ntt["peak"]

    cpu = None
    if d.world == 1 and d.rank == 0 and not args.no_cpu_baseline:
        host = host_info()
        threads = host["nproc"] or 1
        v, sec, desc = cpu_sample(threads, shape=(N, C_, T_))
        cpu = {"value": v, "unit": "corr/s", "cores": threads, "kind": "port",
               "sample": desc, "sample_seconds": sec, "host": host}
        # The reference's CPU bench runs one thread per party (its OpenMP
        # pragma is not compiled in): one whole block step on one thread
        # (its 256 keys and 2 of the 36 products).
        one = CpuExpansion((N, C_, T_))
        sec1 = one.step(0, 1)
        cpu["one_thread"] = {"value": one.corr_per_step() / sec1, "cores": 1,
                             "sample": "one whole block (1/16 of the expansion's keys) and 2 "
                                       "of its 36 products on 1 thread",
                             "sample_seconds": sec1}

    serve = None
    if d.world == 1 and args.serve_requests > 0:
        serve = run_serving(L, args.serve_requests)
    polymul = run_polymul(L) if d.world == 1 and args.polymul else None

    # The plain per-stage GPU path (the >=5x denominator): the reference's
    # own kernels, compiled unmodified (oracle/_ref), driven one request at a
    # time like GPU_baseline/e2e_full_bench.cu's serial arm.  A baseline leg
    # after the timed region; of this library only the step-4 products run
    # in it (the reference tree lacks its GPU-NTT backend).
    plain = None
    if d.world == 1 and args.plain_gpu and N == 1 << 20:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import plain_gpu_bench
        plain = plain_gpu_bench.run(L, N, C_, T_, iters=2)
        if plain:
            plain["value_over_plain"] = value / plain["corr_per_s"]
            if e2e:
                plain["e2e_over_plain"] = e2e["value"] / plain["corr_per_s"]
            if serve:
                plain["served_capacity_over_plain"] = (
                    serve["headline_saturating"]["batched"]["corr_per_s"] / plain["corr_per_s"])

    if d.rank == 0:
        stage_means = [float(np.mean([s[i] for s in stages])) for i in range(4)] if stages else None
        line = {
            "metric": METRIC, "value": value, "unit": "corr/s", "n_gpus": d.world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": value / PUBLISHED, "dtype": "u64",
            "data": "synthetic",
            "config": {"workload": f"pcg-ole expansion N=2^{N.bit_length() - 1} c={C_} t={T_} "
                                   "w=1 chacha8 (one party, keyed DPF from the GPU dealer)",
                       "N": N, "c": C_, "t": T_, "w": W_, "keys": K, "leaves": K * D,
                       "public_a": ("a_0 .. a_{c-1} uniform" if args.a0_public
                                    else "a_0 = 1, a_1 .. a_{c-1} uniform"),
                       "parallelism": f"replicas x{d.world}",
                       "l2": "flushed between timed steps (256 MiB write)",
                       "cuda_graph": bool(args.graph), "leaf_cta_threads": leaf_tpb,
                       "leaf_leaves_per_thread": leaf_lpt,
                       "leaf_shape": "pinned" if args.leaf_shape else "autotuned",
                       "vs_baseline_ref": "1x L40S serial arm 5.46M corr/s "
                                          "(GPU_baseline/final_l40s/e2e_arms.csv:32)"},
            "stage_ms": dict(zip(["tops", "leaf_gather", "x", "ntt"], stage_means))
            if stage_means else None,
            "bit_exact_ole_relation": verified,
            "gpu_launches": int(launches),
            "clocks": clk, "roofline": roofline, "roofline_ntt": roofline_ntt,
            "e2e": e2e, "cpu_baseline": cpu, "serve": serve, "poly_mul": polymul,
            "plain_gpu": plain,
        }
        print(json.dumps(line), flush=True)
    e.close()


def run_arx_variants(L):
    """The ARX probe (two ChaCha8 states per thread, every SM full) with a
    chosen set of the quarter round's four adds issued as multiply-adds on
    the FMA pipe; median T int-ops/s of 7 launches per variant."""
    masks = [("none", 0x00000000), ("1 of 8 (add 0, every other QR)", 0x10101010),
             ("add 0 (1/4)", 0x11111111), ("add 1 (1/4)", 0x22222222),
             ("adds 0,1 (1/2)", 0x33333333), ("adds 0,2 (1/2)", 0x55555555),
             ("3 of 8 (adds 0,2 / 0)", 0x15151515), ("3 of 4", 0x77777777),
             ("all 4", 0xFFFFFFFF)]
    out = []
    for name, m in masks:
        g = L.arx_peak_variant(m)
        out.append({"adds_on_fma": name, "mask": f"{m:08x}",
                    "tops_median": float(np.median(g)) / 1e3})
    return out


def run_polymul(L, batch=16, logN=20, steps=10, warmup=3, seed=11):
    """Batched negacyclic product c = a*b mod (X^N + 1, p), 16 x 2^20 words of
    seeded uniform [0, p) inputs, through pcgb_poly_mul_device (forward column
    and row passes of both operands, fused pointwise product and inverse row
    pass, inverse column pass).  The operands (2 x 128 MiB) exceed L2, so no
    flush is needed.  Algorithmic HBM bytes: read a and b, write c."""
    N = 1 << logN
    rng = np.random.default_rng(seed)
    a = rng.integers(0, L.P, batch * N, dtype=np.uint64)
    b = rng.integers(0, L.P, batch * N, dtype=np.uint64)
    d_a, d_b, d_c = L.to_device(a), L.to_device(b), L.DeviceBuffer(8 * batch * N)
    for _ in range(warmup):
        L.poly_mul_device(d_c.ptr, d_a.ptr, d_b.ptr, batch, N)
    L.synchronize()
    evs = [(L.Event(), L.Event()) for _ in range(steps)]
    for s0, s1 in evs:
        s0.record()
        L.poly_mul_device(d_c.ptr, d_a.ptr, d_b.ptr, batch, N)
        s1.record()
    L.synchronize()
    ms = [s0.elapsed_ms(s1) for s0, s1 in evs]
    med = float(np.median(ms))
    nbytes = 24 * batch * N
    out = {"workload": f"{batch} x 2^{logN} negacyclic products, uniform [0,p) inputs",
           "ms_median": med, "ms_min": float(min(ms)),
           "roofline": {"bound": "hbm", "achieved": nbytes / (med * 1e-3) / 1e9,
                        "peak": hbm_peak(), "peak_source": hbm_peak_source()[1],
                        "unit": "GB/s", "bytes": nbytes}}
    out["roofline"]["frac"] = out["roofline"]["achieved"] / out["roofline"]["peak"]
    # Per-pass accounting (8 B read + 8 B written per word in each of the two
    # passes of the three transforms, pointwise fused): 96 B per element.
    out["roofline"]["bytes_per_pass_accounting"] = 96 * batch * N
    out["roofline"]["frac_per_pass_accounting"] = (96 * batch * N / (med * 1e-3) / 1e9 /
                                                   out["roofline"]["peak"])
    out["roofline"]["bound_by"] = ("64-bit integer multiplies (FMA-heavy pipe, math-pipe "
                                   "throttle the top stall; profiles/ntt_polymul_16x2e20.txt)")

    # Mixed lengths in one call (five launches for the batch): 6 x 2^20,
    # 5 x 2^18, 5 x 2^16, interleaved, through pcgb_poly_mul_device_multi.
    import ctypes as C
    sizes = [1 << 20, 1 << 16, 1 << 18] * 5 + [1 << 20]
    bufs = [(L.to_device(rng.integers(0, L.P, n, dtype=np.uint64)),
             L.to_device(rng.integers(0, L.P, n, dtype=np.uint64)), L.DeviceBuffer(8 * n))
            for n in sizes]
    arr = lambda k: (C.c_void_p * len(sizes))(*[bb[k].ptr for bb in bufs])
    pa, pb, pc, pn = arr(0), arr(1), arr(2), (C.c_int * len(sizes))(*sizes)

    def multi():
        rc = L.lib.pcgb_poly_mul_device_multi(len(sizes), pc, pa, pb, pn, None)
        if rc:
            raise RuntimeError(L.lib.pcgb_last_error().decode())

    for _ in range(warmup):
        multi()
    L.synchronize()
    l0 = L.launch_count()
    multi()
    L.synchronize()
    launches = L.launch_count() - l0
    for s0, s1 in evs:
        s0.record()
        multi()
        s1.record()
    L.synchronize()
    mm = float(np.median([s0.elapsed_ms(s1) for s0, s1 in evs]))
    mbytes = 24 * sum(sizes)
    out["mixed"] = {"workload": "16 products: 6 x 2^20, 5 x 2^18, 5 x 2^16 in one call",
                    "ms_median": mm, "launches_per_call": int(launches),
                    "achieved_gbs": mbytes / (mm * 1e-3) / 1e9,
                    "frac_hbm": mbytes / (mm * 1e-3) / 1e9 / hbm_peak()}
    return out


SERVE_SHAPES = [(1 << lg, c, t) for lg in (14, 16, 18, 20, 22) for c in (2, 4) for t in (8, 16, 32)]


def run_serving(L, n_req, seed=2025, util=0.85, n_sat=None):
    """Serving stream (N in {2^14..2^22}, c in {2,4}, t in {8,16,32}, Poisson
    arrivals): continuous batching (4 streams) vs one request at a time on the
    same seeded trace.  Every request deals fresh keys and noise on the GPU;
    the a_i plans of all 30 shapes are resident before the trace starts.

    Three traces, each run by both servers:
      latency     arrivals at `util` of one-at-a-time capacity (p50/p99);
      saturating  the same requests, all queued at t = 0: the served
                  capacity (corr/s = correlations / makespan);
      headline    n_sat requests of N=2^20, c=4, t=16 queued at t = 0."""
    rng = np.random.default_rng(seed)
    n_sat = n_sat or max(16, min(64, n_req // 8))
    batched = L.Server(n_streams=4, a_seed=A_SEED)
    single = L.Server(n_streams=1, max_in_flight=1, a_seed=A_SEED)
    for shp in SERVE_SHAPES:
        batched.prepare(*shp)
        single.prepare(*shp)
    # Warm both servers on every shape (first launches, pool growth), then
    # calibrate the arrival rate on the exact mean one-at-a-time service time
    # of the uniform shape mix: one timed request per shape.
    warm = [(N, c, t, 0, 900 + i, 0.0) for i, (N, c, t) in enumerate(SERVE_SHAPES)]
    batched.run_trace(warm)
    single.run_trace(warm)
    res = single.run_trace([(N, c, t, 0, 1000 + i, 0.0) for i, (N, c, t) in enumerate(SERVE_SHAPES)])
    svc = float(np.mean([r.done_s - r.start_s for r in res]))
    rate = util / svc
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_req))
    trace = []
    for i in range(n_req):
        N, c, t = SERVE_SHAPES[rng.integers(len(SERVE_SHAPES))]
        trace.append((N, c, t, int(rng.integers(2)), int(rng.integers(1, 2**62)),
                      float(arrivals[i])))
    saturating = [(N, c, t, p, sd, 0.0) for N, c, t, p, sd, _ in trace]
    headline = [(1 << 20, 4, 16, 0, 5000 + i, 0.0) for i in range(n_sat)]

    def served(srv, tr):
        rs = srv.run_trace(tr, timeout_s=1800)
        lat = np.array([r.done_s - r.submit_s for r in rs]) * 1e3
        span = max(r.done_s for r in rs) - min(r.submit_s for r in rs)
        return rs, {"p50_ms": float(np.percentile(lat, 50)),
                    "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()),
                    "corr_per_s": float(sum(x[0] for x in tr) / span), "makespan_s": span}

    out = {"latency": {}, "saturating": {}, "headline_saturating": {}}
    digests = {}
    for name, srv in (("batched", batched), ("one_at_a_time", single)):
        rs, out["latency"][name] = served(srv, trace)
        digests[name] = [(r.digest_x, r.digest_z) for r in rs]
        rs, out["saturating"][name] = served(srv, saturating)
        digests[name + "_sat"] = [(r.digest_x, r.digest_z) for r in rs]
        _, out["headline_saturating"][name] = served(srv, headline)
    batched.close()
    single.close()
    out["bit_exact_alone_vs_mix"] = (digests["batched"] == digests["one_at_a_time"] ==
                                     digests["batched_sat"] == digests["one_at_a_time_sat"])
    out["requests"] = n_req
    out["headline_requests"] = n_sat
    out["arrival_rate_per_s"] = rate
    out["mean_service_ms_one_at_a_time"] = svc * 1e3
    out["trace"] = (f"seeded {n_req}-request sample of the 10,000-request stream: N uniform over "
                    "2^14..2^22, c in {2,4}, t in {8,16,32}; latency trace with Poisson "
                    f"arrivals at {util:.0%} of one-at-a-time capacity; saturating trace: the "
                    "same requests all queued at t = 0")
    out["speedup_p99"] = (out["latency"]["one_at_a_time"]["p99_ms"] /
                          out["latency"]["batched"]["p99_ms"])
    out["capacity_gain"] = (out["saturating"]["batched"]["corr_per_s"] /
                            out["saturating"]["one_at_a_time"]["corr_per_s"])
    return out


# DRAM bytes of one leaf-gather launch, from an ncu capture of the N=2^18,
# c=4, t=16 case at 128 threads x 8 leaves per thread: 269.8 MB read for the
# 4096 x 2^15 / 8 frontier nodes (16 B each), 14.8 MB written for the
# 10 x 2^18 g' words (8 B each; part of them still in L2 at kernel end).
LEAF_READ_BYTES_PER_NODE = 269.8e6 / (4096 * 2 ** 15 / 8)
LEAF_WRITE_BYTES_PER_WORD = 14.8e6 / (10 * 2 ** 18)


def hbm_peak():
    """HBM copy bandwidth in GB/s: the measured figure of this pool's B200s
    (MEASURED_PEAKS.json) when present, else the pool's earlier measured
    fallback of 6650 GB/s."""
    return hbm_peak_source()[0]


def hbm_peak_source():
    try:
        return (float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]),
                "MEASURED_PEAKS.json hbm_gbs (measured)")
    except Exception:
        return 6650.0, "fallback 6650 GB/s (MEASURED_PEAKS.json absent)"


def main():
    args = parse()
    d = Dist()
    try:
        if args.impl == "reference":
            run_reference(args, d)
        elif args.arx_variants:
            import pcg_b200 as L
            if d.rank == 0:
                print(json.dumps({"arx_variants": run_arx_variants(L)}), flush=True)
        elif args.polymul_only:
            import pcg_b200 as L
            if d.rank == 0:
                print(json.dumps({"poly_mul": run_polymul(L, steps=args.steps,
                                                          warmup=args.warmup)}), flush=True)
        else:
            run_ours(args, d)
    finally:
        d.close()


if __name__ == "__main__":
    main()
