"""Multi-rank plumbing of bench.py on CPU: two gloo ranks on 127.0.0.1.

bench.py runs one process per GPU under torch.distributed.run, times on each
rank and reports the maximum over ranks; only rank 0 prints.  The expansion
shards as independent replicas (no data-path collective), so the host logic
is all that needs covering here: the max-reduction, the barrier and the
reference arm's rank-0-only behaviour.
"""
import json
import multiprocessing as mp
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    d = bench.Dist()
    try:
        got = d.max(10.0 * rank + 3.0)
        d.barrier()
        q.put((rank, got))
    finally:
        d.close()


def test_dist_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = dict(q.get(timeout=5) for _ in range(2))
    assert res == {0: 13.0, 1: 13.0}


def test_reference_arm_prints_once_under_torchrun():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py",
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] == "port"


if __name__ == "__main__":
    sys.exit(pytest.main([__file__, "-q"]))


def _z_rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import numpy as np
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        sys.path.insert(0, os.path.join(ROOT, "pcg-square_b200"))
        from pcg_b200 import P
        from pcg_b200.shard import allreduce_z
        z = np.random.default_rng(rank).integers(P - 1000, P, 257, dtype=np.uint64)
        z[:5] = [0, 1, P - 1, P - 2, rank]
        t = torch.from_numpy(z.view(np.int64).copy())
        allreduce_z(t)
        q.put((rank, t.numpy().view(np.uint64).tolist()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [3, 8])
def test_shard_z_sum_is_exact_beyond_four_ranks(world):
    """pcg_b200.shard.allreduce_z: the partial z's (values near p, where a
    plain uint64 all-reduce of 8 of them would overflow) sum mod p exactly on
    every rank."""
    import numpy as np
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_z_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=300) for _ in range(world))
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    sys.path.insert(0, os.path.join(ROOT, "pcg-square_b200"))
    from pcg_b200 import P
    parts = []
    for r in range(world):
        z = np.random.default_rng(r).integers(P - 1000, P, 257, dtype=np.uint64)
        z[:5] = [0, 1, P - 1, P - 2, r]
        parts.append([int(v) for v in z])
    want = [sum(col) % P for col in zip(*parts)]
    for r in range(world):
        assert got[r] == want, r
