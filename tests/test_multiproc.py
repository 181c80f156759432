"""Multi-rank plumbing of bench.py on CPU (gloo, world size 2).

The path does not shard inside a pair: N GPUs run N independent replicas and
the bench reports the units all ranks processed divided by the slowest
rank's time.  These tests cover that reduction and the reference arm's
rank handling (rank 0 prints one line, the others exit 0 without work)."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        ms = [12.5, 20.0][rank]  # the second rank is the slow one
        m = bench.max_over_ranks_of(dist, ms)
        q.put((rank, m, bench.replica_value(world, 199, 5, m)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert [g[1] for g in got] == [20.0, 20.0]
    # 2 ranks x 199 pairs x 5 steps in 20 ms
    assert all(abs(g[2] - 2 * 199 * 5 / 0.020) < 1e-6 for g in got)


def test_reference_arm_two_ranks():
    env = dict(os.environ, OMP_NUM_THREADS="2")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0", "--frames", "3",
           "--cpu-seconds", "0.5"]
    out = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
