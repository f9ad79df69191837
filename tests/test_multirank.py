"""The N > 1 path on the CPU with gloo, world size 2.

The time step does not shard (each rank runs an independent replica; no data-path
collective), so what multi-rank code exists is the bench's bookkeeping: the max over ranks
of the timed region, the whole-job rate, and the reference arm that only rank 0 runs.
"""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    # each rank timed its own replica; the job is as slow as the slowest rank
    ms = [120.0, 150.0][rank]
    m = bench.max_over_ranks(ms, dist, "cpu")
    rate = bench.job_rate(1000, 10, world, m / 1e3)
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, m, rate))


def test_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [150.0, 150.0]
    # 2 replicas x 1000 nodes x 10 steps in 0.15 s
    assert res[0][2] == pytest.approx(2 * 1000 * 10 / 0.15 / 1e9)
    assert res[0][2] == res[1][2]


def test_reference_arm_rank0_only():
    """Under torchrun with two ranks the reference arm prints one line, from rank 0."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
           "--warmup", "0", "--config", "flat"]
    env = dict(os.environ, OMP_NUM_THREADS="4")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["steps"] == 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"
    assert line["value"] > 0
