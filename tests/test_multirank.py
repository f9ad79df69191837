"""The N > 1 paths on the CPU with gloo.

* The bench runs independent replicas (no data-path collective): the max over ranks of
  the timed region, the whole-job rate, and the reference arm that only rank 0 runs.
* A domain decomposed along y (dynfd3dcuda_b200.decomp.DistributedSlab): the routing of
  the halo messages between three ranks, with stand-ins for the library's pack and
  unpack that move one field of column numbers, so that every ghost column must end up
  holding the global column it stands for.
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


def _slab_worker(rank, world, port, out):
    import datetime

    import numpy as np
    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    from dynfd3dcuda_b200.decomp import DistributedSlab

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    nj, nz = 5, 4
    j0 = rank * nj
    # one field (nz, nj + 6): own columns hold their global column number, ghosts NaN
    f = np.full((nz, nj + 6), np.nan)
    f[:, 3:3 + nj] = np.arange(j0, j0 + nj)[None, :]

    def pack(what, side, t):
        cols = f[:, 3:6] if side == 0 else f[:, nj:nj + 3]
        t.copy_(torch.from_numpy(np.ascontiguousarray(cols, np.float32).ravel()))

    def unpack(what, side, t):
        cols = t.numpy().reshape(nz, 3)
        if side == 0:
            f[:, 0:3] = cols
        else:
            f[:, nj + 3:nj + 6] = cols

    slab = DistributedSlab(None, dist, nfloats=nz * 3, pack=pack, unpack=unpack)
    slab.exchange(0)
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, f[0].tolist()))


def test_slab_halo_routing_gloo():
    import math

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    world, nj = 3, 5
    procs = [ctx.Process(target=_slab_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    for r in range(world):
        row = res[r]
        j0 = r * nj
        assert row[3:3 + nj] == list(range(j0, j0 + nj))
        # ghosts beside a neighbour hold its columns; at the domain's ends they stay unset
        if r > 0:
            assert row[0:3] == [j0 - 3, j0 - 2, j0 - 1]
        else:
            assert all(math.isnan(v) for v in row[0:3])
        if r < world - 1:
            assert row[nj + 3:nj + 6] == [j0 + nj, j0 + nj + 1, j0 + nj + 2]
        else:
            assert all(math.isnan(v) for v in row[nj + 3:nj + 6])
