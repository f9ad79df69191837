"""A domain decomposed along y into slabs with halo exchange between RK stages equals the
same domain run whole (the reference's multi-rank path, mod_mpi.cu / mod_mpi_fault.cu).

The slabs run in one process on cuda:0, each its own context, the messages moved through
device buffers between stages (no kernel of one slab waits on another's).  Compared with
the single context after a number of steps: the wavefield of every slab's own columns and
the on-fault planes.  The rupture sensor is left out of the comparison: like the
reference's per-rank sensor it is not evaluated within two columns of a slab's ends (it
feeds only its output)."""
import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    s = np.abs(b).max()
    return np.abs(a - b).max() / (s if s > 0 else 1.0)


@pytest.mark.parametrize("name,PY,steps", [("sw_flat", 2, 30), ("sw_flat", 4, 30), ("rs_flat", 2, 30),
                                           ("sw_curved", 2, 25), ("media_cj", 2, 40)])
def test_slabs_equal_whole_domain(name, PY, steps):
    import dynfd3dcuda_b200 as dfd
    from dynfd3dcuda_b200.decomp import LocalSlabs

    p, fx, st, layers, w0, meta = cases.get_case(name)
    whole = dfd.Simulation(p, fx, st, layers)
    slabs = LocalSlabs(p, fx, st, layers, PY)
    for it in range(steps):
        for irk in range(4):
            whole.stage(it, irk)
        slabs.step(it)
    whole.synchronize()
    slabs.synchronize()
    W, Ws = whole.wave(), slabs.wave()
    errs = {"wave": rel(Ws[..., 3:-3], W[..., 3:-3])}
    for nm in ("slip", "Vs1", "Vs2", "Tn", "Ts1", "Ts2", "State", "init_t0"):
        errs[nm] = rel(slabs.fault(nm), whole.fault(nm))
    print(name, PY, {k: f"{v:.1e}" for k, v in errs.items()})
    for k, v in errs.items():
        assert v < 1e-6, (k, v)
    whole.close()
    slabs.close()


def _dist_worker(rank, world, port, name, steps, out):
    import datetime
    import os
    import sys

    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "tests", "golden")):
        sys.path.insert(0, p)
    import cases as cs
    import dynfd3dcuda_b200 as dfd
    from dynfd3dcuda_b200.decomp import DistributedSlab, slab_job

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    p, fx, st, layers, w0, meta = cs.get_case(name)
    sim = dfd.Simulation(slab_job(p, world, rank), fx, st, layers, device=0)
    slab = DistributedSlab(sim, dist, device="cuda:0")
    slab.setup()
    for it in range(steps):
        slab.step(it)
    sim.synchronize()
    res = {"wave": sim.wave()[..., 3:-3], "slip": sim.fault("slip"), "Vs1": sim.fault("Vs1")}
    sim.close()
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, res))


def test_distributed_slabs_gloo_on_one_gpu():
    """Two processes, each one slab on cuda:0, the messages through host memory by gloo
    (no kernel of one process waits on the other's: the host exchanges between stages)."""
    import socket

    import torch.multiprocessing as mp

    import dynfd3dcuda_b200 as dfd

    name, steps, world = "sw_flat", 20, 2
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_dist_worker, args=(r, world, port, name, steps, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=600) for _ in procs)
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    p, fx, st, layers, w0, meta = cases.get_case(name)
    whole = dfd.Simulation(p, fx, st, layers)
    for it in range(steps):
        for irk in range(4):
            whole.stage(it, irk)
    whole.synchronize()
    W = whole.wave()[..., 3:-3]
    Ws = np.concatenate([res[r]["wave"] for r in range(world)], axis=-1)
    assert rel(Ws, W) < 1e-6
    for nm in ("slip", "Vs1"):
        a = np.concatenate([res[r][nm] for r in range(world)], axis=-1)
        assert rel(a, whole.fault(nm)) < 1e-6, nm
    whole.close()
