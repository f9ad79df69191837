"""A rupture domain decomposed along y into slabs, one context per slab.

The reference splits its domain over MPI ranks (PX x PY x PZ, set_params.cu) and, before
every RK stage, swaps the three boundary columns of the wavefield and of the fault's
split-node state with the neighbouring ranks (exchange_wave and exchange_fault,
mod_mpi.cu:104-281, mod_mpi_fault.cu:87-237); the metric's ghost columns are swapped once
(exchange_array, main.cu:277-297).  Here a domain splits along y into PY slabs of NY / PY
columns: each slab is a context built from the domain's global job and input arrays with
slabs_y = PY and its slab_y (the PML, the sponge, the masks and the output files follow the slab's
place), and the library packs and unpacks the messages in device memory
(dfd_halo_pack / dfd_halo_unpack).  How a message travels is the caller's:

  LocalSlabs        every slab in this process (one GPU or several): device-to-device
                    copies through one buffer per slab pair.
  DistributedSlab   one slab per process of a torch.distributed group: device tensors
                    with NCCL (the messages cross NVLink), host tensors with gloo.

Stepping goes stage by stage: exchange(irk), then dfd_stage on every slab.
"""
import numpy as np

from . import HALO_SETUP, Simulation


def slab_job(job, PY, rank):
    """The job of slab rank of a domain split into PY slabs along y."""
    j = dict(job)
    j["slabs_y"] = int(PY)
    j["slab_y"] = int(rank)
    return j


class LocalSlabs:
    """The PY slabs of one domain in this process; device d of devices holds slab d."""

    def __init__(self, job, fxyz, stress, layers, PY, devices=None):
        import torch

        self.PY = PY
        devices = devices or [0] * PY
        self.sims = [Simulation(slab_job(job, PY, r), fxyz, stress, layers, device=devices[r]) for r in range(PY)]
        n = max(s.halo_floats() for s in self.sims)
        self._bufs = [torch.empty(n, dtype=torch.float32, device=f"cuda:{devices[r]}") for r in range(PY - 1)]
        self.exchange(HALO_SETUP)

    def exchange(self, what):
        """Swap the boundary columns of every neighbouring pair (what: HALO_SETUP or the
        RK stage about to run)."""
        for r in range(self.PY - 1):
            lo, hi, b = self.sims[r], self.sims[r + 1], self._bufs[r]
            lo.halo_pack(what, 1, b.data_ptr())
            lo.synchronize()
            hi.halo_unpack(what, 0, b.data_ptr())
            hi.synchronize()
            hi.halo_pack(what, 0, b.data_ptr())
            hi.synchronize()
            lo.halo_unpack(what, 1, b.data_ptr())
            lo.synchronize()

    def step(self, it):
        for irk in range(4):
            self.exchange(irk)
            for s in self.sims:
                s.stage(it, irk)

    def run(self, it0, nsteps):
        for it in range(it0, it0 + nsteps):
            self.step(it)

    def synchronize(self):
        for s in self.sims:
            s.synchronize()

    def fault(self, name):
        """An on-fault plane (NZ, NY) of the whole domain."""
        return np.concatenate([s.fault(name) for s in self.sims], axis=-1)

    def wave(self):
        """The wavefield (9, nx, nz, NY + 6) of the whole domain, ghost columns at its ends."""
        parts = [s.wave() for s in self.sims]
        mid = [p[..., 3:-3] for p in parts]
        return np.concatenate([parts[0][..., :3]] + mid + [parts[-1][..., -3:]], axis=-1)

    def close(self):
        for s in self.sims:
            s.close()


class DistributedSlab:
    """Slab dist.get_rank() of a domain split over the ranks of a torch.distributed group.

    With the NCCL backend the messages are device tensors (packed and sent without leaving
    the GPU); with gloo they are staged through host memory.  pack(what, side, tensor) and
    unpack(what, side, tensor) default to the slab's library calls; a test may pass its own
    to check the message routing without a GPU."""

    def __init__(self, sim, dist, device=None, nfloats=None, pack=None, unpack=None):
        import torch

        self.sim, self.dist = sim, dist
        self.rank, self.size = dist.get_rank(), dist.get_world_size()
        self.cuda = dist.get_backend() == "nccl"
        n = nfloats if nfloats is not None else sim.halo_floats()
        where = device if self.cuda else "cpu"
        self._send = [torch.empty(n, dtype=torch.float32, device=where) for _ in range(2)]
        self._recv = [torch.empty(n, dtype=torch.float32, device=where) for _ in range(2)]
        self._dev = None
        if not self.cuda and sim is not None:
            self._dev = torch.empty(n, dtype=torch.float32, device=device)
        self._pack = pack or self._lib_pack
        self._unpack = unpack or self._lib_unpack

    def _lib_pack(self, what, side, t):
        if self.cuda:
            self.sim.halo_pack(what, side, t.data_ptr())
            self.sim.synchronize()
        else:
            self.sim.halo_pack(what, side, self._dev.data_ptr())
            self.sim.synchronize()
            t.copy_(self._dev)

    def _lib_unpack(self, what, side, t):
        if self.cuda:
            self.sim.halo_unpack(what, side, t.data_ptr())
        else:
            self._dev.copy_(t)
            self.sim.halo_unpack(what, side, self._dev.data_ptr())
        self.sim.synchronize()

    def neighbours(self):
        """(rank below, rank above) along y, None at the domain's ends."""
        return (self.rank - 1 if self.rank > 0 else None, self.rank + 1 if self.rank < self.size - 1 else None)

    def exchange(self, what):
        """Swap boundary columns with both neighbours: every send is posted with its
        matching receive in one batch, so no pair of ranks waits on the other's order."""
        below, above = self.neighbours()
        ops = []
        P2P = self.dist.P2POp
        if below is not None:
            self._pack(what, 0, self._send[0])
            ops += [P2P(self.dist.isend, self._send[0], below), P2P(self.dist.irecv, self._recv[0], below)]
        if above is not None:
            self._pack(what, 1, self._send[1])
            ops += [P2P(self.dist.isend, self._send[1], above), P2P(self.dist.irecv, self._recv[1], above)]
        if ops:
            for req in self.dist.batch_isend_irecv(ops):
                req.wait()
            if self.cuda:
                # NCCL's wait orders the current stream only; the unpack runs on the
                # context's own stream
                import torch

                torch.cuda.current_stream().synchronize()
        if below is not None:
            self._unpack(what, 0, self._recv[0])
        if above is not None:
            self._unpack(what, 1, self._recv[1])

    def setup(self):
        self.exchange(HALO_SETUP)

    def step(self, it):
        for irk in range(4):
            self.exchange(irk)
            self.sim.stage(it, irk)
