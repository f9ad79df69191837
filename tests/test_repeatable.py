"""Runs of the same job in one process are identical, bit for bit.

Every volume node is updated by one thread of one kernel per stage, with no atomics in
its arithmetic, so a job run twice gives the same bits.  The library uploads host arrays
(the initial wavefield of dfd_set_wave, the PML and sponge profiles, the grid) on the
context's stepping stream and waits for them: a plain cudaMemcpy from pageable memory
runs on the legacy default stream, can still be in flight when it returns, and is not
ordered with the context's non-blocking streams, so the first kernels of a run could read
a partly copied wavefield.  That showed only once kernels were already loaded in the
process (later runs launched sooner), as differences at every node after 40 steps.
"""
import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tile", ["1", "0"])
def test_repeated_runs_identical(monkeypatch, tile):
    import dynfd3dcuda_b200 as dfd

    NX, NY, NZ = 24, 40, 24
    job = dict(NX=NX, NY=NY, NZ=NZ, DH=100.0, DT=0.004, TMAX=10.0, PML_N=5, PML_velocity=6000.0,
               INPORT_GRID_TYPE=0, Rupture=0, FreeSurface=1)
    w0 = cases.smooth_wave(NX, NY, NZ, seed=5).astype(np.float32)
    monkeypatch.setenv("DFD_TILE", tile)
    out = []
    for _ in range(4):
        sim = dfd.Simulation(job)
        sim.set_wave(w0)
        sim.run(0, 40)
        sim.synchronize()
        out.append(sim.wave())
        sim.close()
    assert np.abs(out[0]).max() > 0
    for w in out[1:]:
        assert np.array_equal(w, out[0])


def test_repeated_rupture_runs_identical():
    """The same with a fault (slip weakening on a curved grid, 30 steps)."""
    import dynfd3dcuda_b200 as dfd

    p, fx, st, layers, w0, meta = cases.get_case("sw_curved")
    res = []
    for _ in range(3):
        sim = dfd.Simulation(p, fx, st, layers)
        sim.run(0, 30)
        sim.synchronize()
        res.append((sim.wave(), sim.fault("slip"), sim.fault("Vs1")))
        sim.close()
    for r in res[1:]:
        for a, b in zip(r, res[0]):
            assert np.array_equal(a, b)
