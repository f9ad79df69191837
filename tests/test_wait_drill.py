"""The bounded waits of the TMA-tiled volume kernels, exercised without faulting the GPU.

The interior kernel's computing warps wait on mbarriers that its copy-issuing warp arms
with each TMA copy.  Every such wait is bounded: when it runs out, the kernel sets the
context's error flag and returns, and the host reports the failure instead of hanging.
The test drill (dfd_test_wait_drill) makes the copy-issuing warp issue nothing, so no copy
is ever in flight and the first wait runs out after a short bounded poll.  The drilled
context then reports DFD_ERR_CUDA and keeps it (sticky); a new context on the same device
steps normally and matches an undrilled run bit for bit."""
import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu

# a volume case whose interior box holds several tiles, so the interior kernel runs
OVER = {"NX": 40, "NY": 100, "NZ": 52, "Rupture": 0}


def make():
    import dynfd3dcuda_b200 as dfd

    p, fx, st, layers, w0, meta = cases.get_case("vol_curved")
    job = dict(p)
    job.update(OVER)
    fx = cases.curved_geometry(job["NY"], job["NZ"], job["DH"], hill_amp=300.0, hill_width=600.0, seed=3)
    sim = dfd.Simulation(job, fx, None, None)
    sim.set_wave(cases.smooth_wave(job["NX"], job["NY"], job["NZ"], seed=4).astype(np.float32))
    return sim


def test_wait_runs_out_and_is_reported():
    import dynfd3dcuda_b200 as dfd

    sim = make()
    sim.test_wait_drill(True)
    sim.stage(0, 0)
    with pytest.raises(dfd.DfdError) as e:
        sim.synchronize()
    assert e.value.status == 2  # DFD_ERR_CUDA
    assert "TMA copy did not complete" in str(e.value)
    # the error is sticky in the drilled context
    with pytest.raises(dfd.DfdError):
        sim.synchronize()
    sim.close()

    # the device is unaffected: fresh contexts step normally and agree bit for bit
    a, b = make(), make()
    for it in range(3):
        a.run(it, 1)
        for irk in range(4):
            b.stage(it, irk)
    a.synchronize()
    b.synchronize()
    wa, wb = a.wave(), b.wave()
    assert np.isfinite(wa).all()
    assert np.array_equal(wa, wb)
    a.close()
    b.close()
