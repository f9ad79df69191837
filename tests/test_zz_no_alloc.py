"""The allocation-free slice entry point (dfd_get_slice_noalloc) against dfd_get_slice.

Both gather Vx, Vy, Vz on one grid slice with the same kernel; the no-alloc entry uses the
library's static device buffer instead of a temporary cudaMalloc.  The comparison is exact
(tolerance 0): the same values are copied, only the staging buffer differs.
"""
import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu


def test_noalloc_slice_matches_allocating_slice():
    import dynfd3dcuda_b200 as dfd

    p, fx, st, layers, w0, meta = cases.get_case("sw_flat")
    sim = dfd.Simulation(dict(p), fx, st, layers)
    sim.run(0, 10)
    sim.synchronize()
    for axis, index in ((0, p["NX"] // 2), (0, 5), (1, p["NY"] // 3), (2, p["NZ"] - 1), (2, 0)):
        ref = sim.slice(axis, index)
        a = sim.slice_noalloc(axis, index)
        b = sim.slice_noalloc(axis, index)
        assert np.abs(ref).max() > 0 or axis == 2
        np.testing.assert_array_equal(a, ref)
        np.testing.assert_array_equal(b, ref)
    sim.close()


def test_noalloc_slice_rejects_oversize():
    import dynfd3dcuda_b200 as dfd

    job = {"NX": 1450, "NY": 1000, "NZ": 8, "DH": 100.0, "DT": 0.005, "TMAX": 1.0,
           "Rupture": 0, "usePML": 0, "FreeSurface": 0}
    sim = dfd.Simulation(job, precompute=False)
    assert 3 * 1450 * 1000 > dfd.SLICE_SCRATCH_FLOATS
    with pytest.raises(dfd.DfdError) as e:
        sim.slice_noalloc(2, 0)
    assert e.value.status == 1  # DFD_ERR_PARAM
    assert "static gather buffer" in str(e.value)
    # a slice within the limit still works on the same context
    s = sim.slice_noalloc(0, 3)
    assert s.shape == (3, 8, 1000) and not s.any()
    sim.close()
