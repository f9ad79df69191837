"""Errors of the FP32 GPU path against the FP64 oracle on the Cartesian slip-weakening job
at its full size (200 x 100 x 100 nodes), over its first 100 steps (0.8 s; the full job
runs 1000, whose figures config_errors.py produces): rupture time, final slip and peak
slip rate tracked every step on both sides."""
import pytest

pytestmark = pytest.mark.gpu


def test_flat_job_against_fp64_oracle(oracle_lib):
    import config_errors as ce

    job, fx, st, layers = ce.job_of("flat")
    steps = 100
    a = ce.run_gpu(job, fx, st, layers, steps)
    b = ce.run_oracle(job, fx, st, layers, steps)
    r = ce.compare(a, b, job["DT"])
    print(r)
    assert r["ruptured_nodes"] > 300
    # rupture times agree to the step; a node crossing the 1 mm/s threshold in the very last
    # step may be counted on one side only
    assert r["rupture_time_max_abs_steps"] <= 1.0
    assert r["ruptured_in_one_run_only"] <= 0.01 * r["ruptured_nodes"]
    # slip-weakening tolerance of the parity tests (relative to the field maximum)
    assert r["final_slip_max_rel"] < 2e-4
    assert r["peak_slip_rate_max_rel"] < 2e-4
