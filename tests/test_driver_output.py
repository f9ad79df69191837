"""The drop-in driver executable and the NetCDF outputs, on the GPU.

The driver (dynfd3dcuda_b200/dfd_b200) reads the same params.json and NetCDF inputs as
the reference's executable and writes fault_mpi000000.nc and wave_{yz,xz,xy}_mpi000000.nc
with the reference's variable names, one record per EXPORT_TIME_SKIP steps, written before
the step (main.cu:425-437, io_fault.cu, io_wave_*.cu).  The records must equal the state
that the Python mirror of the C ABI reads before the same steps.
"""
import json
import os
import subprocess

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "dynfd3dcuda_b200", "dfd_b200")


def test_driver_writes_reference_outputs(tmp_path):
    from scipy.io import netcdf_file

    import dynfd3dcuda_b200 as dfd

    job, meta = cases.write_inputs("sw_flat", str(tmp_path))
    job.update(EXPORT_TIME_SKIP=5, EXPORT_WAVE_SLICE_X=job["NX"] // 2, EXPORT_WAVE_SLICE_Y=30,
               EXPORT_WAVE_SLICE_Z=job["NZ"] - 1, TMAX=0.2 + 0.004)
    with open(tmp_path / "params.json", "w") as f:
        json.dump(job, f)
    r = subprocess.run([EXE, str(tmp_path / "params.json")], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    NT = int(np.float32(job["TMAX"]) / np.float32(job["DT"]))
    assert NT == 25

    p, fx, st, _, _, _ = cases.get_case("sw_flat")
    sim = dfd.Simulation(dict(job), fx, st, None)
    recs = {k: [] for k in ("Vs1", "Vs2", "Tn", "Ts1", "Ts2", "slip", "State", "rup_sensor")}
    slices = []
    for it in range(NT):
        if it % 5 == 0:
            for k in recs:
                recs[k].append(sim.fault(k))
            slices.append([sim.slice(0, job["NX"] // 2), sim.slice(1, 30), sim.slice(2, job["NZ"] - 1)])
        sim.step(it)
    t0 = sim.fault("init_t0")
    sim.close()

    with netcdf_file(tmp_path / "fault_mpi000000.nc", "r", mmap=False) as f:
        v = f.variables
        assert v["Vs1"].shape == (NT // 5, job["NZ"], job["NY"])
        for nc, k in (("Vs1", "Vs1"), ("Vs2", "Vs2"), ("tn", "Tn"), ("ts1", "Ts1"), ("ts2", "Ts2"), ("Us0", "slip"),
                      ("State", "State"), ("rup_sensor", "rup_sensor")):
            np.testing.assert_array_equal(np.asarray(v[nc][:]), np.stack(recs[k]), err_msg=nc)
        assert np.asarray(v["y"][:]).shape == (job["NZ"], job["NY"])
        # rupture times as of the last record (written before step 20)
        assert np.asarray(v["init_t0"][:]).shape == t0.shape
    for a, name in enumerate(("wave_yz", "wave_xz", "wave_xy")):
        with netcdf_file(tmp_path / f"{name}_mpi000000.nc", "r", mmap=False) as f:
            for c, comp in enumerate(("Vx", "Vy", "Vz")):
                got = np.asarray(f.variables[comp][:])
                want = np.stack([s[a][c] for s in slices])
                np.testing.assert_array_equal(got, want, err_msg=f"{name}/{comp}")


def test_async_output_matches_state(tmp_path):
    """dfd_output_write only queues a record (snapshot on the stepping stream, copy and
    file writes behind it): twelve records written before twelve graph-replayed steps with
    no synchronisation between them (both staging slots reused, the writer queue full)
    equal, bit for bit, the state a second identical run reads before each step."""
    from scipy.io import netcdf_file

    import dynfd3dcuda_b200 as dfd

    p, fx, st, _, _, _ = cases.get_case("sw_flat")
    job = dict(p)
    job.update(EXPORT_WAVE_SLICE_X=job["NX"] // 2, EXPORT_WAVE_SLICE_Y=30, EXPORT_WAVE_SLICE_Z=job["NZ"] - 1)
    a = dfd.Simulation(dict(job), fx, st, None)
    a.output_open(str(tmp_path))
    for it in range(12):
        a.output_write(it)
        a.run(it, 1)
    a.output_close()
    a.close()

    b = dfd.Simulation(dict(job), fx, st, None)
    want = {k: [] for k in ("Vs1", "slip", "State")}
    slices = []
    for it in range(12):
        for k in want:
            want[k].append(b.fault(k))
        slices.append([b.slice(0, job["NX"] // 2), b.slice(1, 30), b.slice(2, job["NZ"] - 1)])
        b.run(it, 1)
    b.close()
    with netcdf_file(tmp_path / "fault_mpi000000.nc", "r", mmap=False) as f:
        for nc, k in (("Vs1", "Vs1"), ("Us0", "slip"), ("State", "State")):
            np.testing.assert_array_equal(np.asarray(f.variables[nc][:]), np.stack(want[k]), err_msg=nc)
    for ax, name in enumerate(("wave_yz", "wave_xz", "wave_xy")):
        with netcdf_file(tmp_path / f"{name}_mpi000000.nc", "r", mmap=False) as f:
            for c, comp in enumerate(("Vx", "Vy", "Vz")):
                np.testing.assert_array_equal(np.asarray(f.variables[comp][:]), np.stack([s[ax][c] for s in slices]),
                                              err_msg=f"{name}/{comp}")


def test_fetch_outputs_matches_state():
    """dfd_fetch_outputs snapshots the eight per-step output planes on the stepping
    stream and copies them to the host on a side stream: six fetches, each followed by a
    step, hold the state a second run reads before the same steps."""
    import dynfd3dcuda_b200 as dfd

    p, fx, st, _, _, _ = cases.get_case("sw_flat")
    a = dfd.Simulation(dict(p), fx, st, None)
    nf = p["NY"] * p["NZ"]
    bufs = [np.zeros((8, nf), np.float32) for _ in range(6)]
    for it in range(6):
        a.fetch_outputs(bufs[it].ctypes.data)
        a.run(it, 1)
    a.synchronize()
    a.close()
    b = dfd.Simulation(dict(p), fx, st, None)
    names = ("Vs1", "Vs2", "Tn", "Ts1", "Ts2", "slip", "State", "init_t0")
    for it in range(6):
        for r, k in enumerate(names):
            np.testing.assert_array_equal(bufs[it][r], b.fault(k).ravel(), err_msg=f"step {it} {k}")
        b.run(it, 1)
    b.close()


def test_driver_thermal_pressurisation_records(tmp_path):
    """Friction_type 3 through the driver: TP_hy comes from the init file's TP_hy variable
    (init.cu:999-1003) and every record holds temperature and pore pressure at the fault
    (io_fault.cu:263-265), equal to what the C ABI reads before the same steps."""
    from scipy.io import netcdf_file

    import dynfd3dcuda_b200 as dfd

    job, meta = cases.write_inputs("tp_flat", str(tmp_path))
    job.update(EXPORT_TIME_SKIP=4, TMAX=0.16 + 0.004)
    with open(tmp_path / "params.json", "w") as f:
        json.dump(job, f)
    r = subprocess.run([EXE, str(tmp_path / "params.json")], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    NT = int(np.float32(job["TMAX"]) / np.float32(job["DT"]))
    assert NT == 20

    p, fx, st, _, _, _ = cases.get_case("tp_flat")
    sim = dfd.Simulation(dict(job), fx, st, None)
    want = {k: [] for k in ("TP_T", "TP_P", "slip")}
    for it in range(NT):
        if it % 4 == 0:
            for k in want:
                want[k].append(sim.fault(k))
        sim.step(it)
    sim.close()
    assert np.stack(want["TP_P"]).max() > 1e3  # the pore pressure has started to rise by the last record
    with netcdf_file(tmp_path / "fault_mpi000000.nc", "r", mmap=False) as f:
        for nc, k in (("TP_T", "TP_T"), ("TP_P", "TP_P"), ("Us0", "slip")):
            np.testing.assert_array_equal(np.asarray(f.variables[nc][:]), np.stack(want[k]), err_msg=nc)
