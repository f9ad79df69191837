"""The C ABI without a GPU: every symbol the header declares is exported, the parameter
struct matches its ctypes mirror, job parsing follows the reference's set_params.cu, and
bad jobs are rejected on the host before any device work.

The reference's job files are read from the reference checkout named by the environment
variable DFD_REFERENCE when it is set (this only adds cases; the hand-written jobs below
always run).
"""
import ctypes
import glob
import json
import os
import re

import numpy as np
import pytest

import dynfd3dcuda_b200 as dfd

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "dfd_b200.h")
REF_ROOT = os.environ.get("DFD_REFERENCE", "")
REF_JOBS = sorted(glob.glob(os.path.join(REF_ROOT, "jobs", "*", "params.json"))) if REF_ROOT else []


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(dfd_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol():
    names = declared_functions()
    assert len(names) >= 30, names
    L = dfd.lib()
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_params_struct_matches_mirror():
    assert dfd.lib().dfd_params_size() == ctypes.sizeof(dfd.DfdParams)


def test_defaults_follow_reference():
    s = dfd.DfdParams()
    assert dfd.lib().dfd_params_default(ctypes.byref(s)) == 0
    # set_params.cu:60-103 and the PML block :263-267
    assert (s.NX, s.NY, s.NZ) == (100, 90, 80)
    assert s.TMAX == 1.0 and s.DT == 0.01 and s.DH == 100.0
    assert (s.mu_s, s.mu_d, s.Dc, s.C0) == (0.677, 0.525, 0.4, 0.0)
    assert (s.PML_N, s.PML_velocity, s.PML_bmax, s.PML_fc) == (20, 3000.0, 3.0, 1.0)
    assert s.EXPORT_TIME_SKIP == 1 and s.DAMP_N == 20
    assert (s.bi_vp1, s.bi_vs1, s.bi_rho1) == (6000.0, 3464.0, 2670.0)
    assert (s.rupture, s.free_surface, s.use_pml, s.use_cerjan, s.normal_refine) == (1, 1, 1, 0, 1)
    assert s.OUT == b"output" and s.Fault_geometry == b"Fault_geometry.nc"
    assert s.NT == 100
    assert s.TP_n == 1  # set_params.cu:103


def load_json(tmp_path, job):
    f = tmp_path / "params.json"
    f.write_text(json.dumps(job) if isinstance(job, dict) else job)
    s = dfd.DfdParams()
    r = dfd.lib().dfd_params_load_json(str(f).encode(), ctypes.byref(s))
    return r, s


def test_json_keys_and_quirks(tmp_path):
    job = {"NX": 300, "NY": 400, "NZ": 200, "DH": 100.0, "DT": 0.006, "TMAX": 5.0031,
           "Friction_type": 1, "RS_V0": 1e-6, "RS_Vini": 1e-12, "RS_f0": 0.6, "RS_fw": 0.2, "RS_L": 0.02,
           "rho1": 2500.0, "bi_vs2": 3000.0, "PML_N": 12, "PML_velocity": 6000.0, "Fault_grid": [51, 350, 51, 200],
           "Asp_grid": [1, 2, 3, 4], "OUT": "out_dir", "EXPORT_TIME_SKIP": 5, "useCerjan": 1, "FreeSurface": 0,
           "PX": 2, "PY": 4, "PZ": 2, "igpu": 3, "TP_n": 64}
    r, s = load_json(tmp_path, job)
    assert r == 0
    assert (s.NX, s.NY, s.NZ, s.Friction_type, s.PML_N, s.EXPORT_TIME_SKIP) == (300, 400, 200, 1, 12, 5)
    assert s.bi_rho1 == 2500.0            # "rho1" is read into the bimaterial density
    assert (s.V0, s.Vini, s.f0, s.fw, s.L) == (1e-6, 1e-12, 0.6, 0.2, 0.02)
    assert list(s.Fault_grid) == [51, 350, 51, 200] and list(s.Asp_grid) == [1, 2, 3, 4]
    assert s.OUT == b"out_dir" and s.use_cerjan == 1 and s.free_surface == 0
    assert s.TP_n == 64
    # NT = (int)(TMAX / DT) in single precision (set_params.cu:286-295)
    assert s.NT == int(np.float32(5.0031) / np.float32(0.006))
    # unknown and multi-rank keys are accepted and leave the defaults alone: a reference
    # job's PX/PY/PZ do not split the domain (the caller sets slabs_y / slab_y)
    assert s.mu_s == 0.677
    assert (s.slabs_y, s.slab_y) == (1, 0)


@pytest.mark.parametrize("path", REF_JOBS, ids=[os.path.basename(os.path.dirname(p)) for p in REF_JOBS])
def test_reference_jobs_parse(tmp_path, path):
    src = json.load(open(path))
    s = dfd.DfdParams()
    assert dfd.lib().dfd_params_load_json(path.encode(), ctypes.byref(s)) == 0
    for key, attr in (("NX", "NX"), ("NY", "NY"), ("NZ", "NZ"), ("PML_N", "PML_N"), ("Friction_type", "Friction_type")):
        if key in src:
            assert getattr(s, attr) == int(src[key]), key
    for key, attr in (("DH", "DH"), ("DT", "DT"), ("TMAX", "TMAX"), ("mu_s", "mu_s"), ("mu_d", "mu_d"), ("Dc", "Dc")):
        if key in src:
            assert getattr(s, attr) == pytest.approx(float(src[key]), rel=0, abs=0), key
    assert s.NT == int(np.float32(s.TMAX) / np.float32(s.DT))


def test_malformed_and_missing_json(tmp_path):
    r, _ = load_json(tmp_path, '{"NX": 10,, }')
    assert r == 3  # DFD_ERR_IO
    s = dfd.DfdParams()
    assert dfd.lib().dfd_params_load_json(str(tmp_path / "nope.json").encode(), ctypes.byref(s)) == 3


# Friction_type 3 at the reference's default TP_n = 1: the column spacing width / (TP_n - 1)
# is infinite and the reference's heat source is NaN
@pytest.mark.parametrize("bad", [{"PML_N": 31}, {"Friction_type": 3}, {"Friction_type": 3, "TP_n": 5000},
                                 {"Friction_type": 4}, {"NX": 4}, {"DT": 0.0},
                                 {"EXPORT_TIME_SKIP": 0}, {"PML_N": 60, "NY": 100},
                                 # slabs of a domain split along y: NY a multiple of slabs_y,
                                 # slab_y in range, slabs wide enough for the PML and halo
                                 {"slabs_y": 3}, {"slabs_y": 2, "slab_y": 2}, {"slabs_y": 0},
                                 {"slabs_y": 5, "PML_N": 20}])
def test_bad_jobs_rejected_before_device_work(bad):
    """dfd_create validates the job on the host and returns DFD_ERR_PARAM without touching a GPU."""
    job = {"NX": 100, "NY": 100, "NZ": 100}
    job.update(bad)
    p = dfd.params_struct(job)
    h = ctypes.c_void_p()
    assert dfd.lib().dfd_create(ctypes.byref(p), 0, ctypes.byref(h)) == 1
    assert not h.value


def test_error_strings():
    L = dfd.lib()
    seen = set()
    for code in range(8):
        s = L.dfd_error_string(code)
        assert s and s not in seen
        seen.add(s)


def test_no_gpu_fails_loudly():
    """Without a usable GPU the product path reports a CUDA error; it never falls back to the CPU."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    p = dfd.params_struct({"NX": 16, "NY": 16, "NZ": 16, "PML_N": 2, "DAMP_N": 2})
    with pytest.raises(dfd.DfdError) as e:
        dfd.Simulation({"NX": 16, "NY": 16, "NZ": 16, "PML_N": 2, "DAMP_N": 2})
    assert e.value.status == 2  # DFD_ERR_CUDA
    h = ctypes.c_void_p()
    assert dfd.lib().dfd_create(ctypes.byref(p), 0, ctypes.byref(h)) == 2
