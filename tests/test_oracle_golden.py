"""Pin the CPU oracle against the reference's own CUDA build.

The golden fixtures in tests/golden/*.npz were produced by tests/golden/make_golden.py,
which runs the reference sources (compiled for sm_100a by oracle/Makefile with the
single-rank MPI / NetCDF-classic shims) on the seeded cases of tests/golden/cases.py.
"_dp" fixtures come from the reference's own FP64 build (-DDoublePrecision), "_sp" from
its default FP32 build.  The FP64 oracle must reproduce both.
"""
import numpy as np
import pytest

import cases


# relative max-error tolerances (of the field's max magnitude).  FP64-vs-FP64 is limited by
# the fixtures' FP32 storage (the oracle reproduces the reference's single-precision sqrtf
# in its vector norm, device.cu:84-89, which on a rough fault moves rate-and-state results
# by 1e-3); the FP32 reference adds its own rounding, most for rate and state (exp/sinh of
# state over a = 0.01) and most of all on the rough fault.
TOL = {
    ("vol_small", "dp"): 1e-6, ("vol_small", "sp"): 2e-6,
    ("vol_curved", "dp"): 1e-6, ("vol_curved", "sp"): 2e-6,
    ("sw_flat", "dp"): 1e-6, ("sw_flat", "sp"): 1e-5,
    ("sw_flat_nr", "dp"): 1e-6, ("sw_flat_nr", "sp"): 1e-5,
    ("sw_curved", "dp"): 3e-5, ("sw_curved", "sp"): 1e-4,
    ("rs_flat", "dp"): 3e-5, ("rs_flat", "sp"): 3e-4,
    ("sw_cerjan", "dp"): 1e-6, ("sw_cerjan", "sp"): 1e-5,
    ("tp_flat", "dp"): 1e-5, ("tp_flat", "sp"): 3e-4,
    ("rs_aging", "dp"): 1e-6, ("rs_aging", "sp"): 1e-3,
    ("rs_curved", "dp"): 1e-5, ("rs_curved", "sp"): 3e-3,
    ("media_cj", "sp"): 1e-4,  # no FP64 fixture: the reference's FP64 build misreads Media1D
}


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    s = np.abs(b).max()
    return np.abs(a - b).max() / (s if s > 0 else 1.0)


def sensor_mask(ts1):
    """Nodes where the rupture sensor (jumps of second differences of Ts1 over Ts1^2,
    rup_sensor.cu:8-95) is well conditioned: |Ts1| above 5 % of its maximum."""
    a = np.abs(np.asarray(ts1, np.float64))
    return a > 5e-2 * a.max()


@pytest.mark.parametrize("name,var", sorted(TOL))
def test_oracle_matches_reference(oracle_lib, name, var):
    g = np.load(f"{cases.__file__[:-8]}/{name}_{var}.npz")
    p, fx, st, layers, w0, meta = cases.get_case(name)
    o = oracle_lib.Oracle(p, fx, st, layers, double=True)
    if w0 is not None:
        o.set("W", w0)
    NX, NY, NZ = p["NX"], p["NY"], p["NZ"]
    nx, ny, nz = NX + 6, NY + 6, NZ + 6
    i0 = nx // 2
    tol = TOL[(name, var)]
    J0, J1 = (int(v) for v in g["jblock"]) if "jblock" in g.files else (24, 52)
    if var == "dp":
        M = o.get("M").reshape(13, nx, nz, ny)
        assert rel(M[:, i0 - 1:i0 + 2], g["M_planes"]) < 1e-6
        if not meta["volume"]:
            assert (o.get("united").reshape(NZ, NY) == g["united"]).all()
            assert (o.get("faultgrid").reshape(NZ, NY) == g["faultgrid"]).all()
            for nm in ("D21_1", "matPlus2Min1", "matT1toVxm", "matVztoVxp", "matMin2Plus5"):
                assert rel(o.get(nm).reshape(nz, ny, 9)[:, J0:J1], g[nm]) < 1e-6, nm
            assert rel(o.get("vec_n").reshape(nz, ny, 3)[:, J0:J1], g["vec_n"]) < 1e-6
            for nm in ("matVx2Vz1", "matPlus2Min2f", "matMin2Plus3f"):
                assert rel(o.get(nm).reshape(ny, 9), g[nm]) < 1e-6, nm
    it = 0
    for s in g["steps"]:
        while it < s:
            (o.step_volume if meta["volume"] else o.step)(it)
            it += 1
        W = o.wave()
        ws = np.stack([[W[f].sum(), np.sqrt((W[f] ** 2).sum()), np.abs(W[f]).max()] for f in range(9)])
        assert rel(ws[:, 1:], g[f"Wsum_s{s}"][:, 1:]) < tol
        if not meta["volume"]:
            for nm in ("slip", "Vs1", "Vs2", "Tn", "Ts1", "Ts2", "State"):
                assert rel(o.get(nm).reshape(NZ, NY), g[f"{nm}_s{s}"]) < tol, (nm, s)
            # rupture times are identical to the step
            t0 = o.get("init_t0").reshape(NZ, NY)
            assert np.abs(t0 - g[f"init_t0_s{s}"]).max() < 0.5 * p["DT"]
            if f"rup_sensor_s{s}" in g:  # rupture sensor of the step start, where well conditioned
                m = sensor_mask(o.get("Ts1").reshape(NZ, NY))
                assert rel(o.get("rup_sensor").reshape(NZ, NY)[m], g[f"rup_sensor_s{s}"][m]) < tol, ("rup_sensor", s)
            for nm in ("TP_T", "TP_P"):  # thermal pressurisation: the point on the fault
                if f"{nm}_s{s}" in g:
                    assert rel(o.get(nm).reshape(-1, NZ, NY)[0], g[f"{nm}_s{s}"]) < tol, (nm, s)
    if meta["volume"]:
        assert rel(o.wave(), g["W_final"]) < tol
    else:
        assert rel(o.wave()[:, i0 - 3:i0 + 4, :, J0:J1], g["W_block"]) < tol
        assert rel(o.get("FW").reshape(9, 2, nz, ny)[..., J0:J1], g["FW_block"]) < tol
        for nm in ("T11", "T12", "T13"):
            assert rel(o.get(nm).reshape(7, nz, ny)[..., J0:J1], g[f"{nm}_block"]) < tol, nm
        fg = p["Fault_grid"]
        for nm in ("TP_T", "TP_P"):  # whole columns over the non-united block
            if f"{nm}_cols" in g:
                col = o.get(nm).reshape(-1, NZ, NY)[:, fg[2] - 1:fg[3], fg[0] - 1:fg[1]]
                assert rel(col, g[f"{nm}_cols"]) < tol, nm
