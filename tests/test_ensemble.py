"""The batched ensemble (dfd_ens_*): scenarios of uneven grid sizes, slip weakening and
rate and state mixed, stepped together with one batched launch per kernel and RK stage.
Each scenario must end where the single-scenario path puts it, whatever the unit length
and tile shape the autotuner picks.  The batched kernels evaluate the same expressions as the single
ones but are compiled as other kernels, so the compiler may fuse a multiply and an add
differently: agreement is to FP32 rounding (1e-5 of each field's maximum, as between the
tiled and the plain interior kernels), not bit for bit."""
import numpy as np
import pytest

import cases

TOL = 1e-5


def close(a, b, msg):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(np.abs(a).max(), 1e-30)
    assert np.abs(a - b).max() <= TOL * scale, (msg, np.abs(a - b).max() / scale)

pytestmark = pytest.mark.gpu


def make(i):
    import dynfd3dcuda_b200 as dfd

    # the configuration's generator at test size: uneven grids (the y extent keeps room
    # for the non-united fault area inside the 30-node borders)
    p, _, _ = cases.ensemble_case(i, seed=7, size=(28, 44), steps=40)
    p["NY"] = 72 + p["NY"] % 16
    p["NZ"] = max(p["NZ"], 40)
    p["Fault_grid"] = [31, p["NY"] - 30, 31, p["NZ"]]
    fx = cases.flat_geometry(p["NY"], p["NZ"], p["DH"])
    if p["Friction_type"] == 0:
        st = cases.sw_stress(fx, p["Fault_grid"], tn=-120e6, ts=-66e6, patch=(0.0, -500.0, 600.0), patch_ts=-95e6,
                             Dc=p["Dc"], mu_d=0.525)
    else:
        st = cases.sw_stress(fx, p["Fault_grid"], tn=-120e6, ts=-40e6)
        st = cases.rs_fields(st, fx, seed=11 + i, L=0.02, patch=(0.0, -500.0, 600.0), patch_dtau=45e6)
        # load the patch within the test's few steps
        p["smooth_load_T"] = 0.05
    return p, fx, st


def state(sim):
    return sim.wave(), {k: sim.fault(k) for k in ("slip", "Vs1", "Tn", "State")}


@pytest.mark.parametrize("chunk,rows", [(0, 8), (8, 8), (0, 4)])
def test_ensemble_matches_single_runs(chunk, rows):
    import dynfd3dcuda_b200 as dfd

    specs = [make(i) for i in range(5)]
    singles = [dfd.Simulation(p, fx, st, None) for p, fx, st in specs]
    batch = [dfd.Simulation(p, fx, st, None) for p, fx, st in specs]
    ens = dfd.Ensemble(batch)
    ens.set_chunk(chunk)
    ens.set_tile_rows(rows)
    steps = 24
    ens.run(0, steps)
    ens.synchronize()
    for s in singles:
        s.run(0, steps)
    for i, (a, b) in enumerate(zip(singles, batch)):
        wa, fa = state(a)
        wb, fb = state(b)
        assert np.abs(wa).max() > 0
        for f in range(9):
            close(wa[f], wb[f], f"scenario {i} field {f}")
        for k in fa:
            close(fa[k], fb[k], f"scenario {i} {k}")
    assert ens.nodes() == sum(p["NX"] * p["NY"] * p["NZ"] for p, _, _ in specs)
    ens.close()
    for s in singles + batch:
        s.close()


def test_autotune_keeps_results():
    import dynfd3dcuda_b200 as dfd

    specs = [make(i) for i in range(3)]
    a = [dfd.Simulation(p, fx, st, None) for p, fx, st in specs]
    b = [dfd.Simulation(p, fx, st, None) for p, fx, st in specs]
    ens = dfd.Ensemble(a)
    times, best, it = ens.autotune(0, candidates=(0, 8, 16), steps=2)
    # every tile shape (rows 8 and 4) with every unit length, 1 + 2 steps each
    assert set(times) == {(r, c) for r in (8, 4) for c in (0, 8, 16)}
    assert best in times and it == 3 * len(times)
    ens.run(it, 3)
    ens.synchronize()
    for s in b:
        s.run(0, it + 3)
    for x, y in zip(a, b):
        close(x.fault("slip"), y.fault("slip"), "slip")
        wx, wy = x.wave(), y.wave()
        for f in range(9):
            close(wx[f], wy[f], f"field {f}")
    ens.close()


def test_ensemble_thermal_pressurisation():
    """A thermal-pressurisation scenario (Friction_type 3) in a batch: its column update
    runs once per step before the batched stages and its pore pressure enters the batched
    friction law; it ends where it ends alone."""
    import dynfd3dcuda_b200 as dfd

    specs = [make(i) for i in range(3)]
    p, fx, st = specs[1]  # a rate-and-state scenario
    hy = np.full(st.shape[1:], 1e-4, np.float32)
    specs[1] = (dict(p, Friction_type=3, TP_n=40), fx, np.concatenate([st, hy[None]]))
    singles = [dfd.Simulation(p, fx, st, None) for p, fx, st in specs]
    batch = [dfd.Simulation(p, fx, st, None) for p, fx, st in specs]
    ens = dfd.Ensemble(batch)
    steps = 24
    ens.run(0, steps)
    ens.synchronize()
    for s in singles:
        s.run(0, steps)
    assert singles[1].fault("TP_P").max() > 0
    for i, (a, b) in enumerate(zip(singles, batch)):
        wa, fa = state(a)
        wb, fb = state(b)
        for f in range(9):
            close(wa[f], wb[f], f"scenario {i} field {f}")
        for k in fa:
            close(fa[k], fb[k], f"scenario {i} {k}")
    for nm in ("TP_T", "TP_P"):
        close(singles[1].tp_columns(nm), batch[1].tp_columns(nm), nm)
    ens.close()
    for s in singles + batch:
        s.close()
