"""Errors of the FP32 GPU path against the FP64 oracle at the benchmark configurations.

Rupture time (init_t0), final slip and peak slip rate (the time maximum of the slip-rate
magnitude sqrt(Vs1^2 + Vs2^2), tracked after every step on both sides) of a run on the
GPU through the C ABI and of the same run in the FP64 CPU restatement (oracle/), which
is pinned to the reference's own CUDA build by test_oracle_golden.py.  Test
infrastructure: the product never imports it.

Configurations (the jobs of bench.py and tests/golden/cases.py):
  flat           200 (strike) x 100 x 100, DH 100 m, Cartesian, slip weakening, PML 12,
                 DT 8 ms (1000 steps in full)
  curved_coarse  the curved-grid job (400 x 300 x 200 at DH 100 m) over the same physical
                 domain at DH 200 m: 200 x 150 x 100 nodes, 60-degree dip, Gaussian hills,
                 DT 12 ms (750 steps in full, the 9 s of the 1500-step job)
  rough          300 x 200 x 150 rate and state (slip law) on a self-similar rough fault,
                 run on seed 23 (600 steps in full); --learned trains the guess network
                 on the plain solver's samples of seed 11 first, as bench.py does

usage:
  python tests/config_errors.py gpu    --config C --steps N [--learned] --out A.npz
  python tests/config_errors.py oracle --config C --steps N --out B.npz
  python tests/config_errors.py compare A.npz B.npz
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for _p in (ROOT, os.path.join(HERE, "golden"), os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)


def job_of(config):
    """(job, fxyz, stress, layers) of a named configuration."""
    import bench
    import cases

    if config == "flat":
        job, fx, st, layers, _ = bench.workload("flat")
        return job, fx, st, layers
    if config == "curved_coarse":
        NX, NY, NZ, DH = 150, 200, 100, 200.0
        fg = [26, 175, 26, 100]
        job = dict(NX=NX, NY=NY, NZ=NZ, DH=DH, DT=0.012, TMAX=9.006, PML_N=12, PML_velocity=6000.0,
                   PML_bmax=2.5, PML_fc=1.592356687898089, INPORT_GRID_TYPE=1, INPORT_STRESS_TYPE=1,
                   Friction_type=0, Fault_grid=fg, mu_s=0.76, mu_d=0.448, Dc=0.5, C0=0.2e6)
        fx = cases.curved_geometry(NY, NZ, DH, dip_deg=60.0, hill_amp=500.0, hill_width=5e3, nhills=2, seed=2024)
        n = cases.surface_normal(fx, DH)
        st = cases.depth_stress(fx, fg, grad=7378.0, ratio=0.55, normal=n, patch=(0.0, -8.0e3, 1.5e3))
        return job, fx, st, None
    if config == "rough":
        job, fx, st, _, _, _ = cases.rs_rough_case(300, 200, 150, seed=23, steps=600)
        return job, fx, st, None
    raise SystemExit(f"unknown configuration {config}")


def trained_net(dfd, steps=600, every=7, epochs=4):
    """The guess network of bench.py's learned_rs: samples of the plain solver on seed 11."""
    import cases

    job, fx, st, _, _, _ = cases.rs_rough_case(300, 200, 150, seed=11, steps=steps)
    sim = dfd.Simulation(job, fx, st, None)
    sim.newton_record(12_000_000, every)
    sim.run(0, steps)
    samples = sim.newton_samples(12_000_000)
    sim.close()
    w, _ = dfd.train_guess_net(samples, epochs=epochs, batch=8192, lr=3e-3, seed=1)
    return w


def track(step, get, steps, NZ, NY):
    """Run steps steps; return final slip, rupture time and peak slip rate."""
    psr = np.zeros((NZ, NY))
    for it in range(steps):
        step(it)
        v = np.hypot(get("Vs1"), get("Vs2"))
        np.maximum(psr, v, out=psr)
    return {"slip": get("slip"), "init_t0": get("init_t0"), "psr": psr}


def run_gpu(job, fx, st, layers, steps, net=None):
    import dynfd3dcuda_b200 as dfd

    sim = dfd.Simulation(job, fx, st, layers)
    if net is not None:
        sim.set_guess_net(net)
    NZ, NY = job["NZ"], job["NY"]
    out = track(lambda it: sim.run(it, 1), lambda nm: sim.fault(nm).astype(np.float64), steps, NZ, NY)
    out["newton"] = np.array(sim.newton_stats())
    out["rs_stats"] = np.array(sim.rs_solve_stats())
    sim.close()
    return out


def run_oracle(job, fx, st, layers, steps):
    import oracle

    o = oracle.Oracle(job, fx, st, layers, double=True)
    NZ, NY = job["NZ"], job["NY"]
    return track(o.step, lambda nm: o.get(nm).reshape(NZ, NY), steps, NZ, NY)


def compare(a, b, dt):
    """Error statistics of run a against the reference run b (the FP64 oracle)."""
    both = (a["init_t0"] >= 0) & (b["init_t0"] >= 0)
    only = int(((a["init_t0"] >= 0) != (b["init_t0"] >= 0)).sum())
    dt0 = np.abs(a["init_t0"] - b["init_t0"])[both]
    smax = np.abs(b["slip"]).max()
    pmax = np.abs(b["psr"]).max()
    return {"ruptured_nodes": int((b["init_t0"] >= 0).sum()),
            "rupture_time_max_abs_s": float(dt0.max()) if dt0.size else 0.0,
            "rupture_time_max_abs_steps": float(dt0.max() / dt) if dt0.size else 0.0,
            "rupture_time_nodes_differing": int((dt0 > 0.5 * dt).sum()),
            "ruptured_in_one_run_only": only,
            "final_slip_max_m": float(smax),
            "final_slip_max_rel": float(np.abs(a["slip"] - b["slip"]).max() / smax) if smax > 0 else 0.0,
            "peak_slip_rate_max_m_s": float(pmax),
            "peak_slip_rate_max_rel": float(np.abs(a["psr"] - b["psr"]).max() / pmax) if pmax > 0 else 0.0}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("mode", choices=["gpu", "oracle", "compare"])
    ap.add_argument("files", nargs="*")
    ap.add_argument("--config", default="flat")
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--learned", action="store_true")
    ap.add_argument("--out")
    a = ap.parse_args()
    if a.mode == "compare":
        A, B = (dict(np.load(f, allow_pickle=False)) for f in a.files[:2])
        res = compare(A, B, float(B["dt"]))
        res["a"], res["b"], res["steps"] = a.files[0], a.files[1], int(B["steps"])
        print(json.dumps(res), flush=True)
        return
    job, fx, st, layers = job_of(a.config)
    t0 = time.time()
    if a.mode == "gpu":
        import dynfd3dcuda_b200 as dfd

        net = trained_net(dfd) if a.learned else None
        out = run_gpu(job, fx, st, layers, a.steps, net)
    else:
        out = run_oracle(job, fx, st, layers, a.steps)
    out.update(dt=np.array(job["DT"]), steps=np.array(a.steps), config=np.array(a.config),
               seconds=np.array(time.time() - t0))
    np.savez_compressed(a.out, **out)
    print(f"{a.mode} {a.config} {a.steps} steps: {time.time() - t0:.1f} s -> {a.out}", flush=True)


if __name__ == "__main__":
    main()
