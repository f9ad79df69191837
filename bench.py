#!/usr/bin/env python
"""Benchmark: grid-point-steps per second of the curved-grid rupture time step on B200.

Workload (default, --config large): the large single domain the HBM roofline is quoted
on -- 1000 (strike) x 600 (normal) x 300 (depth) nodes = 180 M at DH = 50 m, a 1-D
layered medium (vs 2000 to 3600 m/s over depth, Media1D table), a curved non-planar
vertical fault 50 km x 15 km (seeded along-strike bumps), normal stress 7378 Pa/m of
depth and shear 0.55 x normal, slip-weakening friction, a 20-node PML plus a 20-node
Cerjan sponge, free surface, DT = 4 ms.  --config curved: the curved-grid job, 400 x 300 x
200 nodes at DH = 100 m with a 60-degree dipping fault and Gaussian-hill topography.
Inputs are seeded synthetic data in the reference's file layouts (tests/golden/cases.py);
each of the four volume buffers (6.7 GB for the large domain) is far larger than the
126 MB L2, so no explicit flush is needed between steps.

  value      Gpt-steps/s of the stepping loop on the device: K steps replayed from the
             CUDA graphs, timed with CUDA events on the stepping stream, max over ranks
  e2e        the same metric through the C ABI end to end: context creation, upload of the
             job's host arrays from pinned memory, setup, K steps, and every step a copy of
             the eight on-fault output planes back to pinned host memory (the reference
             writes them every step, main.cu:425-437)
  roofline   the dominant kernel, the TMA-tiled interior volume kernel: 768 algorithmic
             bytes per node per step (39/57/57/39 floats over the four RK stages) over the
             nodes it updates, divided by its event-timed duration on its stream (an
             instrumented pass of up to 200 steps after the timed region, stages launched
             one by one with events around the kernel), against the measured HBM copy
             bandwidth; volume_phase gives the same over all nodes and the volume phase
  cpu_baseline / --impl reference: the OpenMP FP32 CPU restatement of the same scheme
             (oracle/), the reference having no CPU path, on a bounded sample of steps

usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
       [--config large|curved|flat|profile|ensemble] [--scenarios S] [--split]

--split: one domain split along y over the N GPUs (strong scaling, halo exchange over
NCCL before every RK stage) instead of the default N independent replicas.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "tests", "golden"), os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

ALG_BYTES_PER_NODE_STEP = 768  # 192 floats: stages 39 + 57 + 57 + 39 (stencil input, metric, RK registers)
LAUNCHES_PER_STEP = 22         # rupture sensor + 4 x (fault node + interior + PML + free-surface rows + fault band) + step counter


def workload(name):
    """(job, fxyz, stress, layers, label) of a benchmark configuration."""
    import cases

    if name == "curved":
        NX, NY, NZ, DH = 300, 400, 200, 100.0
        fg = [51, 350, 51, 200]
        # DT = 6 ms: the 60-degree sheared, normal-refined grid has hmin = 32 m, so the
        # reference's stability limit 1.3 hmin / vpmax (main.cu:323) is 6.94 ms
        job = dict(NX=NX, NY=NY, NZ=NZ, DH=DH, DT=0.006, TMAX=9.003, PML_N=12, PML_velocity=6000.0,
                   PML_bmax=2.5, PML_fc=1.592356687898089, INPORT_GRID_TYPE=1, INPORT_STRESS_TYPE=1,
                   Friction_type=0, Fault_grid=fg, mu_s=0.76, mu_d=0.448, Dc=0.5, C0=0.2e6,
                   EXPORT_WAVE_SLICE_X=NX // 2, EXPORT_WAVE_SLICE_Y=NY // 2, EXPORT_WAVE_SLICE_Z=NZ - 1)
        fx = cases.curved_geometry(NY, NZ, DH, dip_deg=60.0, hill_amp=500.0, hill_width=5e3, nhills=2, seed=2024)
        n = cases.surface_normal(fx, DH)
        st = cases.depth_stress(fx, fg, grad=7378.0, ratio=0.55, normal=n, patch=(0.0, -8.0e3, 1.5e3))
        label = "curved-grid SW rupture 400x300x200 (strike x normal x depth), dh=100 m, dip 60, hills, PML 12"
        return job, fx, st, None, label
    if name == "flat":
        NX, NY, NZ, DH = 100, 200, 100, 100.0
        fg = [26, 175, 26, 100]
        job = dict(NX=NX, NY=NY, NZ=NZ, DH=DH, DT=0.008, TMAX=8.004, PML_N=12, PML_velocity=6000.0,
                   INPORT_GRID_TYPE=1, INPORT_STRESS_TYPE=1, Friction_type=0, Fault_grid=fg, mu_s=0.677,
                   mu_d=0.525, Dc=0.4, C0=0.0, NormalRefine=0)
        fx = cases.flat_geometry(NY, NZ, DH)
        st = cases.sw_stress(fx, fg, patch=(0.0, -7.5e3, 1.5e3), patch_ts=-81.6e6)
        label = "Cartesian SW rupture 200x100x100 (strike x normal x depth), dh=100 m, PML 12"
        return job, fx, st, None, label
    if name == "profile":
        # mid-size case for ncu captures: 6.5 M nodes, each volume buffer 0.24 GB (> L2)
        NX, NY, NZ, DH = 160, 256, 160, 100.0
        fg = [41, 216, 41, 160]
        job = dict(NX=NX, NY=NY, NZ=NZ, DH=DH, DT=0.008, TMAX=8.004, PML_N=12, PML_velocity=6000.0,
                   INPORT_GRID_TYPE=1, INPORT_STRESS_TYPE=1, Friction_type=0, Fault_grid=fg, mu_s=0.677,
                   mu_d=0.525, Dc=0.4, C0=0.0, NormalRefine=0)
        fx = cases.flat_geometry(NY, NZ, DH)
        st = cases.sw_stress(fx, fg, patch=(0.0, -6.0e3, 1.5e3), patch_ts=-81.6e6)
        label = "profiling case: Cartesian SW rupture 256x160x160, dh=100 m, PML 12"
        return job, fx, st, None, label
    if name in ("large", "large_profile"):
        # large_profile: the same configuration on 320 x 160 x 160 nodes (8.2 M, about 3 GB
        # on the device) for ncu captures, whose per-node traffic scales to the full domain
        if name == "large":
            NX, NY, NZ, DH = 600, 1000, 300, 50.0
            fg, pz = [101, 900, 61, 300], -7.5e3
        else:
            NX, NY, NZ, DH = 160, 320, 160, 50.0
            fg, pz = [41, 280, 41, 160], -4.0e3
        depth = np.linspace(0, 15e3, 16)
        vs = np.linspace(2000.0, 3600.0, 16)
        layers = np.stack([depth, 2670.0 + 0 * depth, np.sqrt(3.0) * vs, vs], 1).astype(np.float32)
        job = dict(NX=NX, NY=NY, NZ=NZ, DH=DH, DT=0.004, TMAX=8.002, PML_N=20, PML_velocity=6236.0,
                   INPORT_GRID_TYPE=1, INPORT_STRESS_TYPE=1, Friction_type=0, Fault_grid=fg, mu_s=0.677,
                   mu_d=0.525, Dc=0.4, C0=0.0, useCerjan=1, DAMP_N=20)
        fx = cases.curved_geometry(NY, NZ, DH, dip_deg=90.0, hill_amp=0.0, seed=7)
        rng = np.random.default_rng(7)
        jj = np.arange(NY)[None, :]
        # along-strike bumps of the same wavelengths (in metres) on both grid sizes
        fx[0] = (200.0 * np.sin(2 * np.pi * jj / 1000 * rng.uniform(1, 3)) + 0 * fx[0]).astype(np.float32)
        n = cases.surface_normal(fx, DH)
        st = cases.depth_stress(fx, fg, grad=7378.0, ratio=0.55, normal=n, mu_s=0.677, mu_d=0.525, Dc=0.4, C0=0.0,
                                patch=(0.0, pz, 1.5e3))
        label = (f"large curved-fault SW rupture {NY}x{NX}x{NZ} ({NX * NY * NZ / 1e6:.0f} M nodes), dh=50 m, "
                 "1-D layered, PML 20 + Cerjan")
        return job, fx, st, layers, label
    raise SystemExit(f"unknown config {name}")


class Clocks:
    """nvidia-smi sampling of SM clock and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        if vis:
            ids = [v.strip() for v in vis.split(",") if v.strip()]
            if index < len(ids):
                index = ids[index]
        self.index = index
        self.proc = None
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        load = [s for s in sm if s > 0.5 * smax] or sm
        reasons = set()
        for r in rows:
            for name, val in (("hw_slowdown", r[5]), ("hw_thermal_slowdown", r[6]), ("sw_thermal_slowdown", r[7]),
                              ("sw_power_cap", r[8])):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": smax, "samples": len(rows),
                "reasons": sorted(reasons)}


def cpu_baseline(job, fx, st, layers, budget_s=25.0, max_steps=None):
    """FP32 OpenMP CPU restatement on the same job for a bounded number of steps."""
    import oracle

    threads = oracle.threads()
    t0 = time.time()
    o = oracle.Oracle(job, fx, st, layers, double=False)
    setup = time.time() - t0
    npts = job["NX"] * job["NY"] * job["NZ"]
    done, t_step = 0, 0.0
    while True:
        t1 = time.time()
        o.step(done)
        t_step += time.time() - t1
        done += 1
        if t_step > budget_s or (max_steps and done >= max_steps) or (t_step / done) * (done + 1) > 3 * budget_s:
            break
    del o
    return {"value": npts * done / t_step / 1e9, "unit": "Gpt-steps/s", "cores": threads, "kind": "port",
            "sample": f"{done} time steps of the full workload grid after a {setup:.1f} s setup "
                      f"(FP32 oracle/dfd_oracle.cpp, OpenMP {threads} threads)"}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            m = json.load(f)
        return float(m["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def traffic_per_node():
    """DRAM bytes per node per step of the volume kernel from the committed ncu summary."""
    try:
        with open(os.path.join(ROOT, "profiles", "volume_traffic.json")) as f:
            return float(json.load(f)["dram_bytes_per_node_step"])
    except (OSError, KeyError, ValueError):
        return None


def max_over_ranks(x, dist, device):
    """The slowest rank's figure: all-reduce MAX over the process group (identity alone)."""
    import torch

    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(npts, steps, world, seconds):
    """Whole-job Gpt-steps/s: every rank advances its own replica of npts nodes by steps
    steps, and the job takes as long as its slowest rank."""
    return npts * steps * world / seconds / 1e9


def run_reference(args, rank):
    if rank != 0:
        return
    job, fx, st, layers, label = workload(args.config)
    npts = job["NX"] * job["NY"] * job["NZ"]
    import oracle

    o = oracle.Oracle(job, fx, st, layers, double=False)
    for it in range(args.warmup):
        o.step(it)
    t0 = time.time()
    done = 0
    while done < args.steps:
        o.step(args.warmup + done)
        done += 1
        el = time.time() - t0
        if el > 90.0:
            break
    el = time.time() - t0
    v = npts * done / el / 1e9
    cores = oracle.threads()
    line = {"impl": "reference", "metric": "Gpt-steps/s", "value": v, "unit": "Gpt-steps/s", "n_gpus": args.gpus,
            "steps": done, "warmup": args.warmup, "ms_per_step": 1e3 * el / done, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": label, "nodes": npts},
            "cpu_baseline": {"value": v, "unit": "Gpt-steps/s", "cores": cores, "kind": "port",
                             "sample": f"{done} of {args.steps} requested steps (capped at 90 s) on {cores} threads; "
                                       "the reference has no CPU implementation, this is the OpenMP FP32 "
                                       "restatement of its scheme"},
            "e2e": {"value": v, "unit": "Gpt-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def active_fault_nodes(job):
    """Fault nodes that run the friction solve: the non-united ones (init.cu:806-816)."""
    NY, NZ = job["NY"], job["NZ"]
    nj = sum(1 for j in range(NY) if 30 < j + 1 < NY - 30)
    free = job.get("FreeSurface", 1)
    nk = sum(1 for k in range(NZ) if k + 1 > 30 and (free or k + 1 < NZ - 30))
    return nj * nk


def learned_rs(dfd, steps=600, every=7, epochs=4, device=0):
    """The learned Newton guess on the rate-and-state rough-fault configuration
    (300 x 200 x 150, slip law): record plain-solver samples on one seed, train the MLP on
    the GPU, then run another seed with the plain and with the learned guess and compare
    the fault node kernel time, the clock cycles of the solve section alone (guess,
    network, Newton iterations), Newton iterations per solve, the residual test's
    acceptance and the final slip."""
    import cases

    job, fx, st, _, _, _ = cases.rs_rough_case(300, 200, 150, seed=11, steps=steps)
    sim = dfd.Simulation(job, fx, st, None, device=device)
    sim.newton_record(12_000_000, every)
    sim.run(0, steps)
    samples = sim.newton_samples(12_000_000)
    sim.close()
    t0 = time.perf_counter()
    w, hist = dfd.train_guess_net(samples, epochs=epochs, batch=8192, lr=3e-3, seed=1)
    train_s = time.perf_counter() - t0
    job, fx, st, _, _, _ = cases.rs_rough_case(300, 200, 150, seed=23, steps=steps)
    nact = active_fault_nodes(job)
    out = {"config": "rate-and-state slip law, self-similar rough fault 300x200x150 (strike x normal x depth), "
                     f"dh=100 m, a log-uniform 0.01-0.02, {steps} steps; trained on seed 11, run on seed 23",
           "train_samples": int(len(samples)), "epochs": epochs, "train_s": train_s,
           "loss_per_epoch": [float(v) for v in hist]}
    slips = {}
    nprof = 40  # steps with the solve section timed (clock64 around guess, network and Newton)
    for name, net in (("plain", None), ("learned", w)):
        sim = dfd.Simulation(job, fx, st, None, device=device)
        if net is not None:
            sim.set_guess_net(net)
        sim.run(0, 5)
        sim.synchronize()
        it0, cap0 = sim.newton_stats()
        acc0, fb0, _, _ = sim.rs_solve_stats()
        total_ms, vol_ms, _ = sim.run_timed(5, steps - 5 - nprof)
        node_ms = sim.fault_node_ms()
        it1, cap1 = sim.newton_stats()
        acc1, fb1, _, _ = sim.rs_solve_stats()
        nst = steps - 5 - nprof
        solves = nact * 4 * nst
        sim.rs_profile(timing=True)
        sim.run(steps - nprof, nprof)
        _, _, cyc, _ = sim.rs_solve_stats()
        slips[name] = sim.fault("slip").astype(np.float64)
        out[name] = {"node_kernel_us_per_stage": 1e3 * node_ms / (4 * nst),
                     "newton_iterations_per_solve": (it1 - it0) / solves,
                     "solve_cycles_per_node": cyc,
                     "unconverged_solves": int(cap1 - cap0), "step_ms": total_ms / nst}
        if net is not None:
            out[name]["guesses_accepted"] = int(acc1 - acc0)
            out[name]["guesses_fell_back"] = int(fb1 - fb0)
        sim.close()
    p, l = out["plain"], out["learned"]
    out["speedup_node_kernel"] = p["node_kernel_us_per_stage"] / l["node_kernel_us_per_stage"]
    out["speedup_solve_section"] = p["solve_cycles_per_node"] / l["solve_cycles_per_node"]
    out["speedup_newton_iterations"] = p["newton_iterations_per_solve"] / l["newton_iterations_per_solve"]
    s0 = np.abs(slips["plain"]).max()
    out["final_slip_max_m"] = float(s0)
    out["slip_rel_diff_learned_vs_plain"] = float(np.abs(slips["learned"] - slips["plain"]).max() / max(s0, 1e-30))
    return out


def run_ensemble(args, dfd, local):
    """Batched ensemble (64 scenarios, grids of 100-300 nodes per axis, slip weakening and
    rate and state mixed): aggregate Gpt-steps/s of the whole batch, after the autotuner has
    picked the tile shape and the unit length of the interior kernel."""
    import cases
    import torch

    n = args.scenarios
    specs = [cases.ensemble_case(i) for i in range(n)]
    nodes = sum(p["NX"] * p["NY"] * p["NZ"] for p, _, _ in specs)
    need = sum((p["NX"] + 6) * (p["NY"] + 8) * (p["NZ"] + 6) * 4 * (36 + 13 + 8) for p, _, _ in specs)
    free, _ = torch.cuda.mem_get_info(local)
    if need > 0.92 * free:
        raise SystemExit(f"ensemble needs about {need / 1e9:.0f} GB, {free / 1e9:.0f} GB free")
    t0 = time.perf_counter()
    sims = [dfd.Simulation(p, fx, st, None, device=local) for p, fx, st in specs]
    ens = dfd.Ensemble(sims)
    setup_s = time.perf_counter() - t0
    times, best, it = ens.autotune(0, candidates=(0, 32, 64, 128), steps=2, rows=(8, 4))
    ens.run(it, args.warmup)
    ens.synchronize()
    it += args.warmup
    clk = Clocks(local)
    clk.start()
    ms = ens.run_timed(it, args.steps)
    clocks = clk.stop()
    value = job_rate(nodes, args.steps, 1, ms / 1e3)
    nf = sum(p["NY"] * p["NZ"] for p, _, _ in specs)
    # per step: 6 batched launches a stage (fault node, interior, PML, two groups of
    # free-surface-row boxes, fault band), the rupture sensor of each rupture scenario,
    # thermal pressurisation of each Friction_type 3 scenario, the step counter
    n_rup = sum(1 for p, _, _ in specs if int(p.get("Rupture", 1)))
    n_tp = sum(1 for p, _, _ in specs if int(p.get("Rupture", 1)) and int(p.get("Friction_type", 0)) == 3)
    ens_launches = 4 * 6 + n_rup + n_tp + 1
    line = {"metric": "Gpt-steps/s", "value": value, "unit": "Gpt-steps/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"batched ensemble: {n} scenarios, grids 100-300 nodes per axis, dh=100 m, "
                                   "stress drop 2-8 MPa, Dc/L 0.2-0.8 m, slip weakening and rate and state mixed",
                       "nodes": nodes, "fault_nodes": nf, "scenarios": n, "parallelism": "one batched launch "
                       "per kernel and RK stage, CUDA graph per step",
                       "l2": "inputs larger than L2; no flush"},
            "autotune": {"layout_ms": {f"rows {r}, unit planes {c}": v for (r, c), v in times.items()},
                         "chosen": {"tile_rows": best[0], "unit_planes": best[1]}},
            "setup_s": setup_s, "gpu_launches": ens_launches * args.steps, "clocks": clocks}
    ens.close()
    for s in sims:
        s.close()
    print(json.dumps(line), flush=True)


def run_split(args, dfd, local, rank, world, dist):
    """One domain split along y over the ranks (strong scaling): each rank holds a slab of
    NY / N columns and swaps its boundary columns with its neighbours over NCCL before
    every RK stage (dynfd3dcuda_b200.decomp).  Stage-by-stage stepping (the exchange sits
    between the stages), timed between two full synchronisations with CUDA events, max
    over ranks."""
    import torch

    from dynfd3dcuda_b200.decomp import DistributedSlab, slab_job

    job, fx, st, layers, label = workload(args.config)
    npts = job["NX"] * job["NY"] * job["NZ"]
    sim = dfd.Simulation(slab_job(job, world, rank), fx, st, layers, device=local)
    if dist is not None:
        slab = DistributedSlab(sim, dist, device=f"cuda:{local}")
        slab.setup()
        step = slab.step
    else:
        def step(it):
            for irk in range(4):
                sim.stage(it, irk)
    for it in range(args.warmup):
        step(it)
    sim.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clk = Clocks(local)
    clk.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for it in range(args.warmup, args.warmup + args.steps):
        step(it)
    sim.synchronize()
    e1.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), dist, f"cuda:{local}")
    sim.close()
    line = {"metric": "Gpt-steps/s", "value": npts * args.steps / (ms / 1e3) / 1e9, "unit": "Gpt-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": label + f", split along y into {world} slabs", "nodes": npts,
                       "parallelism": f"y-slabs x{world}, halo exchange over NCCL before every RK stage"},
            "gpu_launches": (LAUNCHES_PER_STEP + (8 if world > 1 else 0)) * args.steps, "clocks": clocks}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="large", choices=["curved", "flat", "profile", "large", "large_profile", "ensemble"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--scenarios", type=int, default=64, help="scenarios of the ensemble configuration")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned Newton-guess comparison")
    ap.add_argument("--split", action="store_true",
                    help="one domain split along y over the GPUs (strong scaling) instead of replicas")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch
    import dynfd3dcuda_b200 as dfd

    torch.cuda.set_device(local)
    if args.config == "ensemble":
        if rank == 0:
            run_ensemble(args, dfd, local)
        return
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    if args.split:
        run_split(args, dfd, local, rank, world, dist)
        return
    job, fx, st, layers, label = workload(args.config)
    npts = job["NX"] * job["NY"] * job["NZ"]

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    # ---------------- device-resident throughput (replica per rank, no data-path collective)
    sim = dfd.Simulation(job, fx, st, layers, device=local)
    sim.run(0, args.warmup)
    sim.synchronize()
    barrier()
    clk = Clocks(local)
    clk.start()
    # the timed region: K steps replayed from the CUDA graphs (the production path),
    # CUDA events on the stepping stream
    total_ms = sim.run_graph_timed(args.warmup, args.steps)
    clocks = clk.stop()
    barrier()
    max_ms = max_over_ranks(total_ms, dist, f"cuda:{local}")
    value = job_rate(npts, args.steps, world, max_ms / 1e3)
    # instrumented pass for the kernel figures: the same stages launched one by one with
    # CUDA events around the interior kernel and the volume phase of every stage
    ksteps = min(args.steps, 200)
    _, vol_ms, _ = sim.run_timed(args.warmup + args.steps, ksteps)
    int_ms, int_nodes = sim.interior_stats()
    sim.check_finite()
    sim.close()

    # ---------------- end to end through the C ABI from pinned host memory
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).pin_memory()  # noqa: E731
    hfx, hst = pin(fx), pin(st)
    hlay = pin(layers) if layers is not None else None
    nf = job["NY"] * job["NZ"]
    hout = torch.empty((2, 8, nf), dtype=torch.float32).pin_memory()
    barrier()
    t0 = time.perf_counter()
    e = dfd.Simulation(job, hfx.numpy(), hst.numpy(), hlay.numpy() if hlay is not None else None, device=local)
    for s in range(args.steps):
        e.run(s, 1)
        e.fetch_outputs(hout[s % 2].data_ptr())
        if s % 2 == 1:
            e.synchronize()
    e.synchronize()
    e2e_s = time.perf_counter() - t0
    e.close()
    e2e_s = max_over_ranks(e2e_s, dist, f"cuda:{local}")
    h2d = (hfx.numel() + hst.numel() + (hlay.numel() if hlay is not None else 0)) * 4 / args.steps
    d2h = 8 * nf * 4

    peak, peak_kind = peaks()
    buf_gb = 9 * (job["NX"] + 6) * (job["NY"] + 8) * (job["NZ"] + 6) * 4 / 1e9
    # dominant kernel: the interior (TMA-tiled) volume kernel, timed live with CUDA events on
    # its stream; its algorithmic bytes are 768 per node per step over the nodes it updates
    launches = 4 * ksteps
    achieved = ALG_BYTES_PER_NODE_STEP * int_nodes * ksteps / (int_ms / 1e3) / 1e9
    phase = ALG_BYTES_PER_NODE_STEP * npts * ksteps / (vol_ms / 1e3) / 1e9
    tpn = traffic_per_node()
    line = {
        "metric": "Gpt-steps/s", "value": value, "unit": "Gpt-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": label, "nodes": npts, "fault_nodes": nf, "parallelism": f"replicas x{world}",
                   "l2": f"inputs larger than L2 (each 9-field buffer {buf_gb:.2f} GB); no flush"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": tpn * int_nodes / 4 if tpn else None,
                     "kernel": "volume_tile_kernel (interior box, TMA-tiled)", "peak_source": peak_kind,
                     "bytes_per_node_step": ALG_BYTES_PER_NODE_STEP, "nodes_per_launch": int_nodes,
                     "algorithmic_bytes_per_launch": ALG_BYTES_PER_NODE_STEP * int_nodes / 4,
                     "launch_us": 1e3 * int_ms / launches,
                     "timed": f"instrumented pass of {ksteps} steps after the timed region (per-kernel CUDA events, "
                              "stages launched one by one)",
                     "volume_phase": {"achieved": phase, "frac": phase / peak, "ms_per_step": vol_ms / ksteps,
                                      "covers": "all volume nodes: tiled interior, tiled PML slabs, "
                                                "free-surface rows, fault band (one stream)"}},
        "e2e": {"value": job_rate(npts, args.steps, world, e2e_s), "unit": "Gpt-steps/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "includes": "create + host-array upload + FP64 setup + steps + per-step output fetch"},
        "gpu_launches": LAUNCHES_PER_STEP * args.steps,
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_learned:
        line["learned_rs"] = learned_rs(dfd, device=local)
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(job, fx, st, layers)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
