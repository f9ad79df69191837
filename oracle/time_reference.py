"""Time the reference's own CUDA build on a benchmark workload -- measurement
infrastructure, not part of the product.

Writes the workload of bench.py (its params.json, Fault_geometry / Fault_init_stress
NetCDF files and Media1D table, in the reference's formats) to a scratch directory and
runs oracle/_ref/refharness_<variant> --time on it: the reference's launchers in the
order of its driver (main.cu:420-535), per-stage cudaDeviceSynchronize included, output
I/O excluded.  Prints one JSON line with the stepping loop's wall time.

usage: python oracle/time_reference.py --config curved|flat|large [--steps N] [--variant sp|dp]
"""
import argparse
import json
import os
import re
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path[:0] = [ROOT, os.path.join(ROOT, "tests", "golden")]


def main():
    import bench
    import cases

    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="curved")
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--variant", default="sp")
    a = ap.parse_args()
    job, fx, st, layers, label = bench.workload(a.config)
    nr = "" if int(job.get("NormalRefine", 1)) else "_nr"
    cj = "_cj" if int(job.get("useCerjan", 0)) else ""
    exe = os.path.join(HERE, "_ref", f"refharness_{a.variant}{nr}{cj}")
    with tempfile.TemporaryDirectory() as td:
        cases.write_job(td, job, fx, st, layers)
        r = subprocess.run([exe, os.path.join(td, "params.json"), td, str(a.steps), "0", "--time"],
                           capture_output=True, text=True)
    m = re.search(r"refharness timing: (\d+) steps in ([0-9.]+) s", r.stdout)
    if r.returncode != 0 or not m:
        raise SystemExit(f"reference run failed (rc {r.returncode}):\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}")
    steps, secs = int(m.group(1)), float(m.group(2))
    npts = job["NX"] * job["NY"] * job["NZ"]
    print(json.dumps({"impl": "reference CUDA build", "variant": os.path.basename(exe), "workload": label,
                      "nodes": npts, "steps": steps, "seconds": secs, "ms_per_step": 1e3 * secs / steps,
                      "gpt_steps_per_s": npts * steps / secs / 1e9}), flush=True)


if __name__ == "__main__":
    main()
