"""Generate the golden fixtures from the reference's own CUDA build.

Runs oracle/_ref/refharness_{sp,dp}[_nr] (the reference sources compiled for sm_100a
by oracle/Makefile, driven in the order of the reference driver) on every case of
cases.py and stores a compact subset of the dumped state as tests/golden/<case>_<var>.npz:

  every dump step : all on-fault 2-D arrays (the rupture sensor included), per-field
                    checksums of the wavefield and of the PML auxiliary arrays; with
                    thermal pressurisation (Friction_type
                    3) temperature and pore pressure at the fault
  final step      : the wavefield (full for the volume cases, the seven x-planes around
                    the fault over the rupture block otherwise), split-node state and the
                    traction layers over the same block; thermal-pressurisation columns
                    over the non-united block
  setup (dp only) : metric planes around the fault and the fault coefficient tables

Needs a GPU (the reference is CUDA-only).  usage:
    python tests/golden/make_golden.py --out DIR [--cases a,b] [--variants sp,dp]
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
import cases  # noqa: E402

# block of padded j indices kept for the rupture cases (the non-united nodes plus the
# stencil halo on the 76-node grids); a case may name its own block (meta "jblock")
JBLOCK = (24, 52)


def load_dumps(d):
    out = {}
    with open(os.path.join(d, "manifest.txt")) as f:
        for line in f:
            name, step, n, elem = line.split()
            n, elem, step = int(n), int(elem), int(step)
            if name in ("united", "faultgrid", "rup_index_y"):
                dt = np.int32
            else:
                dt = np.float64 if elem == 8 else np.float32
            out[(name, step)] = np.fromfile(os.path.join(d, f"{name}.s{step}.bin"), dtype=dt)
    return out


def checksums(a):
    a = a.astype(np.float64)
    return np.array([a.sum(), np.sqrt((a * a).sum()), np.abs(a).max()])


def run_case(name, variant, outdir):
    p, fx, st, layers, w0, meta = cases.get_case(name)
    with tempfile.TemporaryDirectory() as td:
        job, meta = cases.write_inputs(name, td)
        nr = "" if int(p.get("NormalRefine", 1)) else "_nr"
        cj = "_cj" if int(p.get("useCerjan", 0)) else ""
        exe = os.path.join(ROOT, "oracle", "_ref", f"refharness_{variant}{nr}{cj}")
        cmd = [exe, os.path.join(td, "params.json"), td, str(meta["steps"]), str(meta["every"])]
        if meta["volume"]:
            cmd.append("--volume")
        if w0 is not None:
            cmd += ["--init-wave", os.path.join(td, "wave0.f64")]
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
        if r.returncode != 0:
            raise RuntimeError(f"{name}/{variant}: harness failed rc={r.returncode}\n{r.stdout}\n{r.stderr}")
        dumps = load_dumps(td)
    NX, NY, NZ = p["NX"], p["NY"], p["NZ"]
    nx, ny, nz = NX + 6, NY + 6, NZ + 6
    i0 = nx // 2
    J0, J1 = meta.get("jblock", JBLOCK)
    steps = sorted({s for (_, s) in dumps if s >= 0})
    last = steps[-1]
    save = {"params": np.array(json.dumps(p)), "steps": np.array(steps), "variant": np.array(variant),
            "jblock": np.array([J0, J1])}
    for s in steps:
        W = dumps[("W", s)].reshape(9, nx, nz, ny)
        save[f"Wsum_s{s}"] = np.stack([checksums(W[f]) for f in range(9)])
        for aux in ("aux_x1", "aux_y1", "aux_z1"):
            if (aux, s) in dumps:
                save[f"{aux}sum_s{s}"] = checksums(dumps[(aux, s)])
        if not meta["volume"]:
            for nm in ("slip", "hslip", "Vs1", "Vs2", "Tn", "Ts1", "Ts2", "State", "init_t0", "tTn", "tTs1", "tTs2"):
                save[f"{nm}_s{s}"] = dumps[(nm, s)].astype(np.float32).reshape(NZ, NY)
            if ("rup_sensor", s) in dumps:
                save[f"rup_sensor_s{s}"] = dumps[("rup_sensor", s)].astype(np.float32).reshape(NZ, NY)
            for nm in ("TP_T", "TP_P"):
                if (nm, s) in dumps:  # thermal pressurisation: the on-fault point of each column
                    save[f"{nm}_s{s}"] = dumps[(nm, s)].astype(np.float32).reshape(-1, NZ, NY)[0]
    W = dumps[("W", last)].reshape(9, nx, nz, ny)
    if meta["volume"]:
        save["W_final"] = W.astype(np.float32)
    else:
        save["W_block"] = W[:, i0 - 3:i0 + 4, :, J0:J1].astype(np.float32)
        save["FW_block"] = dumps[("FW", last)].reshape(9, 2, nz, ny)[..., J0:J1].astype(np.float32)
        for nm in ("T11", "T12", "T13"):
            save[f"{nm}_block"] = dumps[(nm, last)].reshape(7, nz, ny)[..., J0:J1].astype(np.float32)
        for nm in ("hT11", "hT12", "hT13"):
            save[f"{nm}_block"] = dumps[(nm, last)].reshape(nz, ny)[:, J0:J1].astype(np.float32)
        fg = p["Fault_grid"]
        for nm in ("TP_T", "TP_P"):
            if (nm, last) in dumps:  # whole columns over the non-united block
                col = dumps[(nm, last)].reshape(-1, NZ, NY)
                save[f"{nm}_cols"] = col[:, fg[2] - 1:fg[3], fg[0] - 1:fg[1]].astype(np.float32)
    if variant.startswith("dp"):
        M = dumps[("M", -1)].reshape(13, nx, nz, ny)
        save["M_planes"] = M[:, i0 - 1:i0 + 2].astype(np.float32)
        save["matVx2Vz_top"] = dumps[("matVx2Vz", -1)].astype(np.float32)
        if not meta["volume"]:
            for nm in ("vec_n", "vec_s1", "vec_s2"):
                save[nm] = dumps[(nm, -1)].reshape(nz, ny, 3)[:, J0:J1].astype(np.float32)
            for nm in ("D21_1", "D33_2", "matPlus2Min1", "matMin2Plus5", "matT1toVxm", "matVztoVxp"):
                save[nm] = dumps[(nm, -1)].reshape(nz, ny, 9)[:, J0:J1].astype(np.float32)
            for nm in ("matVx2Vz1", "matPlus2Min2f", "matMin2Plus3f"):
                save[nm] = dumps[(nm, -1)].reshape(ny, 9).astype(np.float32)
            for nm in ("united", "faultgrid", "rup_index_y"):
                save[nm] = dumps[(nm, -1)].reshape(NZ, NY)
            save["str_peak"] = dumps[("str_peak", -1)].reshape(NZ, NY).astype(np.float32)
    fn = os.path.join(outdir, f"{name}_{variant}.npz")
    np.savez_compressed(fn, **save)
    return fn


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--cases", default=",".join(cases.CASES))
    ap.add_argument("--variants", default="sp,dp")
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    for c in a.cases.split(","):
        allowed = cases.get_case(c)[5].get("variants", ("sp", "dp"))
        for v in a.variants.split(","):
            if v not in allowed:
                continue
            fn = run_case(c, v, a.out)
            print(f"wrote {fn} ({os.path.getsize(fn) / 1e3:.0f} kB)", flush=True)


if __name__ == "__main__":
    main()
