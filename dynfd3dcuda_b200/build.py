"""Build the CUDA extension in-tree: libdfd_b200.so (C ABI) and the dfd_b200 driver.

nvcc -gencode arch=compute_100a,code=sm_100a for every .cu; objects go to
dynfd3dcuda_b200/_build/, the shared library and the executable next to this file.
Rebuilds only what changed (mtime), in parallel.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libdfd_b200.so")
EXE = os.path.join(HERE, "dfd_b200")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU = ["dfd_volume.cu", "dfd_tile.cu", "dfd_pml.cu", "dfd_fault.cu", "dfd_mlp.cu", "dfd_precompute.cu", "dfd_setup.cu", "dfd_api.cu"]
CPP = ["dfd_host.cpp", "dfd_netcdf.cpp"]
HEADERS = ["dfd_internal.cuh", "dfd_stencil.cuh", "dfd_tma.cuh", "dfd_mlp.cuh", "dfd_host.h"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r.stderr


def build(verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    hdrs = [os.path.join(SRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "dfd_b200.h")]
    jobs = []
    objs = []
    for f in CU + CPP:
        src = os.path.join(SRC, f)
        obj = os.path.join(OBJ, f + ".o")
        objs.append(obj)
        if _stale(obj, [src] + hdrs):
            if f.endswith(".cu"):
                cmd = [nvcc()] + ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-c", src, "-o", obj]
            else:
                cmd = ["g++", "-O3", "-std=c++17", "-fPIC", "-I/usr/local/cuda/include", "-c", src, "-o", obj]
            jobs.append(cmd)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        for msg in ex.map(_run, jobs):
            if verbose and msg:
                print(msg, file=sys.stderr)
    if _stale(LIB, objs):
        _run([nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"])
    drv = os.path.join(SRC, "dfd_driver.cpp")
    if _stale(EXE, [drv, LIB] + hdrs):
        _run(["g++", "-O2", "-std=c++17", drv, "-o", EXE, "-L" + HERE, "-ldfd_b200", "-Wl,-rpath,$ORIGIN"])
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
