"""Builds the partitioner in-tree.

Outputs:
  gpu-heipa_b200/lib/libgpuheipa.so   C ABI (include/gpuheipa.h), sm_100a kernels
  gpu-heipa_b200/bin/GPU-HeiPa         CLI (partitioning)
  gpu-heipa_b200/bin/GPU-HeiProMap     CLI (process mapping)

CUDA sources are compiled with nvcc -gencode arch=compute_100a,code=sm_100a;
host sources with g++ (OpenMP). Objects go to gpu-heipa_b200/_build/ and are
rebuilt when a source or any header is newer.
"""
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib", "libgpuheipa.so")
BIN = os.path.join(HERE, "bin")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--extended-lambda", "-Xcompiler", "-fPIC,-fopenmp",
                     "-Xptxas", "-warn-spills"]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-fopenmp", "-Wall", "-Wno-unused-function", "-ffp-contract=off"]


def _newest(paths):
    return max(os.path.getmtime(p) for p in paths) if paths else 0.0


def _headers():
    return (glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + glob.glob(os.path.join(HERE, "csrc", "*.h")) +
            glob.glob(os.path.join(HERE, "host", "*.h")) + glob.glob(os.path.join(ROOT, "include", "*.h")))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: " + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build(verbose=False, jobs=None):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    os.makedirs(BIN, exist_ok=True)
    hdr_time = _newest(_headers())
    cu = sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))
    cpp = sorted(glob.glob(os.path.join(HERE, "host", "*.cpp")))
    jobs_list = []
    objs = []
    for src in cu + cpp:
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr_time):
            continue
        if src.endswith(".cu"):
            cmd = [NVCC] + NVCC_FLAGS + ["-c", src, "-o", obj]
        else:
            cmd = ["g++"] + CXX_FLAGS + ["-I/usr/local/cuda/include", "-c", src, "-o", obj]
        jobs_list.append(cmd)
    logs = []
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        for out in ex.map(_run, jobs_list):
            logs.append(out)
    if verbose:
        for l in logs:
            if l.strip():
                print(l)
    if jobs_list or not os.path.exists(LIB):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-Xcompiler", "-fopenmp", "-lgomp"])
    lib_time = os.path.getmtime(LIB)
    for app in ("GPU-HeiPa", "GPU-HeiProMap"):
        src = os.path.join(HERE, "apps", app + ".cpp")
        out = os.path.join(BIN, app)
        if not os.path.exists(src):
            continue
        app_hdr = _newest(glob.glob(os.path.join(HERE, "apps", "*.h")))
        if os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(src), lib_time, hdr_time, app_hdr):
            continue
        _run(["g++", "-O2", "-std=c++17", "-Wall", "-I" + os.path.join(ROOT, "include"), src, "-o", out,
              "-L" + os.path.dirname(LIB), "-lgpuheipa", "-Wl,-rpath,$ORIGIN/../lib"])
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIB)
